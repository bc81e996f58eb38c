// Workset pairs from voxel blocks.
//
// Where several points share voxels (dense clusters), the digital Voronoi
// diagram holds one site per voxel: the other points of a voxel ("missing"
// points, GDelHost.cu:246-303) start from the voxel leader alone, and the
// leaders see only one point of each neighbouring voxel. Their initial stars are
// far from the final ones, and splaying builds them at several times the cost
// of an initial insertion. These two kernels add, for every point s of a voxel
// that holds several points, the K points nearest to s among the points of the
// 3x3x3 voxel block around s's voxel (pairs already in the worksets aside) as
// workset pairs of both points. (A point alone in its voxel is already paired
// with the leader of every occupied voxel around it by the Voronoi pairs; it
// gets the other points of those voxels when they select it.)
//
// Splaying needs symmetric worksets (b in a's history means a in b's, or on
// its way), so every pair is pushed both ways, and never twice: the selection
// of a point is "distance at most its threshold" (the K-th smallest block
// distance), and the pair (s, v) is pushed by s when v is in s's selection and
// either v > s or s is beyond v's threshold, else by v. The squared distance of
// a pair is the same float from both sides (the differences only change sign).
// Every selected pair is pushed once, except where the side the rule leaves it
// to never gathered the other (beyond the caps below); such a pair is left to
// splaying. Which pairs are added only changes the work splaying has left: the
// stars are decided by the exact predicates whatever their candidates
// (tests/test_block_rule.py restates the rule and checks it on the CPU).
//
// k_block_sel: warp per point; the block's occupied voxels (a voxel whose site
//   is itself; its points are the run of equal Morton keys from its leader) in
//   order of distance from the centre voxel, at most BLOCK_RUN points of each
//   and BLOCK_MAX in all; the K-th smallest squared distance by a bisection of
//   its float bits; the selection (minus the worksets' pairs) into a row of the
//   insertion-request array, free until splaying starts.
// k_block_push: warp per point, lane per selected point: the pushes.
#include "g4d_internal.cuh"

namespace g4d {

constexpr int BLOCK_RUN = 16;   // points taken from one voxel
constexpr int BLOCK_MAX = 128;  // block points considered (4 per lane)
constexpr int SEL_ROW = INBOX_CAP;  // selection row: ids in [0, SEL_ROW-1), count in the last entry
constexpr uint32_t INF_BITS = 0x7f800000u;

// The 27 voxels of the 3x3x3 block by distance from its centre (own voxel,
// faces, edges, corners): (dx+1) + 3 (dy+1) + 9 (dz+1).
__constant__ uint8_t c_block_order[27] = {13, 4,  10, 12, 14, 16, 22, 1,  3,  5,  7,  9,  11, 15,
                                          17, 19, 21, 23, 25, 0,  2,  6,  8,  18, 20, 24, 26};

__device__ __forceinline__ float dist2(double4 a, double4 b) {
    const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
    return (float)(dx * dx + dy * dy + dz * dz);
}

// Where point s's grid lies: one cloud (width D.G at offset 0), or a batch,
// where point s belongs to slot key >> 30, whose grid has width slotG[k] and
// starts at voxel slotVox[k] of the stacked grids.
struct GridOf {
    const int* slotG;        // null: one cloud
    const long long* slotVox;
    __device__ __forceinline__ void locate(const Dev& D, unsigned long long key, int* G, size_t* base) const {
        if (!slotG) { *G = D.G; *base = 0; return; }
        const int k = (int)(key >> 30);
        *G = slotG[k];
        *base = (size_t)slotVox[k];
    }
};

template <class KeyT>
__global__ void __launch_bounds__(128) k_block_sel(Dev D, const KeyT* __restrict__ keys, GridOf go,
                                                   const uint32_t* __restrict__ grid, const int* __restrict__ map,
                                                   int k_sel, int* __restrict__ sel, float* __restrict__ thr) {
    __shared__ int ids[4][BLOCK_MAX];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned full = 0xffffffffu;
    for (int s = blockIdx.x * 4 + w; s < D.n; s += gridDim.x * 4) {
        // only points of voxels with several points select: elsewhere the
        // Voronoi pairs already join every occupied neighbouring voxel
        const KeyT ks = keys[s];
        if (!((s > 0 && keys[s - 1] == ks) || (s + 1 < D.n && keys[s + 1] == ks))) {
            if (lane == 0) thr[s] = -1.0f;
            continue;
        }
        int G;
        size_t gbase;
        go.locate(D, (unsigned long long)ks, &G, &gbase);
        const uint32_t e = D.vox[s];
        int lead = 0, run = 0;
        if (lane < 27) {
            const int o = c_block_order[lane];
            const int xx = (int)vx(e) + o % 3 - 1, yy = (int)vy(e) + (o / 3) % 3 - 1, zz = (int)vz(e) + o / 9 - 1;
            if (xx >= 0 && yy >= 0 && zz >= 0 && xx < G && yy < G && zz < G) {
                const size_t u = gbase + ((size_t)zz * G + yy) * G + xx;
                if (grid[u] == enc_vox((uint32_t)xx, (uint32_t)yy, (uint32_t)zz)) {
                    lead = map[u];
                    const KeyT k = keys[lead];
                    run = 1;
                    while (run < BLOCK_RUN && lead + run < D.n && keys[lead + run] == k) ++run;
                }
            }
        }
        int incl = run;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int t = __shfl_up_sync(full, incl, d);
            if (lane >= d) incl += t;
        }
        const int total = min(__shfl_sync(full, incl, 31), BLOCK_MAX);
        if (total <= 1) {  // s alone in its block
            if (lane == 0) thr[s] = -1.0f;
            continue;
        }
        __syncwarp();  // the previous point's reads of ids are done
        const int before = incl - run;
        const int take = max(0, min(run, BLOCK_MAX - before));
        for (int j = 0; j < take; ++j) ids[w][before + j] = lead + j;
        __syncwarp();
        const double4 ps = D.P[s];
        uint32_t db[4];
        int id[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int i = lane + 32 * k;
            id[k] = i < total ? ids[w][i] : -1;
            if (id[k] == s) id[k] = -1;
            db[k] = id[k] >= 0 ? __float_as_uint(dist2(ps, D.P[id[k]])) : 0xffffffffu;
        }
        int valid = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) valid += __popc(__ballot_sync(full, id[k] >= 0));
        // threshold: the k_sel-th smallest distance (all of them when fewer)
        uint32_t t = INF_BITS;
        if (valid > k_sel) {
            uint32_t lo = 0, hi = INF_BITS;  // smallest t with count(d <= t) >= k_sel
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                int c = 0;
#pragma unroll
                for (int k = 0; k < 4; ++k) c += __popc(__ballot_sync(full, db[k] <= mid));
                if (c >= k_sel) hi = mid; else lo = mid + 1;
            }
            t = lo;
        }
        // the selection, minus the pairs already in s's workset
        bool pick[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) pick[k] = id[k] >= 0 && db[k] <= t;
        const int bc = min(D.bucketCount[s], BUCKET_CAP);
        const int* bk = D.bucket + (size_t)s * BUCKET_CAP;
        const int b0 = lane < bc ? bk[lane] : -1, b1 = lane + 32 < bc ? bk[lane + 32] : -1;
        for (int j = 0; j < bc; ++j) {
            const int b = __shfl_sync(full, j < 32 ? b0 : b1, j & 31);
#pragma unroll
            for (int k = 0; k < 4; ++k) pick[k] = pick[k] && id[k] != b;
        }
        int* row = sel + (size_t)s * SEL_ROW;
        int cnt = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const unsigned m = __ballot_sync(full, pick[k]);
            const int pos = cnt + __popc(m & ((1u << lane) - 1u));
            if (pick[k] && pos < SEL_ROW - 1) row[pos] = id[k];
            cnt += __popc(m);
        }
        if (lane == 0) {
            row[SEL_ROW - 1] = min(cnt, SEL_ROW - 1);
            thr[s] = __uint_as_float(t);
        }
    }
}

__global__ void __launch_bounds__(128) k_block_push(Dev D, const int* __restrict__ sel,
                                                    const float* __restrict__ thr) {
    const int lane = threadIdx.x & 31;
    for (int s = blockIdx.x * 4 + (threadIdx.x >> 5); s < D.n; s += gridDim.x * 4) {
        if (!(thr[s] >= 0.0f)) continue;
        const int* row = sel + (size_t)s * SEL_ROW;
        const int cnt = row[SEL_ROW - 1];
        const double4 ps = D.P[s];
        int pushed = 0;
        for (int j = lane; j < cnt; j += 32) {
            const int v = row[j];
            if (v > s || !(dist2(ps, D.P[v]) <= thr[v])) {
                bucket_push(D, s, v);
                bucket_push(D, v, s);
                ++pushed;
            }
        }
        pushed = __reduce_add_sync(0xffffffffu, pushed);
        if (lane == 0 && pushed) atomicAdd(&D.ctr->block_pairs, pushed);
    }
}

__global__ void k_workset_total(Dev D) {
    unsigned long long t = 0;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < D.n; s += gridDim.x * blockDim.x)
        t += (unsigned long long)max(min(D.bucketCount[s], BUCKET_CAP), MIN_WORKSET);
    for (int d = 16; d > 0; d >>= 1) t += __shfl_xor_sync(0xffffffffu, t, d);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(&D.ctr->cand_total, t);
}

void launch_workset_total(const Launch& L, const Dev& D) {
    int b = (D.n + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    cudaMemsetAsync(&D.ctr->cand_total, 0, sizeof(unsigned long long), L.stream);
    k_workset_total<<<b, 256, 0, L.stream>>>(D);
    ++*L.launches;
}

void launch_block_pairs(const Launch& L, const Dev& D, const uint32_t* grid, const int* map, int k_sel) {
    int b = (D.n + 3) / 4;
    if (b > 148 * 16) b = 148 * 16;
    float* thr = reinterpret_cast<float*>(D.inboxCount);
    k_block_sel<uint32_t><<<b, 128, 0, L.stream>>>(D, D.mkey, GridOf{nullptr, nullptr}, grid, map, k_sel, D.inbox, thr);
    k_block_push<<<b, 128, 0, L.stream>>>(D, D.inbox, thr);
    *L.launches += 2;
}

void launch_block_pairs_batch(const Launch& L, const Dev& D, const uint32_t* grids, const int* maps,
                              const unsigned long long* skey, const int* slotG, const long long* slotVox, int k_sel) {
    int b = (D.n + 3) / 4;
    if (b > 148 * 16) b = 148 * 16;
    float* thr = reinterpret_cast<float*>(D.inboxCount);
    k_block_sel<unsigned long long><<<b, 128, 0, L.stream>>>(D, skey, GridOf{slotG, slotVox}, grids, maps, k_sel,
                                                             D.inbox, thr);
    k_block_push<<<b, 128, 0, L.stream>>>(D, D.inbox, thr);
    *L.launches += 2;
}

}  // namespace g4d
