// Candidate pairs of the learned star proposal and their features.
//
// For every point s the candidates are the distinct Voronoi sites within
// Chebyshev distance 2 of s's voxel (a 5x5x5 block of the digital Voronoi grid),
// each resolved to its point v (the voxel leader), v != s, that is not already
// in s's initial workset (the Voronoi pairs and missing-point pairs put there
// before the proposal runs): the network only decides which further pairs to
// add. Each unordered pair is scored once: from s when s < v, or from s when
// s is not its voxel's leader (then s is no site, and v's block cannot name
// it); a leader s > v is left to v's block, which names s because the
// Chebyshev distance of their voxels is symmetric. Features of (s, v),
// in grid units so that they do not depend on the cloud's extent:
//   0..2  (v - s) / 2           offset
//   3     |v - s| / 4           distance
//   4     voxels of the block whose site is v, / 16
//   5     distinct sites in the block, / 16
//   6..15 zero (padding to one K=16 MMA step)
// One warp per point; rows are reserved with one atomic per point, so their
// order is arbitrary.
#include <cuda_bf16.h>

#include <cstdint>

#include "g4d_internal.cuh"

namespace g4d {

constexpr int RING_PER_STAR = 64;  // at most this many candidates per point

__global__ void __launch_bounds__(128) k_ring(Dev D, Ring R) {
    __shared__ uint32_t hs[4][256];   // block sites, open addressing
    __shared__ int hc[4][256];        // voxels per site
    __shared__ int list[4][128];      // occupied slots
    __shared__ int nlist[4];
    __shared__ int wset[4][BUCKET_CAP];  // s's initial workset
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int G = R.cols.G;
    const int warps = gridDim.x * 4;
    for (int s = blockIdx.x * 4 + w; s < D.n; s += warps) {
        __syncwarp();
        for (int k = lane; k < 256; k += 32) { hs[w][k] = MARKER; hc[w][k] = 0; }
        if (lane == 0) nlist[w] = 0;
        const int bc = min(D.bucketCount[s], BUCKET_CAP);
        for (int k = lane; k < bc; k += 32) wset[w][k] = D.bucket[(size_t)s * BUCKET_CAP + k];
        const bool leader = s == 0 || D.mkey[s - 1] != D.mkey[s];
        __syncwarp();
        const uint32_t e = D.vox[s];
        const int x = (int)vx(e), y = (int)vy(e), z = (int)vz(e);
        for (int i = lane; i < 125; i += 32) {
            const int xx = x + i % 5 - 2, yy = y + (i / 5) % 5 - 2, zz = z + i / 25 - 2;
            if (xx < 0 || yy < 0 || zz < 0 || xx >= G || yy >= G || zz >= G) continue;
            const uint32_t site = R.grid[((size_t)zz * G + yy) * G + xx];
            if (site == MARKER) continue;
            uint32_t slot = (site * 2654435761u) >> 24;
            for (int probe = 0; probe < 256; ++probe) {
                const uint32_t old = atomicCAS(&hs[w][slot], MARKER, site);
                if (old == MARKER || old == site) {
                    atomicAdd(&hc[w][slot], 1);
                    if (old == MARKER) list[w][atomicAdd(&nlist[w], 1)] = (int)slot;
                    break;
                }
                slot = (slot + 1) & 255u;
            }
        }
        __syncwarp();
        const int nd = nlist[w];
        const double4 ps = D.P[s];
        int base = 0, taken = 0;
        for (int j0 = 0; j0 < nd; j0 += 32) {
            const int j = j0 + lane;
            int v = -1, slot = 0;
            if (j < nd) {
                slot = list[w][j];
                v = site_to_id(R.cols, hs[w][slot]);
                if (v == s || (leader && v < s)) v = -1;
                for (int k = 0; k < bc && v >= 0; ++k)
                    if (wset[w][k] == v) v = -1;
            }
            const unsigned m = __ballot_sync(0xffffffffu, v >= 0);
            int cnt = __popc(m);
            if (taken + cnt > RING_PER_STAR) cnt = RING_PER_STAR - taken;
            if (cnt <= 0) break;
            if (lane == 0) base = atomicAdd(R.rows, cnt);
            base = __shfl_sync(0xffffffffu, base, 0);
            const int k = __popc(m & ((1u << lane) - 1u));
            if (v >= 0 && k < cnt && base + k < R.cap) {
                const int row = base + k;
                const double4 pv = D.P[v];
                const double dx = (pv.x - ps.x) * R.scale, dy = (pv.y - ps.y) * R.scale, dz = (pv.z - ps.z) * R.scale;
                const float f[6] = {(float)(dx * 0.5), (float)(dy * 0.5), (float)(dz * 0.5),
                                    (float)(sqrt(dx * dx + dy * dy + dz * dz) * 0.25), hc[w][slot] * (1.f / 16.f),
                                    nd * (1.f / 16.f)};
                __align__(16) __nv_bfloat16 h[16];
                for (int q = 0; q < 16; ++q) h[q] = __float2bfloat16_rn(q < 6 ? f[q] : 0.f);
                uint4* dst = reinterpret_cast<uint4*>(R.x + (size_t)row * 16);
                dst[0] = reinterpret_cast<const uint4*>(h)[0];
                dst[1] = reinterpret_cast<const uint4*>(h)[1];
                R.pair[row] = make_int2(s, v);
            }
            taken += cnt;
        }
    }
}

// candidates the network accepts join both points' initial worksets (the
// build kernel removes duplicates)
__global__ void k_prop_merge(Dev D, const int2* __restrict__ pair, const float* __restrict__ logits,
                             const int* __restrict__ rows, int cap, float threshold) {
    const int n = min(*rows, cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!(logits[i] > threshold)) continue;
        const int2 p = pair[i];
        bucket_push(D, p.x, p.y);
        bucket_push(D, p.y, p.x);
        atomicAdd(&D.ctr->proposed, 1);
    }
}

void launch_ring(const Launch& L, const Dev& D, const Ring& R) {
    int b = (D.n + 3) / 4;
    if (b > 148 * 16) b = 148 * 16;
    k_ring<<<b < 1 ? 1 : b, 128, 0, L.stream>>>(D, R);
    ++*L.launches;
}

void launch_prop_merge(const Launch& L, const Dev& D, const int2* pair, const float* logits, const int* rows,
                       int cap, float threshold) {
    int b = (cap + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    k_prop_merge<<<b < 1 ? 1 : b, 256, 0, L.stream>>>(D, pair, logits, rows, cap, threshold);
    ++*L.launches;
}

}  // namespace g4d
