// Digital Voronoi diagram on the G^3 grid and the candidate Delaunay edges it
// implies.
//
// The reference computes the exact Euclidean distance transform with PBA
// (PBA/pba3DHost.cu:200-295, PBA/pba3DKernel.h:80-579): seed the grid,
// flood along z, Maurer proximate-site stack along y, colour, transpose, repeat
// for x, then replace site coordinates by point ids. Here the same three axis
// phases are re-planned for B200:
//   z: seeding fused with the flood. Sites are bucketed per (x,y) column by a
//      radix sort, so each column is written once (4 B/voxel, no memset, no read).
//   y: one CTA stages a TX x G slab (x-runs of TX voxels, one row per y) in
//      shared memory and every thread resolves one voxel by an outward search
//      that stops as soon as d^2 >= best (exact; 4 B read + 4 B write per voxel).
//   x: same with G x TY contiguous rows (no transposes).
// Sites stay encoded as voxel coordinates; they become point ids only for the
// emitted pairs (a lookup in the column-sorted site list).
//
// Batches: the grids of all clouds with the same G are stacked (grid k of the
// stack at offset k*G^3, its columns at k*G^2 in the column index), and each
// kernel takes the stack depth K as its last grid dimension, so one launch per
// grid size serves every cloud of that size. One cloud is a stack of depth 1.
#include "g4d_internal.cuh"

namespace g4d {

#ifndef PBA_U
#define PBA_U 2  // search distances per loop iteration in the y and x passes
#endif

template <class KeyT>
__global__ void __launch_bounds__(128) k_pba_z(int G, const KeyT* __restrict__ ckey, const int* __restrict__ cs,
                                               const int* __restrict__ ce, uint32_t* __restrict__ out) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 4 + threadIdx.y;
    if (x >= G || y >= G) return;
    const size_t plane = (size_t)G * G;
    const size_t c = (size_t)blockIdx.z * plane + (size_t)y * G + x;
    int i = cs[c];
    const int e = ce[c];
    uint32_t* o = out + (size_t)blockIdx.z * plane * G + (size_t)y * G + x;
    // empty columns run the same loop so that the warp stays together: each
    // store is then one full 128-byte line (a store split by divergence
    // writes partial sectors, which L2 fills from DRAM first)
    const bool empty = i >= e;
    int prev = -(1 << 20);
    int next = empty ? (1 << 20) : (int)(ckey[i] & 1023u);
    for (int z = 0; z < G; ++z) {
        while (next <= z) {
            prev = next;
            ++i;
            next = i < e ? (int)(ckey[i] & 1023u) : (1 << 20);
        }
        const int zs = (z - prev <= next - z) ? prev : next;
        const uint32_t v = empty ? MARKER : enc_vox(x, y, zs);
        __syncwarp();
        o[z * plane] = v;
    }
}

// y pass: TX consecutive x-columns at fixed z. The slab is staged transposed
// (one line per x, pitch G+1 so the transposing stores are conflict-free), a
// warp resolves 32 consecutive voxels of one line (neighbouring voxels have
// similar search lengths, so the warp stays converged), and results go
// through a second, row-major tile so the global stores are coalesced.
template <int TX>
__global__ void __launch_bounds__(256) k_pba_y(int G, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    extern __shared__ uint32_t smem_pba[];
    uint32_t* lines = smem_pba;                     // [TX][G+1]
    uint32_t* res = smem_pba + (size_t)TX * (G + 1);  // [G][TX+1]
    const int x0 = blockIdx.x * TX;
    const int z = blockIdx.y;
    const size_t zoff = ((size_t)blockIdx.z * G + z) * G * G;
    const int total = G * TX;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int yy = k / TX, xx = k % TX;
        lines[xx * (G + 1) + yy] = in[zoff + (size_t)yy * G + x0 + xx];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int xx = k / G, y = k % G;
        const uint32_t* line = lines + xx * (G + 1);
        uint32_t best = line[y];
        int bestd = best != MARKER ? (z - (int)vz(best)) * (z - (int)vz(best)) : 0x7fffffff;
        // PBA_U distances per iteration (2 PBA_U loads in flight); the visiting
        // order (y - d before y + d, d ascending) and the strict improvement
        // rule are those of a one-step search, so ties resolve the same way
        for (int d = 1; d * d < bestd; d += PBA_U) {
            if (y - d < 0 && y + d >= G) break;
            uint32_t c[2 * PBA_U];
#pragma unroll
            for (int q = 0; q < PBA_U; ++q) {
                c[2 * q] = y - d - q >= 0 ? line[y - d - q] : MARKER;
                c[2 * q + 1] = y + d + q < G ? line[y + d + q] : MARKER;
            }
#pragma unroll
            for (int q = 0; q < 2 * PBA_U; ++q) {
                if (c[q] == MARKER) continue;
                const int dy = d + (q >> 1), dz = z - (int)vz(c[q]);
                const int dd = dy * dy + dz * dz;
                if (dd < bestd) { bestd = dd; best = c[q]; }
            }
        }
        res[y * (TX + 1) + xx] = best;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int yy = k / TX, xx = k % TX;
        out[zoff + (size_t)yy * G + x0 + xx] = res[yy * (TX + 1) + xx];
    }
}

// x pass: TY contiguous rows of G voxels at fixed z
template <int TY>
__global__ void __launch_bounds__(256) k_pba_x(int G, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    extern __shared__ uint32_t tile[];
    const int y0 = blockIdx.x * TY;
    const int z = blockIdx.y;
    const size_t base = ((size_t)blockIdx.z * G + z) * G * G + (size_t)y0 * G;
    const int total = G * TY;
    const uint4* in4 = reinterpret_cast<const uint4*>(in + base);
    uint4* t4 = reinterpret_cast<uint4*>(tile);
    for (int k = threadIdx.x; k < total / 4; k += blockDim.x) t4[k] = in4[k];
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int row = k / G, x = k % G;
        const int y = y0 + row;
        const uint32_t* line = tile + row * G;
        uint32_t best = line[x];
        int bestd = 0x7fffffff;
        if (best != MARKER) {
            const int dy = y - (int)vy(best), dz = z - (int)vz(best);
            bestd = dy * dy + dz * dz;
        }
        for (int d = 1; d * d < bestd; d += PBA_U) {  // as in the y pass
            if (x - d < 0 && x + d >= G) break;
            uint32_t c[2 * PBA_U];
#pragma unroll
            for (int q = 0; q < PBA_U; ++q) {
                c[2 * q] = x - d - q >= 0 ? line[x - d - q] : MARKER;
                c[2 * q + 1] = x + d + q < G ? line[x + d + q] : MARKER;
            }
#pragma unroll
            for (int q = 0; q < 2 * PBA_U; ++q) {
                if (c[q] == MARKER) continue;
                const int dx = d + (q >> 1), dy = y - (int)vy(c[q]), dz = z - (int)vz(c[q]);
                const int dd = dx * dx + dy * dy + dz * dz;
                if (dd < bestd) { bestd = dd; best = c[q]; }
            }
        }
        out[base + k] = best;
    }
}


#ifndef PAIR_HASH_LOG2
#define PAIR_HASH_LOG2 11
#endif
#ifndef PAIR_ZC_DEF
#define PAIR_ZC_DEF 16
#endif
#ifndef PAIR_WARPS_DEF
#define PAIR_WARPS_DEF 4
#endif
constexpr int PAIR_HASH = 1 << PAIR_HASH_LOG2;  // block hash entries (8 bytes each)
constexpr int PAIR_PROBES = 32;
constexpr int PAIR_ZC = PAIR_ZC_DEF;            // cube planes per block
constexpr int PAIR_WARPS = PAIR_WARPS_DEF;      // warps per block, one row of x each

template <class KeyT>
__device__ __forceinline__ void pair_hash_insert(unsigned long long* hs, unsigned long long key, const Dev& D,
                                                 const Cols<KeyT>& C) {
    unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> (64 - PAIR_HASH_LOG2));
    for (int probe = 0; probe < PAIR_PROBES; ++probe) {
        const unsigned long long old = atomicCAS(&hs[h], ~0ull, key);
        if (old == ~0ull || old == key) return;
        h = (h + 1) & (PAIR_HASH - 1);
    }
    // crowded table (dense regions hold thousands of pairs per block): emit
    // directly instead of probing further
    const int ia = site_to_id(C, (uint32_t)(key >> 32)), ib = site_to_id(C, (uint32_t)key);
    if (ia >= 0 && ib >= 0) { bucket_push(D, ia, ib); bucket_push(D, ib, ia); }
}

// Candidate Delaunay edges: every two distinct sites of a 2x2x2 voxel cube in
// which at least four sites meet (a digital Voronoi vertex: its sites are
// pairwise Voronoi neighbours; the reference reads the same cubes and emits
// around digital Voronoi vertices, GDelKernels.cu:137-299). One thread sweeps a
// column of cubes along z, keeping the previous voxel plane in registers and
// loading the plane after the next one ahead of use (4 loads per cube,
// coalesced over x). The distinct sites of a cube are a bit mask computed
// without branches (bit i: voxel i differs from voxels 0..i-1), so every lane
// does the same few dozen instructions per cube. Vertex cubes are rare (about
// 5% of the cubes): a lane queues the site set of each one (skipping a repeat
// of its previous set) in a per-warp queue, and every 32 queued cubes the warp
// emits their pairs, one cube per lane, into a block-local hash that removes
// duplicates before the per-star scatter.
// all pairs of one queued vertex cube into the block hash
template <class KeyT>
__device__ __forceinline__ void emit_cube(unsigned long long* hs, const uint32_t* q, int ns, const Dev& D,
                                          const Cols<KeyT>& C) {
    for (int i = 0; i < ns; ++i)
        for (int j = i + 1; j < ns; ++j) {
            const uint32_t lo = q[i] < q[j] ? q[i] : q[j], hi = q[i] < q[j] ? q[j] : q[i];
            pair_hash_insert(hs, ((unsigned long long)lo << 32) | hi, D, C);
        }
}

constexpr int PAIR_QUEUE = 64;  // queued vertex cubes per warp

// bit i set when v[i] differs from v[0..i-1]; v[0..3] is the lower plane
__device__ __forceinline__ uint32_t distinct_mask(const uint32_t (&v)[8]) {
    uint32_t m = 1u;
#pragma unroll
    for (int i = 1; i < 8; ++i) {
        bool fresh = true;
#pragma unroll
        for (int j = 0; j < i; ++j) fresh = fresh && (v[i] != v[j]);
        m |= (uint32_t)fresh << i;
    }
    return m;
}

template <class KeyT>
__global__ void __launch_bounds__(32 * PAIR_WARPS) k_pairs(Dev D, const uint32_t* __restrict__ stack, Cols<KeyT> C, int nzc) {
    __shared__ unsigned long long hs[PAIR_HASH];
    __shared__ uint32_t qs[PAIR_WARPS][PAIR_QUEUE][8];  // site sets of vertex cubes
    __shared__ uint8_t qn[PAIR_WARPS][PAIR_QUEUE];
    const int G = C.G;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (int k = tid; k < PAIR_HASH; k += 32 * PAIR_WARPS) hs[k] = ~0ull;
    __syncthreads();
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * PAIR_WARPS + threadIdx.y;
    const int kk = blockIdx.z / nzc;  // grid of the stack
    const int z0 = (blockIdx.z - kk * nzc) * PAIR_ZC;
    const size_t plane = (size_t)G * G;
    const uint32_t* grid = stack + (size_t)kk * plane * G;
    C.start += (size_t)kk * plane;
    C.end += (size_t)kk * plane;
    const int lane = threadIdx.x, w = threadIdx.y;
    // every lane of the warp walks the same z range so the warp collectives
    // below stay converged; lanes past the grid edge carry no pairs (they read
    // column 0, which is in bounds)
    const bool active = x < G - 1 && y < G - 1;
    const int zend = min(z0 + PAIR_ZC, G - 1);
    if (y < G - 1 && z0 < G - 1) {
        const uint32_t* g = grid + (size_t)y * G + (active ? x : 0);
        uint32_t v[8];
        {
            const size_t o = (size_t)z0 * plane;
            v[0] = g[o]; v[1] = g[o + 1]; v[2] = g[o + G]; v[3] = g[o + G + 1];
        }
        // plane z0+1 exists: z0 < G-1
        uint32_t n0, n1, n2, n3;
        {
            const size_t o = (size_t)(z0 + 1) * plane;
            n0 = g[o]; n1 = g[o + 1]; n2 = g[o + G]; n3 = g[o + G + 1];
        }
        unsigned long long last = 0;  // signature of the set this lane queued last
        int qc = 0;                   // queued cubes of this warp (same in every lane)
        for (int z = z0; z < zend; ++z) {
            v[4] = n0; v[5] = n1; v[6] = n2; v[7] = n3;
            if (z + 1 < zend) {  // the plane after the next one, loaded ahead of use
                const size_t o = (size_t)(z + 2) * plane;
                n0 = g[o]; n1 = g[o + 1]; n2 = g[o + G]; n3 = g[o + G + 1];
            }
            bool cand = false;
            uint32_t m = 0;
            // a warp whose cubes all lie inside one Voronoi cell each skips the mask
            const bool mixed = (v[1] != v[0]) | (v[2] != v[0]) | (v[3] != v[0]) | (v[4] != v[0]) |
                               (v[5] != v[0]) | (v[6] != v[0]) | (v[7] != v[0]);
            if (__any_sync(0xffffffffu, active && mixed)) {
                m = distinct_mask(v);
                if (active && __popc(m) >= 4) {
                    // consecutive cubes around one Voronoi vertex repeat its set
                    unsigned long long sum = 0, xr = 0;
#pragma unroll
                    for (int k = 0; k < 8; ++k)
                        if (m >> k & 1u) { sum += v[k]; xr ^= (unsigned long long)v[k] * 0x9E3779B97F4A7C15ull; }
                    const unsigned long long sig = (sum << 32) ^ xr ^ (unsigned long long)__popc(m);
                    cand = sig != last;
                    last = sig;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, cand);
            if (cand) {
                const int pos = qc + __popc(bal & ((1u << lane) - 1u));
                int ns = 0;
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    if (m >> k & 1u) qs[w][pos][ns++] = v[k];
                qn[w][pos] = (uint8_t)ns;
            }
            qc += __popc(bal);
            if (qc >= 32) {  // one queued cube per lane
                __syncwarp();
                emit_cube(hs, qs[w][lane], qn[w][lane], D, C);
                __syncwarp();
                for (int k = 32 + lane; k < qc; k += 32) {
                    for (int q = 0; q < qn[w][k]; ++q) qs[w][k - 32][q] = qs[w][k][q];
                    qn[w][k - 32] = qn[w][k];
                }
                qc -= 32;
                __syncwarp();
            }
            v[0] = v[4]; v[1] = v[5]; v[2] = v[6]; v[3] = v[7];
        }
        __syncwarp();
        if (lane < qc) emit_cube(hs, qs[w][lane], qn[w][lane], D, C);
    }
    __syncthreads();
    for (int k = tid; k < PAIR_HASH; k += 32 * PAIR_WARPS) {
        const unsigned long long key = hs[k];
        if (key == ~0ull) continue;
        const int ia = site_to_id(C, (uint32_t)(key >> 32)), ib = site_to_id(C, (uint32_t)key);
        if (ia >= 0 && ib >= 0) {
            bucket_push(D, ia, ib);
            bucket_push(D, ib, ia);
        }
    }
}

// Points that share a voxel with a smaller Morton index are absent from the
// digital diagram; each is paired with its voxel's leader (GDelKernels.cu:109-135).
template <class KeyT>
__global__ void k_missing(Dev D, const KeyT* __restrict__ mkey) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += gridDim.x * blockDim.x) {
        const KeyT k = mkey[i];
        if (i == 0 || mkey[i - 1] != k) continue;
        int j = i - 1;
        while (j > 0 && mkey[j - 1] == k) --j;
        bucket_push(D, i, j);
        bucket_push(D, j, i);
    }
}

void launch_pba_z(const Launch& L, const Dev& D, uint32_t* out) {
    dim3 b(32, 4), g((D.G + 31) / 32, (D.G + 3) / 4, 1);
    k_pba_z<<<g, b, 0, L.stream>>>(D.G, D.ckey, D.colStart, D.colEnd, out);
    ++*L.launches;
}

void launch_pba_z_stack(const Launch& L, int G, int K, const unsigned long long* ckey, const int* cs, const int* ce,
                        uint32_t* out) {
    dim3 b(32, 4), g((G + 31) / 32, (G + 3) / 4, K);
    k_pba_z<<<g, b, 0, L.stream>>>(G, ckey, cs, ce, out);
    ++*L.launches;
}

void launch_pba_y(const Launch& L, int G, const uint32_t* in, uint32_t* out) { launch_pba_y_stack(L, G, 1, in, out); }

void launch_pba_y_stack(const Launch& L, int G, int K, const uint32_t* in, uint32_t* out) {
    // two tiles of TX*G voxels: about 34 KB for G >= 256
    const int TX = G >= 512 ? 8 : (G >= 256 ? 16 : 32);
    const size_t sm = ((size_t)TX * (G + 1) + (size_t)G * (TX + 1)) * 4;
    switch (TX) {
#define G4D_Y(T)                                                                                  \
    case T:                                                                                       \
        cudaFuncSetAttribute(k_pba_y<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm); \
        k_pba_y<T><<<dim3(G / T, G, K), 256, sm, L.stream>>>(G, in, out);                         \
        break;
        G4D_Y(8) G4D_Y(16) G4D_Y(32)
#undef G4D_Y
        default: break;
    }
    ++*L.launches;
}

void launch_pba_x(const Launch& L, int G, const uint32_t* in, uint32_t* out) { launch_pba_x_stack(L, G, 1, in, out); }

void launch_pba_x_stack(const Launch& L, int G, int K, const uint32_t* in, uint32_t* out) {
    // TY rows of G voxels: 32 KB of shared memory per block
    const int TY = G >= 1024 ? 8 : (G >= 512 ? 16 : (G >= 256 ? 32 : (8192 / G < G ? 8192 / G : G)));
    const size_t sm = (size_t)G * TY * 4;
    switch (TY) {
#define G4D_X(T)                                                                                   \
    case T:                                                                                        \
        cudaFuncSetAttribute(k_pba_x<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);  \
        k_pba_x<T><<<dim3(G / T, G, K), 256, sm, L.stream>>>(G, in, out);                          \
        break;
        G4D_X(8) G4D_X(16) G4D_X(32) G4D_X(64) G4D_X(128) G4D_X(256)
#undef G4D_X
        default: break;
    }
    ++*L.launches;
}

void launch_pairs(const Launch& L, const Dev& D, const uint32_t* grid) {
    const int G = D.G;
    const int nzc = (G - 1 + PAIR_ZC - 1) / PAIR_ZC;
    dim3 b(32, PAIR_WARPS), g((G - 1 + 31) / 32, (G - 1 + PAIR_WARPS - 1) / PAIR_WARPS, nzc);
    k_pairs<<<g, b, 0, L.stream>>>(D, grid, Cols<uint32_t>{D.ckey, D.cid, D.colStart, D.colEnd, G}, nzc);
    ++*L.launches;
}

void launch_pairs_stack(const Launch& L, const Dev& D, const uint32_t* stack, int G, int K,
                        const unsigned long long* ckey, const int* cid, const int* cs, const int* ce) {
    const int nzc = (G - 1 + PAIR_ZC - 1) / PAIR_ZC;
    dim3 b(32, PAIR_WARPS), g((G - 1 + 31) / 32, (G - 1 + PAIR_WARPS - 1) / PAIR_WARPS, nzc * K);
    k_pairs<<<g, b, 0, L.stream>>>(D, stack, Cols<unsigned long long>{ckey, cid, cs, ce, G}, nzc);
    ++*L.launches;
}

void launch_missing(const Launch& L, const Dev& D) {
    int blocks = (D.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_missing<<<blocks, 256, 0, L.stream>>>(D, D.mkey);
    ++*L.launches;
}

void launch_missing_u64(const Launch& L, const Dev& D, const unsigned long long* mkey) {
    int blocks = (D.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_missing<<<blocks, 256, 0, L.stream>>>(D, mkey);
    ++*L.launches;
}

}  // namespace g4d
