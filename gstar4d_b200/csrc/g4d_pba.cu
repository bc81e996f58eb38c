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
#include "g4d_internal.cuh"

namespace g4d {

__global__ void __launch_bounds__(128) k_pba_z(int G, const uint32_t* __restrict__ ckey, const int* __restrict__ cs,
                                               const int* __restrict__ ce, uint32_t* __restrict__ out) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 4 + threadIdx.y;
    if (x >= G || y >= G) return;
    const int c = y * G + x;
    int i = cs[c];
    const int e = ce[c];
    const size_t plane = (size_t)G * G;
    uint32_t* o = out + (size_t)y * G + x;
    if (i >= e) {
        for (int z = 0; z < G; ++z) o[z * plane] = MARKER;
        return;
    }
    int prev = -(1 << 20);
    int next = (int)(ckey[i] & 1023u);
    for (int z = 0; z < G; ++z) {
        while (next <= z) {
            prev = next;
            ++i;
            next = i < e ? (int)(ckey[i] & 1023u) : (1 << 20);
        }
        const int zs = (z - prev <= next - z) ? prev : next;
        o[z * plane] = enc_vox(x, y, zs);
    }
}

// y pass: tile[y][tx], TX consecutive x at fixed z
template <int TX>
__global__ void __launch_bounds__(256) k_pba_y(int G, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    extern __shared__ uint32_t tile[];
    const int x0 = blockIdx.x * TX;
    const int z = blockIdx.y;
    const size_t zoff = (size_t)z * G * G;
    const int total = G * TX;
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int yy = k / TX, xx = k % TX;
        tile[k] = in[zoff + (size_t)yy * G + x0 + xx];
    }
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int y = k / TX, xx = k % TX;
        uint32_t best = MARKER;
        int bestd = 0x7fffffff;
        for (int d = 0;; ++d) {
            if (d * d >= bestd) break;
            const int ya = y - d, yb = y + d;
            if (ya < 0 && yb >= G) break;
            if (ya >= 0) {
                const uint32_t s = tile[ya * TX + xx];
                if (s != MARKER) {
                    const int dz = z - (int)vz(s);
                    const int dd = d * d + dz * dz;
                    if (dd < bestd) { bestd = dd; best = s; }
                }
            }
            if (d > 0 && yb < G) {
                const uint32_t s = tile[yb * TX + xx];
                if (s != MARKER) {
                    const int dz = z - (int)vz(s);
                    const int dd = d * d + dz * dz;
                    if (dd < bestd) { bestd = dd; best = s; }
                }
            }
        }
        out[zoff + (size_t)y * G + x0 + xx] = best;
    }
}

// x pass: TY contiguous rows of G voxels at fixed z
template <int TY>
__global__ void __launch_bounds__(256) k_pba_x(int G, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    extern __shared__ uint32_t tile[];
    const int y0 = blockIdx.x * TY;
    const int z = blockIdx.y;
    const size_t base = (size_t)z * G * G + (size_t)y0 * G;
    const int total = G * TY;
    const uint4* in4 = reinterpret_cast<const uint4*>(in + base);
    uint4* t4 = reinterpret_cast<uint4*>(tile);
    for (int k = threadIdx.x; k < total / 4; k += blockDim.x) t4[k] = in4[k];
    __syncthreads();
    for (int k = threadIdx.x; k < total; k += blockDim.x) {
        const int row = k / G, x = k % G;
        const int y = y0 + row;
        const uint32_t* line = tile + row * G;
        uint32_t best = MARKER;
        int bestd = 0x7fffffff;
        for (int d = 0;; ++d) {
            if (d * d >= bestd) break;
            const int xa = x - d, xb = x + d;
            if (xa < 0 && xb >= G) break;
            if (xa >= 0) {
                const uint32_t s = line[xa];
                if (s != MARKER) {
                    const int dy = y - (int)vy(s), dz = z - (int)vz(s);
                    const int dd = d * d + dy * dy + dz * dz;
                    if (dd < bestd) { bestd = dd; best = s; }
                }
            }
            if (d > 0 && xb < G) {
                const uint32_t s = line[xb];
                if (s != MARKER) {
                    const int dy = y - (int)vy(s), dz = z - (int)vz(s);
                    const int dd = d * d + dy * dy + dz * dz;
                    if (dd < bestd) { bestd = dd; best = s; }
                }
            }
        }
        out[base + k] = best;
    }
}

// site (packed voxel) -> point id of the voxel's leader (smallest Morton index)
__device__ __forceinline__ int site_to_id(const Dev& D, uint32_t e) {
    const int c = (int)(vy(e) * (uint32_t)D.G + vx(e));
    const uint32_t z = vz(e);
    for (int j = D.colStart[c], je = D.colEnd[c]; j < je; ++j)
        if ((D.ckey[j] & 1023u) == z) return D.cid[j];
    return -1;
}

__device__ __forceinline__ void push_bucket(const Dev& D, int a, int b) {
    const int pos = atomicAdd(&D.bucketCount[a], 1);
    if (pos < BUCKET_CAP) D.bucket[(size_t)a * BUCKET_CAP + pos] = b;
}

constexpr int PAIR_HASH = 2048;
constexpr int PAIR_ZC = 8;

// Every two distinct sites meeting in a 2x2x2 voxel cube are a candidate
// Delaunay edge (the reference reads the same cubes, GDelKernels.cu:137-299).
// Block-local dedupe in a shared-memory hash before the per-star scatter.
__global__ void __launch_bounds__(256) k_pairs(Dev D, const uint32_t* __restrict__ grid) {
    __shared__ unsigned long long hs[PAIR_HASH];
    const int G = D.G;
    for (int k = threadIdx.y * 32 + threadIdx.x; k < PAIR_HASH; k += 256) hs[k] = ~0ull;
    __syncthreads();
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    const int z0 = blockIdx.z * PAIR_ZC;
    const size_t plane = (size_t)G * G;
    if (x < G - 1 && y < G - 1) {
        for (int zi = 0; zi < PAIR_ZC; ++zi) {
            const int z = z0 + zi;
            if (z >= G - 1) break;
            uint32_t s[8];
            int ns = 0;
            for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dx = 0; dx < 2; ++dx) {
                        const uint32_t v = __ldg(&grid[(size_t)(z + dz) * plane + (size_t)(y + dy) * G + x + dx]);
                        bool dup = false;
                        for (int k = 0; k < ns; ++k) dup |= (s[k] == v);
                        if (!dup) s[ns++] = v;
                    }
            for (int a = 0; a < ns; ++a)
                for (int b = a + 1; b < ns; ++b) {
                    const uint32_t lo = s[a] < s[b] ? s[a] : s[b], hi = s[a] < s[b] ? s[b] : s[a];
                    const unsigned long long key = ((unsigned long long)lo << 32) | hi;
                    unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ull) >> 53) & (PAIR_HASH - 1);
                    bool placed = false;
                    for (int probe = 0; probe < PAIR_HASH; ++probe) {
                        const unsigned long long old = atomicCAS(&hs[h], ~0ull, key);
                        if (old == ~0ull || old == key) { placed = true; break; }
                        h = (h + 1) & (PAIR_HASH - 1);
                    }
                    if (!placed) {  // table full: emit directly
                        const int ia = site_to_id(D, lo), ib = site_to_id(D, hi);
                        if (ia >= 0 && ib >= 0) { push_bucket(D, ia, ib); push_bucket(D, ib, ia); }
                    }
                }
        }
    }
    __syncthreads();
    for (int k = threadIdx.y * 32 + threadIdx.x; k < PAIR_HASH; k += 256) {
        const unsigned long long key = hs[k];
        if (key == ~0ull) continue;
        const int ia = site_to_id(D, (uint32_t)(key >> 32)), ib = site_to_id(D, (uint32_t)key);
        if (ia >= 0 && ib >= 0) {
            push_bucket(D, ia, ib);
            push_bucket(D, ib, ia);
        }
    }
}

// Points that share a voxel with a smaller Morton index are absent from the
// digital diagram; each is paired with its voxel's leader (GDelKernels.cu:109-135).
__global__ void k_missing(Dev D) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += gridDim.x * blockDim.x) {
        const uint32_t k = D.mkey[i];
        if (i == 0 || D.mkey[i - 1] != k) continue;
        int j = i - 1;
        while (j > 0 && D.mkey[j - 1] == k) --j;
        push_bucket(D, i, j);
        push_bucket(D, j, i);
    }
}

void launch_pba_z(const Launch& L, const Dev& D, uint32_t* out) {
    dim3 b(32, 4), g((D.G + 31) / 32, (D.G + 3) / 4);
    k_pba_z<<<g, b, 0, L.stream>>>(D.G, D.ckey, D.colStart, D.colEnd, out);
    ++*L.launches;
}

void launch_pba_y(const Launch& L, int G, const uint32_t* in, uint32_t* out) {
    if (G >= 1024) {
        constexpr int TX = 16;
        const size_t sm = (size_t)G * TX * 4;
        cudaFuncSetAttribute(k_pba_y<TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pba_y<TX><<<dim3(G / TX, G), 256, sm, L.stream>>>(G, in, out);
    } else {
        constexpr int TX = 32;
        const size_t sm = (size_t)G * TX * 4;
        cudaFuncSetAttribute(k_pba_y<TX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pba_y<TX><<<dim3(G / TX, G), 256, sm, L.stream>>>(G, in, out);
    }
    ++*L.launches;
}

void launch_pba_x(const Launch& L, int G, const uint32_t* in, uint32_t* out) {
    // TY rows of G voxels: 32 KB of shared memory per block
    const int TY = G >= 1024 ? 8 : (G >= 512 ? 16 : (G >= 256 ? 32 : (8192 / G < G ? 8192 / G : G)));
    const size_t sm = (size_t)G * TY * 4;
    switch (TY) {
#define G4D_X(T)                                                                                   \
    case T:                                                                                        \
        cudaFuncSetAttribute(k_pba_x<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);  \
        k_pba_x<T><<<dim3(G / T, G), 256, sm, L.stream>>>(G, in, out);                             \
        break;
        G4D_X(8) G4D_X(16) G4D_X(32) G4D_X(64) G4D_X(128) G4D_X(256)
#undef G4D_X
        default: break;
    }
    ++*L.launches;
}

void launch_pairs(const Launch& L, const Dev& D, const uint32_t* grid) {
    const int G = D.G;
    dim3 b(32, 8), g((G - 1 + 31) / 32, (G - 1 + 7) / 8, (G - 1 + PAIR_ZC - 1) / PAIR_ZC);
    k_pairs<<<g, b, 0, L.stream>>>(D, grid);
    ++*L.launches;
}

void launch_missing(const Launch& L, const Dev& D) {
    int blocks = (D.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_missing<<<blocks, 256, 0, L.stream>>>(D);
    ++*L.launches;
}

}  // namespace g4d
