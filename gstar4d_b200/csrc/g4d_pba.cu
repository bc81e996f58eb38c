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
//   y, x: one thread per line builds the lower envelope of the line's
//      candidates and colours the line from it (O(G) per line, no transposes;
//      k_pba_env_y / k_pba_env_x below).
// Sites stay encoded as voxel coordinates; the pair scan turns them into point
// ids through a voxel -> leader map written into the free second grid.
//
// Batches: the grids of all clouds with the same G are stacked (grid k of the
// stack at offset k*G^3, its columns at k*G^2 in the column index), and each
// kernel takes the stack depth K as its last grid dimension, so one launch per
// grid size serves every cloud of that size. One cloud is a stack of depth 1.
#include <type_traits>

#include "g4d_internal.cuh"

namespace g4d {


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



// ---------------------------------------------------------------------------
// y and x passes as lower envelopes (one thread per line, O(G) per line).
//
// Along a line, candidate p (a voxel whose site came from the earlier passes)
// gives every voxel q the squared distance (q - p)^2 + f_p, f_p the squared
// distance of its site across the line. The nearest site of each voxel is the
// lowest of these parabolas: the lower convex hull of the points
// (p, F_p = f_p + p^2), built in one sweep with a stack (Felzenszwalb and
// Huttenlocher's envelope, the role of PBA's proximate-site stacks,
// pba3DKernel.h:200-420), then read off in a second sweep. The sweep goes
// downwards, so the stack is a list linked towards larger p; its links are
// written into the input word of each stacked candidate (the input is
// scratch), packed with the site coordinates the line does not fix. The
// colouring sweep goes upwards along those links. Each thread keeps the two
// top entries in registers, so a pop costs one load (of the new second).
// Distances are exact; among equidistant sites the choice is free (only the
// distance of the digital diagram is specified).
// ---------------------------------------------------------------------------
constexpr uint32_t ENV_END = 2047;  // end of a list (11-bit link)

// Products of height differences (< 3 G^2) and position differences (< G):
// 32-bit up to G = 512, 64-bit beyond.
template <bool WIDE>
using EnvInt = typename std::conditional<WIDE, long long, int>::type;

// first position y at which candidate n (height fn) is at most as far as
// candidate c (height fc), c < n: (n - c)(2y - n - c) >= fn - fc
__device__ __forceinline__ int env_switch(int c, int fc, int n, int fn) {
    const int A = n - c;
    const int N = fn - fc + A * (n + c);  // switch when 2 y A >= N
    int q = N / (2 * A);
    if (q * 2 * A < N) ++q;
    return q;
}

// One line of G voxels. Ops supplies: next_in(q), the input word of position
// q (q = G-1 .. 0 in turn); put(q, w), the word left at q after pass 1 (the
// same order); at(p), the word of an earlier position p > q (a stacked,
// packed word); fin(w), the height of an input site; fpk(w), the height of a
// packed word; link(w), its next position; pack(w, next); site(p, w), the
// output site of packed word w at position p; emit(y, site) for y = 0 .. G-1
// in turn. Pass 1 keeps the top two stack entries in registers; pass 2 moves
// to the next envelope entry at precomputed switch positions.
template <bool WIDE, class Ops>
__device__ __forceinline__ void env_line(int G, Ops& o) {
    using I = EnvInt<WIDE>;
    int top = (int)ENV_END, sec = (int)ENV_END;
    I Ft = 0, D = 0;  // F of the top; F_second - F_top
    int E = 0;        // second - top
    uint32_t wt = 0, ws = 0;
    for (int q = G - 1; q >= 0; --q) {
        const uint32_t w = o.next_in(q);  // q descending
        if (w == MARKER) {
            o.put(q, w);
            continue;
        }
        const I Fq = (I)o.fin(w) + (I)q * q;
        // pop the top while its region between q and the second is empty:
        // (F_t - F_q)(s - t) >= (F_s - F_t)(t - q)
        while (sec != (int)ENV_END && (Ft - Fq) * (I)E >= D * (I)(top - q)) {
            top = sec; Ft = Ft + D; wt = ws;
            sec = o.link(ws);
            if (sec != (int)ENV_END) {
                ws = o.at(sec);
                D = (I)o.fpk(ws) + (I)sec * sec - Ft;
                E = sec - top;
            }
        }
        const uint32_t wq = o.pack(w, top);
        o.put(q, wq);
        sec = top; ws = wt; D = Ft - Fq; E = top - q;
        top = q; Ft = Fq; wt = wq;
    }
    if (top == (int)ENV_END) {  // no site in this line
        for (int y = 0; y < G; ++y) o.emit(y, MARKER);
        return;
    }
    int cur = top, fc = o.fpk(wt), nx = o.link(wt), fn = 0, T = 1 << 30;
    uint32_t wc = wt, wn = 0;
    if (nx != (int)ENV_END) {
        wn = o.at(nx);
        fn = o.fpk(wn);
        T = env_switch(cur, fc, nx, fn);
    }
    for (int y = 0; y < G; ++y) {
        while (y >= T) {
            cur = nx; wc = wn; fc = fn;
            nx = o.link(wc);
            T = 1 << 30;
            if (nx != (int)ENV_END) {
                wn = o.at(nx);
                fn = o.fpk(wn);
                T = env_switch(cur, fc, nx, fn);
            }
        }
        o.emit(y, o.site(cur, wc));
    }
}

// y pass (after the z flood): line (x, z) along y; the site of candidate p is
// (x, p, zs), f_p = (z - zs)^2; packed word zs | next << 10. Lanes take
// consecutive x, so every row access of a warp is one 128-byte line.
struct EnvY {
    uint32_t* line;
    uint32_t* res;
    int st;  // one row along y (G words; offsets within a line fit in 32 bits)
    int x, z;
    uint32_t ahead;  // input word of the next position, loaded ahead of use
    __device__ uint32_t next_in(int q) {
        const uint32_t w = ahead;
        if (q > 0) ahead = line[(q - 1) * st];
        return w;
    }
    __device__ uint32_t at(int p) const { return line[p * st]; }
    __device__ void put(int p, uint32_t w) const {
        if (w != MARKER) line[p * st] = w;
    }
    __device__ int fin(uint32_t w) const { const int d = z - (int)vz(w); return d * d; }
    __device__ int fpk(uint32_t w) const { const int d = z - (int)(w & 1023u); return d * d; }
    __device__ int link(uint32_t w) const { return (int)((w >> 10) & 2047u); }
    __device__ uint32_t pack(uint32_t w, int next) const { return vz(w) | ((uint32_t)next << 10); }
    __device__ uint32_t site(int p, uint32_t w) const { return enc_vox((uint32_t)x, (uint32_t)p, w & 1023u); }
    __device__ void emit(int y, uint32_t v) const {
        __syncwarp();  // one full line per warp store
        res[y * st] = v;
    }
};

template <bool WIDE>
__global__ void __launch_bounds__(128) k_pba_env_y(int G, uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int z = blockIdx.y * 4 + threadIdx.y;
    if (x >= G || z >= G) return;
    const size_t plane = (size_t)G * G;
    const size_t off = (size_t)blockIdx.z * plane * G + (size_t)z * plane + x;
    EnvY o{in + off, out + off, G, x, z, in[off + (size_t)(G - 1) * G]};
    env_line<WIDE>(G, o);
}

// x pass (after the y pass): line (y, z) along x; the site of candidate p is
// (p, ys, zs), f_p = (y - ys)^2 + (z - zs)^2; packed word ys | zs << 10 |
// next << 20. Lanes take consecutive y, each walking its own contiguous row,
// so words move four at a time (16-byte accesses): pass 1 reads the next group
// ahead, keeps the current group in registers and writes it back when it is
// done; pass 2 writes four sites at once.
struct EnvX {
    uint32_t* line;
    uint32_t* res;
    int y, z;
    int g0;                 // first position of the group in registers
    uint32_t g[4];          // its words (packed once stacked)
    uint4 ahead;            // the group below it
    uint32_t o0, o1, o2;    // pass 2: sites of the group being emitted
    __device__ uint32_t gsel(int d) const { return d == 0 ? g[0] : (d == 1 ? g[1] : (d == 2 ? g[2] : g[3])); }
    __device__ uint32_t next_in(int q) {
        if ((q & 3) == 3) {
            const uint4 v = g0 < 0 ? *reinterpret_cast<const uint4*>(line + q - 3) : ahead;
            g[0] = v.x; g[1] = v.y; g[2] = v.z; g[3] = v.w;
            g0 = q - 3;
            if (g0 > 0) ahead = *reinterpret_cast<const uint4*>(line + g0 - 4);
        }
        return gsel(q - g0);
    }
    __device__ void put(int q, uint32_t w) {
        const int d = q - g0;
        g[0] = d == 0 ? w : g[0];
        g[1] = d == 1 ? w : g[1];
        g[2] = d == 2 ? w : g[2];
        g[3] = d == 3 ? w : g[3];
        if (d == 0) {
            *reinterpret_cast<uint4*>(line + g0) = make_uint4(g[0], g[1], g[2], g[3]);
            g0 = 1 << 20;  // nothing in registers until the next group
        }
    }
    __device__ uint32_t at(int p) const {
        const int d = p - g0;
        return (d >= 0 && d < 4) ? gsel(d) : line[p];
    }
    __device__ int fin(uint32_t w) const {
        const int dy = y - (int)vy(w), dz = z - (int)vz(w);
        return dy * dy + dz * dz;
    }
    __device__ int fpk(uint32_t w) const {
        const int dy = y - (int)(w & 1023u), dz = z - (int)((w >> 10) & 1023u);
        return dy * dy + dz * dz;
    }
    __device__ int link(uint32_t w) const { return (int)((w >> 20) & 2047u); }
    __device__ uint32_t pack(uint32_t w, int next) const { return vy(w) | (vz(w) << 10) | ((uint32_t)next << 20); }
    __device__ uint32_t site(int p, uint32_t w) const { return enc_vox((uint32_t)p, w & 1023u, (w >> 10) & 1023u); }
    __device__ void emit(int x, uint32_t v) {
        const int d = x & 3;
        if (d == 0) o0 = v;
        else if (d == 1) o1 = v;
        else if (d == 2) o2 = v;
        else *reinterpret_cast<uint4*>(res + x - 3) = make_uint4(o0, o1, o2, v);
    }
};

template <bool WIDE>
__global__ void __launch_bounds__(128) k_pba_env_x(int G, uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    const int y = blockIdx.x * 32 + threadIdx.x;
    const int z = blockIdx.y * 4 + threadIdx.y;
    if (y >= G || z >= G) return;
    const size_t plane = (size_t)G * G;
    const size_t off = (size_t)blockIdx.z * plane * G + (size_t)z * plane + (size_t)y * G;
    EnvX o;
    o.line = in + off;
    o.res = out + off;
    o.y = y;
    o.z = z;
    o.g0 = -1;  // the first group is loaded directly
    o.ahead = make_uint4(0, 0, 0, 0);
    o.o0 = o.o1 = o.o2 = 0;
    env_line<WIDE>(G, o);
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
    if (C.map) C.map += (size_t)kk * plane * G;
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

void launch_pba_y(const Launch& L, int G, uint32_t* in, uint32_t* out) { launch_pba_y_stack(L, G, 1, in, out); }

// `in` is scratch: the envelope passes keep their stacks in it
void launch_pba_y_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out) {
    if (G > 512) k_pba_env_y<true><<<dim3(G / 32, G / 4, K), dim3(32, 4), 0, L.stream>>>(G, in, out);
    else k_pba_env_y<false><<<dim3(G / 32, G / 4, K), dim3(32, 4), 0, L.stream>>>(G, in, out);
    ++*L.launches;
}

void launch_pba_x(const Launch& L, int G, uint32_t* in, uint32_t* out) { launch_pba_x_stack(L, G, 1, in, out); }

void launch_pba_x_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out) {
    if (G > 512) k_pba_env_x<true><<<dim3(G / 32, G / 4, K), dim3(32, 4), 0, L.stream>>>(G, in, out);
    else k_pba_env_x<false><<<dim3(G / 32, G / 4, K), dim3(32, 4), 0, L.stream>>>(G, in, out);
    ++*L.launches;
}

// leader id at the voxel of every leader (the first point of its voxel in
// Morton order), for site_to_id; other voxels of the map are never read
__global__ void k_site_map(const uint32_t* __restrict__ vox, const uint32_t* __restrict__ mkey, int n, int G,
                           int* __restrict__ map) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i > 0 && mkey[i - 1] == mkey[i]) continue;
        const uint32_t e = vox[i];
        map[((size_t)vz(e) * G + vy(e)) * G + vx(e)] = i;
    }
}

// the same for a batch pass: point i of slot k = skey >> 30 maps into its grid
// at slotVox[k]; leaders are the first of equal sort keys
__global__ void k_b_site_map(const uint32_t* __restrict__ vox, const unsigned long long* __restrict__ skey,
                             const int* __restrict__ slotG, const long long* __restrict__ slotVox, int n,
                             int* __restrict__ map) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i > 0 && skey[i - 1] == skey[i]) continue;
        const int k = (int)(skey[i] >> 30);
        const size_t G = (size_t)slotG[k];
        const uint32_t e = vox[i];
        map[(size_t)slotVox[k] + ((size_t)vz(e) * G + vy(e)) * G + vx(e)] = i;
    }
}

void launch_site_map(const Launch& L, const Dev& D, int* map) {
    int blocks = (D.n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_site_map<<<blocks, 256, 0, L.stream>>>(D.vox, D.mkey, D.n, D.G, map);
    ++*L.launches;
}

void launch_b_site_map(const Launch& L, const uint32_t* vox, const unsigned long long* skey, const int* slotG,
                       const long long* slotVox, int n, int* map) {
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    k_b_site_map<<<blocks, 256, 0, L.stream>>>(vox, skey, slotG, slotVox, n, map);
    ++*L.launches;
}

void launch_pairs(const Launch& L, const Dev& D, const uint32_t* grid, int* map) {
    const int G = D.G;
    const int nzc = (G - 1 + PAIR_ZC - 1) / PAIR_ZC;
    dim3 b(32, PAIR_WARPS), g((G - 1 + 31) / 32, (G - 1 + PAIR_WARPS - 1) / PAIR_WARPS, nzc);
    k_pairs<<<g, b, 0, L.stream>>>(D, grid, Cols<uint32_t>{D.ckey, D.cid, D.colStart, D.colEnd, G, map}, nzc);
    ++*L.launches;
}

void launch_pairs_stack(const Launch& L, const Dev& D, const uint32_t* stack, int* map, int G, int K,
                        const unsigned long long* ckey, const int* cid, const int* cs, const int* ce) {
    const int nzc = (G - 1 + PAIR_ZC - 1) / PAIR_ZC;
    dim3 b(32, PAIR_WARPS), g((G - 1 + 31) / 32, (G - 1 + PAIR_WARPS - 1) / PAIR_WARPS, nzc * K);
    k_pairs<<<g, b, 0, L.stream>>>(D, stack, Cols<unsigned long long>{ckey, cid, cs, ce, G, map}, nzc);
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
