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
//   y, x: tiles of 8 lines staged in shared memory, one warp per line
//      building the line's lower envelope from 32 band hulls merged in a tree
//      and colouring the line from it (k_pba_env below; no transposes).
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
// y and x passes: the exact 1D lower envelope of every line, on tiles of lines
// staged in shared memory.
//
// Along a line, candidate p (a voxel whose site came from the earlier passes)
// gives every voxel q the squared distance (q - p)^2 + f_p, f_p the squared
// distance of its site across the line. The nearest site of each voxel is the
// lowest of these parabolas, i.e. the lower convex hull of the points
// (p, F_p = f_p + p^2) (Felzenszwalb and Huttenlocher's envelope; PBA's
// proximate-site stacks and band merge, pba3DKernel.h:200-420, compute the
// same hull). Each warp stages LPW whole lines in shared memory (one coalesced
// read of every voxel) and splits every line into B = 32 / LPW bands, one lane
// per band:
//  1. lane (line i, band b) builds the hull of its band left to right, with
//     the stack kept in place in the staged words;
//  2. the bands of a line are merged pairwise in log2(B) levels, each merge by
//     one lane walking to the lower common tangent of the two chains and
//     cutting them there (every walk step removes a point; with B <= 8 the
//     walks are a few steps, measured on the benchmark clouds);
//  3. lane (i, b) colours its band: a binary search over the surviving hull
//     points (addressed by rank through the bands' surviving runs) finds the
//     point nearest to the band's first voxel, since the distance to a fixed
//     voxel is convex along the hull (no division), then it walks forward,
//     writing each site straight to the output (the y pass with 8 lines per
//     warp: 8 consecutive x, one 32-byte sector per band per store; the x pass:
//     4 sites per 16-byte store).
// The words are site voxels, and the position of a candidate along the line is
// one of its own coordinates (y in the y pass, x in the x pass), so the hull
// holds words only. Distances are exact; among equidistant sites the choice is
// free (only the distance of the digital diagram is specified); collinear hull
// points are dropped.
// ---------------------------------------------------------------------------

// Products of height differences (< 4 G^2) and position differences (< G):
// 32-bit up to G = 512, 64-bit beyond.
template <bool WIDE>
using EnvInt = typename std::conditional<WIDE, long long, int>::type;

template <int AXIS>
struct EnvLine {
    int a, b;  // the line's fixed coordinates: (x, z) for the y pass (AXIS 1), (y, z) for the x pass (AXIS 0)
    __device__ __forceinline__ int pos(uint32_t w) const { return AXIS ? (int)vy(w) : (int)vx(w); }
    __device__ __forceinline__ int f(uint32_t w) const {
        const int dz = b - (int)vz(w);
        if (AXIS) return dz * dz;
        const int dy = a - (int)vy(w);
        return dy * dy + dz * dz;
    }
    __device__ __forceinline__ int height(uint32_t w) const { const int p = pos(w); return f(w) + p * p; }
    __device__ __forceinline__ int dist(int q, uint32_t w) const { const int d = q - pos(w); return d * d + f(w); }
};

// (pb - pa)(Fc - Fa) - (Fb - Fa)(pc - pa) > 0: b lies strictly below the
// segment from a to c (positions pa < pb < pc)
template <bool WIDE>
__device__ __forceinline__ bool below(int pa, int Fa, int pb, int Fb, int pc, int Fc) {
    using I = EnvInt<WIDE>;
    return (I)(pb - pa) * (I)(Fc - Fa) - (I)(Fb - Fa) * (I)(pc - pa) > 0;
}

// Staged line layout: band b of a line at word b (Lb + 1) (one padding word
// per band), lines S = G + B words apart. With Lb a multiple of 32 the 32
// lanes of a warp, one per (line, band), read 32 different banks.
template <int LPW>
struct EnvTile {
    static constexpr int B = 32 / LPW;
    int Lb, S;
    __device__ __forceinline__ int idx(int q) const { return q + q / Lb; }  // position -> word within the line
};

template <int LPW>
__host__ __device__ constexpr size_t env_warp_smem(int G) {
    return (size_t)LPW * (size_t)(G + 32 / LPW) * 4 + (size_t)LPW * (32 / LPW) * 2 * 4;
}

// The envelope of the LPW lines staged in A (line i at A + i S), colouring
// written through emit(i, q, site) for q = 0 .. G-1 of each band in turn.
template <int AXIS, bool WIDE, int LPW, class Emit>
__device__ __forceinline__ void env_lines(int G, const EnvTile<LPW>& T, uint32_t* A, int* lo, int* hi, int l0,
                                          int c1, Emit& emit) {
    constexpr int B = EnvTile<LPW>::B;
    const int lane = threadIdx.x & 31;
    const int i = lane % LPW, b = lane / LPW;
    const int Lb = T.Lb;
    uint32_t* line = A + i * T.S;
    int* lo_i = lo + i * B;
    int* hi_i = hi + i * B;
    const EnvLine<AXIS> ln{l0 + i, c1};
    // 1. the hull of this lane's band, in place
    {
        uint32_t* band = line + b * (Lb + 1);
        int cnt = 0, ps = 0, Fs = 0, pt = 0, Ft = 0;
        for (int k = 0; k < Lb; ++k) {
            const uint32_t w = band[k];
            if (w == MARKER) continue;
            const int p = ln.pos(w), F = ln.height(w);
            while (cnt >= 2 && !below<WIDE>(ps, Fs, pt, Ft, p, F)) {
                --cnt;
                pt = ps;
                Ft = Fs;
                if (cnt >= 2) {
                    const uint32_t v = band[cnt - 2];
                    ps = ln.pos(v);
                    Fs = ln.height(v);
                }
            }
            band[cnt++] = w;
            ps = pt;
            Fs = Ft;
            pt = p;
            Ft = F;
        }
        lo_i[b] = 0;
        hi_i[b] = cnt;
    }
    __syncwarp();
    // 2. merge neighbouring groups of s bands of the same line
#pragma unroll
    for (int s = 1; s < B; s <<= 1) {
        if ((b & (2 * s - 1)) == 0) {
            const int g = b, gm = g + s, ge = g + 2 * s;
            int ta = gm - 1, tb = gm;
            while (ta >= g && lo_i[ta] == hi_i[ta]) --ta;
            while (tb < ge && lo_i[tb] == hi_i[tb]) ++tb;
            if (ta >= g && tb < ge) {
                int ia = hi_i[ta] - 1, ib = lo_i[tb];
                uint32_t w = line[ta * (Lb + 1) + ia];
                int pa = ln.pos(w), Fa = ln.height(w);
                w = line[tb * (Lb + 1) + ib];
                int pb = ln.pos(w), Fb = ln.height(w);
                for (;;) {
                    bool moved = false;
                    // b moves right while its successor is on or below the line a-b
                    for (;;) {
                        int tn = tb, in_ = ib + 1;
                        if (in_ >= hi_i[tn]) {
                            ++tn;
                            while (tn < ge && lo_i[tn] == hi_i[tn]) ++tn;
                            if (tn >= ge) break;
                            in_ = lo_i[tn];
                        }
                        const uint32_t wn = line[tn * (Lb + 1) + in_];
                        const int pn = ln.pos(wn), Fn = ln.height(wn);
                        if (below<WIDE>(pa, Fa, pb, Fb, pn, Fn)) break;
                        tb = tn; ib = in_; pb = pn; Fb = Fn;
                        moved = true;
                    }
                    // a moves left while it is on or above the segment from its predecessor to b
                    for (;;) {
                        int tp = ta, ip = ia - 1;
                        if (ip < lo_i[tp]) {
                            --tp;
                            while (tp >= g && lo_i[tp] == hi_i[tp]) --tp;
                            if (tp < g) break;
                            ip = hi_i[tp] - 1;
                        }
                        const uint32_t wp = line[tp * (Lb + 1) + ip];
                        const int pp = ln.pos(wp), Fp = ln.height(wp);
                        if (below<WIDE>(pp, Fp, pa, Fa, pb, Fb)) break;
                        ta = tp; ia = ip; pa = pp; Fa = Fp;
                        moved = true;
                    }
                    if (!moved) break;
                }
                // cut both chains at the tangent
                hi_i[ta] = ia + 1;
                for (int t = ta + 1; t < gm; ++t) hi_i[t] = lo_i[t];
                lo_i[tb] = ib;
                for (int t = gm; t < tb; ++t) lo_i[t] = hi_i[t];
            }
        }
        __syncwarp();
    }
    // 3. colour this lane's band from the hull, addressed by rank r through the
    // surviving runs [lo, hi) of the line's bands
    int P[B + 1];
    P[0] = 0;
#pragma unroll
    for (int t = 0; t < B; ++t) P[t + 1] = P[t] + hi_i[t] - lo_i[t];
    const int K = P[B];
    auto word = [&](int r) {  // selects instead of an indexed array: P stays in registers
        int t = 0, pt = 0;
#pragma unroll
        for (int u = 1; u < B; ++u)
            if (r >= P[u]) { t = u; pt = P[u]; }
        return line[t * (Lb + 1) + lo_i[t] + (r - pt)];
    };
    const int q0 = b * Lb;
    if (K == 0) {
        for (int j = 0; j < Lb; ++j) emit(i, q0 + j, MARKER);
        return;
    }
    int kl = 0, kh = K - 1;  // the first hull point whose successor is not nearer to q0
    while (kl < kh) {
        const int m = (kl + kh) >> 1;
        if (ln.dist(q0, word(m + 1)) >= ln.dist(q0, word(m))) kh = m;
        else kl = m + 1;
    }
    // walk the hull over the band: point r is the nearest from q0 until the
    // first position sw at which point r + 1 is at least as near,
    //   (q - p1)^2 + f1 <= (q - p0)^2 + f0  <=>  2 q (p1 - p0) >= F1 - F0,
    // so sw = ceil((F1 - F0) / (2 (p1 - p0))): a float quotient (both operands
    // are exact in float) corrected by two integer tests
    int r = kl;
    uint32_t we = word(r);
    int pe = ln.pos(we), Fe = ln.height(we);
    auto next_switch = [&](int& sw, uint32_t& wn, int& pn, int& Fn) {
        if (r + 1 >= K) {
            sw = 1 << 30;
            return;
        }
        wn = word(r + 1);
        pn = ln.pos(wn);
        Fn = ln.height(wn);
        const int num = Fn - Fe, den = 2 * (pn - pe);
        int t = (int)ceilf((float)num / (float)den);
        if ((long long)t * den < num) ++t;
        if ((long long)(t - 1) * den >= num) --t;
        sw = t;
    };
    int sw;
    uint32_t wn = 0;
    int pn = 0, Fn = 0;
    next_switch(sw, wn, pn, Fn);
    const int q1 = q0 + Lb;
    int q = q0;
    while (q < q1) {
        // the run of voxels nearest to point r inside this band
        const int e = sw < q1 ? (sw > q ? sw : q) : q1;
        for (; q < e; ++q) emit(i, q, we);
        if (q >= q1) break;
        ++r;
        we = wn;
        pe = pn;
        Fe = Fn;
        next_switch(sw, wn, pn, Fn);
    }
}

// y pass output: site of voxel (x0 + i, q, z); with LPW = 8 the lanes of one
// band store 8 consecutive words
struct EmitY {
    uint32_t* out;  // &out[z][0][x0]
    int G;
    __device__ __forceinline__ void operator()(int i, int q, uint32_t v) const { out[(size_t)q * G + i] = v; }
};

// x pass output: site of voxel (q, y0 + i, z), four consecutive sites per
// 16-byte store (band starts are multiples of 4)
struct EmitX {
    uint32_t* out;  // &out[z][y0][0]
    int G;
    uint32_t v0, v1, v2;
    __device__ __forceinline__ void operator()(int i, int q, uint32_t v) {
        const int d = q & 3;
        if (d == 0) v0 = v;
        else if (d == 1) v1 = v;
        else if (d == 2) v2 = v;
        else *reinterpret_cast<uint4*>(out + (size_t)i * G + q - 3) = make_uint4(v0, v1, v2, v);
    }
};

// Block (t, z, k): W warps, warp w stages lines l0 .. l0 + LPW - 1, l0 =
// (t W + w) LPW, of plane z of grid k of the stack. AXIS 1: lines (x = l0 + i,
// z) along y, rows of LPW words; AXIS 0: lines (y = l0 + i, z) along x, read as
// 16-byte vectors.
template <int AXIS, bool WIDE, int LPW, int W>
__global__ void __launch_bounds__(32 * W) k_pba_env(int G, const uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
    G4D_DYN_SMEM(env_smem_raw);
    constexpr int B = EnvTile<LPW>::B;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    EnvTile<LPW> T{G / B, G + B};
    uint32_t* A = reinterpret_cast<uint32_t*>(env_smem_raw) + (size_t)warp * LPW * T.S;
    int* lo = reinterpret_cast<int*>(reinterpret_cast<uint32_t*>(env_smem_raw) + (size_t)W * LPW * T.S) +
              warp * 2 * LPW * B;
    int* hi = lo + LPW * B;
    const size_t plane = (size_t)G * G;
    const size_t gbase = (size_t)blockIdx.z * plane * G + (size_t)blockIdx.y * plane;
    const int l0 = (blockIdx.x * W + warp) * LPW;
    // Staging: 16-byte chunks, a batch of 8 loads per lane in flight before
    // any is stored. AXIS 1: chunk c holds 4 words of row y = c / (LPW / 4)
    // (lines 4h .. 4h + 3, h = c % (LPW / 4)); AXIS 0: chunk c holds words
    // 4c .. 4c + 3 of the tile's rows (line 4c / G, positions 4c % G ..).
    constexpr int BATCH = 8;
    const int nchunk = LPW * G / 4;
    const uint4* src = AXIS ? reinterpret_cast<const uint4*>(in + gbase + l0)
                            : reinterpret_cast<const uint4*>(in + gbase + (size_t)l0 * G);
    for (int c0 = 0; c0 < nchunk; c0 += 32 * BATCH) {
        uint4 v[BATCH];
#pragma unroll
        for (int k = 0; k < BATCH; ++k) {
            const int c = c0 + k * 32 + lane;
            if (c < nchunk) {
                if constexpr (AXIS) v[k] = src[(size_t)(c / (LPW / 4)) * (G / 4) + c % (LPW / 4)];
                else v[k] = src[c];
            }
        }
#pragma unroll
        for (int k = 0; k < BATCH; ++k) {
            const int c = c0 + k * 32 + lane;
            if (c >= nchunk) continue;
            if constexpr (AXIS) {
                const int y = c / (LPW / 4), h = c % (LPW / 4);
                uint32_t* d = A + 4 * h * T.S + T.idx(y);
                d[0] = v[k].x;
                d[T.S] = v[k].y;
                d[2 * T.S] = v[k].z;
                d[3 * T.S] = v[k].w;
            } else {
                const int i = (c * 4) / G, x = (c * 4) % G;
                uint32_t* d = A + i * T.S + T.idx(x);  // x .. x + 3 lie in one band
                d[0] = v[k].x;
                d[1] = v[k].y;
                d[2] = v[k].z;
                d[3] = v[k].w;
            }
        }
    }
    __syncwarp();
    if (AXIS) {
        EmitY em{out + gbase + l0, G};
        env_lines<AXIS, WIDE, LPW>(G, T, A, lo, hi, l0, (int)blockIdx.y, em);
    } else {
        EmitX em{out + gbase + (size_t)l0 * G, G, 0, 0, 0};
        env_lines<AXIS, WIDE, LPW>(G, T, A, lo, hi, l0, (int)blockIdx.y, em);
    }
}

// ---------------------------------------------------------------------------
// The same passes with one thread per line (the other candidate of the
// per-grid-width tuning in g4d_api.cu): no staging, the envelope's stack kept
// as a list linked through the input words in global memory (the input is
// scratch), full occupancy. On the 8M-point 1024^3 cloud this is the faster
// form; at 512^3 and below the tiles are.
//
// Candidate p gives every voxel q of the line the squared distance
// (q - p)^2 + f_p; the lower envelope is built in one downward sweep with a
// stack whose links are written into the input word of each stacked candidate,
// packed with the site coordinates the line does not fix, and read off in an
// upward sweep at precomputed switch positions. Each thread keeps the two top
// entries in registers, so a pop costs one load (of the new second).
// ---------------------------------------------------------------------------
constexpr uint32_t ENV_END = 2047;  // end of a list (11-bit link)

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
__global__ void __launch_bounds__(128) k_pba_line_y(int G, uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
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
__global__ void __launch_bounds__(128) k_pba_line_x(int G, uint32_t* __restrict__ in, uint32_t* __restrict__ out) {
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
// probes of a pair insert before it goes to the worksets directly: inside
// dense clusters nearly every cube holds eight sites and the block's pairs
// outnumber the table, where a long probe walk costs more than the duplicate
// pushes it saves
#ifndef PAIR_PROBES_DEF
#define PAIR_PROBES_DEF 4
#endif
constexpr int PAIR_PROBES = PAIR_PROBES_DEF;
constexpr int PAIR_BATCH = 4;  // hash entries per thread in flight in the final scatter
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
// coalesced over x). Each 2x2 face gets its distinct-site count and its
// smallest and largest site once (the two cubes that share it reuse them).
// A cube holds fewer than four sites when its faces' counts add up to less
// than four, or when both faces hold the same two sites (a cube on a Voronoi
// wall, the common case away from clusters). The cubes left (near Voronoi
// edges and vertices, and inside dense clusters) go to a per-warp queue;
// every 32 queued cubes the warp takes one per lane, computes its distinct
// sites and emits the pairs of the vertex cubes, spread over the lanes, into a
// block-local hash that removes duplicates before the per-star scatter.
constexpr int PAIR_QUEUE = 64;  // queued cubes per warp

struct Face {
    int n;           // distinct sites
    uint32_t lo, hi;  // smallest and largest site
};

__device__ __forceinline__ Face face_of(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    Face f;
    f.n = 1 + (b != a) + (c != a && c != b) + (d != a && d != b && d != c);
    f.lo = min(min(a, b), min(c, d));
    f.hi = max(max(a, b), max(c, d));
    return f;
}

// The 32 queued cubes qs[0..32) of a warp, one per lane: each lane reduces its
// cube to its distinct sites (in place); the pairs of the vertex cubes (four
// or more sites: n(n-1)/2 pairs, up to 28) are then spread over the lanes, 32
// at a time, so that a cube of eight sites does not hold up the warp. Pair k
// of a cube is (i, j) in colexicographic order: j(j-1)/2 <= k < j(j+1)/2,
// i = k - j(j-1)/2.
template <class KeyT>
__device__ __forceinline__ void emit_queued(unsigned long long* hs, uint32_t (*qs)[8], int* qoff, int lane, int nq,
                                            const Dev& D, const Cols<KeyT>& C) {
    int np = 0;
    if (lane < nq) {
        uint32_t* q = qs[lane];
        uint32_t v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = q[k];
        int ns = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            bool fresh = true;
#pragma unroll
            for (int j = 0; j < i; ++j) fresh = fresh && (v[i] != v[j]);
            if (fresh) q[ns++] = v[i];
        }
        np = ns >= 4 ? ns * (ns - 1) / 2 : 0;
    }
    int incl = np;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += t;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    qoff[lane] = incl - np;
    __syncwarp();
    for (int p = lane; p < total; p += 32) {
        // the last cube whose first pair is at or before p (it has pairs)
        int c = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
            if (qoff[c + step] <= p) c += step;
        const int k = p - qoff[c];
        int j = 1;
        while ((j + 1) * j / 2 <= k) ++j;
        const int i = k - j * (j - 1) / 2;
        const uint32_t a = qs[c][i], b = qs[c][j];
        pair_hash_insert(hs, a < b ? ((unsigned long long)a << 32) | b : ((unsigned long long)b << 32) | a, D, C);
    }
    __syncwarp();
}

template <class KeyT>
__global__ void __launch_bounds__(32 * PAIR_WARPS) k_pairs(Dev D, const uint32_t* __restrict__ stack, Cols<KeyT> C, int nzc) {
    __shared__ unsigned long long hs[PAIR_HASH];
    __shared__ uint32_t qs[PAIR_WARPS][PAIR_QUEUE][8];  // voxel sites of queued cubes
    __shared__ int qoff[PAIR_WARPS][32];                // first pair of each of 32 queued cubes
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
    // below stay converged; lanes past the grid edge queue nothing (they read
    // column 0, which is in bounds)
    const bool active = x < G - 1 && y < G - 1;
    const int zend = min(z0 + PAIR_ZC, G - 1);
    if (y < G - 1 && z0 < G - 1) {
        const uint32_t* g = grid + (size_t)y * G + (active ? x : 0);
        uint32_t v0, v1, v2, v3;
        {
            const size_t o = (size_t)z0 * plane;
            v0 = g[o]; v1 = g[o + 1]; v2 = g[o + G]; v3 = g[o + G + 1];
        }
        // plane z0+1 exists: z0 < G-1
        uint32_t n0, n1, n2, n3;
        {
            const size_t o = (size_t)(z0 + 1) * plane;
            n0 = g[o]; n1 = g[o + 1]; n2 = g[o + G]; n3 = g[o + G + 1];
        }
        Face fl = face_of(v0, v1, v2, v3);
        int qc = 0;  // queued cubes of this warp (same in every lane)
        for (int z = z0; z < zend; ++z) {
            const uint32_t u0 = n0, u1 = n1, u2 = n2, u3 = n3;
            if (z + 1 < zend) {  // the plane after the next one, loaded ahead of use
                const size_t o = (size_t)(z + 2) * plane;
                n0 = g[o]; n1 = g[o + 1]; n2 = g[o + G]; n3 = g[o + G + 1];
            }
            const Face fu = face_of(u0, u1, u2, u3);
            const bool wall = fl.n == 2 && fu.n == 2 && fl.lo == fu.lo && fl.hi == fu.hi;
            const bool maybe = active && fl.n + fu.n >= 4 && !wall;
            const unsigned bal = __ballot_sync(0xffffffffu, maybe);
            if (bal) {
                if (maybe) {
                    uint32_t* q = qs[w][qc + __popc(bal & ((1u << lane) - 1u))];
                    q[0] = v0; q[1] = v1; q[2] = v2; q[3] = v3;
                    q[4] = u0; q[5] = u1; q[6] = u2; q[7] = u3;
                }
                qc += __popc(bal);
                if (qc >= 32) {  // one queued cube per lane
                    __syncwarp();
                    emit_queued(hs, qs[w], qoff[w], lane, 32, D, C);
                    for (int k = 32 + lane; k < qc; k += 32)
#pragma unroll
                        for (int i = 0; i < 8; ++i) qs[w][k - 32][i] = qs[w][k][i];
                    qc -= 32;
                    __syncwarp();
                }
            }
            v0 = u0; v1 = u1; v2 = u2; v3 = u3;
            fl = fu;
        }
        __syncwarp();
        emit_queued(hs, qs[w], qoff[w], lane, qc, D, C);
    }
    __syncthreads();
    // the block's distinct pairs to both stars' worksets, PAIR_BATCH entries per
    // thread at a time so that their map loads and workset atomics overlap
    for (int k0 = tid; k0 < PAIR_HASH; k0 += PAIR_BATCH * 32 * PAIR_WARPS) {
        int ia[PAIR_BATCH], ib[PAIR_BATCH];
#pragma unroll
        for (int j = 0; j < PAIR_BATCH; ++j) {
            const int k = k0 + j * 32 * PAIR_WARPS;
            const unsigned long long key = k < PAIR_HASH ? hs[k] : ~0ull;
            ia[j] = ib[j] = -1;
            if (key != ~0ull) {
                ia[j] = site_to_id(C, (uint32_t)(key >> 32));
                ib[j] = site_to_id(C, (uint32_t)key);
            }
        }
        int pa[PAIR_BATCH], pb[PAIR_BATCH];
#pragma unroll
        for (int j = 0; j < PAIR_BATCH; ++j) {
            const bool ok = ia[j] >= 0 && ib[j] >= 0;
            pa[j] = ok ? atomicAdd(&D.bucketCount[ia[j]], 1) : -1;
            pb[j] = ok ? atomicAdd(&D.bucketCount[ib[j]], 1) : -1;
        }
#pragma unroll
        for (int j = 0; j < PAIR_BATCH; ++j) {
            if (pa[j] >= 0) bucket_put(D, ia[j], ib[j], pa[j]);
            if (pb[j] >= 0) bucket_put(D, ib[j], ia[j], pb[j]);
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

template <int AXIS, int LPW, int W>
static void launch_tiles(const Launch& L, int G, int K, const uint32_t* in, uint32_t* out) {
    const size_t sm = W * env_warp_smem<LPW>(G);
    const dim3 grid(G / (LPW * W), G, K), block(32 * W);
    if (G > 512) {
        cudaFuncSetAttribute(k_pba_env<AXIS, true, LPW, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pba_env<AXIS, true, LPW, W><<<grid, block, sm, L.stream>>>(G, in, out);
    } else {
        cudaFuncSetAttribute(k_pba_env<AXIS, false, LPW, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k_pba_env<AXIS, false, LPW, W><<<grid, block, sm, L.stream>>>(G, in, out);
    }
    ++*L.launches;
}

int pba_default_form(int G) { return G >= 1024 ? PBA_LINES : PBA_TILES_4; }

bool pba_form_ok(int form, int G) { return form >= 0 && form < PBA_FORMS && (form != PBA_TILES_2 || G >= 64); }

// `in` is scratch: the line form keeps its stacks in it
void launch_pba_y_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out, int form) {
    if (!pba_form_ok(form, G)) form = pba_default_form(G);
    if (form == PBA_LINES) {
        const dim3 grid(G / 32, G / 4, K), block(32, 4);
        if (G > 512) k_pba_line_y<true><<<grid, block, 0, L.stream>>>(G, in, out);
        else k_pba_line_y<false><<<grid, block, 0, L.stream>>>(G, in, out);
        ++*L.launches;
    } else if (form == PBA_TILES_4) {
        launch_tiles<1, 4, 4>(L, G, K, in, out);
    } else {
        launch_tiles<1, 4, 2>(L, G, K, in, out);
    }
}

void launch_pba_x_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out, int form) {
    if (!pba_form_ok(form, G)) form = pba_default_form(G);
    if (form == PBA_LINES) {
        const dim3 grid(G / 32, G / 4, K), block(32, 4);
        if (G > 512) k_pba_line_x<true><<<grid, block, 0, L.stream>>>(G, in, out);
        else k_pba_line_x<false><<<grid, block, 0, L.stream>>>(G, in, out);
        ++*L.launches;
    } else if (form == PBA_TILES_4) {
        launch_tiles<0, 4, 4>(L, G, K, in, out);
    } else {
        launch_tiles<0, 2, 2>(L, G, K, in, out);
    }
}

void launch_pba_y(const Launch& L, int G, uint32_t* in, uint32_t* out, int form) {
    launch_pba_y_stack(L, G, 1, in, out, form);
}

void launch_pba_x(const Launch& L, int G, uint32_t* in, uint32_t* out, int form) {
    launch_pba_x_stack(L, G, 1, in, out, form);
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
