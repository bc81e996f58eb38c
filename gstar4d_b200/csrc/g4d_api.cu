// C ABI and host orchestration (C++).
//
// Replaces the reference's facade and host drivers (GDelaunay/GDelaunay.cpp:
// 47-104, GDelHost.cu:136-1630): status codes instead of exit(-1), one context
// per host thread, a CUDA stream per context, CUB for the radix sorts and scans
// the reference did with Thrust, and one host read of a few counters per
// splaying round instead of dozens of implicit device->host reads.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "g4d_internal.cuh"

using namespace g4d;

namespace {

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes + bytes / 8 + 256;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) { p = nullptr; return e; }
        cap = want;
        return cudaSuccess;
    }
    template <class T>
    T* as() const { return reinterpret_cast<T*>(p); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

enum BufId {
    B_XYZ, B_GRIDSRC, B_MM, B_KEYS, B_VALS, B_VOXIN, B_MKEY, B_ORDER, B_P, B_VOX, B_CKEY0, B_CID0, B_CKEY,
    B_CID, B_COLS, B_COLE, B_GA, B_GB, B_BUCKET, B_BCOUNT, B_HH, B_TRI, B_HDR, B_INBOX, B_ICOUNT, B_WLINS,
    B_WLEMIT, B_WLEMIT2, B_DROWN, B_DROWN2, B_CTR, B_CNT, B_BASE, B_TETS, B_CUB, B_BAD, B_LIDX, B_LHH, B_LTRI,
    B_WLINSL, B_WLPROM, B_SKEY0, B_SKEY, B_GIDX, B_LOCAL, B_BCKEY0, B_BCKEY, B_SLOTS, B_MMB, B_TC, B_TETS2, B_OVF, B_OVF2, B_NUM
};

}  // namespace

struct g4d_ctx {
    g4d_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    Buf b[B_NUM];
    std::string err;
    // results of the last compute
    int n = 0;
    int G = 0;
    int ntet = 0;
    int large_cap = 0;   // large-class star slots allocated
    int large_used = 0;  // stars promoted to the large class by the last compute
    long long launches = 0;
    g4d_stats stats{};
    std::vector<g4d_tet> host_tets;
    // gdel-style state
    std::vector<double> gdel_points;
    bool gdel_ready = false;
    cudaEvent_t ev[8];
};

namespace {

g4d_status fail(g4d_ctx* c, g4d_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return s;
}

#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return fail(ctx, e_ == cudaErrorMemoryAllocation ? G4D_ERR_NOMEM : G4D_ERR_CUDA, \
                                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

int auto_grid(int n) {
    // about 134 voxels per point (the reference's default density), power of two
    const double want = std::cbrt(134.0 * (double)n);
    int G = 32;
    while (G < want && G < 1024) G <<= 1;
    return G;
}

Dev make_dev(g4d_ctx* ctx) {
    Dev D{};
    D.n = ctx->n;
    D.G = ctx->G;
    D.P = ctx->b[B_P].as<double4>();
    D.vox = ctx->b[B_VOX].as<uint32_t>();
    D.mkey = ctx->b[B_MKEY].as<uint32_t>();
    D.ckey = ctx->b[B_CKEY].as<uint32_t>();
    D.cid = ctx->b[B_CID].as<int>();
    D.colStart = ctx->b[B_COLS].as<int>();
    D.colEnd = ctx->b[B_COLE].as<int>();
    D.hh = ctx->b[B_HH].as<int>();
    D.tri = ctx->b[B_TRI].as<uint2>();
    D.hdr = ctx->b[B_HDR].as<StarHdr>();
    D.bucket = ctx->b[B_BUCKET].as<int>();
    D.bucketCount = ctx->b[B_BCOUNT].as<int>();
    D.inbox = ctx->b[B_INBOX].as<int>();
    D.inboxCount = ctx->b[B_ICOUNT].as<int>();
    D.wlIns = ctx->b[B_WLINS].as<int>();
    D.wlEmit = ctx->b[B_WLEMIT].as<int>();
    D.wlEmitNext = ctx->b[B_WLEMIT2].as<int>();
    D.drown = ctx->b[B_DROWN].as<int2>();
    D.drownNext = ctx->b[B_DROWN2].as<int2>();
    D.drownCap = (int)(ctx->b[B_DROWN].cap / sizeof(int2));
    D.ctr = ctx->b[B_CTR].as<Counters>();
    D.lidx = ctx->b[B_LIDX].as<int>();
    D.lhh = ctx->b[B_LHH].as<int>();
    D.ltri = ctx->b[B_LTRI].as<uint4>();
    D.largeCap = ctx->large_cap;
    D.wlInsL = ctx->b[B_WLINSL].as<int>();
    D.wlPromote = ctx->b[B_WLPROM].as<int>();
    D.anyLarge = 0;
    D.ovf = ctx->b[B_OVF].as<int2>();
    D.ovfNext = ctx->b[B_OVF2].as<int2>();
    D.ovfCap = (int)(std::min(ctx->b[B_OVF].cap, ctx->b[B_OVF2].cap) / sizeof(int2));
    D.cloudOff = nullptr;
    D.nclouds = 0;
    return D;
}

// Grow the large-star storage to hold `need` stars, keeping the stars already
// promoted (their slots are referenced by lidx).
g4d_status grow_large(g4d_ctx* ctx, Dev& D, int used, int need) {
    if (need <= ctx->large_cap) return G4D_OK;
    int cap = std::max(std::max(need, 2 * ctx->large_cap), 1024);
    cap = std::min(cap, std::max(ctx->n, 1));
    if (cap < need) return fail(ctx, G4D_ERR_CAPACITY, "large star storage for %d stars exceeds %d", need, cap);
    const size_t hb = sizeof(int) * (size_t)LHSLOTS, tb = sizeof(uint4) * (size_t)LTSTRIDE;
    void *nh = nullptr, *nt = nullptr, *nl = nullptr;
    CK(cudaMalloc(&nh, hb * cap));
    CK(cudaMalloc(&nt, tb * cap));
    CK(cudaMalloc(&nl, sizeof(int) * (size_t)cap));
    if (used > 0) {
        CK(cudaMemcpyAsync(nh, ctx->b[B_LHH].p, hb * used, cudaMemcpyDeviceToDevice, ctx->stream));
        CK(cudaMemcpyAsync(nt, ctx->b[B_LTRI].p, tb * used, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    CK(cudaStreamSynchronize(ctx->stream));
    ctx->b[B_LHH].release();
    ctx->b[B_LTRI].release();
    ctx->b[B_WLINSL].release();
    ctx->b[B_LHH].p = nh; ctx->b[B_LHH].cap = hb * cap;
    ctx->b[B_LTRI].p = nt; ctx->b[B_LTRI].cap = tb * cap;
    ctx->b[B_WLINSL].p = nl; ctx->b[B_WLINSL].cap = sizeof(int) * (size_t)cap;
    ctx->large_cap = cap;
    D.lhh = ctx->b[B_LHH].as<int>();
    D.ltri = ctx->b[B_LTRI].as<uint4>();
    D.wlInsL = ctx->b[B_WLINSL].as<int>();
    D.largeCap = cap;
    return G4D_OK;
}

g4d_status check_err(g4d_ctx* ctx, unsigned e) {
    if (!e) return G4D_OK;
    if (e & 0x100u) return fail(ctx, G4D_ERR_ARG, "grid coordinates outside [1, G-2]");
    if (e & ERR_PRECISION) {
        Counters h{};
        cudaMemcpy(&h, ctx->b[B_CTR].p, sizeof(Counters), cudaMemcpyDeviceToHost);
        return fail(ctx, G4D_ERR_PRECISION,
                    "coordinates span too wide an exponent range for exact predicates; first input: "
                    "(%.17g %.17g %.17g) (%.17g %.17g %.17g) (%.17g %.17g %.17g) (%.17g %.17g %.17g) "
                    "(%.17g %.17g %.17g) ids %d %d %d %d %d",
                    h.dbg_pts[0], h.dbg_pts[1], h.dbg_pts[2], h.dbg_pts[3], h.dbg_pts[4], h.dbg_pts[5],
                    h.dbg_pts[6], h.dbg_pts[7], h.dbg_pts[8], h.dbg_pts[9], h.dbg_pts[10], h.dbg_pts[11],
                    h.dbg_pts[12], h.dbg_pts[13], h.dbg_pts[14], h.dbg_ids[0], h.dbg_ids[1], h.dbg_ids[2],
                    h.dbg_ids[3], h.dbg_ids[4]);
    }
    if (e & ERR_CAPACITY)
        return fail(ctx, G4D_ERR_CAPACITY, "a star exceeded %d points / %d triangles (large class)", LHMAX, LTMAX);
    if (e & ERR_DROWNCAP) return fail(ctx, G4D_ERR_CAPACITY, "drowned or overflow request list capacity exceeded");
    return fail(ctx, G4D_ERR_INTERNAL, "star topology error (flags 0x%x)", e);
}

float ms_between(cudaEvent_t a, cudaEvent_t b) {
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    return t;
}

// Stage 1: order. xyz on device (input order). grid_src: device array of grid
// coordinates or nullptr (then xyz is scaled like Application::_scalePoint).
g4d_status run_order(g4d_ctx* ctx, const double* d_xyz, const double* d_grid_src, int n) {
    Launch L{ctx->stream, &ctx->launches};
    const int G = ctx->G;
    CK(ctx->b[B_MM].ensure(64));
    CK(ctx->b[B_KEYS].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_VALS].ensure(sizeof(int) * n));
    CK(ctx->b[B_VOXIN].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_MKEY].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_ORDER].ensure(sizeof(int) * n));
    CK(ctx->b[B_P].ensure(sizeof(double4) * n));
    CK(ctx->b[B_VOX].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_CKEY0].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_CID0].ensure(sizeof(int) * n));
    CK(ctx->b[B_CKEY].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_CID].ensure(sizeof(int) * n));
    CK(ctx->b[B_CTR].ensure(sizeof(Counters)));
    CK(cudaMemsetAsync(ctx->b[B_CTR].p, 0, sizeof(Counters), ctx->stream));
    unsigned long long* mm = ctx->b[B_MM].as<unsigned long long>();
    unsigned* err = &ctx->b[B_CTR].as<Counters>()->err;
    if (!d_grid_src) {
        CK(cudaMemsetAsync(mm, 0xff, 8, ctx->stream));
        CK(cudaMemsetAsync(mm + 1, 0, 8, ctx->stream));
        launch_minmax(L, d_xyz, n, mm);
    }
    launch_scale_morton(L, d_xyz, d_grid_src, n, G, d_grid_src ? nullptr : mm, ctx->b[B_KEYS].as<uint32_t>(),
                        ctx->b[B_VALS].as<int>(), ctx->b[B_VOXIN].as<uint32_t>(), err);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ctx->b[B_KEYS].as<uint32_t>(), ctx->b[B_MKEY].as<uint32_t>(),
                                       ctx->b[B_VALS].as<int>(), ctx->b[B_ORDER].as<int>(), n, 0, 30, ctx->stream));
    CK(ctx->b[B_CUB].ensure(tmp));
    CK(cub::DeviceRadixSort::SortPairs(ctx->b[B_CUB].p, tmp, ctx->b[B_KEYS].as<uint32_t>(),
                                       ctx->b[B_MKEY].as<uint32_t>(), ctx->b[B_VALS].as<int>(),
                                       ctx->b[B_ORDER].as<int>(), n, 0, 30, ctx->stream));
    ++ctx->launches;
    launch_gather(L, d_xyz, ctx->b[B_VOXIN].as<uint32_t>(), ctx->b[B_ORDER].as<int>(), n, ctx->b[B_P].as<double4>(),
                  ctx->b[B_VOX].as<uint32_t>(), nullptr);
    launch_colkeys(L, ctx->b[B_VOX].as<uint32_t>(), n, G, ctx->b[B_CKEY0].as<uint32_t>(), ctx->b[B_CID0].as<int>());
    tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ctx->b[B_CKEY0].as<uint32_t>(), ctx->b[B_CKEY].as<uint32_t>(),
                                       ctx->b[B_CID0].as<int>(), ctx->b[B_CID].as<int>(), n, 0, 30, ctx->stream));
    CK(ctx->b[B_CUB].ensure(tmp));
    CK(cub::DeviceRadixSort::SortPairs(ctx->b[B_CUB].p, tmp, ctx->b[B_CKEY0].as<uint32_t>(),
                                       ctx->b[B_CKEY].as<uint32_t>(), ctx->b[B_CID0].as<int>(),
                                       ctx->b[B_CID].as<int>(), n, 0, 30, ctx->stream));
    ++ctx->launches;
    const size_t G2 = (size_t)G * G;
    CK(ctx->b[B_COLS].ensure(sizeof(int) * G2));
    CK(ctx->b[B_COLE].ensure(sizeof(int) * G2));
    CK(cudaMemsetAsync(ctx->b[B_COLS].p, 0, sizeof(int) * G2, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_COLE].p, 0, sizeof(int) * G2, ctx->stream));
    launch_colranges(L, ctx->b[B_CKEY].as<uint32_t>(), n, G, ctx->b[B_COLS].as<int>(), ctx->b[B_COLE].as<int>());
    return G4D_OK;
}

// Star buffers for n points (every star starts in the small class).
g4d_status alloc_stars(g4d_ctx* ctx, int n) {
    CK(ctx->b[B_BUCKET].ensure(sizeof(int) * (size_t)n * BUCKET_CAP));
    CK(ctx->b[B_BCOUNT].ensure(sizeof(int) * n));
    CK(ctx->b[B_HH].ensure(sizeof(int) * (size_t)n * HSLOTS));
    CK(ctx->b[B_TRI].ensure(sizeof(uint2) * (size_t)n * TSTRIDE));
    CK(ctx->b[B_HDR].ensure(sizeof(StarHdr) * n));
    CK(ctx->b[B_INBOX].ensure(sizeof(int) * (size_t)n * INBOX_CAP));
    CK(ctx->b[B_ICOUNT].ensure(sizeof(int) * n));
    CK(ctx->b[B_WLINS].ensure(sizeof(int) * n));
    CK(ctx->b[B_WLEMIT].ensure(sizeof(int) * 2 * (size_t)n));
    CK(ctx->b[B_WLEMIT2].ensure(sizeof(int) * 2 * (size_t)n));
    CK(ctx->b[B_DROWN].ensure(sizeof(int2) * 16 * (size_t)n));
    CK(ctx->b[B_DROWN2].ensure(sizeof(int2) * 16 * (size_t)n));
    CK(ctx->b[B_CNT].ensure(sizeof(int) * (n + 1)));
    CK(ctx->b[B_BASE].ensure(sizeof(int) * (n + 1)));
    CK(ctx->b[B_BAD].ensure(64));
    CK(ctx->b[B_LIDX].ensure(sizeof(int) * n));
    CK(ctx->b[B_WLPROM].ensure(sizeof(int) * n));
    CK(ctx->b[B_OVF].ensure(sizeof(int2) * 4 * (size_t)n));
    CK(ctx->b[B_OVF2].ensure(sizeof(int2) * 4 * (size_t)n));
    return G4D_OK;
}

// Initial stars and the splaying loop (worksets already in the buckets).
g4d_status run_splay(g4d_ctx* ctx, Dev& D) {
    Launch L{ctx->stream, &ctx->launches};
    const int n = D.n;
    CK(cudaMemsetAsync(ctx->b[B_ICOUNT].p, 0, sizeof(int) * n, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_INBOX].p, 0xff, sizeof(int) * (size_t)n * INBOX_CAP, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_LIDX].p, 0xff, sizeof(int) * n, ctx->stream));
    launch_star_build(L, D);
    cudaEventRecord(ctx->ev[3], ctx->stream);

    Counters h{};
    Counters* dctr = D.ctr;
    CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    g4d_status st = check_err(ctx, h.err);
    if (st) return st;
    int emitCount = h.emit_next, drownCount = h.drown_next, ovfCount = h.ovf_next;
    // the lists produced by the build become the current ones
    std::swap(D.wlEmit, D.wlEmitNext);
    std::swap(D.drown, D.drownNext);
    std::swap(D.ovf, D.ovfNext);
    CK(cudaMemsetAsync(&dctr->emit_next, 0, 2 * sizeof(int), ctx->stream));  // emit_next, drown_next
    CK(cudaMemsetAsync(&dctr->ovf_next, 0, sizeof(int), ctx->stream));
    int loops = 0;
    const int max_loops = 4000;
    for (;; ++loops) {
        if (loops >= max_loops) return fail(ctx, G4D_ERR_TIMEOUT, "splaying did not converge in %d loops", max_loops);
        if (ovfCount) launch_requeue(L, D, std::min(ovfCount, D.ovfCap));
        if (drownCount) launch_proof(L, D, drownCount);
        if (emitCount) launch_emit(L, D, emitCount);
        CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        st = check_err(ctx, h.err);
        if (st) return st;
        if (h.ins_count == 0 && h.ins_count_large == 0) break;
        ovfCount = h.ovf_next;  // requests that found a full inbox this round
        if (h.ins_count) launch_star_insert(L, D, h.ins_count);
        if (h.ins_count_large) launch_star_insert_large(L, D, D.wlInsL, std::min(h.ins_count_large, D.largeCap));
        CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        st = check_err(ctx, h.err);
        if (st) return st;
        if (h.promote_count) {
            // stars that outgrew the small class: move them, then replay their round
            st = grow_large(ctx, D, h.large_next, h.large_next + h.promote_count);
            if (st) return st;
            launch_promote(L, D, h.promote_count);
            D.anyLarge = 1;
            launch_star_insert_large(L, D, D.wlPromote, h.promote_count);
            CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
            CK(cudaStreamSynchronize(ctx->stream));
            st = check_err(ctx, h.err);
            if (st) return st;
        }
        emitCount = h.emit_next;
        drownCount = h.drown_next;
        std::swap(D.wlEmit, D.wlEmitNext);
        std::swap(D.drown, D.drownNext);
        std::swap(D.ovf, D.ovfNext);
        // ins_count, emit_next, drown_next, ins_count_large, promote_count
        CK(cudaMemsetAsync(dctr, 0, 5 * sizeof(int), ctx->stream));
        CK(cudaMemsetAsync(&dctr->ovf_next, 0, sizeof(int), ctx->stream));
    }
    cudaEventRecord(ctx->ev[4], ctx->stream);
    ctx->stats.loops = loops;
    ctx->stats.splay_insertions = (long long)h.insertions;
    ctx->stats.proofs = (long long)h.proofs_total;
    ctx->stats.exact_predicates = (long long)h.exact;
    ctx->large_used = h.large_next;

    if (ctx->cfg.do_check) {
        unsigned long long* bad = ctx->b[B_BAD].as<unsigned long long>();
        CK(cudaMemsetAsync(bad, 0, 8, ctx->stream));
        launch_check(L, D, bad);
        unsigned long long hb = 0;
        CK(cudaMemcpyAsync(&hb, bad, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        if (hb) return fail(ctx, G4D_ERR_INTERNAL, "stars are not consistent (%llu missing triangles)", hb);
    }
    return G4D_OK;
}

// Tetrahedra of all stars: count, scan, write (ids mapped through
// sorted_to_input when given).
g4d_status run_extract(g4d_ctx* ctx, const Dev& D, const int* sorted_to_input) {
    Launch L{ctx->stream, &ctx->launches};
    const int n = D.n;
    int* cnt = ctx->b[B_CNT].as<int>();
    int* base = ctx->b[B_BASE].as<int>();
    launch_tet_count(L, D, cnt);
    size_t tmp = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tmp, cnt, base, n + 1, ctx->stream));
    CK(ctx->b[B_CUB].ensure(tmp));
    CK(cudaMemsetAsync(cnt + n, 0, sizeof(int), ctx->stream));
    CK(cub::DeviceScan::ExclusiveSum(ctx->b[B_CUB].p, tmp, cnt, base, n + 1, ctx->stream));
    ++ctx->launches;
    int ntet = 0;
    CK(cudaMemcpyAsync(&ntet, base + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(ctx->b[B_TETS].ensure(sizeof(g4d_tet) * (size_t)std::max(ntet, 1)));
    launch_tet_write(L, D, base, ctx->b[B_TETS].as<g4d_tet>(), sorted_to_input);
    cudaEventRecord(ctx->ev[5], ctx->stream);
    Counters h{};
    CK(cudaMemcpyAsync(&h, D.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    g4d_status st = check_err(ctx, h.err);
    if (st) return st;
    ctx->ntet = ntet;
    ctx->stats.tets = ntet;
    return G4D_OK;
}

// Stages 2-5: digital Voronoi, stars, splaying, extraction.
g4d_status run_compute(g4d_ctx* ctx, bool map_to_input) {
    Launch L{ctx->stream, &ctx->launches};
    const int n = ctx->n, G = ctx->G;
    const size_t G3 = (size_t)G * G * G;
    CK(ctx->b[B_GA].ensure(sizeof(uint32_t) * G3));
    CK(ctx->b[B_GB].ensure(sizeof(uint32_t) * G3));
    g4d_status st = alloc_stars(ctx, n);
    if (st) return st;
    Dev D = make_dev(ctx);
    // equalise the two drowned buffers' capacity
    D.drownCap = (int)std::min(ctx->b[B_DROWN].cap, ctx->b[B_DROWN2].cap) / (int)sizeof(int2);

    cudaEventRecord(ctx->ev[1], ctx->stream);
    // digital Voronoi diagram
    uint32_t* gA = ctx->b[B_GA].as<uint32_t>();
    uint32_t* gB = ctx->b[B_GB].as<uint32_t>();
    launch_pba_z(L, D, gA);
    launch_pba_y(L, G, gA, gB);
    launch_pba_x(L, G, gB, gA);
    cudaEventRecord(ctx->ev[2], ctx->stream);
    // worksets
    CK(cudaMemsetAsync(ctx->b[B_BCOUNT].p, 0, sizeof(int) * n, ctx->stream));
    launch_pairs(L, D, gA);
    launch_missing(L, D);
    st = run_splay(ctx, D);
    if (st) return st;
    return run_extract(ctx, D, map_to_input ? ctx->b[B_ORDER].as<int>() : nullptr);
}

void finish_stats(g4d_ctx* ctx) {
    g4d_stats& s = ctx->stats;
    s.t_init_ms = ms_between(ctx->ev[0], ctx->ev[1]);
    s.t_pba_ms = ms_between(ctx->ev[1], ctx->ev[2]);
    s.t_star_ms = ms_between(ctx->ev[2], ctx->ev[3]);
    s.t_splay_ms = ms_between(ctx->ev[3], ctx->ev[4]);
    s.t_out_ms = ms_between(ctx->ev[4], ctx->ev[5]);
    s.t_total_ms = ms_between(ctx->ev[0], ctx->ev[5]);
    s.grid_size = ctx->G;
    s.gpu_launches = ctx->launches;
    s.large_stars = ctx->large_used;
}

g4d_status check_n(g4d_ctx* ctx, int n) {
    if (!ctx) return G4D_ERR_ARG;
    if (n < 5) return fail(ctx, G4D_ERR_ARG, "need at least 5 points (got %d)", n);
    if (n >= (1 << 30)) return fail(ctx, G4D_ERR_ARG, "too many points (%d)", n);
    return G4D_OK;
}

g4d_status pick_grid(g4d_ctx* ctx, int n) {
    int G = ctx->cfg.grid_size > 0 ? ctx->cfg.grid_size : auto_grid(n);
    if (G < 32 || G > 1024 || (G & (G - 1)))
        return fail(ctx, G4D_ERR_ARG, "grid size must be a power of two in [32, 1024] (got %d)", G);
    ctx->G = G;
    return G4D_OK;
}

// full device pipeline on d_xyz (input order)
g4d_status run_all_device(g4d_ctx* ctx, const double* d_xyz, const double* d_grid_src, int n, bool map_to_input) {
    ctx->n = n;
    ctx->launches = 0;
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    g4d_status st = pick_grid(ctx, n);
    if (st) return st;
    cudaEventRecord(ctx->ev[0], ctx->stream);
    st = run_order(ctx, d_xyz, d_grid_src, n);
    if (st) return st;
    st = run_compute(ctx, map_to_input);
    if (st) return st;
    finish_stats(ctx);
    return G4D_OK;
}

// ---------------------------------------------------------------------------
// Batches: one pass ("wave") triangulates many clouds together. The clouds of
// a wave are ordered by grid width; clouds of equal width form one stack of
// grids, so every PBA and pair kernel runs once per distinct width, and the
// star and splaying kernels run once over all points of the wave (stars only
// ever reference points of their own cloud). A wave holds at most
// kWavePoints points and kWaveVoxels voxels per grid buffer.
// ---------------------------------------------------------------------------

constexpr long long kWavePoints = 8LL << 20;
constexpr long long kWaveVoxels = 4LL << 30;

int bits_for(unsigned long long v) {
    int b = 0;
    while ((1ull << b) <= v && b < 63) ++b;
    return b;
}

struct BatchOut {
    g4d_tet* tets = nullptr;
    size_t count = 0, cap = 0;
};

// clouds[c0..c1) of the batch, grid widths in Gc; appends the wave's
// tetrahedra (cloud order, cloud-local ids) to out and fills tet counts.
g4d_status run_wave(g4d_ctx* ctx, const double* d_xyz, const int64_t* offs, int c0, int c1, const int* Gc,
                    BatchOut& out, int64_t* tet_counts) {
    Launch L{ctx->stream, &ctx->launches};
    const int ns = c1 - c0;
    // slots: clouds ordered by grid width (stable)
    std::vector<int> slot_cloud(ns);
    for (int k = 0; k < ns; ++k) slot_cloud[k] = c0 + k;
    std::stable_sort(slot_cloud.begin(), slot_cloud.end(), [&](int a, int b) { return Gc[a] < Gc[b]; });
    std::vector<long long> slotIn(ns), slotCol(ns);
    std::vector<int> slotW(ns + 1), slotG(ns);
    struct Stack { int G, k0, K; long long col, vox; };
    std::vector<Stack> stacks;
    long long cols = 0, voxels = 0;
    slotW[0] = 0;
    for (int k = 0; k < ns; ++k) {
        const int c = slot_cloud[k], G = Gc[c];
        slotIn[k] = offs[c];
        slotW[k + 1] = slotW[k] + (int)(offs[c + 1] - offs[c]);
        slotG[k] = G;
        if (stacks.empty() || stacks.back().G != G) stacks.push_back({G, k, 0, cols, voxels});
        stacks.back().K++;
        slotCol[k] = cols;
        cols += (long long)G * G;
        voxels += (long long)G * G * G;
    }
    const int n = slotW[ns];
    ctx->n = n;
    // device copies of the slot tables: slotIn, slotCol, dst (int64), slotW, slotG, tc (int32)
    const size_t i64b = sizeof(long long) * ns, i32b = sizeof(int) * (ns + 1);
    CK(ctx->b[B_SLOTS].ensure(3 * i64b + 3 * i32b + 64));
    char* sb = ctx->b[B_SLOTS].as<char>();
    long long* d_slotIn = reinterpret_cast<long long*>(sb);
    long long* d_slotCol = reinterpret_cast<long long*>(sb + i64b);
    long long* d_dst = reinterpret_cast<long long*>(sb + 2 * i64b);
    int* d_slotW = reinterpret_cast<int*>(sb + 3 * i64b);
    int* d_slotG = reinterpret_cast<int*>(sb + 3 * i64b + i32b);
    int* d_tc = reinterpret_cast<int*>(sb + 3 * i64b + 2 * i32b);
    CK(cudaMemcpyAsync(d_slotIn, slotIn.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_slotCol, slotCol.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_slotW, slotW.data(), i32b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_slotG, slotG.data(), sizeof(int) * ns, cudaMemcpyHostToDevice, ctx->stream));

    // order
    CK(ctx->b[B_MMB].ensure(sizeof(unsigned long long) * 2 * ns));
    CK(ctx->b[B_SKEY0].ensure(sizeof(unsigned long long) * n));
    CK(ctx->b[B_SKEY].ensure(sizeof(unsigned long long) * n));
    CK(ctx->b[B_VALS].ensure(sizeof(int) * n));
    CK(ctx->b[B_ORDER].ensure(sizeof(int) * n));
    CK(ctx->b[B_VOXIN].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_GIDX].ensure(sizeof(long long) * n));
    CK(ctx->b[B_P].ensure(sizeof(double4) * n));
    CK(ctx->b[B_VOX].ensure(sizeof(uint32_t) * n));
    CK(ctx->b[B_LOCAL].ensure(sizeof(int) * n));
    CK(ctx->b[B_BCKEY0].ensure(sizeof(unsigned long long) * n));
    CK(ctx->b[B_BCKEY].ensure(sizeof(unsigned long long) * n));
    CK(ctx->b[B_CID0].ensure(sizeof(int) * n));
    CK(ctx->b[B_CID].ensure(sizeof(int) * n));
    CK(ctx->b[B_COLS].ensure(sizeof(int) * cols));
    CK(ctx->b[B_COLE].ensure(sizeof(int) * cols));
    CK(ctx->b[B_GA].ensure(sizeof(uint32_t) * voxels));
    CK(ctx->b[B_GB].ensure(sizeof(uint32_t) * voxels));
    CK(ctx->b[B_CTR].ensure(sizeof(Counters)));
    CK(cudaMemsetAsync(ctx->b[B_CTR].p, 0, sizeof(Counters), ctx->stream));
    g4d_status st = alloc_stars(ctx, n);
    if (st) return st;
    unsigned* err = &ctx->b[B_CTR].as<Counters>()->err;
    cudaEventRecord(ctx->ev[0], ctx->stream);
    unsigned long long* skey0 = ctx->b[B_SKEY0].as<unsigned long long>();
    unsigned long long* skey = ctx->b[B_SKEY].as<unsigned long long>();
    launch_b_order(L, d_xyz, ns, d_slotIn, d_slotW, d_slotG, ctx->b[B_MMB].as<unsigned long long>(), skey0,
                   ctx->b[B_VALS].as<int>(), ctx->b[B_VOXIN].as<uint32_t>(), ctx->b[B_GIDX].as<long long>(), err);
    const int kbits = 30 + bits_for((unsigned long long)ns);
    size_t tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, skey0, skey, ctx->b[B_VALS].as<int>(), ctx->b[B_ORDER].as<int>(),
                                       n, 0, kbits, ctx->stream));
    CK(ctx->b[B_CUB].ensure(tmp));
    CK(cub::DeviceRadixSort::SortPairs(ctx->b[B_CUB].p, tmp, skey0, skey, ctx->b[B_VALS].as<int>(),
                                       ctx->b[B_ORDER].as<int>(), n, 0, kbits, ctx->stream));
    ++ctx->launches;
    launch_b_gather(L, d_xyz, ctx->b[B_GIDX].as<long long>(), ctx->b[B_VOXIN].as<uint32_t>(),
                    ctx->b[B_ORDER].as<int>(), skey, d_slotW, n, ctx->b[B_P].as<double4>(),
                    ctx->b[B_VOX].as<uint32_t>(), ctx->b[B_LOCAL].as<int>());
    unsigned long long* ckey0 = ctx->b[B_BCKEY0].as<unsigned long long>();
    unsigned long long* ckey = ctx->b[B_BCKEY].as<unsigned long long>();
    launch_b_colkeys(L, ctx->b[B_VOX].as<uint32_t>(), skey, d_slotG, d_slotCol, n, ckey0, ctx->b[B_CID0].as<int>());
    const int cbits = 10 + bits_for((unsigned long long)cols);
    tmp = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp, ckey0, ckey, ctx->b[B_CID0].as<int>(), ctx->b[B_CID].as<int>(), n,
                                       0, cbits, ctx->stream));
    CK(ctx->b[B_CUB].ensure(tmp));
    CK(cub::DeviceRadixSort::SortPairs(ctx->b[B_CUB].p, tmp, ckey0, ckey, ctx->b[B_CID0].as<int>(),
                                       ctx->b[B_CID].as<int>(), n, 0, cbits, ctx->stream));
    ++ctx->launches;
    int* cs = ctx->b[B_COLS].as<int>();
    int* ce = ctx->b[B_COLE].as<int>();
    CK(cudaMemsetAsync(cs, 0, sizeof(int) * cols, ctx->stream));
    CK(cudaMemsetAsync(ce, 0, sizeof(int) * cols, ctx->stream));
    launch_colranges_u64(L, ckey, n, cs, ce);

    Dev D = make_dev(ctx);
    D.drownCap = (int)std::min(ctx->b[B_DROWN].cap, ctx->b[B_DROWN2].cap) / (int)sizeof(int2);
    D.G = 0;
    D.cloudOff = d_slotW;
    D.nclouds = ns;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    uint32_t* gA = ctx->b[B_GA].as<uint32_t>();
    uint32_t* gB = ctx->b[B_GB].as<uint32_t>();
    for (const Stack& S : stacks) {
        launch_pba_z_stack(L, S.G, S.K, ckey, cs + S.col, ce + S.col, gA + S.vox);
        launch_pba_y_stack(L, S.G, S.K, gA + S.vox, gB + S.vox);
        launch_pba_x_stack(L, S.G, S.K, gB + S.vox, gA + S.vox);
    }
    cudaEventRecord(ctx->ev[2], ctx->stream);
    CK(cudaMemsetAsync(ctx->b[B_BCOUNT].p, 0, sizeof(int) * n, ctx->stream));
    for (const Stack& S : stacks)
        launch_pairs_stack(L, D, gA + S.vox, S.G, S.K, ckey, ctx->b[B_CID].as<int>(), cs + S.col, ce + S.col);
    launch_missing_u64(L, D, skey);
    st = run_splay(ctx, D);
    if (st) return st;
    st = run_extract(ctx, D, nullptr);
    if (st) return st;
    // per-cloud counts and output offsets in cloud order
    const int ntet = ctx->ntet;
    launch_b_slot_tets(L, ctx->b[B_BASE].as<int>(), d_slotW, ns, d_tc);
    std::vector<int> tc(ns);
    CK(cudaMemcpyAsync(tc.data(), d_tc, sizeof(int) * ns, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<long long> cnt_cloud(ns), dst(ns);
    for (int k = 0; k < ns; ++k) cnt_cloud[slot_cloud[k] - c0] = tc[k];
    std::vector<long long> off_cloud(ns + 1, 0);
    for (int c = 0; c < ns; ++c) off_cloud[c + 1] = off_cloud[c] + cnt_cloud[c];
    for (int k = 0; k < ns; ++k) dst[k] = off_cloud[slot_cloud[k] - c0];
    for (int c = 0; c < ns; ++c) tet_counts[c0 + c] = cnt_cloud[c];
    CK(cudaMemcpyAsync(d_dst, dst.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    CK(ctx->b[B_TETS2].ensure(sizeof(g4d_tet) * (size_t)std::max(ntet, 1)));
    launch_b_localize(L, ctx->b[B_TETS].as<g4d_tet>(), ntet, skey, ctx->b[B_LOCAL].as<int>(),
                      ctx->b[B_BASE].as<int>(), d_slotW, d_dst, ctx->b[B_TETS2].as<g4d_tet>());
    // host output
    if (out.count + (size_t)ntet > out.cap) {
        size_t ncap = std::max(out.cap * 2, out.count + (size_t)ntet);
        g4d_tet* p = (g4d_tet*)realloc(out.tets, sizeof(g4d_tet) * std::max<size_t>(ncap, 1));
        if (!p) return fail(ctx, G4D_ERR_NOMEM, "host allocation of %zu tetrahedra failed", ncap);
        out.tets = p;
        out.cap = ncap;
    }
    CK(cudaMemcpyAsync(out.tets + out.count, ctx->b[B_TETS2].p, sizeof(g4d_tet) * (size_t)ntet,
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    out.count += ntet;
    return G4D_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

void g4d_default_config(g4d_config* cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof(*cfg));
    cfg->seed = 0;
    cfg->run_num = 1;
    cfg->grid_size = 0;
    cfg->point_num = 100000;
    cfg->facet_max = -1;
    cfg->pred_thread_num = -1;
    cfg->pred_block_num = -1;
    cfg->do_sorting = 1;
}

const char* g4d_status_string(g4d_status s) {
    switch (s) {
        case G4D_OK: return "ok";
        case G4D_ERR_ARG: return "invalid argument";
        case G4D_ERR_NOMEM: return "out of memory";
        case G4D_ERR_TIMEOUT: return "iteration cap reached";
        case G4D_ERR_INTERNAL: return "internal consistency error";
        case G4D_ERR_CUDA: return "CUDA error";
        case G4D_ERR_CAPACITY: return "star capacity exceeded";
        case G4D_ERR_PRECISION: return "coordinate exponent range too wide";
        case G4D_ERR_NODEVICE: return "no sm_100 device";
    }
    return "unknown";
}

g4d_status g4d_create(g4d_ctx** out, const g4d_config* cfg) {
    if (!out) return G4D_ERR_ARG;
    *out = nullptr;
    g4d_ctx* ctx = new (std::nothrow) g4d_ctx();
    if (!ctx) return G4D_ERR_NOMEM;
    if (cfg) ctx->cfg = *cfg; else g4d_default_config(&ctx->cfg);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        delete ctx;
        return G4D_ERR_NODEVICE;
    }
    ctx->device = ctx->cfg.device;
    if (ctx->device < 0 || ctx->device >= count || cudaSetDevice(ctx->device) != cudaSuccess) {
        delete ctx;
        return G4D_ERR_NODEVICE;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, ctx->device);
    if (prop.major != 10) {
        delete ctx;
        return G4D_ERR_NODEVICE;
    }
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return G4D_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    *out = ctx;
    return G4D_OK;
}

void g4d_destroy(g4d_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->b) b.release();
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* g4d_last_error(const g4d_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

g4d_status g4d_triangulate_device(g4d_ctx* ctx, const double* d_xyz, int n, const g4d_tet** d_tets, int* ntet,
                                  g4d_stats* stats) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!d_xyz || !d_tets || !ntet) return fail(ctx, G4D_ERR_ARG, "null argument");
    cudaSetDevice(ctx->device);
    st = run_all_device(ctx, d_xyz, nullptr, n, ctx->cfg.index_space == 0);
    if (st) return st;
    *d_tets = ctx->b[B_TETS].as<g4d_tet>();
    *ntet = ctx->ntet;
    if (stats) *stats = ctx->stats;
    return G4D_OK;
}

g4d_status g4d_triangulate_to(g4d_ctx* ctx, const double* xyz, int n, g4d_tet* out, int cap, int* ntet,
                              int* sorted_to_input, g4d_stats* stats) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!xyz || !ntet) return fail(ctx, G4D_ERR_ARG, "null argument");
    cudaSetDevice(ctx->device);
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)n));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    st = run_all_device(ctx, ctx->b[B_XYZ].as<double>(), nullptr, n, ctx->cfg.index_space == 0);
    if (st) return st;
    *ntet = ctx->ntet;
    if (out) {
        if (cap < ctx->ntet) return fail(ctx, G4D_ERR_ARG, "output buffer too small (%d < %d)", cap, ctx->ntet);
        CK(cudaMemcpyAsync(out, ctx->b[B_TETS].p, sizeof(g4d_tet) * (size_t)ctx->ntet, cudaMemcpyDeviceToHost,
                           ctx->stream));
    }
    if (sorted_to_input)
        CK(cudaMemcpyAsync(sorted_to_input, ctx->b[B_ORDER].p, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost,
                           ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (stats) *stats = ctx->stats;
    return G4D_OK;
}

g4d_status g4d_triangulate(g4d_ctx* ctx, const double* xyz, int n, g4d_tet** tets, int* ntet, int* sorted_to_input,
                           g4d_stats* stats) {
    if (!tets) return fail(ctx, G4D_ERR_ARG, "null argument");
    *tets = nullptr;
    int nt = 0;
    g4d_status st = g4d_triangulate_to(ctx, xyz, n, nullptr, 0, &nt, sorted_to_input, stats);
    if (st) return st;
    g4d_tet* out = (g4d_tet*)malloc(sizeof(g4d_tet) * (size_t)std::max(nt, 1));
    if (!out) return fail(ctx, G4D_ERR_NOMEM, "host allocation of %d tetrahedra failed", nt);
    CK(cudaMemcpyAsync(out, ctx->b[B_TETS].p, sizeof(g4d_tet) * (size_t)nt, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    *tets = out;
    *ntet = nt;
    return G4D_OK;
}

// -------- reference-shaped entry points ----------------------------------------

g4d_status g4d_gdel_init(g4d_ctx* ctx, double* points, double* scaled, int n) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!points) return fail(ctx, G4D_ERR_ARG, "null points");
    cudaSetDevice(ctx->device);
    ctx->n = n;
    ctx->launches = 0;
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    st = pick_grid(ctx, n);
    if (st) return st;
    const size_t bytes = sizeof(double) * 3 * (size_t)n;
    CK(ctx->b[B_XYZ].ensure(bytes));
    CK(ctx->b[B_GRIDSRC].ensure(bytes));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, points, bytes, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->b[B_GRIDSRC].p, scaled ? scaled : points, bytes, cudaMemcpyHostToDevice, ctx->stream));
    cudaEventRecord(ctx->ev[0], ctx->stream);
    st = run_order(ctx, ctx->b[B_XYZ].as<double>(), ctx->b[B_GRIDSRC].as<double>(), n);
    if (st) return st;
    // like PointData::init (GDelData.cu:125-130): hand back the sorted order
    std::vector<int> order(n);
    CK(cudaMemcpyAsync(order.data(), ctx->b[B_ORDER].p, sizeof(int) * n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    Counters h{};
    CK(cudaMemcpy(&h, ctx->b[B_CTR].p, sizeof(Counters), cudaMemcpyDeviceToHost));
    st = check_err(ctx, h.err);
    if (st) return st;
    std::vector<double> tmp(3 * (size_t)n);
    for (int i = 0; i < n; ++i) memcpy(&tmp[3 * (size_t)i], points + 3 * (size_t)order[i], sizeof(double) * 3);
    memcpy(points, tmp.data(), bytes);
    if (scaled) {
        for (int i = 0; i < n; ++i) memcpy(&tmp[3 * (size_t)i], scaled + 3 * (size_t)order[i], sizeof(double) * 3);
        memcpy(scaled, tmp.data(), bytes);
    }
    ctx->gdel_ready = true;
    return G4D_OK;
}

g4d_status g4d_gdel_compute(g4d_ctx* ctx, double* t_pba, double* t_star, double* t_splay, double* t_out) {
    if (!ctx) return G4D_ERR_ARG;
    if (!ctx->gdel_ready) return fail(ctx, G4D_ERR_ARG, "g4d_gdel_init was not called");
    cudaSetDevice(ctx->device);
    g4d_status st = run_compute(ctx, false);
    if (st) return st;
    finish_stats(ctx);
    if (t_pba) *t_pba = ctx->stats.t_pba_ms;
    if (t_star) *t_star = ctx->stats.t_star_ms;
    if (t_splay) *t_splay = ctx->stats.t_splay_ms;
    if (t_out) *t_out = ctx->stats.t_out_ms;
    ctx->host_tets.resize((size_t)ctx->ntet);
    CK(cudaMemcpyAsync(ctx->host_tets.data(), ctx->b[B_TETS].p, sizeof(g4d_tet) * (size_t)ctx->ntet,
                       cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return G4D_OK;
}

g4d_status g4d_get_tetra(g4d_ctx* ctx, const g4d_tet** tets, int* ntet) {
    if (!ctx || !tets || !ntet) return G4D_ERR_ARG;
    *tets = ctx->host_tets.data();
    *ntet = (int)ctx->host_tets.size();
    return G4D_OK;
}

g4d_status g4d_gdel_deinit(g4d_ctx* ctx) {
    if (!ctx) return G4D_ERR_ARG;
    ctx->gdel_ready = false;
    ctx->host_tets.clear();
    ctx->host_tets.shrink_to_fit();
    return G4D_OK;
}

g4d_status g4d_triangulate_batch(g4d_ctx* ctx, const double* xyz, const int64_t* cloud_offsets, int nclouds,
                                 g4d_tet** tets, int64_t** tet_offsets, g4d_stats* stats) {
    if (!ctx) return G4D_ERR_ARG;
    if (!xyz || !cloud_offsets || nclouds < 0 || !tets || !tet_offsets) return fail(ctx, G4D_ERR_ARG, "null argument");
    *tets = nullptr;
    *tet_offsets = nullptr;
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<int> Gc(std::max(nclouds, 1));
    for (int c = 0; c < nclouds; ++c) {
        const int64_t n = cloud_offsets[c + 1] - cloud_offsets[c];
        if (n < 5 || n >= (1 << 30)) return fail(ctx, G4D_ERR_ARG, "cloud %d has %lld points (need 5 or more)", c, (long long)n);
        const int G = ctx->cfg.grid_size > 0 ? ctx->cfg.grid_size : auto_grid((int)n);
        if (G < 32 || G > 1024 || (G & (G - 1)))
            return fail(ctx, G4D_ERR_ARG, "grid size must be a power of two in [32, 1024] (got %d)", G);
        Gc[c] = G;
    }
    const int64_t total = nclouds ? cloud_offsets[nclouds] - cloud_offsets[0] : 0;
    if (nclouds && cloud_offsets[0] != 0) return fail(ctx, G4D_ERR_ARG, "cloud_offsets[0] must be 0");
    ctx->launches = 0;
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)std::max<int64_t>(total, 1)));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)total, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int64_t> counts(nclouds, 0);
    BatchOut out;
    g4d_stats acc{};
    int large = 0;
    for (int c0 = 0; c0 < nclouds;) {
        int c1 = c0;
        long long pts = 0, vox = 0;
        while (c1 < nclouds) {
            const long long n = cloud_offsets[c1 + 1] - cloud_offsets[c1];
            const long long v = (long long)Gc[c1] * Gc[c1] * Gc[c1];
            if (c1 > c0 && (pts + n > kWavePoints || vox + v > kWaveVoxels)) break;
            pts += n;
            vox += v;
            ++c1;
        }
        g4d_status st = run_wave(ctx, ctx->b[B_XYZ].as<double>(), cloud_offsets, c0, c1, Gc.data(), out,
                                 counts.data());
        if (st) { free(out.tets); return st; }
        acc.t_pba_ms += ms_between(ctx->ev[1], ctx->ev[2]);
        acc.t_star_ms += ms_between(ctx->ev[2], ctx->ev[3]);
        acc.t_splay_ms += ms_between(ctx->ev[3], ctx->ev[4]);
        acc.t_out_ms += ms_between(ctx->ev[4], ctx->ev[5]);
        acc.splay_insertions += ctx->stats.splay_insertions;
        acc.proofs += ctx->stats.proofs;
        acc.exact_predicates += ctx->stats.exact_predicates;
        acc.loops = std::max(acc.loops, ctx->stats.loops);
        large += ctx->large_used;
        c0 = c1;
    }
    int64_t* offs = (int64_t*)malloc(sizeof(int64_t) * (nclouds + 1));
    if (!offs) { free(out.tets); return fail(ctx, G4D_ERR_NOMEM, "host allocation failed"); }
    offs[0] = 0;
    for (int c = 0; c < nclouds; ++c) offs[c + 1] = offs[c] + counts[c];
    if (!out.tets) out.tets = (g4d_tet*)malloc(sizeof(g4d_tet));
    *tets = out.tets;
    *tet_offsets = offs;
    acc.tets = (int)std::min<size_t>(out.count, 0x7fffffff);
    acc.gpu_launches = ctx->launches;
    acc.large_stars = large;
    acc.t_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->stats = acc;
    if (stats) *stats = acc;
    return G4D_OK;
}

g4d_status g4d_eval_predicates(g4d_ctx* ctx, int kind, const double* pts, const int* idx, int count, int8_t* out) {
    if (!ctx || !pts || !out || count < 0 || kind < 0 || kind > 2 || (kind == 1 && !idx)) return G4D_ERR_ARG;
    if (count == 0) return G4D_OK;
    cudaSetDevice(ctx->device);
    const int per = kind == 0 ? 12 : 15;
    void *dp = nullptr, *di = nullptr, *dout = nullptr, *derr = nullptr;
    CK(cudaMalloc(&dp, sizeof(double) * per * (size_t)count));
    CK(cudaMalloc(&dout, (size_t)count));
    CK(cudaMalloc(&derr, sizeof(unsigned)));
    if (kind == 1) CK(cudaMalloc(&di, sizeof(int) * 5 * (size_t)count));
    CK(cudaMemcpyAsync(dp, pts, sizeof(double) * per * (size_t)count, cudaMemcpyHostToDevice, ctx->stream));
    if (kind == 1) CK(cudaMemcpyAsync(di, idx, sizeof(int) * 5 * (size_t)count, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(derr, 0, sizeof(unsigned), ctx->stream));
    Launch L{ctx->stream, &ctx->launches};
    launch_eval_pred(L, kind, (const double*)dp, (const int*)di, count, (int8_t*)dout, (unsigned*)derr);
    unsigned herr = 0;
    CK(cudaMemcpyAsync(out, dout, (size_t)count, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&herr, derr, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(dp);
    cudaFree(dout);
    cudaFree(derr);
    if (di) cudaFree(di);
    if (herr) return fail(ctx, G4D_ERR_PRECISION, "coordinates span too wide an exponent range");
    return G4D_OK;
}

g4d_status g4d_voronoi(g4d_ctx* ctx, const double* xyz, int n, int grid, uint32_t* sites) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!xyz || !sites) return fail(ctx, G4D_ERR_ARG, "null argument");
    if (grid < 32 || grid > 1024 || (grid & (grid - 1))) return fail(ctx, G4D_ERR_ARG, "bad grid %d", grid);
    cudaSetDevice(ctx->device);
    ctx->n = n;
    ctx->G = grid;
    const size_t G3 = (size_t)grid * grid * grid;
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)n));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    st = run_order(ctx, ctx->b[B_XYZ].as<double>(), nullptr, n);
    if (st) return st;
    CK(ctx->b[B_GA].ensure(sizeof(uint32_t) * G3));
    CK(ctx->b[B_GB].ensure(sizeof(uint32_t) * G3));
    Launch L{ctx->stream, &ctx->launches};
    Dev D = make_dev(ctx);
    launch_pba_z(L, D, ctx->b[B_GA].as<uint32_t>());
    launch_pba_y(L, grid, ctx->b[B_GA].as<uint32_t>(), ctx->b[B_GB].as<uint32_t>());
    launch_pba_x(L, grid, ctx->b[B_GB].as<uint32_t>(), ctx->b[B_GA].as<uint32_t>());
    CK(cudaMemcpyAsync(sites, ctx->b[B_GA].p, sizeof(uint32_t) * G3, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return G4D_OK;
}

void* g4d_stream(g4d_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

void g4d_free(void* p) { free(p); }

}  // extern "C"
