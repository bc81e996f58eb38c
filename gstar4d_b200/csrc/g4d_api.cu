// C ABI and host orchestration (C++).
//
// Replaces the reference's facade and host drivers (GDelaunay/GDelaunay.cpp:
// 47-104, GDelHost.cu:136-1630): status codes instead of exit(-1), one context
// per host thread, CUDA streams per context (the pipeline, containment proofs
// beside emission, batch results to host), CUB for the radix sorts and scans
// the reference did with Thrust, and two host reads of a few counters per
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
#include <map>
#include <random>
#include <vector>

#include "g4d_internal.cuh"

using namespace g4d;

namespace {

// Allocation-failure injection for tests: with G4D_FAIL_ALLOC_AFTER=k in the
// environment when a context is created, its workspace allocations after the
// first k fail as if the device were out of memory (G4D_ERR_NOMEM).
struct AllocBudget {
    long long left = -1;  // allocations still allowed; -1: no limit
    bool take() {
        if (left < 0) return true;
        if (left == 0) return false;
        --left;
        return true;
    }
};

struct Buf {
    void* p = nullptr;
    size_t cap = 0;
    AllocBudget* budget = nullptr;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        if (budget && !budget->take()) return cudaErrorMemoryAllocation;
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
    B_WLINSL, B_WLPROM, B_SKEY0, B_SKEY, B_GIDX, B_LOCAL, B_BCKEY0, B_BCKEY, B_SLOTS, B_MMB, B_TC, B_TETS2, B_OVF, B_OVF2, B_KMASK, B_BOUT, B_OCC, B_WLEXACT, B_WLBIG,
    B_MLP_P, B_MLP_G, B_MLP_M1, B_MLP_M2, B_MLP_AUX, B_RING_PAIR, B_RING_X, B_RING_Y, B_RING_LOGIT, B_TILES,
    B_DIAG_X, B_DIAG_Y, B_DIAG_P, B_DIAG_G, B_FIX, B_FACE, B_XYZ32, B_CHECK, B_CHECKOUT, B_CHKP, B_CHKT, B_NUM
};

}  // namespace

struct g4d_ctx {
    g4d_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // batch results to host while the next pass computes
    cudaStream_t side = nullptr;         // proofs beside emission
    cudaEvent_t fork = nullptr, join = nullptr;
    Buf b[B_NUM];
    AllocBudget budget;
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
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};  // the PBA form tuner's own timing events
    std::map<int, int> tuned;  // autotuner: (size bucket, distribution class) -> grid width
    std::map<int, int> pba_form;  // autotuner: grid width -> fastest PBA pass form
    int next_grid = 0;         // tuned width for the next single-cloud call (0: none)
    int block_k = BLOCK_K_DEFAULT;  // voxel-block workset pairs per point (0: none)
    // learned star proposal
    bool has_model = false;
    int adam_step = 0;
    std::vector<float> mlp;    // host copy of the parameters
    int ring_rows = 0;         // candidate rows of the last ring pass
    std::vector<int64_t> batch_offsets;  // tet offsets of the last device batch
    // the tetrahedra in B_TETS belong to the last single-cloud call (not a batch)
    bool has_result = false;
    bool result_mapped = false;  // ... and use input indices (else Morton indices)
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

// A failed call is reported and its (non-sticky) error cleared, so that it
// does not resurface in a later call on the same thread.
#define CK(call)                                                                                     \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) {                                                                     \
            (void)cudaGetLastError();                                                                \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? G4D_ERR_NOMEM : G4D_ERR_CUDA,         \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);         \
        }                                                                                            \
    } while (0)

// Wait for a stream, then surface any kernel launch error since the last
// check: a launch that failed (configuration, resources) is reported only by
// cudaGetLastError, not by the later calls.
#define CK_SYNC(stream)                     \
    do {                                    \
        CK(cudaStreamSynchronize(stream));  \
        CK(cudaGetLastError());             \
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
    D.wlExact = ctx->b[B_WLEXACT].as<int>();
    D.wlBig = ctx->b[B_WLBIG].as<int>();
    D.anyLarge = 0;
    D.keptMask = ctx->b[B_KMASK].as<uint32_t>();
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
    CK_SYNC(ctx->stream);
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
    if (e & ERR_DROWNCAP) return fail(ctx, G4D_ERR_CAPACITY, "drowned list capacity exceeded");
    if (e & ERR_OVFCAP) return fail(ctx, G4D_ERR_CAPACITY, "overflow request list capacity exceeded");
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
    CK(ctx->b[B_WLEXACT].ensure(sizeof(int) * n));
    CK(ctx->b[B_WLBIG].ensure(sizeof(int) * n));
    CK(ctx->b[B_OVF].ensure(sizeof(int2) * (8 * (size_t)n + 1024)));
    CK(ctx->b[B_OVF2].ensure(sizeof(int2) * (8 * (size_t)n + 1024)));
    CK(ctx->b[B_KMASK].ensure(sizeof(uint32_t) * (TSTRIDE / 32) * (size_t)n));
    return G4D_OK;
}

// Entries both drowned lists hold (their byte sizes may pass 2 GiB).
int drown_cap(const g4d_ctx* ctx) {
    return (int)std::min<size_t>(std::min(ctx->b[B_DROWN].cap, ctx->b[B_DROWN2].cap) / sizeof(int2), 0x7fffffff);
}

// Grow both overflow request lists to hold `need` entries, keeping the
// current list's first `keep` entries.
g4d_status grow_ovf(g4d_ctx* ctx, Dev& D, int keep, size_t need) {
    void *a = nullptr, *b = nullptr;
    CK(cudaMalloc(&a, sizeof(int2) * need));
    CK(cudaMalloc(&b, sizeof(int2) * need));
    if (keep > 0) CK(cudaMemcpyAsync(a, D.ovf, sizeof(int2) * keep, cudaMemcpyDeviceToDevice, ctx->stream));
    CK_SYNC(ctx->stream);
    ctx->b[B_OVF].release();
    ctx->b[B_OVF2].release();
    ctx->b[B_OVF].p = a; ctx->b[B_OVF].cap = sizeof(int2) * need;
    ctx->b[B_OVF2].p = b; ctx->b[B_OVF2].cap = sizeof(int2) * need;
    D.ovf = static_cast<int2*>(a);
    D.ovfNext = static_cast<int2*>(b);
    D.ovfCap = (int)std::min<size_t>(need, 0x7fffffff);
    return G4D_OK;
}

// After the worksets are formed: if the overflow request list ran out, grow it
// and ask for the worksets to be formed again (*again).
g4d_status worksets_fit(g4d_ctx* ctx, Dev& D, int attempt, bool* again) {
    Counters h{};
    CK(cudaMemcpyAsync(&h, D.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    *again = false;
    if (h.ovf_next <= D.ovfCap) {
        // every candidate the initial build inserts may drown: room for all
        const size_t need = std::min<size_t>(std::max<size_t>(16 * (size_t)D.n, h.cand_total + 1024), 0x7fffffff);
        if (need > (size_t)D.drownCap) {
            CK(ctx->b[B_DROWN].ensure(sizeof(int2) * need));
            CK(ctx->b[B_DROWN2].ensure(sizeof(int2) * need));
            D.drown = ctx->b[B_DROWN].as<int2>();
            D.drownNext = ctx->b[B_DROWN2].as<int2>();
            D.drownCap = drown_cap(ctx);
        }
        return G4D_OK;
    }
    if (attempt >= 2) return fail(ctx, G4D_ERR_CAPACITY, "overflow request list capacity exceeded");
    g4d_status st = grow_ovf(ctx, D, 0, 2 * (size_t)h.ovf_next + (size_t)D.n);
    if (st) return st;
    CK(cudaMemsetAsync(&D.ctr->ovf_next, 0, sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(&D.ctr->proposed, 0, sizeof(int), ctx->stream));
    CK(cudaMemsetAsync(&D.ctr->block_pairs, 0, sizeof(int), ctx->stream));
    h.err &= ~(unsigned)ERR_OVFCAP;
    CK(cudaMemcpyAsync(&D.ctr->err, &h.err, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
    CK_SYNC(ctx->stream);
    *again = true;
    return G4D_OK;
}

// Initial stars and the splaying loop (worksets already in the buckets).
g4d_status run_splay(g4d_ctx* ctx, Dev& D) {
    Launch L{ctx->stream, &ctx->launches};
    const int n = D.n;
    CK(cudaMemsetAsync(ctx->b[B_ICOUNT].p, 0, sizeof(int) * n, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_INBOX].p, 0xff, sizeof(int) * (size_t)n * INBOX_CAP, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_LIDX].p, 0xff, sizeof(int) * n, ctx->stream));
    Counters h{};
    Counters* dctr = D.ctr;
    auto read = [&]() -> g4d_status {
        CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
        CK_SYNC(ctx->stream);
        return check_err(ctx, h.err);
    };
    // initial stars: filter-only, then the exact kernel for the stars it left,
    // then the large class for stars too big for the small one
    launch_star_build(L, D, nullptr, n, false);
    g4d_status st = read();
    if (st) return st;
    if (h.exact_next) {
        launch_star_build(L, D, D.wlExact, h.exact_next, true);
        if ((st = read())) return st;
    }
    if (h.build_big) {
        st = grow_large(ctx, D, h.large_next, h.large_next + h.build_big);
        if (st) return st;
        D.anyLarge = 1;
        launch_star_build_large(L, D, D.wlBig, h.build_big);
        if ((st = read())) return st;
    }
    cudaEventRecord(ctx->ev[3], ctx->stream);
    CK(cudaMemsetAsync(&dctr->exact_next, 0, 2 * sizeof(int), ctx->stream));  // exact_next, build_big
    const unsigned long long built = h.insertions;  // initial workset insertions
    int emitCount = h.emit_next, drownCount = h.drown_next, ovfCount = h.ovf_next;
    // the lists produced by the build become the current ones
    std::swap(D.wlEmit, D.wlEmitNext);
    std::swap(D.drown, D.drownNext);
    std::swap(D.ovf, D.ovfNext);
    CK(cudaMemsetAsync(&dctr->emit_next, 0, 2 * sizeof(int), ctx->stream));  // emit_next, drown_next
    CK(cudaMemsetAsync(&dctr->ovf_next, 0, sizeof(int), ctx->stream));
    int loops = 0;
    const int max_loops = ctx->cfg.max_splay_loops > 0 ? ctx->cfg.max_splay_loops : 4000;
    for (;; ++loops) {
        if (loops >= max_loops) return fail(ctx, G4D_ERR_TIMEOUT, "splaying did not converge in %d loops", max_loops);
        // emission phase; it only adds (deduplicated) inbox requests, so when the
        // overflow list ran out it is grown and the phase repeated
        for (int attempt = 0;; ++attempt) {
            // proofs on the side stream next to emission: both only add
            // deduplicated inbox requests
            if (drownCount) {
                CK(cudaEventRecord(ctx->fork, ctx->stream));
                CK(cudaStreamWaitEvent(ctx->side, ctx->fork, 0));
                Launch Ls{ctx->side, &ctx->launches};
                launch_proof(Ls, D, drownCount);
                CK(cudaEventRecord(ctx->join, ctx->side));
            }
            if (ovfCount) launch_requeue(L, D, ovfCount);
            if (emitCount) launch_emit(L, D, emitCount);
            if (drownCount) CK(cudaStreamWaitEvent(ctx->stream, ctx->join, 0));
            CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
            CK_SYNC(ctx->stream);
            if (!(h.err & ERR_OVFCAP) || attempt >= 3) break;
            st = grow_ovf(ctx, D, ovfCount, 2 * (size_t)h.ovf_next + (size_t)D.n);
            if (st) return st;
            CK(cudaMemsetAsync(&dctr->ovf_next, 0, sizeof(int), ctx->stream));
            const unsigned clear = ~(unsigned)ERR_OVFCAP;
            h.err &= clear;
            CK(cudaMemcpyAsync(&dctr->err, &h.err, sizeof(unsigned), cudaMemcpyHostToDevice, ctx->stream));
        }
        st = check_err(ctx, h.err);
        if (st) return st;
        if (h.ins_count == 0 && h.ins_count_large == 0) break;
        if (loops == 0 && D.anyLarge && h.ins_count) {
            // requests queued during the build may target stars built large
            launch_reroute(L, D, h.ins_count);
            if ((st = read())) return st;
        }
        ovfCount = h.ovf_next;  // requests that found a full inbox this round
        if (h.ins_count) launch_star_insert(L, D, D.wlIns, h.ins_count, false);
        if (h.ins_count_large) launch_star_insert_large(L, D, D.wlInsL, std::min(h.ins_count_large, D.largeCap));
        if ((st = read())) return st;
        if (h.exact_next) {  // stars the filter-only kernel could not decide
            launch_star_insert(L, D, D.wlExact, h.exact_next, true);
            if ((st = read())) return st;
        }
        if (h.promote_count) {
            // stars that outgrew the small class: move them, then replay their round
            st = grow_large(ctx, D, h.large_next, h.large_next + h.promote_count);
            if (st) return st;
            launch_promote(L, D, h.promote_count);
            D.anyLarge = 1;
            launch_star_insert_large(L, D, D.wlPromote, h.promote_count);
            CK(cudaMemcpyAsync(&h, dctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
            CK_SYNC(ctx->stream);
            st = check_err(ctx, h.err);
            if (st) return st;
        }
        emitCount = h.emit_next;
        drownCount = h.drown_next;
        std::swap(D.wlEmit, D.wlEmitNext);
        std::swap(D.drown, D.drownNext);
        std::swap(D.ovf, D.ovfNext);
        // ins_count, emit_next, drown_next, ins_count_large, promote_count, exact_next, build_big
        CK(cudaMemsetAsync(dctr, 0, 7 * sizeof(int), ctx->stream));
        CK(cudaMemsetAsync(&dctr->ovf_next, 0, sizeof(int), ctx->stream));
    }
    cudaEventRecord(ctx->ev[4], ctx->stream);
    ctx->stats.loops = loops;
    ctx->stats.star_insertions = (long long)built;
    ctx->stats.splay_insertions = (long long)(h.insertions - built);
    ctx->stats.proofs = (long long)h.proofs_total;
    ctx->stats.exact_predicates = (long long)h.exact;
    ctx->stats.proposed = h.proposed;
    ctx->stats.block_pairs = h.block_pairs;
    ctx->large_used = h.large_next;

    if (ctx->cfg.do_check) {
        unsigned long long* bad = ctx->b[B_BAD].as<unsigned long long>();
        CK(cudaMemsetAsync(bad, 0, 8, ctx->stream));
        launch_check(L, D, bad);
        unsigned long long hb = 0;
        CK(cudaMemcpyAsync(&hb, bad, 8, cudaMemcpyDeviceToHost, ctx->stream));
        CK_SYNC(ctx->stream);
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
    CK_SYNC(ctx->stream);
    CK(ctx->b[B_TETS].ensure(sizeof(g4d_tet) * (size_t)std::max(ntet, 1)));
    // at most one queued link per (tetrahedron, vertex slot)
    CK(ctx->b[B_FIX].ensure(sizeof(int2) * 4 * (size_t)std::max(ntet, 1)));
    CK(ctx->b[B_FACE].ensure(sizeof(int4) * (size_t)std::max(ntet, 1)));
    launch_tet_write(L, D, base, ctx->b[B_TETS].as<g4d_tet>(), sorted_to_input, ctx->b[B_FACE].as<int4>(), ntet,
                     ctx->b[B_FIX].as<int2>());
    launch_tet_fix(L, D, ctx->b[B_TETS].as<g4d_tet>(), ctx->b[B_FIX].as<int2>());
    cudaEventRecord(ctx->ev[5], ctx->stream);
    Counters h{};
    CK(cudaMemcpyAsync(&h, D.ctr, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    g4d_status st = check_err(ctx, h.err);
    if (st) return st;
    ctx->ntet = ntet;
    ctx->stats.tets = ntet;
    return G4D_OK;
}

// ---------------------------------------------------------------------------
// Learned star proposal (host side)
// ---------------------------------------------------------------------------

double dkey_inv_host(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    double d;
    memcpy(&d, &b, sizeof(d));
    return d;
}

struct MlpAux {
    float loss;
    unsigned err;
    int rows;
};

// candidate rows of the 5x5x5 Voronoi block around every point, with labels
// from the final stars when `labels`
g4d_status run_ring(g4d_ctx* ctx, const Dev& D, bool labels) {
    Launch L{ctx->stream, &ctx->launches};
    const int n = D.n, G = D.G;
    const size_t cap = 24 * (size_t)n + 1024;
    CK(ctx->b[B_MLP_AUX].ensure(sizeof(MlpAux)));
    CK(ctx->b[B_RING_PAIR].ensure(sizeof(int2) * cap));
    CK(ctx->b[B_RING_X].ensure(sizeof(uint16_t) * 16 * cap));
    CK(ctx->b[B_RING_LOGIT].ensure(sizeof(float) * cap));
    if (labels) CK(ctx->b[B_RING_Y].ensure(sizeof(float) * cap));
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    CK(cudaMemsetAsync(aux, 0, sizeof(MlpAux), ctx->stream));
    // grid units per coordinate unit, as in the scaling of the points
    unsigned long long mm[2] = {0, 0};
    CK(cudaMemcpyAsync(mm, ctx->b[B_MM].p, sizeof(mm), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    const double range = dkey_inv_host(mm[1]) - dkey_inv_host(mm[0]);
    Ring R;
    R.grid = ctx->b[B_GA].as<uint32_t>();
    // grid B holds the voxel -> leader map from the pair scan of this cloud
    R.cols = Cols<uint32_t>{D.ckey, D.cid, D.colStart, D.colEnd, G, ctx->b[B_GB].as<int>()};
    R.scale = (mm[1] && range > 0) ? (double)(G - 3) / range : 1.0;
    R.cap = (int)cap;
    R.rows = &aux->rows;
    R.pair = ctx->b[B_RING_PAIR].as<int2>();
    R.x = ctx->b[B_RING_X].as<uint16_t>();
    R.y = labels ? ctx->b[B_RING_Y].as<float>() : nullptr;
    launch_ring(L, D, R);
    if (labels) launch_ring_labels(L, D, R.pair, R.rows, R.cap, R.y);
    MlpAux h{};
    CK(cudaMemcpyAsync(&h, aux, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    ctx->ring_rows = std::min(h.rows, R.cap);
    return G4D_OK;
}

// score the candidates and add the accepted ones to the initial worksets
g4d_status run_proposal(g4d_ctx* ctx, const Dev& D) {
    if (!ctx->cfg.proposal || !ctx->has_model) return G4D_OK;
    Launch L{ctx->stream, &ctx->launches};
    g4d_status st = run_ring(ctx, D, false);
    if (st) return st;
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    if (ctx->ring_rows > 0)
        launch_mlp_infer(L, ctx->b[B_MLP_P].as<float>(), ctx->b[B_RING_X].as<uint16_t>(), ctx->ring_rows,
                         ctx->b[B_RING_LOGIT].as<float>(), &aux->err);
    launch_prop_merge(L, D, ctx->b[B_RING_PAIR].as<int2>(), ctx->b[B_RING_LOGIT].as<float>(), &aux->rows,
                      ctx->ring_rows, 0.0f);
    return G4D_OK;
}

// The y and x passes in the form tuned for this grid width: the first grid
// of a width on a context times every form (the z pass rebuilds the input
// before each, since the line form uses it as scratch) and keeps the fastest;
// later grids of that width use it. All forms give exact distances.
// G4D_PBA_FORM=<0..2> in the environment at context creation fixes the form.
int pba_form_for(g4d_ctx* ctx, const Dev& D, uint32_t* gA, uint32_t* gB) {
    const int G = D.G;
    if (ctx->pba_form.count(G)) return ctx->pba_form[G];
    Launch L{ctx->stream, &ctx->launches};
    cudaEvent_t a = ctx->tune_ev[0], b = ctx->tune_ev[1];
    int best = pba_default_form(G);
    float best_ms = 1e30f;
    for (int f = 0; f < PBA_FORMS; ++f) {
        if (!pba_form_ok(f, G)) continue;
        float ms = 0.f;
        for (int rep = 0; rep < 2; ++rep) {  // the first run of a form also loads its kernels
            launch_pba_z(L, D, gA);
            cudaEventRecord(a, ctx->stream);
            launch_pba_y(L, G, gA, gB, f);
            launch_pba_x(L, G, gB, gA, f);
            cudaEventRecord(b, ctx->stream);
            if (cudaEventSynchronize(b) != cudaSuccess) return best;
            cudaEventElapsedTime(&ms, a, b);
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = f;
        }
    }
    ctx->pba_form[G] = best;
    return best;
}

// Stages 2-5: digital Voronoi, stars, splaying, extraction.
g4d_status run_compute(g4d_ctx* ctx, bool map_to_input) {
    ctx->has_result = false;
    ctx->result_mapped = map_to_input;
    Launch L{ctx->stream, &ctx->launches};
    const int n = ctx->n, G = ctx->G;
    const size_t G3 = (size_t)G * G * G;
    CK(ctx->b[B_GA].ensure(sizeof(uint32_t) * G3));
    CK(ctx->b[B_GB].ensure(sizeof(uint32_t) * G3));
    g4d_status st = alloc_stars(ctx, n);
    if (st) return st;
    Dev D = make_dev(ctx);
    // equalise the two drowned buffers' capacity
    D.drownCap = drown_cap(ctx);

    uint32_t* gA = ctx->b[B_GA].as<uint32_t>();
    uint32_t* gB = ctx->b[B_GB].as<uint32_t>();
    const int form = pba_form_for(ctx, D, gA, gB);
    ctx->stats.pba_form = form;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    // digital Voronoi diagram
    launch_pba_z(L, D, gA);
    launch_pba_y(L, G, gA, gB, form);
    launch_pba_x(L, G, gB, gA, form);
    cudaEventRecord(ctx->ev[2], ctx->stream);
    // worksets (repeated with a longer overflow list if theirs ran out)
    for (int attempt = 0;; ++attempt) {
        CK(cudaMemsetAsync(ctx->b[B_BCOUNT].p, 0, sizeof(int) * n, ctx->stream));
        // grid B is free after the x pass: it becomes the voxel -> leader map
        launch_site_map(L, D, reinterpret_cast<int*>(gB));
        launch_pairs(L, D, gA, reinterpret_cast<int*>(gB));
        launch_missing(L, D);
        if (ctx->block_k > 0) launch_block_pairs(L, D, gA, reinterpret_cast<const int*>(gB), ctx->block_k);
        st = run_proposal(ctx, D);
        if (st) return st;
        launch_workset_total(L, D);
        bool again = false;
        st = worksets_fit(ctx, D, attempt, &again);
        if (st) return st;
        if (ctx->cfg.proposal && ctx->has_model) {  // the stream is idle after worksets_fit
            MlpAux h{};
            CK(cudaMemcpy(&h, ctx->b[B_MLP_AUX].p, sizeof(h), cudaMemcpyDeviceToHost));
            if (h.err)
                return fail(ctx, G4D_ERR_TIMEOUT, "tensor-core inference kernel timed out waiting (0x%x)", h.err);
        }
        if (!again) break;
    }
    st = run_splay(ctx, D);
    if (st) return st;
    st = run_extract(ctx, D, map_to_input ? ctx->b[B_ORDER].as<int>() : nullptr);
    ctx->has_result = st == G4D_OK;
    return st;
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
    int G = ctx->cfg.grid_size > 0 ? ctx->cfg.grid_size : (ctx->next_grid > 0 ? ctx->next_grid : auto_grid(n));
    ctx->next_grid = 0;
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

// Device-side batch output: tetrahedra of all waves back to back (cloud order
// within each wave, waves in cloud order), grown by copying when needed.
g4d_status reserve_out(g4d_ctx* ctx, size_t used, size_t need) {
    Buf& o = ctx->b[B_BOUT];
    if (need * sizeof(g4d_tet) <= o.cap && o.p) return G4D_OK;
    const size_t want = std::max(need, used + used / 2) * sizeof(g4d_tet) + 256;
    void* np = nullptr;
    CK(cudaMalloc(&np, want));
    if (used && o.p) CK(cudaMemcpyAsync(np, o.p, used * sizeof(g4d_tet), cudaMemcpyDeviceToDevice, ctx->stream));
    CK_SYNC(ctx->stream);
    if (ctx->copy_stream) CK_SYNC(ctx->copy_stream);  // host copies out of the old buffer
    o.release();
    o.p = np;
    o.cap = want;
    return G4D_OK;
}

// One wave over the clouds cl[0..ns) (grid widths Gc[cloud]): their tetrahedra,
// in list order with cloud-local ids, are written to the batch output from
// element `at` on; tet_counts[cloud] receives each cloud's count.
g4d_status run_wave(g4d_ctx* ctx, const double* d_xyz, const int64_t* offs, const int* cl, int ns, const int* Gc,
                    size_t at, int64_t* tet_counts, size_t* wave_tets) {
    Launch L{ctx->stream, &ctx->launches};
    // slots: clouds ordered by grid width (stable)
    std::vector<int> slot_cloud(cl, cl + ns);
    std::vector<int> list_pos(ns);
    std::stable_sort(slot_cloud.begin(), slot_cloud.end(), [&](int a, int b) { return Gc[a] < Gc[b]; });
    std::vector<long long> slotIn(ns), slotCol(ns), slotVox(ns);
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
        slotVox[k] = voxels;
        cols += (long long)G * G;
        voxels += (long long)G * G * G;
    }
    const int n = slotW[ns];
    ctx->n = n;
    // device copies of the slot tables: slotIn, slotCol, dst, slotVox (int64), slotW, slotG, tc (int32)
    const size_t i64b = sizeof(long long) * ns, i32b = sizeof(int) * (ns + 1);
    CK(ctx->b[B_SLOTS].ensure(4 * i64b + 3 * i32b + 64));
    char* sb = ctx->b[B_SLOTS].as<char>();
    long long* d_slotIn = reinterpret_cast<long long*>(sb);
    long long* d_slotCol = reinterpret_cast<long long*>(sb + i64b);
    long long* d_dst = reinterpret_cast<long long*>(sb + 2 * i64b);
    long long* d_slotVox = reinterpret_cast<long long*>(sb + 3 * i64b);
    int* d_slotW = reinterpret_cast<int*>(sb + 4 * i64b);
    int* d_slotG = reinterpret_cast<int*>(sb + 4 * i64b + i32b);
    int* d_tc = reinterpret_cast<int*>(sb + 4 * i64b + 2 * i32b);
    CK(cudaMemcpyAsync(d_slotIn, slotIn.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_slotCol, slotCol.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(d_slotVox, slotVox.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
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
    D.drownCap = drown_cap(ctx);
    D.G = 0;
    D.cloudOff = d_slotW;
    D.nclouds = ns;
    cudaEventRecord(ctx->ev[1], ctx->stream);
    uint32_t* gA = ctx->b[B_GA].as<uint32_t>();
    uint32_t* gB = ctx->b[B_GB].as<uint32_t>();
    for (const Stack& S : stacks) {
        launch_pba_z_stack(L, S.G, S.K, ckey, cs + S.col, ce + S.col, gA + S.vox);
        const auto tf = ctx->pba_form.find(S.G);  // a width tuned on single clouds, else the default
        const int form = tf != ctx->pba_form.end() ? tf->second : -1;
        launch_pba_y_stack(L, S.G, S.K, gA + S.vox, gB + S.vox, form);
        launch_pba_x_stack(L, S.G, S.K, gB + S.vox, gA + S.vox, form);
    }
    cudaEventRecord(ctx->ev[2], ctx->stream);
    for (int attempt = 0;; ++attempt) {
        CK(cudaMemsetAsync(ctx->b[B_BCOUNT].p, 0, sizeof(int) * n, ctx->stream));
        // the grids B are free after the x passes: they become the voxel -> leader maps
        int* map = reinterpret_cast<int*>(gB);
        launch_b_site_map(L, ctx->b[B_VOX].as<uint32_t>(), skey, d_slotG, d_slotVox, n, map);
        for (const Stack& S : stacks)
            launch_pairs_stack(L, D, gA + S.vox, map + S.vox, S.G, S.K, ckey, ctx->b[B_CID].as<int>(), cs + S.col,
                               ce + S.col);
        launch_missing_u64(L, D, skey);
        if (ctx->block_k > 0)
            launch_block_pairs_batch(L, D, gA, map, skey, d_slotG, d_slotVox, ctx->block_k);
        launch_workset_total(L, D);
        bool again = false;
        st = worksets_fit(ctx, D, attempt, &again);
        if (st) return st;
        if (!again) break;
    }
    st = run_splay(ctx, D);
    if (st) return st;
    st = run_extract(ctx, D, nullptr);
    if (st) return st;
    // per-cloud counts and output offsets in list order
    const int ntet = ctx->ntet;
    launch_b_slot_tets(L, ctx->b[B_BASE].as<int>(), d_slotW, ns, d_tc);
    std::vector<int> tc(ns);
    CK(cudaMemcpyAsync(tc.data(), d_tc, sizeof(int) * ns, cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    std::vector<int> pos_of(ns);  // slot -> position of its cloud in the list
    {
        std::vector<std::pair<int, int>> lp(ns);
        for (int i = 0; i < ns; ++i) lp[i] = {cl[i], i};
        std::sort(lp.begin(), lp.end());
        for (int k = 0; k < ns; ++k) {
            const auto it = std::lower_bound(lp.begin(), lp.end(), std::make_pair(slot_cloud[k], -1));
            pos_of[k] = it->second;
        }
    }
    std::vector<long long> cnt_pos(ns), off_pos(ns + 1, 0), dst(ns);
    for (int k = 0; k < ns; ++k) cnt_pos[pos_of[k]] = tc[k];
    for (int i = 0; i < ns; ++i) off_pos[i + 1] = off_pos[i] + cnt_pos[i];
    for (int k = 0; k < ns; ++k) dst[k] = (long long)at + off_pos[pos_of[k]];
    for (int i = 0; i < ns; ++i) tet_counts[cl[i]] = cnt_pos[i];
    CK(cudaMemcpyAsync(d_dst, dst.data(), i64b, cudaMemcpyHostToDevice, ctx->stream));
    st = reserve_out(ctx, at, at + (size_t)ntet);
    if (st) return st;
    launch_b_localize(L, ctx->b[B_TETS].as<g4d_tet>(), ntet, skey, ctx->b[B_LOCAL].as<int>(),
                      ctx->b[B_BASE].as<int>(), d_slotW, d_dst, ctx->b[B_BOUT].as<g4d_tet>());
    cudaEventRecord(ctx->ev[6], ctx->stream);
    CK(cudaEventSynchronize(ctx->ev[6]));  // stage times are read right after
    *wave_tets = (size_t)ntet;
    return G4D_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: grid width per cloud. The reference fixes G by flag; its default
// density is about 134 voxels per point. Sparse grids make the digital Voronoi
// passes expensive (their cost follows the voxel count), dense ones leave more
// points sharing voxels and more work for splaying. For every (size bucket,
// distribution class) the tuner times waves of up to kTuneClouds sample clouds
// at the density rule's width and at one half and one quarter of it, and keeps
// the fastest; later clouds of that key reuse the choice (per context).
// ---------------------------------------------------------------------------

constexpr int kTuneClouds = 16;

// Distribution class: occupancy of an 8^3 histogram of a strided sample of up
// to 4096 points against what a uniform sample of that size fills.
// 0 = spread out (uniform-like), 1 = intermediate, 2 = concentrated.
int class_of(int filled, int64_t n) {
    const double m = (double)std::min<int64_t>(n, 4096);
    const double expect = 512.0 * (1.0 - std::exp(-m / 512.0));
    const double r = filled / expect;
    return r > 0.6 ? 0 : (r > 0.25 ? 1 : 2);
}

// host restatement of k_b_occupancy (same sample, same arithmetic order)
int occupancy(const double* xyz, int64_t n) {
    const int64_t m = std::min<int64_t>(n, 4096);
    const int64_t step = std::max<int64_t>(1, n / m);
    double lo = xyz[0], hi = xyz[0];
    for (int64_t i = 0; i < m; ++i)
        for (int c = 0; c < 3; ++c) {
            const double v = xyz[3 * (i * step) + c];
            lo = std::min(lo, v);
            hi = std::max(hi, v);
        }
    const double span = hi > lo ? hi - lo : 1.0;
    uint32_t bits[16] = {0};
    for (int64_t i = 0; i < m; ++i) {
        int q[3];
        for (int c = 0; c < 3; ++c) {
            volatile double d = xyz[3 * (i * step) + c] - lo;  // no contraction: the device rounds each step
            volatile double e = 8.0 * d;
            q[c] = std::min(7, (int)(e / span));
        }
        const int cell = (q[2] * 8 + q[1]) * 8 + q[0];
        bits[cell >> 5] |= 1u << (cell & 31);
    }
    int f = 0;
    for (int w = 0; w < 16; ++w) f += __builtin_popcount(bits[w]);
    return f;
}

int tune_key(int64_t n, int dclass) { return bits_for((unsigned long long)n) * 4 + dclass; }

// grid widths for every cloud; tunes the keys not yet in the context's table
g4d_status pick_batch_grids(g4d_ctx* ctx, const double* d_xyz, const int64_t* offs, int nclouds,
                            std::vector<int>& Gc) {
    Gc.assign(std::max(nclouds, 1), 0);
    if (ctx->cfg.grid_size > 0 || ctx->cfg.grid_size == 0) {
        for (int c = 0; c < nclouds; ++c) {
            const int64_t n = offs[c + 1] - offs[c];
            Gc[c] = ctx->cfg.grid_size > 0 ? ctx->cfg.grid_size : auto_grid((int)n);
        }
        return G4D_OK;
    }
    // distribution classes from the device copy of the points
    CK(ctx->b[B_OCC].ensure(sizeof(long long) * (nclouds + 1) + sizeof(int) * nclouds + 64));
    long long* d_offs = ctx->b[B_OCC].as<long long>();
    int* d_occ = reinterpret_cast<int*>(d_offs + nclouds + 1);
    CK(cudaMemcpyAsync(d_offs, offs, sizeof(long long) * (nclouds + 1), cudaMemcpyHostToDevice, ctx->stream));
    Launch L{ctx->stream, &ctx->launches};
    launch_b_occupancy(L, d_xyz, d_offs, nclouds, d_occ);
    std::vector<int> occ(nclouds);
    CK(cudaMemcpyAsync(occ.data(), d_occ, sizeof(int) * nclouds, cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    std::vector<int> key(nclouds);
    std::map<int, std::vector<int>> pending;
    for (int c = 0; c < nclouds; ++c) {
        const int64_t n = offs[c + 1] - offs[c];
        key[c] = tune_key(n, class_of(occ[c], n));
        if (!ctx->tuned.count(key[c])) {
            auto& v = pending[key[c]];
            if ((int)v.size() < kTuneClouds) v.push_back(c);
        }
    }
    for (auto& kv : pending) {
        const std::vector<int>& sample = kv.second;
        long long pts = 0;
        for (int c : sample) pts += offs[c + 1] - offs[c];
        const int g0 = auto_grid((int)std::max<long long>(5, pts / (long long)sample.size()));
        int best = g0;
        float best_ms = 1e30f;
        std::vector<int> Gs(nclouds, 0);
        std::vector<int64_t> cnt(nclouds, 0);
        const double avg = (double)pts / (double)sample.size();
        for (int pass = 0; pass < 4; ++pass) {
            const int g = pass == 0 ? g0 : std::max(32, g0 >> (pass - 1));  // first pass warms up
            if (pass > 1 && g == std::max(32, g0 >> (pass - 2))) break;
            if (pass > 1 && (double)g * g * g < 8.0 * avg) break;  // under 8 voxels per point
            for (int c : sample) Gs[c] = g;
            size_t wt = 0;
            g4d_status st = run_wave(ctx, d_xyz, offs, sample.data(), (int)sample.size(), Gs.data(), 0, cnt.data(), &wt);
            if (st && pass <= 1) return st;
            if (st) break;  // a denser candidate that fails is not taken
            const float ms = ms_between(ctx->ev[0], ctx->ev[6]);
            if (ctx->cfg.log_verbose)
                fprintf(stderr, "autotune: %zu clouds, %.0f points avg, class %d: G=%d %.3f ms%s\n", sample.size(),
                        avg, kv.first & 3, g, ms, pass == 0 ? " (warm-up)" : "");
            if (pass > 0 && ms < best_ms) { best_ms = ms; best = g; }
        }
        ctx->tuned[kv.first] = best;
    }
    for (int c = 0; c < nclouds; ++c) Gc[c] = ctx->tuned[key[c]];
    return G4D_OK;
}

// All waves of a batch whose points are on the device; the tetrahedra end in
// B_BOUT (cloud order) and counts[c] per cloud.
// Optional host destination of a batch: each pass's tetrahedra are copied on
// the copy stream while the next pass computes (as long as they fit in cap).
struct HostSink {
    g4d_tet* out;
    size_t cap;
    bool fits;
};

g4d_status run_batch(g4d_ctx* ctx, const double* d_xyz, const int64_t* offs, int nclouds,
                     std::vector<int64_t>& counts, size_t* total, g4d_stats* acc, HostSink* sink = nullptr) {
    ctx->has_result = false;
    for (int c = 0; c < nclouds; ++c) {
        const int64_t n = offs[c + 1] - offs[c];
        if (n < 5 || n >= (1 << 30))
            return fail(ctx, G4D_ERR_ARG, "cloud %d has %lld points (need 5 or more)", c, (long long)n);
    }
    if (nclouds && offs[0] != 0) return fail(ctx, G4D_ERR_ARG, "cloud_offsets[0] must be 0");
    std::vector<int> Gc;
    g4d_status st = pick_batch_grids(ctx, d_xyz, offs, nclouds, Gc);
    if (st) return st;
    for (int c = 0; c < nclouds; ++c)
        if (Gc[c] < 32 || Gc[c] > 1024 || (Gc[c] & (Gc[c] - 1)))
            return fail(ctx, G4D_ERR_ARG, "grid size must be a power of two in [32, 1024] (got %d)", Gc[c]);
    ctx->launches = 0;
    counts.assign(nclouds, 0);
    // reserve output for about 7 tetrahedra per point (grown if exceeded)
    const int64_t npts = nclouds ? offs[nclouds] : 0;
    st = reserve_out(ctx, 0, (size_t)(7.2 * (double)npts) + 1024);
    if (st) return st;
    size_t at = 0;
    int large = 0;
    std::vector<int> list;
    // G4D_WAVE_POINTS lowers the points per pass (tests use it to get many passes)
    long long wave_points = kWavePoints;
    if (const char* e = getenv("G4D_WAVE_POINTS")) {
        const long long v = atoll(e);
        if (v > 0 && v < kWavePoints) wave_points = v;
    }
    for (int c0 = 0; c0 < nclouds;) {
        int c1 = c0;
        long long pts = 0, vox = 0;
        while (c1 < nclouds) {
            const long long n = offs[c1 + 1] - offs[c1];
            const long long v = (long long)Gc[c1] * Gc[c1] * Gc[c1];
            if (c1 > c0 && (pts + n > wave_points || vox + v > kWaveVoxels)) break;
            pts += n;
            vox += v;
            ++c1;
        }
        list.resize(c1 - c0);
        for (int c = c0; c < c1; ++c) list[c - c0] = c;
        size_t wt = 0;
        st = run_wave(ctx, d_xyz, offs, list.data(), c1 - c0, Gc.data(), at, counts.data(), &wt);
        if (st) return st;
        if (sink && sink->fits) {
            if (at + wt <= sink->cap) {
                CK(cudaEventRecord(ctx->ev[7], ctx->stream));
                CK(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev[7], 0));
                CK(cudaMemcpyAsync(sink->out + at, ctx->b[B_BOUT].as<g4d_tet>() + at, sizeof(g4d_tet) * wt,
                                   cudaMemcpyDeviceToHost, ctx->copy_stream));
            } else {
                sink->fits = false;
            }
        }
        at += wt;
        acc->t_init_ms += ms_between(ctx->ev[0], ctx->ev[1]);
        acc->t_pba_ms += ms_between(ctx->ev[1], ctx->ev[2]);
        acc->t_star_ms += ms_between(ctx->ev[2], ctx->ev[3]);
        acc->t_splay_ms += ms_between(ctx->ev[3], ctx->ev[4]);
        acc->t_out_ms += ms_between(ctx->ev[4], ctx->ev[6]);
        acc->star_insertions += ctx->stats.star_insertions;
        acc->splay_insertions += ctx->stats.splay_insertions;
        acc->proofs += ctx->stats.proofs;
        acc->exact_predicates += ctx->stats.exact_predicates;
        acc->loops = std::max(acc->loops, ctx->stats.loops);
        large += ctx->large_used;
        c0 = c1;
    }
    *total = at;
    acc->tets = (int)std::min<size_t>(at, 0x7fffffff);
    acc->gpu_launches = ctx->launches;
    acc->large_stars = large;
    acc->grid_size = nclouds ? *std::max_element(Gc.begin(), Gc.begin() + nclouds) : 0;
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
    if (cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->join, cudaEventDisableTiming) != cudaSuccess) {
        if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->fork) cudaEventDestroy(ctx->fork);
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        return G4D_ERR_CUDA;
    }
    for (auto& e : ctx->ev) cudaEventCreate(&e);
    for (auto& e : ctx->tune_ev) cudaEventCreate(&e);
    if (const char* f = std::getenv("G4D_PBA_FORM")) {
        const int form = std::atoi(f);
        for (int G = 32; G <= 1024; G *= 2)
            if (pba_form_ok(form, G)) ctx->pba_form[G] = form;
    }
    if (const char* f = std::getenv("G4D_BLOCK_K")) ctx->block_k = std::max(0, std::min(std::atoi(f), 64));
    if (const char* f = std::getenv("G4D_FAIL_ALLOC_AFTER")) {
        ctx->budget.left = std::atoll(f);
        for (auto& b : ctx->b) b.budget = &ctx->budget;
    }
    *out = ctx;
    return G4D_OK;
}

void g4d_destroy(g4d_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->side) cudaStreamSynchronize(ctx->side);
    for (auto& b : ctx->b) b.release();
    for (auto& e : ctx->ev) cudaEventDestroy(e);
    for (auto& e : ctx->tune_ev)
        if (e) cudaEventDestroy(e);
    if (ctx->fork) cudaEventDestroy(ctx->fork);
    if (ctx->join) cudaEventDestroy(ctx->join);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->side) cudaStreamDestroy(ctx->side);
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
    if (ctx->cfg.grid_size < 0 && !ctx->tuned.empty()) {
        // autotuned mode: the distribution class from the device copy of the points
        const long long offs[2] = {0, n};
        CK(ctx->b[B_OCC].ensure(sizeof(long long) * 2 + sizeof(int) + 64));
        long long* d_offs = ctx->b[B_OCC].as<long long>();
        int* d_occ = reinterpret_cast<int*>(d_offs + 2);
        CK(cudaMemcpyAsync(d_offs, offs, sizeof(offs), cudaMemcpyHostToDevice, ctx->stream));
        Launch L{ctx->stream, &ctx->launches};
        launch_b_occupancy(L, d_xyz, d_offs, 1, d_occ);
        int occ = 0;
        CK(cudaMemcpyAsync(&occ, d_occ, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CK_SYNC(ctx->stream);
        const auto it = ctx->tuned.find(tune_key(n, class_of(occ, n)));
        if (it != ctx->tuned.end()) ctx->next_grid = it->second;
    }
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
    if (ctx->cfg.grid_size < 0) {
        // autotuned mode: reuse the width tuned for this size and distribution
        const auto it = ctx->tuned.find(tune_key(n, class_of(occupancy(xyz, n), n)));
        if (it != ctx->tuned.end()) ctx->next_grid = it->second;
    }
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
    CK_SYNC(ctx->stream);
    if (stats) *stats = ctx->stats;
    return G4D_OK;
}

g4d_status g4d_triangulate_to_f32(g4d_ctx* ctx, const float* xyz, int n, g4d_tet* out, int cap, int* ntet,
                                  int* sorted_to_input, g4d_stats* stats) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!xyz || !ntet) return fail(ctx, G4D_ERR_ARG, "null argument");
    cudaSetDevice(ctx->device);
    Launch L{ctx->stream, &ctx->launches};
    // float points (the reference's default RealType) are widened on the
    // device; the triangulation is that of the same values in double
    CK(ctx->b[B_XYZ32].ensure(sizeof(float) * 3 * (size_t)n));
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)n));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ32].p, xyz, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    launch_f32_to_f64(L, ctx->b[B_XYZ32].as<float>(), 3 * (size_t)n, ctx->b[B_XYZ].as<double>());
    if (ctx->cfg.grid_size < 0) {
        // autotuned mode: the tuned width for this size and distribution
        std::vector<double> h(3 * (size_t)n);
        for (size_t i = 0; i < h.size(); ++i) h[i] = xyz[i];
        const auto it = ctx->tuned.find(tune_key(n, class_of(occupancy(h.data(), n), n)));
        if (it != ctx->tuned.end()) ctx->next_grid = it->second;
    }
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
    CK_SYNC(ctx->stream);
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
    CK_SYNC(ctx->stream);
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
    CK_SYNC(ctx->stream);
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
    CK_SYNC(ctx->stream);
    return G4D_OK;
}

g4d_status g4d_get_tetra(g4d_ctx* ctx, const g4d_tet** tets, int* ntet) {
    if (!ctx || !tets || !ntet) return G4D_ERR_ARG;
    *tets = ctx->host_tets.data();
    *ntet = (int)ctx->host_tets.size();
    return G4D_OK;
}

g4d_status g4d_get_stats(const g4d_ctx* ctx, g4d_stats* stats) {
    if (!ctx || !stats) return G4D_ERR_ARG;
    *stats = ctx->stats;
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
    const int64_t total = nclouds ? cloud_offsets[nclouds] : 0;
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)std::max<int64_t>(total, 1)));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)total, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int64_t> counts;
    size_t ntet = 0;
    g4d_stats acc{};
    g4d_status st = run_batch(ctx, ctx->b[B_XYZ].as<double>(), cloud_offsets, nclouds, counts, &ntet, &acc);
    if (st) return st;
    g4d_tet* out = (g4d_tet*)malloc(sizeof(g4d_tet) * std::max<size_t>(ntet, 1));
    int64_t* offs = (int64_t*)malloc(sizeof(int64_t) * (nclouds + 1));
    if (!out || !offs) {
        free(out);
        free(offs);
        return fail(ctx, G4D_ERR_NOMEM, "host allocation of %zu tetrahedra failed", ntet);
    }
    CK(cudaMemcpyAsync(out, ctx->b[B_BOUT].p, sizeof(g4d_tet) * ntet, cudaMemcpyDeviceToHost, ctx->stream));
    offs[0] = 0;
    for (int c = 0; c < nclouds; ++c) offs[c + 1] = offs[c] + counts[c];
    CK_SYNC(ctx->stream);
    *tets = out;
    *tet_offsets = offs;
    acc.t_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->stats = acc;
    if (stats) *stats = acc;
    return G4D_OK;
}

g4d_status g4d_triangulate_batch_to(g4d_ctx* ctx, const double* xyz, const int64_t* cloud_offsets, int nclouds,
                                    g4d_tet* out, int64_t cap, int64_t* tet_offsets, int64_t* ntet,
                                    g4d_stats* stats) {
    if (!ctx) return G4D_ERR_ARG;
    if (!xyz || !cloud_offsets || nclouds < 0 || !out || cap < 0 || !tet_offsets || !ntet)
        return fail(ctx, G4D_ERR_ARG, "null argument");
    *ntet = 0;
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    const int64_t total = nclouds ? cloud_offsets[nclouds] : 0;
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)std::max<int64_t>(total, 1)));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)total, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<int64_t> counts;
    size_t nt = 0;
    g4d_stats acc{};
    HostSink sink{out, (size_t)cap, true};
    g4d_status st = run_batch(ctx, ctx->b[B_XYZ].as<double>(), cloud_offsets, nclouds, counts, &nt, &acc, &sink);
    CK_SYNC(ctx->copy_stream);
    if (st) return st;
    tet_offsets[0] = 0;
    for (int c = 0; c < nclouds; ++c) tet_offsets[c + 1] = tet_offsets[c] + counts[c];
    *ntet = (int64_t)nt;
    if (!sink.fits) return fail(ctx, G4D_ERR_ARG, "output buffer too small (%lld < %zu)", (long long)cap, nt);
    acc.t_total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    ctx->stats = acc;
    if (stats) *stats = acc;
    return G4D_OK;
}

g4d_status g4d_triangulate_batch_device(g4d_ctx* ctx, const double* d_xyz, const int64_t* cloud_offsets,
                                        int nclouds, const g4d_tet** d_tets, const int64_t** tet_offsets,
                                        g4d_stats* stats) {
    if (!ctx) return G4D_ERR_ARG;
    if (!d_xyz || !cloud_offsets || nclouds < 0 || !d_tets || !tet_offsets)
        return fail(ctx, G4D_ERR_ARG, "null argument");
    cudaSetDevice(ctx->device);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<int64_t> counts;
    size_t ntet = 0;
    g4d_stats acc{};
    g4d_status st = run_batch(ctx, d_xyz, cloud_offsets, nclouds, counts, &ntet, &acc);
    if (st) return st;
    ctx->batch_offsets.assign(nclouds + 1, 0);
    for (int c = 0; c < nclouds; ++c) ctx->batch_offsets[c + 1] = ctx->batch_offsets[c] + counts[c];
    *d_tets = ctx->b[B_BOUT].as<g4d_tet>();
    *tet_offsets = ctx->batch_offsets.data();
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
    CK_SYNC(ctx->stream);
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
    const auto tf = ctx->pba_form.find(grid);  // a tuned (or fixed) form for this width, else the default
    const int form = tf != ctx->pba_form.end() ? tf->second : -1;
    launch_pba_z(L, D, ctx->b[B_GA].as<uint32_t>());
    launch_pba_y(L, grid, ctx->b[B_GA].as<uint32_t>(), ctx->b[B_GB].as<uint32_t>(), form);
    launch_pba_x(L, grid, ctx->b[B_GB].as<uint32_t>(), ctx->b[B_GA].as<uint32_t>(), form);
    CK(cudaMemcpyAsync(sites, ctx->b[B_GA].p, sizeof(uint32_t) * G3, cudaMemcpyDeviceToHost, ctx->stream));
    unsigned herr = 0;
    CK(cudaMemcpyAsync(&herr, &ctx->b[B_CTR].as<Counters>()->err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK_SYNC(ctx->stream);
    // coordinates the scaling could not place in [1, G-2] (NaN, infinite, or
    // every coordinate equal) were clamped on the device: report them
    return check_err(ctx, herr);
}

// ---- learned star proposal ------------------------------------------------

static g4d_status mlp_upload(g4d_ctx* ctx) {
    CK(ctx->b[B_MLP_P].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_MLP_G].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_MLP_M1].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_MLP_M2].ensure(sizeof(float) * MLP_NPARAMS));
    CK(cudaMemcpyAsync(ctx->b[B_MLP_P].p, ctx->mlp.data(), sizeof(float) * MLP_NPARAMS, cudaMemcpyHostToDevice,
                       ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_MLP_G].p, 0, sizeof(float) * MLP_NPARAMS, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_MLP_M1].p, 0, sizeof(float) * MLP_NPARAMS, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_MLP_M2].p, 0, sizeof(float) * MLP_NPARAMS, ctx->stream));
    ctx->adam_step = 0;
    ctx->has_model = true;
    return G4D_OK;
}

// He-uniform initialisation (fixed seed), zero biases
static void mlp_init(std::vector<float>& w) {
    w.assign(MLP_NPARAMS, 0.f);
    std::mt19937 rng(20240611u);
    auto fill = [&](int off, int count, int fan_in, float gain) {
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        const float a = gain * std::sqrt(6.f / (float)fan_in);
        for (int i = 0; i < count; ++i) w[off + i] = a * u(rng);
    };
    fill(0, 64 * 16, 6, 1.f);                     // W1 (6 live inputs)
    fill(64 * 16 + 64, 64 * 64, 64, 1.f);         // W2
    fill(64 * 16 + 64 + 64 * 64 + 64, 64 * 64, 64, 1.f);  // W3
    fill(64 * 16 + 64 + 2 * (64 * 64 + 64), 64, 64, 0.1f);  // w4
}

g4d_status g4d_proposal_train(g4d_ctx* ctx, const double* xyz, int n, int epochs, float lr, float* loss_out) {
    g4d_status st = check_n(ctx, n);
    if (st) return st;
    if (!xyz || epochs < 0 || !(lr > 0.f)) return fail(ctx, G4D_ERR_ARG, "bad training arguments");
    cudaSetDevice(ctx->device);
    // labels come from the plain method
    const int saved = ctx->cfg.proposal;
    ctx->cfg.proposal = 0;
    CK(ctx->b[B_XYZ].ensure(sizeof(double) * 3 * (size_t)n));
    CK(cudaMemcpyAsync(ctx->b[B_XYZ].p, xyz, sizeof(double) * 3 * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    st = run_all_device(ctx, ctx->b[B_XYZ].as<double>(), nullptr, n, false);
    ctx->cfg.proposal = saved;
    if (st) return st;
    Dev D = make_dev(ctx);
    D.anyLarge = ctx->large_used > 0;
    st = run_ring(ctx, D, true);
    if (st) return st;
    if (!ctx->has_model) {
        mlp_init(ctx->mlp);
        st = mlp_upload(ctx);
        if (st) return st;
    }
    const int M = ctx->ring_rows;
    const int ntiles = (M + 127) / 128;
    const int per_step = 64;  // tiles per optimizer step (8192 rows)
    Launch L{ctx->stream, &ctx->launches};
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    CK(ctx->b[B_TILES].ensure(sizeof(int) * std::max(ntiles, 1)));
    std::vector<int> order(ntiles);
    std::mt19937 rng(7u + (unsigned)ctx->adam_step);
    float last = 0.f;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = 0; i < ntiles; ++i) order[i] = i;
        std::shuffle(order.begin(), order.end(), rng);
        CK(cudaMemcpyAsync(ctx->b[B_TILES].p, order.data(), sizeof(int) * ntiles, cudaMemcpyHostToDevice,
                           ctx->stream));
        CK(cudaMemsetAsync(aux, 0, sizeof(MlpAux), ctx->stream));
        for (int b0 = 0; b0 < ntiles; b0 += per_step) {
            const int nb = std::min(per_step, ntiles - b0);
            int rows = 0;
            for (int i = b0; i < b0 + nb; ++i) rows += std::min(128, M - 128 * order[i]);
            launch_mlp_train(L, ctx->b[B_MLP_P].as<float>(), ctx->b[B_RING_X].as<uint16_t>(),
                             ctx->b[B_RING_Y].as<float>(), M, ctx->b[B_TILES].as<int>() + b0, nb, 1.f / (float)rows,
                             ctx->b[B_MLP_G].as<float>(), &aux->loss, &aux->err);
            launch_adam(L, ctx->b[B_MLP_P].as<float>(), ctx->b[B_MLP_G].as<float>(), ctx->b[B_MLP_M1].as<float>(),
                        ctx->b[B_MLP_M2].as<float>(), ++ctx->adam_step, lr);
        }
        MlpAux h{};
        CK(cudaMemcpyAsync(&h, aux, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
        CK_SYNC(ctx->stream);
        if (h.err) return fail(ctx, G4D_ERR_TIMEOUT, "tensor-core training kernel timed out waiting (0x%x)", h.err);
        last = M ? h.loss / (float)M : 0.f;
    }
    CK(cudaMemcpyAsync(ctx->mlp.data(), ctx->b[B_MLP_P].p, sizeof(float) * MLP_NPARAMS, cudaMemcpyDeviceToHost,
                       ctx->stream));
    CK_SYNC(ctx->stream);
    if (loss_out) *loss_out = last;
    return G4D_OK;
}

g4d_status g4d_proposal_weights(g4d_ctx* ctx, float* w, int count, int set) {
    if (!ctx) return G4D_ERR_ARG;
    if (!w || count != MLP_NPARAMS)
        return fail(ctx, G4D_ERR_ARG, "the proposal model has %d parameters (got %d)", MLP_NPARAMS, count);
    cudaSetDevice(ctx->device);
    if (set) {
        ctx->mlp.assign(w, w + MLP_NPARAMS);
        g4d_status st = mlp_upload(ctx);
        if (st) return st;
        CK_SYNC(ctx->stream);
        return G4D_OK;
    }
    if (!ctx->has_model) return fail(ctx, G4D_ERR_ARG, "no proposal model (train or set one first)");
    memcpy(w, ctx->mlp.data(), sizeof(float) * MLP_NPARAMS);
    return G4D_OK;
}

// diagnostic: one pass of the training kernel (no update) on given rows
g4d_status g4d_mlp_grad(g4d_ctx* ctx, const uint16_t* x, const float* y, int m, const float* params, float* grads,
                        float* loss) {
    if (!ctx || !x || !y || m < 1 || !params || !grads) return G4D_ERR_ARG;
    cudaSetDevice(ctx->device);
    CK(ctx->b[B_DIAG_X].ensure(sizeof(uint16_t) * 16 * (size_t)m));
    CK(ctx->b[B_DIAG_Y].ensure(sizeof(float) * (size_t)m));
    CK(ctx->b[B_DIAG_P].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_DIAG_G].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_MLP_AUX].ensure(sizeof(MlpAux)));
    CK(cudaMemcpyAsync(ctx->b[B_DIAG_X].p, x, sizeof(uint16_t) * 16 * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->b[B_DIAG_Y].p, y, sizeof(float) * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->b[B_DIAG_P].p, params, sizeof(float) * MLP_NPARAMS, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemsetAsync(ctx->b[B_DIAG_G].p, 0, sizeof(float) * MLP_NPARAMS, ctx->stream));
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    CK(cudaMemsetAsync(aux, 0, sizeof(MlpAux), ctx->stream));
    Launch L{ctx->stream, &ctx->launches};
    launch_mlp_train(L, ctx->b[B_DIAG_P].as<float>(), ctx->b[B_DIAG_X].as<uint16_t>(), ctx->b[B_DIAG_Y].as<float>(),
                     m, nullptr, (m + 127) / 128, 1.f / (float)m, ctx->b[B_DIAG_G].as<float>(), &aux->loss, &aux->err);
    MlpAux h{};
    CK(cudaMemcpyAsync(grads, ctx->b[B_DIAG_G].p, sizeof(float) * MLP_NPARAMS, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&h, aux, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    if (h.err) return fail(ctx, G4D_ERR_TIMEOUT, "tensor-core training kernel timed out waiting (0x%x)", h.err);
    if (loss) *loss = h.loss / (float)m;
    return G4D_OK;
}

// diagnostic: logits of given rows
g4d_status g4d_mlp_infer(g4d_ctx* ctx, const uint16_t* x, int m, const float* params, float* logits) {
    if (!ctx || !x || m < 1 || !params || !logits) return G4D_ERR_ARG;
    cudaSetDevice(ctx->device);
    CK(ctx->b[B_DIAG_X].ensure(sizeof(uint16_t) * 16 * (size_t)m));
    CK(ctx->b[B_DIAG_Y].ensure(sizeof(float) * (size_t)m));
    CK(ctx->b[B_DIAG_P].ensure(sizeof(float) * MLP_NPARAMS));
    CK(ctx->b[B_MLP_AUX].ensure(sizeof(MlpAux)));
    CK(cudaMemcpyAsync(ctx->b[B_DIAG_X].p, x, sizeof(uint16_t) * 16 * (size_t)m, cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaMemcpyAsync(ctx->b[B_DIAG_P].p, params, sizeof(float) * MLP_NPARAMS, cudaMemcpyHostToDevice, ctx->stream));
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    CK(cudaMemsetAsync(aux, 0, sizeof(MlpAux), ctx->stream));
    Launch L{ctx->stream, &ctx->launches};
    launch_mlp_infer(L, ctx->b[B_DIAG_P].as<float>(), ctx->b[B_DIAG_X].as<uint16_t>(), m,
                     ctx->b[B_DIAG_Y].as<float>(), &aux->err);
    MlpAux h{};
    CK(cudaMemcpyAsync(logits, ctx->b[B_DIAG_Y].p, sizeof(float) * (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(&h, aux, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    if (h.err) return fail(ctx, G4D_ERR_TIMEOUT, "tensor-core inference kernel timed out waiting (0x%x)", h.err);
    return G4D_OK;
}

g4d_status g4d_mlp_wait_probe(g4d_ctx* ctx, int limit) {
    if (!ctx || limit < 1) return G4D_ERR_ARG;
    cudaSetDevice(ctx->device);
    CK(ctx->b[B_MLP_AUX].ensure(sizeof(MlpAux)));
    MlpAux* aux = ctx->b[B_MLP_AUX].as<MlpAux>();
    CK(cudaMemsetAsync(aux, 0, sizeof(MlpAux), ctx->stream));
    Launch L{ctx->stream, &ctx->launches};
    launch_mlp_wait_probe(L, limit, &aux->err);
    MlpAux h{};
    CK(cudaMemcpyAsync(&h, aux, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    if (h.err) return fail(ctx, G4D_ERR_TIMEOUT, "tensor-core kernel wait ran out after %d polls (0x%x)", limit, h.err);
    return G4D_OK;
}

namespace {

// the validator over points P (n, Morton order when order is given) and
// device tetrahedra
g4d_status check_on_device(g4d_ctx* ctx, const double4* P, const int* order, const g4d_tet* tets, int ntet, int n,
                           g4d_check_report* report) {
    CK(ctx->b[B_CHECK].ensure(check_scratch_bytes(ntet, n)));
    CK(ctx->b[B_CHECKOUT].ensure(8 * sizeof(unsigned long long)));
    unsigned long long* out = ctx->b[B_CHECKOUT].as<unsigned long long>();
    unsigned* err = reinterpret_cast<unsigned*>(out + 6);
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned), ctx->stream));
    CK(run_mesh_check(ctx->stream, &ctx->launches, P, order, tets, ntet, n, ctx->b[B_CHECK].p, out, err));
    unsigned long long h[7] = {0, 0, 0, 0, 0, 0, 0};
    CK(cudaMemcpyAsync(h, out, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    CK_SYNC(ctx->stream);
    const unsigned herr = (unsigned)h[6];
    if (herr & 0x200u) return fail(ctx, G4D_ERR_INTERNAL, "a tetrahedron has a vertex index outside [0, %d)", n);
    if (herr) return fail(ctx, G4D_ERR_PRECISION, "a validator predicate could not be evaluated exactly");
    report->vertices = (long long)h[0];
    report->edges = (long long)h[1];
    report->triangles = (long long)h[2];
    report->tets = ntet;
    report->euler = report->vertices - report->edges + report->triangles - report->tets;
    report->orient_fail = (long long)h[3];
    report->insphere_fail = (long long)h[4];
    report->adjacency_fail = (long long)h[5];
    return G4D_OK;
}

}  // namespace

g4d_status g4d_check_mesh(g4d_ctx* ctx, g4d_check_report* report) {
    if (!ctx || !report) return G4D_ERR_ARG;
    if (!ctx->has_result) return fail(ctx, G4D_ERR_ARG, "no single-cloud triangulation to check");
    cudaSetDevice(ctx->device);
    return check_on_device(ctx, ctx->b[B_P].as<double4>(), ctx->result_mapped ? ctx->b[B_ORDER].as<int>() : nullptr,
                           ctx->b[B_TETS].as<g4d_tet>(), ctx->ntet, ctx->n, report);
}

g4d_status g4d_check_tets(g4d_ctx* ctx, const double* xyz, int n, const g4d_tet* tets, int ntet,
                          g4d_check_report* report) {
    if (!ctx || !xyz || !report || n < 1 || ntet < 0 || (ntet > 0 && !tets)) return G4D_ERR_ARG;
    cudaSetDevice(ctx->device);
    std::vector<double4> p((size_t)n);
    for (int i = 0; i < n; ++i) p[i] = make_double4(xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2], 0.0);
    CK(ctx->b[B_CHKP].ensure(sizeof(double4) * (size_t)n));
    CK(ctx->b[B_CHKT].ensure(sizeof(g4d_tet) * (size_t)std::max(ntet, 1)));
    CK(cudaMemcpyAsync(ctx->b[B_CHKP].p, p.data(), sizeof(double4) * (size_t)n, cudaMemcpyHostToDevice, ctx->stream));
    if (ntet)
        CK(cudaMemcpyAsync(ctx->b[B_CHKT].p, tets, sizeof(g4d_tet) * (size_t)ntet, cudaMemcpyHostToDevice,
                           ctx->stream));
    g4d_status st = check_on_device(ctx, ctx->b[B_CHKP].as<double4>(), nullptr, ctx->b[B_CHKT].as<g4d_tet>(), ntet,
                                    n, report);
    CK_SYNC(ctx->stream);  // the host copy of the points outlives the upload
    return st;
}

void* g4d_stream(g4d_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

void g4d_free(void* p) { free(p); }

}  // extern "C"
