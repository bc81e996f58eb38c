// Stars and star splaying.
//
// A star is the link of a point in the 4D convex hull of the points lifted to
// (x, y, z, |p|^2): a triangulated 2-sphere of neighbour points (the reference's
// StarData, GDelaunay/GDelData.h:54-85, GDelCommon.h:598-717). The reference
// updates stars with one launch per insertion index across all stars
// (GDelHost.cu:591-743, 1208-1360). Here one warp owns one star for a whole
// round: it stages the star's history hash, coordinates and triangles in shared
// memory, inserts every pending point (beneath test = orient4 < 0 as in
// GDelPredKernels.cu:233-420; hole re-fan as in GDelKernels.cu:622-783) and
// writes the star back once. Between rounds, emission (GDelKernels.cu:818-939)
// and containment proofs (GDelPredKernels.cu:427-538) queue insertions into
// per-star inboxes; the loop ends when no star receives a new point.
//
// Storage classes. The reference grows each star's triangle array on demand
// (GDelData.cu:306-340). Here a star lives in a fixed small slot (127 history
// points, 124 triangles, 2 KB in HBM, 6.7 KB of shared memory while a warp
// works on it) that fits nearly every star; a star that outgrows it during a
// round is left untouched, its inbox kept, and k_promote copies it to a large
// slot (2047 points, 2044 triangles) before the large-class kernel replays the
// round's insertions for it. lidx[s] says which class holds star s.
//
// Every star kernel also exists as a filter-only variant (FP64 filters only,
// 64 registers, 32 warps/SM): a star, proof or count that meets an undecided
// predicate is left untouched and queued for the exact variant.
#include "g4d_internal.cuh"
#include "g4d_predicates.cuh"

namespace g4d {

constexpr int WARPS_PER_BLOCK = 4;
#ifndef FAST_BLOCKS
#define FAST_BLOCKS 8  // blocks per SM of the filter-only star kernels
#endif
#ifndef PROOF_BLOCKS
#define PROOF_BLOCKS 8  // blocks per SM of the filter-only proof kernel
#endif
#ifndef BUILD_BLOCKS
#define BUILD_BLOCKS 7  // launch-bound blocks per SM of the filter-only initial-star kernel
#endif

// ---------------------------------------------------------------------------
// storage classes
// ---------------------------------------------------------------------------

struct SmallStar {
    static constexpr int LOG2_HS = 8, HS = HSLOTS, HM = HMAX, TM = TMAX, TS = TSTRIDE;
    // blocks per SM: FAST_BLOCKS filter-only (64 registers at 8), 4 with the exact path
    static constexpr int WARPS = WARPS_PER_BLOCK, MINB = 4, MINB_FAST = FAST_BLOCKS;
    // the initial build is compiled for one block fewer: it still takes 64
    // registers and runs 8 blocks per SM, but the looser bound gives faster
    // code (8M cloud: initial stars 72.4 -> 70.1 ms), while the same bound on
    // the insertion kernels costs far more (splaying 61.8 -> 78.8 ms)
    static constexpr int MINB_BUILD = BUILD_BLOCKS;
    static constexpr bool LARGE = false;
    using Idx = uint8_t;   // triangle index and coordinate-cache index
    using Slot = uint8_t;  // history slot
    using Rec = uint32_t;  // hole boundary edge: u | w<<9 | o<<18 | oj<<26
    using Tri = uint2;     // packing in g4d_internal.cuh
    __device__ static Rec rec(int u, int w, int o, int oj) {
        return (uint32_t)u | ((uint32_t)w << 9) | ((uint32_t)o << 18) | ((uint32_t)oj << 26);
    }
    __device__ static int rec_u(Rec e) { return (int)(e & 511u); }
    __device__ static int rec_w(Rec e) { return (int)((e >> 9) & 511u); }
    __device__ static int rec_o(Rec e) { return (int)((e >> 18) & 255u); }
    __device__ static int rec_oj(Rec e) { return (int)((e >> 26) & 3u); }
    __device__ static int tv(Tri T, int i) { return tri_v(T, i); }
    __device__ static int to(Tri T, int i) { return tri_o(T, i); }
    __device__ static int tj(Tri T, int i) { return tri_j(T, i); }
    __device__ static int gen(Tri T) { return tri_gen(T); }
    __device__ static bool kept(Tri T) { return (T.x & TRI_KEPT) != 0; }
    __device__ static Tri pack(int v0, int v1, int v2, int g, int o0, int o1, int o2, int j0, int j1, int j2) {
        return tri_pack(v0, v1, v2, g, o0, o1, o2, j0, j1, j2);
    }
    __device__ static int* hash(const Dev& D, int s) { return D.hh + (size_t)s * HS; }
    __device__ static Tri* tris(const Dev& D, int s) { return D.tri + (size_t)s * TS; }
};

// Large-class triangle packing in HBM (16 bytes):
//   x = v0 | v1<<16, y = v2 | gen<<16 | kept<<31, z = o0 | o1<<16,
//   w = o2 | j0<<16 | j1<<18 | j2<<20
struct LargeStar {
    static constexpr int LOG2_HS = 12, HS = LHSLOTS, HM = LHMAX, TM = LTMAX, TS = LTSTRIDE;
    static constexpr int WARPS = 1, MINB = 1, MINB_FAST = 1, MINB_BUILD = 1;  // about 141 KB of shared memory per warp
    static constexpr bool LARGE = true;
    using Idx = uint16_t;
    using Slot = uint16_t;
    using Rec = unsigned long long;  // u | w<<12 | o<<24 | oj<<35
    using Tri = uint4;
    __device__ static Rec rec(int u, int w, int o, int oj) {
        return (Rec)u | ((Rec)w << 12) | ((Rec)o << 24) | ((Rec)oj << 35);
    }
    __device__ static int rec_u(Rec e) { return (int)(e & 4095u); }
    __device__ static int rec_w(Rec e) { return (int)((e >> 12) & 4095u); }
    __device__ static int rec_o(Rec e) { return (int)((e >> 24) & 2047u); }
    __device__ static int rec_oj(Rec e) { return (int)((e >> 35) & 3u); }
    __device__ static int tv(Tri T, int i) {
        return (int)(i == 0 ? (T.x & 0xffffu) : (i == 1 ? (T.x >> 16) : (T.y & 0xffffu)));
    }
    __device__ static int to(Tri T, int i) {
        return (int)(i == 0 ? (T.z & 0xffffu) : (i == 1 ? (T.z >> 16) : (T.w & 0xffffu)));
    }
    __device__ static int tj(Tri T, int i) { return (int)((T.w >> (16 + 2 * i)) & 3u); }
    __device__ static int gen(Tri T) { return (int)((T.y >> 16) & 15u); }
    __device__ static bool kept(Tri T) { return (T.y & 0x80000000u) != 0; }
    __device__ static Tri pack(int v0, int v1, int v2, int g, int o0, int o1, int o2, int j0, int j1, int j2) {
        uint4 T;
        T.x = (uint32_t)v0 | ((uint32_t)v1 << 16);
        T.y = (uint32_t)v2 | ((uint32_t)(g & 15) << 16);
        T.z = (uint32_t)o0 | ((uint32_t)o1 << 16);
        T.w = (uint32_t)o2 | ((uint32_t)j0 << 16) | ((uint32_t)j1 << 18) | ((uint32_t)j2 << 20);
        return T;
    }
    __device__ static int* hash(const Dev& D, int s) { return D.lhh + (size_t)D.lidx[s] * HS; }
    __device__ static Tri* tris(const Dev& D, int s) { return D.ltri + (size_t)D.lidx[s] * TS; }
};

// Per-warp shared-memory image of one star (6.7 KB small, so that 32 warps fit
// on an SM; 141 KB large).
template <class C>
struct WS {
    using Idx = typename C::Idx;
    int hh[C::HS];                 // history hash: point id | link bit, HEMPTY when free
    Idx cix[C::HS];                // slot -> index into the coordinate cache
    double cx[C::HM + 1], cy[C::HM + 1], cz[C::HM + 1];
    typename C::Slot tv[3][C::TS];  // triangle vertices (history slots)
    Idx to[3][C::TS];              // neighbour across the edge opposite each vertex
    uint8_t tj[3][C::TS];          // position of the shared edge inside that neighbour
    uint8_t tf[C::TS];             // bit 7 alive, bits 0..3 creation pass
    Idx efrom[C::HM + 1], eto[C::HM + 1];  // by coordinate-cache index of the edge's vertex
    union {
        typename C::Rec erec[C::TS];  // hole boundary edges (insertion)
        float okey[C::HM + 1];        // squared distances (initial sort, before any insertion)
    };
    Idx blist[C::TS];              // beneath triangles in index order / compaction map
    Idx fstack[C::TS];             // free triangle slots
    typename C::Slot order[C::HM + 1];  // insertion order (slots)
    uint32_t bmask[C::TS / 32];
    uint32_t wasLink[C::HS / 32], insMask[C::HS / 32];
    int nedge, nfree, ntri, nins, nhist, ncoord;
};

// MINB_FAST blocks of 4 warps per SM: their images plus the per-block reservation in 228 KB
static_assert(SmallStar::MINB_FAST * (4 * sizeof(WS<SmallStar>) + 1024) <= 228 * 1024, "small star image too large");
static_assert(sizeof(WS<LargeStar>) + 1024 <= 227 * 1024, "large star image too large");

// Read-only view of any star, whichever class holds it (cross-star lookups).
struct StarView {
    const int* hh;
    const void* tri;
    bool large;
};

struct TriU {
    int v[3], o[3], j[3];
    int gen;
    bool kept;
};

__device__ __forceinline__ StarView star_view(const Dev& D, int s) {
    const int li = D.anyLarge ? D.lidx[s] : -1;
    StarView V;
    V.large = li >= 0;
    if (!V.large) {
        V.hh = D.hh + (size_t)s * HSLOTS;
        V.tri = D.tri + (size_t)s * TSTRIDE;
    } else {
        V.hh = D.lhh + (size_t)li * LHSLOTS;
        V.tri = D.ltri + (size_t)li * LTSTRIDE;
    }
    return V;
}

__device__ __forceinline__ TriU tri_get(const StarView& V, int t) {
    TriU r;
    if (!V.large) {
        const uint2 T = static_cast<const uint2*>(V.tri)[t];
#pragma unroll
        for (int i = 0; i < 3; ++i) { r.v[i] = SmallStar::tv(T, i); r.o[i] = SmallStar::to(T, i); r.j[i] = SmallStar::tj(T, i); }
        r.gen = SmallStar::gen(T);
        r.kept = SmallStar::kept(T);
    } else {
        const uint4 T = static_cast<const uint4*>(V.tri)[t];
#pragma unroll
        for (int i = 0; i < 3; ++i) { r.v[i] = LargeStar::tv(T, i); r.o[i] = LargeStar::to(T, i); r.j[i] = LargeStar::tj(T, i); }
        r.gen = LargeStar::gen(T);
        r.kept = LargeStar::kept(T);
    }
    return r;
}

__device__ __forceinline__ bool tri_kept(const StarView& V, int t) {
    return !V.large ? (static_cast<const uint2*>(V.tri)[t].x >> 31) != 0
                    : (static_cast<const uint4*>(V.tri)[t].y >> 31) != 0;
}

__device__ __forceinline__ void tri_set_kept(const StarView& V, int t, bool keep) {
    uint32_t* w = !V.large ? &const_cast<uint2*>(static_cast<const uint2*>(V.tri))[t].x
                           : &const_cast<uint4*>(static_cast<const uint4*>(V.tri))[t].y;
    const uint32_t x = *w, nx = keep ? (x | TRI_KEPT) : (x & ~TRI_KEPT);
    if (nx != x) *w = nx;
}

// slot of v in a star's history hash (entry in *entry), -1 if absent
__device__ __forceinline__ int view_lookup(const StarView& V, int v, uint32_t* entry) {
    const int log2 = V.large ? LargeStar::LOG2_HS : SmallStar::LOG2_HS;
    const uint32_t mask = (1u << log2) - 1u;
    uint32_t s = ((uint32_t)v * 2654435761u) >> (32 - log2);
    for (uint32_t k = 0; k <= mask; ++k) {
        const uint32_t e = (uint32_t)V.hh[s];
        if ((e & HID) == (uint32_t)v) { *entry = e; return (int)s; }
        if ((e & HID) == HEMPTY) return -1;
        s = (s + 1) & mask;
    }
    return -1;
}

template <class C>
__device__ __forceinline__ double3 wpt(const WS<C>& S, int slot) {
    const int c = S.cix[slot];
    return make_double3(S.cx[c], S.cy[c], S.cz[c]);
}
template <class C>
__device__ __forceinline__ int wid(const WS<C>& S, int slot) { return S.hh[slot] & (int)HID; }

__device__ __forceinline__ bool valid_id(const Dev& D, int v) { return (unsigned)v < (unsigned)D.n; }

__device__ __forceinline__ PredSink sink_of(const Dev& D) {
    PredSink k;
    k.err = &D.ctr->err;
    k.dbg_set = &D.ctr->dbg_set;
    k.dbg_pts = D.ctr->dbg_pts;
    k.dbg_ids = D.ctr->dbg_ids;
    return k;
}

// lifted orientation: exact (never 0) or the FP64 filter alone (0 = undecided)
template <bool EXACT>
__device__ __forceinline__ int pred4(double3 a, double3 b, double3 c, double3 d, double3 e, int ia, int ib, int ic,
                                     int id, int ie, const PredSink& sink, unsigned* exact) {
    if (EXACT) return orient4(a, b, c, d, e, ia, ib, ic, id, ie, sink, exact);
    return orient4_filter(a, b, c, d, e);
}

// The coordinate cache of a filter-only kernel holds coordinates relative to
// the star's point (rounded once, as the filter's own differences would be),
// so the filter needs no subtraction; an exact kernel caches absolute
// coordinates for its big-integer fallback. Both give the exact sign or,
// filter-only, 0 (undecided).
// orient4(a, b, c, star, p): p against the link triangle (a, b, c)
// (`bound`: the filter-only kernels' bound for every coordinate the star has
// cached, orient4_static_bound of their largest magnitude)
template <bool EXACT>
__device__ __forceinline__ int pred_beneath(double3 a, double3 b, double3 c, double3 ps, double3 pp, int ia, int ib,
                                            int ic, int is, int ip, const PredSink& sink, unsigned* exact,
                                            double bound) {
    if (EXACT) return orient4(a, b, c, ps, pp, ia, ib, ic, is, ip, sink, exact);
    return -orient4_filter_rel_bounded(a, b, c, pp, bound);  // the star's point as the base: rows a, b, c, p swap two points
}
// orient4(l0, l1, l2, l3, star)
template <bool EXACT>
__device__ __forceinline__ int pred_cone(double3 a, double3 b, double3 c, double3 d, double3 ps, int ia, int ib,
                                         int ic, int id, int is, const PredSink& sink, unsigned* exact) {
    if (EXACT) return orient4(a, b, c, d, ps, ia, ib, ic, id, is, sink, exact);
    return orient4_filter_rel(a, b, c, d);
}

// point coordinates; an out-of-range id (only possible from a corrupted star)
// raises ERR_TOPOLOGY and reads point 0 instead of leaving the buffer
__device__ __forceinline__ double3 gpt(const Dev& D, int id) {
    if (!valid_id(D, id)) {
        atomicOr(&D.ctr->err, ERR_TOPOLOGY);
        id = 0;
    }
    const double4 p = D.P[id];
    return make_double3(p.x, p.y, p.z);
}

// point range [lo, hi) of the cloud that holds point s
__device__ __forceinline__ void cloud_range(const Dev& D, int s, int* lo, int* hi) {
    if (D.nclouds <= 0) {
        *lo = 0;
        *hi = D.n;
        return;
    }
    int a = 0, b = D.nclouds;  // cloudOff[a] <= s < cloudOff[b]
    while (b - a > 1) {
        const int m = (a + b) >> 1;
        if (D.cloudOff[m] <= s) a = m; else b = m;
    }
    *lo = D.cloudOff[a];
    *hi = D.cloudOff[a + 1];
}

// cache the coordinates of the point in `slot`
template <class C>
__device__ __forceinline__ void ws_cache_coords(WS<C>& S, const Dev& D, int slot, int id, double3 base) {
    const int c = atomicAdd(&S.ncoord, 1);
    const int cc = c < C::HM + 1 ? c : C::HM;
    S.cix[slot] = (typename C::Idx)cc;
    const double4 p = D.P[valid_id(D, id) ? id : 0];
    S.cx[cc] = p.x - base.x;
    S.cy[cc] = p.y - base.y;
    S.cz[cc] = p.z - base.z;
}

// filter bound for every coordinate the warp's star has cached (relative to
// the star's point in the filter-only kernels), the same value in every lane
template <class C>
__device__ __forceinline__ double cache_bound(const WS<C>& S, int lane) {
    double r = 0.0;
    const int nc = min(S.ncoord, C::HM + 1);
    for (int c = lane; c < nc; c += 32) r = fmax(r, fmax(fabs(S.cx[c]), fmax(fabs(S.cy[c]), fabs(S.cz[c]))));
#pragma unroll
    for (int o = 16; o; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    return orient4_static_bound(r);
}

// Membership of v in star `star`: 0 = never inserted, 1 = in the history but
// not in the link, 2 = in the link. The first probe of the small table is
// issued together with the class lookup (lidx), so a small star, the common
// case, costs one round trip instead of two.
struct HistProbe {
    const int* h;
    uint32_t mask, pos, e;
    int r;  // -1 while unresolved
};

__device__ __forceinline__ HistProbe hist_begin(const Dev& D, int star, int v) {
    const int li = D.anyLarge ? D.lidx[star] : -1;
    const uint32_t q = hslot0<SmallStar::LOG2_HS>(v);
    const uint32_t e0 = (uint32_t)D.hh[(size_t)star * HSLOTS + q];
    HistProbe P;
    P.r = -1;
    if (li < 0) {
        P.h = D.hh + (size_t)star * HSLOTS;
        P.mask = HSLOTS - 1;
        P.pos = q;
        P.e = e0;
    } else {
        P.h = D.lhh + (size_t)li * LHSLOTS;
        P.mask = LHSLOTS - 1;
        P.pos = hslot0<LargeStar::LOG2_HS>(v);
        P.e = (uint32_t)P.h[P.pos];
    }
    return P;
}

// resolve with the current entry (probe k) or move to the next slot
__device__ __forceinline__ void hist_step(HistProbe& P, int v, uint32_t k) {
    if ((P.e & HID) == (uint32_t)v) P.r = (P.e & HLINK) ? 2 : 1;
    else if ((P.e & HID) == HEMPTY || k == P.mask) P.r = 0;
    else P.pos = (P.pos + 1) & P.mask;
}

__device__ __forceinline__ int hist_state(const Dev& D, int star, int v) {
    if (!valid_id(D, star)) return 1;  // never asks for an insertion into a bad star
    HistProbe P = hist_begin(D, star, v);
    for (uint32_t k = 0;; ++k) {
        hist_step(P, v, k);
        if (P.r >= 0) return P.r;
        P.e = (uint32_t)P.h[P.pos];
    }
}

// hist_state(a, b) and hist_state(b, a) for valid ids, the two probe
// sequences walked in lockstep so that their loads overlap
__device__ __forceinline__ void hist_state_pair(const Dev& D, int a, int b, int* sab, int* sba) {
    HistProbe A = hist_begin(D, a, b), B = hist_begin(D, b, a);
    for (uint32_t k = 0;; ++k) {
        if (A.r < 0) hist_step(A, b, k);
        if (B.r < 0) hist_step(B, a, k);
        if (A.r >= 0 && B.r >= 0) break;
        if (A.r < 0) A.e = (uint32_t)A.h[A.pos];
        if (B.r < 0) B.e = (uint32_t)B.h[B.pos];
    }
    *sab = A.r;
    *sba = B.r;
}

__device__ __forceinline__ void push_inbox(const Dev& D, int t, int v, bool* overflow) {
    if (!valid_id(D, t) || !valid_id(D, v)) {
        atomicOr(&D.ctr->err, ERR_TOPOLOGY);
        return;
    }
    const int cnt = *((volatile int*)&D.inboxCount[t]);
    const int* box = D.inbox + (size_t)t * INBOX_CAP;
    const int lim = cnt < INBOX_CAP ? cnt : INBOX_CAP;
    for (int k = 0; k < lim; ++k)
        if (((volatile const int*)box)[k] == v) return;
    const int pos = atomicAdd(&D.inboxCount[t], 1);
    if (pos == 0) {
        if (D.anyLarge && D.lidx[t] >= 0) {
            const int w = atomicAdd(&D.ctr->ins_count_large, 1);
            if (w < D.largeCap) D.wlInsL[w] = t;
            else atomicOr(&D.ctr->err, ERR_CAPACITY);
        } else {
            const int w = atomicAdd(&D.ctr->ins_count, 1);
            D.wlIns[w] = t;
        }
    }
    if (pos < INBOX_CAP) {
        D.inbox[(size_t)t * INBOX_CAP + pos] = v;
    } else {
        // the inbox is full: the request waits for the next round
        *overflow = true;
        const int q = atomicAdd(&D.ctr->ovf_next, 1);
        if (q < D.ovfCap) D.ovfNext[q] = make_int2(t, v);
        else atomicOr(&D.ctr->err, ERR_OVFCAP);
    }
}

// --------------------------------------------------------------------------
// warp helpers
// --------------------------------------------------------------------------

// exclusive prefix sum over the warp of v in 0..3 (two ballots of its bits)
__device__ __forceinline__ int warp_excl_scan(int v, int lane, int* total) {
    const unsigned b0 = __ballot_sync(0xffffffffu, v & 1), b1 = __ballot_sync(0xffffffffu, v & 2);
    const unsigned below = (1u << lane) - 1u;
    *total = __popc(b0) + 2 * __popc(b1);
    return __popc(b0 & below) + 2 * __popc(b1 & below);
}

// Insert id v into the shared history hash; returns slot, sets *fresh when new.
template <class C>
__device__ __forceinline__ int ws_hash_insert(WS<C>& S, int v, bool* fresh) {
    uint32_t s = hslot0<C::LOG2_HS>(v);
    for (int k = 0; k < C::HS; ++k) {
        const int old = atomicCAS(&S.hh[s], (int)HEMPTY, v);
        if ((uint32_t)old == HEMPTY) { *fresh = true; return (int)s; }
        if ((old & (int)HID) == v) { *fresh = false; return (int)s; }
        s = (s + 1) & (C::HS - 1);
    }
    *fresh = false;
    return -1;
}

// Insert the point in slot sp into the star held by the warp. Returns 1 when it
// entered the link, 0 when it lies inside the star's cone (drowned), -1 on an
// error (flag raised), -2 when the star's class has no room for the new
// triangles (the caller promotes the star or reports the capacity error), -3
// when a filter-only kernel meets an undecided predicate (nothing changed).
template <class C, bool EXACT>
__device__ int warp_insert(WS<C>& S, int lane, int s, double3 ps, int sp, int gen, const PredSink& sink,
                           unsigned* exact, double bound) {
    using Idx = typename C::Idx;
    unsigned* err = sink.err;
    const double3 pp = wpt(S, sp);
    const int pid = wid(S, sp);
    const int ntri = S.ntri;
    int nb = 0, nedge = 0;
    if (ntri <= 32) {
        // one chunk (the common case): the beneath mask, the triangle's
        // vertices and neighbours stay in registers for the boundary pass
        const int t = lane;
        bool b = false, al = false, und = false;
        int a = 0, bb = 0, c = 0;
        if (t < ntri && (S.tf[t] & 0x80)) {
            al = true;
            a = S.tv[0][t]; bb = S.tv[1][t]; c = S.tv[2][t];
            const int sg = pred_beneath<EXACT>(wpt(S, a), wpt(S, bb), wpt(S, c), ps, pp, wid(S, a), wid(S, bb),
                                               wid(S, c), s, pid, sink, exact, bound);
            b = sg < 0;
            und = sg == 0;
        }
        const unsigned m = __ballot_sync(0xffffffffu, b);
        const int nalive = __popc(__ballot_sync(0xffffffffu, al));
        if (!EXACT && __any_sync(0xffffffffu, und)) return -3;
        nb = __popc(m);
        if (nb == 0) return 0;
        if (nb == nalive) {
            if (lane == 0) {
                atomicOr(err, ERR_TOPOLOGY);
                G4D_TRACE("star %d: point %d beneath all %d triangles\n", s, pid, nalive);
            }
            return -1;
        }
        if (lane == 0) S.bmask[0] = m;
        int o0 = 0, o1 = 0, o2 = 0;
        bool e0 = false, e1 = false, e2 = false;
        if (b) {
            S.blist[__popc(m & ((1u << lane) - 1u))] = (Idx)t;
            o0 = S.to[0][t]; o1 = S.to[1][t]; o2 = S.to[2][t];
            e0 = !((m >> o0) & 1u); e1 = !((m >> o1) & 1u); e2 = !((m >> o2) & 1u);
        }
        int k = warp_excl_scan((int)e0 + (int)e1 + (int)e2, lane, &nedge);
        // edge i is the one opposite vertex i
        if (e0) { if (k < C::TS) S.erec[k] = C::rec(bb, c, o0, S.tj[0][t]); ++k; }
        if (e1) { if (k < C::TS) S.erec[k] = C::rec(c, a, o1, S.tj[1][t]); ++k; }
        if (e2) { if (k < C::TS) S.erec[k] = C::rec(a, bb, o2, S.tj[2][t]); }
    } else {
        int nalive = 0;
        bool undecided = false;
        for (int base = 0; base < ntri; base += 32) {
            const int t = base + lane;
            bool b = false, al = false, und = false;
            if (t < ntri && (S.tf[t] & 0x80)) {
                al = true;
                const int a = S.tv[0][t], bb = S.tv[1][t], c = S.tv[2][t];
                const int sg = pred_beneath<EXACT>(wpt(S, a), wpt(S, bb), wpt(S, c), ps, pp, wid(S, a), wid(S, bb),
                                                   wid(S, c), s, pid, sink, exact, bound);
                b = sg < 0;
                und = sg == 0;
            }
            const unsigned m = __ballot_sync(0xffffffffu, b);
            nalive += __popc(__ballot_sync(0xffffffffu, al));
            if (!EXACT) undecided |= __any_sync(0xffffffffu, und);
            if (lane == 0) S.bmask[base >> 5] = m;
            nb += __popc(m);
        }
        __syncwarp();
        if (!EXACT && undecided) return -3;
        if (nb == 0) return 0;
        if (nb == nalive) {
            if (lane == 0) {
                atomicOr(err, ERR_TOPOLOGY);
                G4D_TRACE("star %d: point %d beneath all %d triangles\n", s, pid, nalive);
            }
            return -1;
        }
        // beneath triangles in index order, and the hole's boundary edges
        int prefix = 0;
        for (int base = 0; base < ntri; base += 32) {
            const unsigned m = S.bmask[base >> 5];
            const int t = base + lane;
            const bool b = (m >> lane) & 1u;
            if (b) S.blist[prefix + __popc(m & ((1u << lane) - 1u))] = (Idx)t;
            prefix += __popc(m);
            // edge i (opposite vertex i) is on the hole boundary when the
            // triangle across it is not beneath
            int o[3] = {0, 0, 0};
            bool e[3] = {false, false, false};
            if (b) {
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    o[i] = S.to[i][t];
                    e[i] = !((S.bmask[o[i] >> 5] >> (o[i] & 31)) & 1u);
                }
            }
            int total;
            int k = nedge + warp_excl_scan((int)e[0] + (int)e[1] + (int)e[2], lane, &total);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (e[i]) {
                    if (k < C::TS) S.erec[k] = C::rec(S.tv[(i + 1) % 3][t], S.tv[(i + 2) % 3][t], o[i], S.tj[i][t]);
                    ++k;
                }
            nedge += total;
        }
    }
    __syncwarp();
    const int B = nedge;
    if (B > C::HM) {  // a disk's boundary visits each link vertex at most once
        if (lane == 0) {
            atomicOr(err, ERR_TOPOLOGY);
            G4D_TRACE("star %d: point %d hole boundary of %d edges\n", s, pid, B);
        }
        return -1;
    }
    const int nfree = S.nfree;
    // the B new triangles reuse the nb holes first, then free slots, then append
    const int extra = B - nb;
    const int from_free = extra > 0 ? (extra < nfree ? extra : nfree) : 0;
    const int appended = extra > 0 ? extra - from_free : 0;
    if (ntri + appended > C::TM) return -2;
    for (int r = lane; r < B; r += 32) {
        const typename C::Rec e = S.erec[r];
        const int u = C::rec_u(e), w = C::rec_w(e);
        int slot;
        if (r < nb) {
            slot = S.blist[r];
        } else {
            const int rr = r - nb;
            slot = rr < nfree ? S.fstack[nfree - 1 - rr] : ntri + (rr - nfree);
        }
        S.efrom[S.cix[u]] = (Idx)slot;
        S.eto[S.cix[w]] = (Idx)slot;
    }
    __syncwarp();
    // new triangle (u, w, p) replaces the beneath triangle across the edge u->w
    for (int r = lane; r < B; r += 32) {
        const typename C::Rec e = S.erec[r];
        const int u = C::rec_u(e), w = C::rec_w(e), o = C::rec_o(e), oj = C::rec_oj(e);
        const int slot = S.efrom[S.cix[u]];
        S.tv[0][slot] = (typename C::Slot)u;
        S.tv[1][slot] = (typename C::Slot)w;
        S.tv[2][slot] = (typename C::Slot)sp;
        S.to[0][slot] = S.efrom[S.cix[w]];  // edge (w, p): the next boundary edge's triangle
        S.tj[0][slot] = 1;
        S.to[1][slot] = S.eto[S.cix[u]];    // edge (p, u): the previous boundary edge's triangle
        S.tj[1][slot] = 0;
        S.to[2][slot] = (Idx)o;      // edge (u, w): the triangle outside the hole
        S.tj[2][slot] = (uint8_t)oj;
        if (oj < 3) {
            S.to[oj][o] = (Idx)slot;
            S.tj[oj][o] = 2;
        }
        S.tf[slot] = (uint8_t)(0x80 | gen);
    }
    __syncwarp();
    if (B < nb) {
        for (int r = B + lane; r < nb; r += 32) {
            const int t = S.blist[r];
            S.tf[t] = 0;
            S.fstack[nfree + (r - B)] = (Idx)t;
        }
    }
    __syncwarp();
    if (lane == 0) {
        if (B < nb) {
            S.nfree = nfree + (nb - B);
        } else {
            S.nfree = nfree - from_free;
            S.ntri = ntri + appended;
        }
    }
    __syncwarp();
    return 1;
}

// cone of the pentachoron (l0..l3, star): the link triangles of the 4-simplex
// (GDelPredKernels.cu:45-158), oriented so that orient4(tri, star, opposite) > 0
// returns 0, or -3 when a filter-only kernel cannot orient the pentachoron
template <class C, bool EXACT>
__device__ int warp_cone(WS<C>& S, int lane, int s, double3 ps, const int* l4, int gen, const PredSink& sink,
                         unsigned* exact) {
    int l[4] = {l4[0], l4[1], l4[2], l4[3]};
    const int o = pred_cone<EXACT>(wpt(S, l[0]), wpt(S, l[1]), wpt(S, l[2]), wpt(S, l[3]), ps, wid(S, l[0]),
                               wid(S, l[1]), wid(S, l[2]), wid(S, l[3]), s, sink, exact);
    if (!EXACT && o == 0) return -3;
    if (o < 0) { const int t = l[0]; l[0] = l[1]; l[1] = t; }
    if (lane < 4) {
        const int F[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
        const int f = lane;
        for (int i = 0; i < 3; ++i) {
            S.tv[i][f] = (typename C::Slot)l[F[f][i]];
            const int b = F[f][i];  // the face omitting vertex F[f][i] shares this edge
            S.to[i][f] = (typename C::Idx)b;
            int j = 0;
            for (int k = 0; k < 3; ++k)
                if (F[b][k] == f) j = k;
            S.tj[i][f] = (uint8_t)j;
        }
        S.tf[f] = (uint8_t)(0x80 | gen);
    }
    if (lane == 0) {
        S.ntri = 4;
        S.nfree = 0;
    }
    __syncwarp();
    return 0;
}

// sort order[0..n) by okey ascending (bitonic over a power of two <= HM + 1)
template <class C>
__device__ void warp_sort_order(WS<C>& S, int lane, int n) {
    int m = 1;
    while (m < n) m <<= 1;
    for (int i = n + lane; i < m; i += 32) { S.okey[i] = 3.0e38f; S.order[i] = 0; }
    __syncwarp();
    for (int k = 2; k <= m; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < m; i += 32) {
                const int p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const float a = S.okey[i], b = S.okey[p];
                    if ((a > b) == up) {
                        S.okey[i] = b; S.okey[p] = a;
                        const auto t = S.order[i]; S.order[i] = S.order[p]; S.order[p] = t;
                    }
                }
            }
            __syncwarp();
        }
}

// Load star s (history, coordinates, triangles) into shared memory.
template <class C>
__device__ void warp_load(WS<C>& S, const Dev& D, int lane, int s, StarHdr h, double3 base) {
    using Idx = typename C::Idx;
    if (lane == 0) {
        S.ncoord = 0;
        S.nins = 0;
    }
    __syncwarp();
    const int* gh = C::hash(D, s);
    for (int k = lane; k < C::HS; k += 32) {
        const int e = gh[k];
        S.hh[k] = e;
        const bool occ = (uint32_t)(e & (int)HID) != HEMPTY;
        // only link vertices are triangle vertices: the coordinates of
        // drowned history entries are never read
        if (occ && (e & (int)HLINK)) ws_cache_coords(S, D, k, e & (int)HID, base);
        const unsigned m = __ballot_sync(0xffffffffu, occ && (e & (int)HLINK) != 0);
        if (lane == 0) { S.wasLink[k >> 5] = m; S.insMask[k >> 5] = 0; }
    }
    const typename C::Tri* gt = C::tris(D, s);
    for (int t = lane; t < h.ntri; t += 32) {
        const typename C::Tri T = gt[t];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            S.tv[i][t] = (typename C::Slot)C::tv(T, i);
            S.to[i][t] = (Idx)C::to(T, i);
            S.tj[i][t] = (uint8_t)C::tj(T, i);
        }
        S.tf[t] = (uint8_t)(0x80 | C::gen(T));
    }
    if (lane == 0) {
        S.ntri = h.ntri;
        S.nhist = h.nhist;
        S.nfree = 0;
    }
    __syncwarp();
}

// Compact triangles, refresh link bits, report drowned points, write back.
// full: the whole history table (a star built here); otherwise only the slots
// that changed (new ids, link bits that flipped), and the triangles only when
// `created` (they changed).
template <class C>
__device__ void warp_store(WS<C>& S, const Dev& D, int lane, int s, int pass, bool created, bool full) {
    using Idx = typename C::Idx;
    const int ntri = S.ntri;
    int nalive = 0;
    // new index of each live triangle (blist reused as the map)
    for (int base = 0; base < ntri; base += 32) {
        const int t = base + lane;
        const bool al = t < ntri && (S.tf[t] & 0x80);
        const unsigned m = __ballot_sync(0xffffffffu, al);
        if (al) S.blist[t] = (Idx)(nalive + __popc(m & ((1u << lane) - 1u)));
        nalive += __popc(m);
    }
    for (int k = lane; k < C::HS; k += 32) S.hh[k] &= (int)HID;
    __syncwarp();
    for (int t = lane; t < ntri; t += 32) {
        if (!(S.tf[t] & 0x80)) continue;
        for (int i = 0; i < 3; ++i) atomicOr(&S.hh[S.tv[i][t]], (int)HLINK);
    }
    __syncwarp();
    typename C::Tri* gt = C::tris(D, s);
    for (int t = lane; t < ntri && (created || full); t += 32) {
        if (!(S.tf[t] & 0x80)) continue;
        gt[S.blist[t]] = C::pack(S.tv[0][t], S.tv[1][t], S.tv[2][t], S.tf[t] & 15, S.blist[S.to[0][t]],
                                 S.blist[S.to[1][t]], S.blist[S.to[2][t]], S.tj[0][t], S.tj[1][t], S.tj[2][t]);
    }
    // drowned: linked before or inserted now, not linked after
    int* gh = C::hash(D, s);
    for (int k = lane; k < C::HS; k += 32) {
        const int e = S.hh[k];
        const bool was = (S.wasLink[k >> 5] >> (k & 31)) & 1u, ins = (S.insMask[k >> 5] >> (k & 31)) & 1u;
        if (full || ins || was != ((e & (int)HLINK) != 0)) gh[k] = e;
        const bool occupied = (uint32_t)(e & (int)HID) != HEMPTY;
        const bool before = was || ins;
        const bool dr = occupied && before && !(e & (int)HLINK);
        const unsigned m = __ballot_sync(0xffffffffu, dr);
        if (m) {
            int base = 0;
            if (lane == 0) base = atomicAdd(&D.ctr->drown_next, __popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (dr) {
                const int pos = base + __popc(m & ((1u << lane) - 1u));
                if (pos < D.drownCap) D.drownNext[pos] = make_int2(s, e & (int)HID);
                else atomicOr(&D.ctr->err, ERR_DROWNCAP);
            }
        }
    }
    if (lane == 0) {
        StarHdr h;
        h.ntri = (uint16_t)nalive;
        h.nhist = (uint16_t)S.nhist;
        h.pass = (uint8_t)pass;
        h.flags = HDR_BUILT;
        h.spare = 0;
        D.hdr[s] = h;
        if (created) {
            const int w = atomicAdd(&D.ctr->emit_next, 1);
            D.wlEmitNext[w] = s;
        }
    }
    __syncwarp();
}

// --------------------------------------------------------------------------
// build: initial star of every point (list == null) or of the listed points
// from its candidate workset (at most BUCKET_CAP + MIN_WORKSET points). A star
// the small class cannot hold (a link of more than 64 points) is listed in
// wlBig and built again in the large class.
// --------------------------------------------------------------------------

__device__ __forceinline__ void defer(int* list, int* counter, int s) {
    const int q = atomicAdd(counter, 1);
    list[q] = s;
}

template <class C, bool EXACT>
__global__ void __launch_bounds__(32 * C::WARPS, EXACT ? C::MINB : C::MINB_BUILD)
    k_star_build(Dev D, const int* list, int count) {
    G4D_DYN_SMEM(smem_raw);
    const int lane = threadIdx.x & 31;
    WS<C>& S = reinterpret_cast<WS<C>*>(smem_raw)[threadIdx.x >> 5];
    const PredSink sink = sink_of(D);
    unsigned* err = sink.err;
    unsigned* exact = &D.ctr->exact;
    const int warps = gridDim.x * C::WARPS;
    for (int w = blockIdx.x * C::WARPS + (threadIdx.x >> 5); w < count; w += warps) {
        const int s = list ? list[w] : w;
        __syncwarp();  // the previous star's shared-memory reads are done
        for (int k = lane; k < C::HS; k += 32) S.hh[k] = (int)HEMPTY;
        for (int k = lane; k < C::HS / 32; k += 32) { S.wasLink[k] = 0; S.insMask[k] = 0; }
        if (lane == 0) { S.nins = 0; S.nhist = 0; S.ntri = 0; S.nfree = 0; S.ncoord = 0; }
        __syncwarp();
        const double3 ps = gpt(D, s);
        const double3 base = EXACT ? make_double3(0.0, 0.0, 0.0) : ps;  // of the coordinate cache
        const double3 rb = EXACT ? ps : make_double3(0.0, 0.0, 0.0);    // cached coordinate -> relative
        // candidates from the bucket
        const int bc = min(D.bucketCount[s], BUCKET_CAP);
        for (int k = lane; k < bc; k += 32) {
            const int v = D.bucket[(size_t)s * BUCKET_CAP + k];
            if (v == s || !valid_id(D, v)) continue;
            bool fresh;
            const int slot = ws_hash_insert(S, v, &fresh);
            if (fresh) {
                const int pos = atomicAdd(&S.nins, 1);
                S.order[pos] = (typename C::Slot)slot;
            }
        }
        __syncwarp();
        const int ncand = S.nins;
        __syncwarp();  // every lane has read the count before lane 0 may change it
        // pumping (GDelKernels.cu:370-477): fewer than MIN_WORKSET candidates borrow
        // from their candidates' worksets, then from the first point ids of the cloud
        if (ncand < MIN_WORKSET) {
            if (lane == 0) {
                int have = ncand;
                for (int i = 0; i < ncand && have < MIN_WORKSET; ++i) {
                    const int c = S.hh[S.order[i]] & (int)HID;
                    const int cc = min(D.bucketCount[c], BUCKET_CAP);
                    for (int k = 0; k < cc && have < MIN_WORKSET; ++k) {
                        const int v = D.bucket[(size_t)c * BUCKET_CAP + k];
                        if (v == s || !valid_id(D, v)) continue;
                        bool fresh;
                        const int slot = ws_hash_insert(S, v, &fresh);
                        if (fresh) S.order[have++] = (typename C::Slot)slot;
                    }
                }
                int lo, hi;
                cloud_range(D, s, &lo, &hi);
                for (int v = lo; v < hi && have < MIN_WORKSET; ++v) {
                    if (v == s) continue;
                    bool fresh;
                    const int slot = ws_hash_insert(S, v, &fresh);
                    if (fresh) S.order[have++] = (typename C::Slot)slot;
                }
                // reciprocal requests for the pumped points
                bool ovf = false;
                for (int i = ncand; i < have; ++i) push_inbox(D, S.hh[S.order[i]] & (int)HID, s, &ovf);
                if (ovf) atomicOr(&D.ctr->overflow, 1);
                S.nins = have;
            }
            __syncwarp();
        }
        const int nins = S.nins;
        if (nins > C::HM || nins < 4) {
            if (lane == 0) {
                atomicOr(err, nins > C::HM ? ERR_CAPACITY : ERR_TOPOLOGY);
                G4D_TRACE("star %d: %d initial candidates\n", s, nins);
            }
            continue;
        }
        // coordinates, distances, insertion order (nearest first)
        for (int i = lane; i < nins; i += 32) {
            const int slot = S.order[i];
            const int id = S.hh[slot] & (int)HID;
            ws_cache_coords(S, D, slot, id, base);
            // the same rounded differences either way
            const double3 p = wpt(S, slot);
            const double dx = p.x - rb.x, dy = p.y - rb.y, dz = p.z - rb.z;
            S.okey[i] = (float)(dx * dx + dy * dy + dz * dz);
            atomicOr(&S.insMask[slot >> 5], 1u << (slot & 31));
        }
        __syncwarp();
        if (nins <= 32) {
            // one candidate per lane: bitonic sort in registers by (distance,
            // slot), padded with +inf
            float key = lane < nins ? S.okey[lane] : 3.0e38f;
            int slot = lane < nins ? (int)S.order[lane] : 0x7fffffff;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const float ok = __shfl_xor_sync(0xffffffffu, key, j);
                    const int os = __shfl_xor_sync(0xffffffffu, slot, j);
                    const bool other_less = ok < key || (ok == key && os < slot);
                    // the lower lane of a pair keeps the smaller in an ascending block
                    const bool keep_small = ((lane & j) == 0) == ((lane & k) == 0);
                    if (keep_small == other_less) { key = ok; slot = os; }
                }
            __syncwarp();
            if (lane < nins) S.order[lane] = (typename C::Slot)slot;
        } else if (nins <= 64) {
            // two candidates per lane (element lane + 32 r in register r): the
            // same network over 64 elements; j = 32 compares a lane's own pair
            float key[2];
            int slot[2];
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                const int i = lane + 32 * r;
                key[r] = i < nins ? S.okey[i] : 3.0e38f;
                slot[r] = i < nins ? (int)S.order[i] : 0x7fffffff;
            }
#pragma unroll
            for (int k = 2; k <= 64; k <<= 1)
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    if (j == 32) {  // k = 64: ascending, register 0 keeps the smaller
                        if (key[1] < key[0] || (key[1] == key[0] && slot[1] < slot[0])) {
                            const float tk = key[0]; key[0] = key[1]; key[1] = tk;
                            const int ts = slot[0]; slot[0] = slot[1]; slot[1] = ts;
                        }
                        continue;
                    }
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        const float ok = __shfl_xor_sync(0xffffffffu, key[r], j);
                        const int os = __shfl_xor_sync(0xffffffffu, slot[r], j);
                        const bool other_less = ok < key[r] || (ok == key[r] && os < slot[r]);
                        const int i = lane + 32 * r;
                        const bool keep_small = ((lane & j) == 0) == ((i & k) == 0);
                        if (keep_small == other_less) { key[r] = ok; slot[r] = os; }
                    }
                }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < 2; ++r)
                if (lane + 32 * r < nins) S.order[lane + 32 * r] = (typename C::Slot)slot[r];
        } else {
            warp_sort_order(S, lane, nins);
        }
        if (lane == 0) S.nhist = nins;
        __syncwarp();
        const int gen = 1;
        int l4[4] = {S.order[0], S.order[1], S.order[2], S.order[3]};
        int r = warp_cone<C, EXACT>(S, lane, s, ps, l4, gen, sink, exact);
        const double bound = EXACT ? 0.0 : cache_bound(S, lane);
        for (int i = 4; i < nins && r >= 0; ++i)
            r = warp_insert<C, EXACT>(S, lane, s, ps, S.order[i], gen, sink, exact, bound);
        if (r == -3 || r == -2) {
            if (lane == 0) {
                if (r == -3) defer(D.wlExact, &D.ctr->exact_next, s);
                else if (!C::LARGE) defer(D.wlBig, &D.ctr->build_big, s);
                else atomicOr(err, ERR_CAPACITY);
            }
            continue;
        }
        if (r < 0) continue;  // error flag raised
        if (C::LARGE) {  // the star gets its large slot now
            int li = 0;
            if (lane == 0) {
                li = atomicAdd(&D.ctr->large_next, 1);
                if (li < D.largeCap) D.lidx[s] = li;
            }
            li = __shfl_sync(0xffffffffu, li, 0);
            __syncwarp();
            if (li >= D.largeCap) {
                if (lane == 0) atomicOr(err, ERR_CAPACITY);
                continue;
            }
        }
        warp_store(S, D, lane, s, gen, true, true);
        if (lane == 0) atomicAdd(&D.ctr->insertions, (unsigned long long)nins);
    }
}

// --------------------------------------------------------------------------
// insertion round: every star with inbox requests. A small star that outgrows
// its class keeps its inbox and joins the promotion list.
// --------------------------------------------------------------------------

template <class C, bool EXACT>
__global__ void __launch_bounds__(32 * C::WARPS, EXACT ? C::MINB : C::MINB_FAST)
    k_star_insert(Dev D, const int* list, int count) {
    G4D_DYN_SMEM(smem_raw);
    const int lane = threadIdx.x & 31;
    WS<C>& S = reinterpret_cast<WS<C>*>(smem_raw)[threadIdx.x >> 5];
    const PredSink sink = sink_of(D);
    unsigned* err = sink.err;
    unsigned* exact = &D.ctr->exact;
    const int warps = gridDim.x * C::WARPS;
    for (int w = blockIdx.x * C::WARPS + (threadIdx.x >> 5); w < count; w += warps) {
        __syncwarp();  // the previous item's shared-memory reads are done
        const int s = list[w];
        if (s < 0) continue;  // moved to the large class's list (k_reroute)
        const StarHdr h = D.hdr[s];
        const double3 ps = gpt(D, s);
        const double3 base = EXACT ? make_double3(0.0, 0.0, 0.0) : ps;  // of the coordinate cache
        warp_load(S, D, lane, s, h, base);
        const int ic = min(D.inboxCount[s], INBOX_CAP);
        int* box = D.inbox + (size_t)s * INBOX_CAP;
        for (int k = lane; k < ic; k += 32) {
            const int v = box[k];
            if (v == s || !valid_id(D, v)) continue;
            bool fresh;
            const int slot = ws_hash_insert(S, v, &fresh);
            if (slot < 0) { atomicOr(err, ERR_CAPACITY); continue; }
            if (fresh) {
                const int pos = atomicAdd(&S.nins, 1);
                S.order[pos < C::HM ? pos : C::HM] = (typename C::Slot)slot;
                ws_cache_coords(S, D, slot, v, base);
                atomicOr(&S.insMask[slot >> 5], 1u << (slot & 31));
            }
        }
        __syncwarp();
        const int nins = S.nins;
        const int nhist0 = S.nhist;
        __syncwarp();  // all lanes read the counts before lane 0 updates them
        bool outgrown = nhist0 + nins > C::HM, undecided = false;
        int any = 0, failed = 0;
        const int gen = (h.pass % 15) + 1;  // 1..15, differs from the stored pass
        if (!outgrown) {
            if (lane == 0) S.nhist = nhist0 + nins;
            __syncwarp();
            const double bound = EXACT ? 0.0 : cache_bound(S, lane);
            for (int i = 0; i < nins && !failed; ++i) {
                const int r = warp_insert<C, EXACT>(S, lane, s, ps, S.order[i], gen, sink, exact, bound);
                outgrown = r == -2;
                undecided = r == -3;
                failed = r < 0;
                any |= r > 0;
            }
        }
        if (undecided) {  // the exact kernel replays this star's round (inbox kept)
            if (lane == 0) defer(D.wlExact, &D.ctr->exact_next, s);
            continue;
        }
        if (outgrown) {
            if (lane == 0) {
                if (C::LARGE) {
                    atomicOr(err, ERR_CAPACITY);
                    G4D_TRACE("star %d: history %d + %d outgrows the large class\n", s, nhist0, nins);
                } else {
                    const int q = atomicAdd(&D.ctr->promote_count, 1);
                    D.wlPromote[q] = s;
                }
            }
            continue;
        }
        if (failed) continue;
        for (int k = lane; k < ic; k += 32) box[k] = -1;  // the inbox is consumed
        if (lane == 0) D.inboxCount[s] = 0;
        warp_store(S, D, lane, s, any ? gen : h.pass, any != 0, false);
        if (lane == 0) atomicAdd(&D.ctr->insertions, (unsigned long long)nins);
    }
}

// --------------------------------------------------------------------------
// promotion: copy small stars to large slots (history re-hashed into 2048
// slots, triangle vertex slots remapped, triangles widened to 16 bytes)
// --------------------------------------------------------------------------

__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK) k_promote(Dev D, int count) {
    __shared__ uint16_t smap[WARPS_PER_BLOCK][HSLOTS];
    const int lane = threadIdx.x & 31;
    uint16_t* map = smap[threadIdx.x >> 5];
    const int warps = gridDim.x * WARPS_PER_BLOCK;
    for (int w = blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5); w < count; w += warps) {
        __syncwarp();
        const int s = D.wlPromote[w];
        int li = 0;
        if (lane == 0) li = atomicAdd(&D.ctr->large_next, 1);
        li = __shfl_sync(0xffffffffu, li, 0);
        if (li >= D.largeCap) {
            if (lane == 0) atomicOr(&D.ctr->err, ERR_CAPACITY);
            continue;
        }
        int* nh = D.lhh + (size_t)li * LHSLOTS;
        for (int k = lane; k < LHSLOTS; k += 32) nh[k] = (int)HEMPTY;
        __syncwarp();
        const int* oh = D.hh + (size_t)s * HSLOTS;
        for (int k = lane; k < HSLOTS; k += 32) {
            const int e = oh[k];
            if ((uint32_t)(e & (int)HID) == HEMPTY) continue;
            uint32_t slot = hslot0<LargeStar::LOG2_HS>(e & (int)HID);
            for (int probe = 0; probe < LHSLOTS; ++probe) {
                if (atomicCAS(&nh[slot], (int)HEMPTY, e) == (int)HEMPTY) break;
                slot = (slot + 1) & (LHSLOTS - 1);
            }
            map[k] = (uint16_t)slot;
        }
        __syncwarp();
        const StarHdr h = D.hdr[s];
        const uint2* ot = D.tri + (size_t)s * TSTRIDE;
        uint4* nt = D.ltri + (size_t)li * LTSTRIDE;
        for (int t = lane; t < h.ntri; t += 32) {
            const uint2 T = ot[t];
            nt[t] = LargeStar::pack(map[tri_v(T, 0)], map[tri_v(T, 1)], map[tri_v(T, 2)], tri_gen(T), tri_o(T, 0),
                                    tri_o(T, 1), tri_o(T, 2), tri_j(T, 0), tri_j(T, 1), tri_j(T, 2));
        }
        __syncwarp();
        if (lane == 0) D.lidx[s] = li;
    }
}

// --------------------------------------------------------------------------
// emission: every link edge (u,v) of a fresh triangle asks that u and v know
// each other (GDelKernels.cu:818-939)
// --------------------------------------------------------------------------

__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK, 16) k_emit(Dev D, int count) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * WARPS_PER_BLOCK;
    for (int w = blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5); w < count; w += warps) {
        const int s = D.wlEmit[w];
        const StarHdr h = D.hdr[s];
        const StarView V = star_view(D, s);
        // ids of the fresh triangles' vertices straight from the history hash
        // (after the first round a star has few fresh triangles, so staging
        // the whole table would read far more than they need)
        const int* ids = V.hh;
        bool ovf = false;
        for (int t = lane; t < h.ntri; t += 32) {
            const TriU T = tri_get(V, t);
            if (T.gen != h.pass) continue;
            const int v0 = ids[T.v[0]] & (int)HID, v1 = ids[T.v[1]] & (int)HID, v2 = ids[T.v[2]] & (int)HID;
            // edges (v0,v1), (v1,v2), (v2,v0), each taken from the triangle
            // that lists it in increasing order
            const int ea[3] = {v0, v1, v2}, eb[3] = {v1, v2, v0};
            bool need[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                need[i] = ea[i] < eb[i];
                if (need[i] && (!valid_id(D, ea[i]) || !valid_id(D, eb[i]))) {
                    atomicOr(&D.ctr->err, ERR_TOPOLOGY);
                    need[i] = false;
                }
            }
            // Histories stay symmetric up to pending requests: every id
            // entered a's history through the initial workset (built from
            // symmetric pairs) or through a request (a <- b), and every place
            // that queues (a <- b) also checks and queues (b <- a) (overflowing
            // requests are re-sent). So b in a's history means a is in b's or
            // on its way, and only when b is missing from a's history does the
            // other direction need a lookup. The three edges' probes go out
            // together.
            HistProbe P[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                P[i].r = 1;
                if (need[i]) P[i] = hist_begin(D, ea[i], eb[i]);
            }
            for (uint32_t k = 0;; ++k) {
                bool open = false;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (P[i].r < 0) {
                        hist_step(P[i], eb[i], k);
                        open |= P[i].r < 0;
                    }
                if (!open) break;
#pragma unroll
                for (int i = 0; i < 3; ++i)
                    if (P[i].r < 0) P[i].e = (uint32_t)P[i].h[P[i].pos];
            }
#pragma unroll
            for (int i = 0; i < 3; ++i)
                if (need[i] && P[i].r == 0) {
                    push_inbox(D, ea[i], eb[i], &ovf);
                    if (hist_state(D, eb[i], ea[i]) == 0) push_inbox(D, eb[i], ea[i], &ovf);
                }
        }
        if (__ballot_sync(0xffffffffu, ovf) && lane == 0) atomicOr(&D.ctr->overflow, 1);
    }
}

// Requests queued while the initial stars were built (pumping) were routed
// before some of their stars were built in the large class: such entries move
// from the small-class list to the large-class list.
__global__ void k_reroute(Dev D, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int s = D.wlIns[i];
        if (s < 0 || D.lidx[s] < 0) continue;
        D.wlIns[i] = -1;
        const int q = atomicAdd(&D.ctr->ins_count_large, 1);
        if (q < D.largeCap) D.wlInsL[q] = s;
        else atomicOr(&D.ctr->err, ERR_CAPACITY);
    }
}

// requests that found a full inbox last round, re-sent while still needed
__global__ void k_requeue(Dev D, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int2 r = D.ovf[i];
        bool ovf = false;
        if (hist_state(D, r.x, r.y) == 0) push_inbox(D, r.x, r.y, &ovf);
    }
}

// --------------------------------------------------------------------------
// containment proofs for drowned points (GDelPredKernels.cu:427-626)
// --------------------------------------------------------------------------

// A proof is needed only while v's star still links back to s, which most
// drowned points' stars no longer do (2.5M proofs from about 35M drowned items
// on the 8M cloud): k_proof_need checks every item, one per thread (the check
// is a remote history probe, so many in flight), and lists those that need a
// proof; the proof kernels take the list, one item per warp.
__global__ void __launch_bounds__(256) k_proof_need(Dev D, const int2* __restrict__ items, int count,
                                                   int2* __restrict__ need, int* __restrict__ nneed) {
    const int lane = threadIdx.x & 31;
    const int steps = (count + 31) & ~31;  // whole warps take part in the list appends
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < steps; i += gridDim.x * blockDim.x) {
        int2 it = make_int2(-1, -1);
        bool keep = false;
        if (i < count) {
            it = items[i];
            keep = valid_id(D, it.x) && valid_id(D, it.y) && hist_state(D, it.y, it.x) == 2;
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        int base = 0;
        if (lane == 0 && m) base = atomicAdd(nneed, __popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (keep) need[base + __popc(m & ((1u << lane) - 1u))] = it;
    }
}

// Proofs of the listed items (count read on the device), one per warp.
// EXACT = false: the FP64 filter alone; an item whose search meets an
// undecided predicate is left untouched and its index queued on wlExact
// (exact_next), for the exact kernel. EXACT = true: the exact predicates, over
// the queued items, or over every item when the queue overflowed (repeating a
// proof only repeats deduplicated requests).
template <bool EXACT>
__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK, EXACT ? 4 : PROOF_BLOCKS)
    k_proof(Dev D, const int2* __restrict__ items, const int* __restrict__ nitems) {
    const int lane = threadIdx.x & 31;
    const PredSink sink = sink_of(D);
    unsigned* err = sink.err;
    unsigned* exact = &D.ctr->exact;
    const int warps = gridDim.x * WARPS_PER_BLOCK;
    int count = *(volatile const int*)nitems;
    bool from_list = false;
    if (EXACT) {
        const int queued = *(volatile int*)&D.ctr->exact_next;
        from_list = queued <= D.n;
        if (from_list) count = queued;
    }
    for (int w = blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5); w < count; w += warps) {
        const int2 item = items[from_list ? D.wlExact[w] : w];
        const int s = item.x, v = item.y;
        const StarHdr h = D.hdr[s];
        if (h.ntri == 0) continue;
        const StarView V = star_view(D, s);
        const int* ids = V.hh;  // the vertices' ids straight from the history hash
        const double3 ps = gpt(D, s), pv = gpt(D, v);
        const int ex = ids[tri_get(V, 0).v[0]] & (int)HID;
        const double3 pe = gpt(D, ex);
        int found_t = 0x7fffffff;
        int pa = -1, pb = -1, pc = -1;
        bool undecided = false;
        for (int base = 0; base < h.ntri; base += 32) {
            const int t = base + lane;
            bool ok = false, und = false;
            int a = -1, b = -1, c = -1;
            if (t < h.ntri) {
                const TriU T = tri_get(V, t);
                a = ids[T.v[0]] & (int)HID; b = ids[T.v[1]] & (int)HID; c = ids[T.v[2]] & (int)HID;
                if (a != ex && b != ex && c != ex) {
                    const double3 qa = gpt(D, a), qb = gpt(D, b), qc = gpt(D, c);
                    const int o0 = pred4<EXACT>(ps, pv, pe, qa, qb, s, v, ex, a, b, sink, exact);
                    const int o1 = pred4<EXACT>(ps, pv, pe, qb, qc, s, v, ex, b, c, sink, exact);
                    und = o0 == 0 || o1 == 0;
                    ok = !und && o0 == o1;
                    if (ok) {
                        const int o2 = pred4<EXACT>(ps, pv, pe, qc, qa, s, v, ex, c, a, sink, exact);
                        und = o2 == 0;
                        ok = !und && o1 == o2;
                    }
                }
            }
            if (!EXACT && __any_sync(0xffffffffu, und)) {
                undecided = true;
                break;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (m) {
                const int src = __ffs(m) - 1;
                found_t = base + src;
                pa = __shfl_sync(0xffffffffu, a, src);
                pb = __shfl_sync(0xffffffffu, b, src);
                pc = __shfl_sync(0xffffffffu, c, src);
                break;
            }
        }
        if (!EXACT && undecided) {
            if (lane == 0) {
                const int q = atomicAdd(&D.ctr->exact_next, 1);
                if (q < D.n) D.wlExact[q] = w;
            }
            continue;
        }
        if (found_t == 0x7fffffff) {
            if (lane == 0) {
                atomicOr(err, ERR_PROOF);
                G4D_TRACE("star %d: no containment proof for %d\n", s, v);
            }
            continue;
        }
        bool ovf = false;
        if (lane < 4) {
            const int q = lane == 0 ? ex : (lane == 1 ? pa : (lane == 2 ? pb : pc));
            if (q != v) {
                if (hist_state(D, v, q) == 0) push_inbox(D, v, q, &ovf);
                if (hist_state(D, q, v) == 0) push_inbox(D, q, v, &ovf);
            }
        }
        const unsigned anyovf = __ballot_sync(0xffffffffu, ovf);
        if (lane == 0) {
            atomicAdd(&D.ctr->proofs_total, 1ull);
            if (anyovf) atomicOr(&D.ctr->overflow, 1);
        }
    }
}

// --------------------------------------------------------------------------
// consistency check (GDelKernels.cu:1193-1271): triangle (a,b,c) of star s must
// appear as the cyclic triangle (b,s,c) in star a
// --------------------------------------------------------------------------

// slot of id v in a class-C history hash, -1 if absent
template <class C>
__device__ __forceinline__ int hash_slot(const int* h, int v) {
    uint32_t s = hslot0<C::LOG2_HS>(v);
    for (int k = 0; k < C::HS; ++k) {
        const uint32_t e = (uint32_t)h[s];
        if ((e & HID) == (uint32_t)v) return (int)s;
        if ((e & HID) == HEMPTY) return -1;
        s = (s + 1) & (C::HS - 1);
    }
    return -1;
}

// index of the triangle with vertex ids {x,y,z} (cyclic x,y,z when `cyclic`)
// in a class-C star, or -1
template <class C>
__device__ __forceinline__ int find_tri_slots(const typename C::Tri* gt, int ntri, int sx, int sy, int sz,
                                              bool cyclic) {
    // four triangles per step, loaded together (clamped to the last one)
    for (int t0 = 0; t0 < ntri; t0 += 4) {
        typename C::Tri T[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) T[u] = gt[min(t0 + u, ntri - 1)];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int a = C::tv(T[u], 0), b = C::tv(T[u], 1), c = C::tv(T[u], 2);
            bool hit;
            if (cyclic) {
                hit = (a == sx && b == sy && c == sz) || (b == sx && c == sy && a == sz) ||
                      (c == sx && a == sy && b == sz);
            } else {
                hit = (a == sx || b == sx || c == sx) && (a == sy || b == sy || c == sy) &&
                      (a == sz || b == sz || c == sz);
            }
            if (hit && t0 + u < ntri) return t0 + u;
        }
    }
    return -1;
}

template <class C>
__device__ __forceinline__ int find_tri_t(const int* h, const typename C::Tri* gt, int ntri, int x, int y, int z,
                                          bool cyclic) {
    const int sx = hash_slot<C>(h, x), sy = hash_slot<C>(h, y), sz = hash_slot<C>(h, z);
    if (sx < 0 || sy < 0 || sz < 0) return -1;
    return find_tri_slots<C>(gt, ntri, sx, sy, sz, cyclic);
}

// small-table slot of v given the entry at its first probe position
__device__ __forceinline__ int hash_slot_small(const int* h, int v, uint32_t e) {
    uint32_t s = hslot0<SmallStar::LOG2_HS>(v);
    for (int k = 0;; ++k) {
        if ((e & HID) == (uint32_t)v) return (int)s;
        if ((e & HID) == HEMPTY || k == SmallStar::HS - 1) return -1;
        s = (s + 1) & (SmallStar::HS - 1);
        e = (uint32_t)h[s];
    }
}

// triangle of `star` with vertex ids {x, y, z} in any order (and its view),
// or -1. The first probes of the small table are issued together with the
// class and size lookups, so a small star's lookup starts one round trip
// earlier.
__device__ __forceinline__ int find_tri_spec(const Dev& D, int star, int x, int y, int z, StarView* Vout) {
    const int li = D.anyLarge ? D.lidx[star] : -1;
    const int* hs = D.hh + (size_t)star * HSLOTS;
    const uint32_t ex = (uint32_t)hs[hslot0<SmallStar::LOG2_HS>(x)];
    const uint32_t ey = (uint32_t)hs[hslot0<SmallStar::LOG2_HS>(y)];
    const uint32_t ez = (uint32_t)hs[hslot0<SmallStar::LOG2_HS>(z)];
    const int ntri = D.hdr[star].ntri;
    StarView V;
    V.large = li >= 0;
    if (V.large) {
        V.hh = D.lhh + (size_t)li * LHSLOTS;
        V.tri = D.ltri + (size_t)li * LTSTRIDE;
        *Vout = V;
        return find_tri_t<LargeStar>(V.hh, static_cast<const uint4*>(V.tri), ntri, x, y, z, false);
    }
    V.hh = hs;
    V.tri = D.tri + (size_t)star * TSTRIDE;
    *Vout = V;
    const int sx = hash_slot_small(hs, x, ex), sy = hash_slot_small(hs, y, ey), sz = hash_slot_small(hs, z, ez);
    if (sx < 0 || sy < 0 || sz < 0) return -1;
    return find_tri_slots<SmallStar>(static_cast<const uint2*>(V.tri), ntri, sx, sy, sz, false);
}

__device__ int find_tri(const Dev& D, int star, int x, int y, int z, bool cyclic) {
    if (!valid_id(D, star)) return -1;
    const StarView V = star_view(D, star);
    const int ntri = D.hdr[star].ntri;
    return V.large ? find_tri_t<LargeStar>(V.hh, static_cast<const uint4*>(V.tri), ntri, x, y, z, cyclic)
                   : find_tri_t<SmallStar>(V.hh, static_cast<const uint2*>(V.tri), ntri, x, y, z, cyclic);
}

__global__ void k_check(Dev D, unsigned long long* bad) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    unsigned long long cnt = 0;
    for (int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); s < D.n; s += warps) {
        const StarHdr h = D.hdr[s];
        const StarView V = star_view(D, s);
        for (int t = lane; t < h.ntri; t += 32) {
            const TriU T = tri_get(V, t);
            const int v[3] = {V.hh[T.v[0]] & (int)HID, V.hh[T.v[1]] & (int)HID, V.hh[T.v[2]] & (int)HID};
            for (int i = 0; i < 3; ++i)
                if (find_tri(D, v[i], v[(i + 1) % 3], s, v[(i + 2) % 3], true) < 0) ++cnt;
        }
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if (lane == 0 && cnt) atomicAdd(bad, cnt);
}

// --------------------------------------------------------------------------
// extraction (GDelHost.cu:1520-1607): owner triangle (star < its 3 vertices) on
// the lower hull, orient3d(v0,v1,v2,star) < 0, is a Delaunay tetrahedron. The
// tetrahedra of star s are numbered base[s] + (rank of the triangle among the
// star's kept triangles); small stars keep a bit mask of their kept triangles
// so that any star's rank is a few popcounts.
// --------------------------------------------------------------------------

// EXACT = false: the orient3d filter alone; a star with an undecided triangle
// is left untouched and queued on wlExact for the exact kernel, which takes
// its count from the device (or every star when the queue overflowed).
template <bool EXACT>
__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK, EXACT ? 1 : 8) k_tet_count(Dev D, int* cnt) {
    const int lane = threadIdx.x & 31;
    const PredSink sink = sink_of(D);
    const int warps = gridDim.x * WARPS_PER_BLOCK;
    int count = D.n;
    bool from_list = false;
    if (EXACT) {
        const int queued = *(volatile int*)&D.ctr->exact_next;
        from_list = queued <= D.n;
        if (from_list) count = queued;
    }
    for (int w = blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5); w < count; w += warps) {
        const int s = from_list ? D.wlExact[w] : w;
        const StarHdr h = D.hdr[s];
        const StarView V = star_view(D, s);
        const int* ids = V.hh;  // the link vertices' ids straight from the history hash
        const double3 ps = gpt(D, s);
        // (an undecided sign leaves the star to the exact kernel, which
        // rewrites every kept bit and the count)
        int c = 0;
        bool undecided = false;
        for (int b0 = 0; b0 < h.ntri; b0 += 32) {
            const int t = b0 + lane;
            bool keep = false, und = false;
            if (t < h.ntri) {
                const TriU T = tri_get(V, t);
                const int a = ids[T.v[0]] & (int)HID, b = ids[T.v[1]] & (int)HID, cc = ids[T.v[2]] & (int)HID;
                if (s < a && s < b && s < cc) {
                    const int sg = EXACT ? orient3d(gpt(D, a), gpt(D, b), gpt(D, cc), ps, sink)
                                         : orient3d_filter(gpt(D, a), gpt(D, b), gpt(D, cc), ps);
                    keep = sg < 0;
                    und = sg == 0;
                }
                tri_set_kept(V, t, keep);
            }
            if (!EXACT && __any_sync(0xffffffffu, und)) {
                undecided = true;
                break;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (!V.large && lane == 0) D.keptMask[(size_t)s * (TSTRIDE / 32) + (b0 >> 5)] = m;
            c += keep;
        }
        if (undecided) {
            if (lane == 0) {
                const int q = atomicAdd(&D.ctr->exact_next, 1);
                if (q < D.n) D.wlExact[q] = s;
            }
            continue;
        }
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) cnt[s] = c;
    }
}

// tet id of triangle ti of `star` when it is kept (a tetrahedron owned by the
// star), else -1
__device__ __forceinline__ int kept_tet_id(const Dev& D, const int* base, int star, const StarView& V, int ti) {
    if (!V.large) {
        const uint32_t* m = D.keptMask + (size_t)star * (TSTRIDE / 32);
        const uint4 mw = *reinterpret_cast<const uint4*>(m);  // TSTRIDE / 32 == 4 words
        const uint32_t w[4] = {mw.x, mw.y, mw.z, mw.w};
        const int q = ti >> 5;
        const uint32_t cur = q == 0 ? w[0] : (q == 1 ? w[1] : (q == 2 ? w[2] : w[3]));
        if (!((cur >> (ti & 31)) & 1u)) return -1;
        int r = __popc(cur & ((1u << (ti & 31)) - 1u));
        r += (q > 0 ? __popc(w[0]) : 0) + (q > 1 ? __popc(w[1]) : 0) + (q > 2 ? __popc(w[2]) : 0);
        return base[star] + r;
    }
    if (!tri_kept(V, ti)) return -1;
    int r = 0;
    for (int t = 0; t < ti; ++t) r += tri_kept(V, t);
    return base[star] + r;
}

// tet id of the kept tetrahedron owned by `star` (its smallest vertex) whose
// other vertices are {x,y,z}, or -1
__device__ int owned_tet_id(const Dev& D, const int* base, int star, int x, int y, int z) {
    if (!valid_id(D, star)) return -1;
    StarView V;
    const int ti = find_tri_spec(D, star, x, y, z, &V);
    return ti < 0 ? -1 : kept_tet_id(D, base, star, V, ti);
}

// star m's link triangle ta and the triangle beyond its edge opposite vertex
// id s: returns that triangle's index and sets *y to its vertex not in {a, b}
template <class C>
__device__ __forceinline__ int across_t(const int* h, const typename C::Tri* gt, int ta, int s, int a, int b, int* y) {
    const typename C::Tri A = gt[ta];
    const int i0 = h[C::tv(A, 0)] & (int)HID, i1 = h[C::tv(A, 1)] & (int)HID;
    const int pos = i0 == s ? 0 : (i1 == s ? 1 : 2);
    const int ni = C::to(A, pos);
    const typename C::Tri N = gt[ni];
    const int n0 = h[C::tv(N, 0)] & (int)HID, n1 = h[C::tv(N, 1)] & (int)HID, n2 = h[C::tv(N, 2)] & (int)HID;
    *y = (n2 != a && n2 != b) ? n2 : ((n1 != a && n1 != b) ? n1 : n0);
    return ni;
}

// Neighbour links between tetrahedra of different owners are resolved once,
// by one side, which writes its own link and queues the other side's on the
// fix list (tet id * 4 + vertex slot, value), applied by k_tet_fix:
//  - across a face that contains the owner s, towards a neighbour owned by a
//    smaller x: left to x (for x's tetrahedron the face is the one opposite
//    its owner, handled below);
//  - across the face (v0, v1, v2) opposite s: through m, the smallest of v0,
//    v1, v2, the link triangle {a, s, b} of star m and the one beyond its
//    edge (a, b), {a, b, y}. If y > m that triangle is the neighbour (owned by
//    m, vertex y opposite the face); otherwise the neighbour is owned by y and
//    the face is opposite y in it too, so the side with the smaller owner
//    does the second lookup and writes both links.
__device__ __forceinline__ void push_fix(const Dev& D, int2* fix, int tet, int slot, int value) {
    const int q = atomicAdd(&D.ctr->fix_next, 1);
    fix[q] = make_int2(tet * 4 + slot, value);
}

// link of tetrahedron `self` (vertices v0, v1, v2, s; s smallest) across the
// face (v0, v1, v2): the neighbour's id, or -1 (no neighbour, or written later
// through the fix list by the neighbour's owner)
__device__ int face_neighbor(const Dev& D, const int* base, int2* fix, int self, int s, int v0, int v1, int v2) {
    const int m = min(v0, min(v1, v2));
    const int a = m == v0 ? v1 : v0, b = m == v2 ? v1 : v2;
    if (!valid_id(D, m)) return -1;
    StarView V;
    const int ta = find_tri_spec(D, m, a, s, b, &V);
    if (ta < 0) return -1;
    int y = -1;
    const int ni = V.large ? across_t<LargeStar>(V.hh, static_cast<const uint4*>(V.tri), ta, s, a, b, &y)
                           : across_t<SmallStar>(V.hh, static_cast<const uint2*>(V.tri), ta, s, a, b, &y);
    if (y > m) {
        const int nid = kept_tet_id(D, base, m, V, ni);
        if (nid < 0) return -1;
        // the neighbour's vertex slot of y
        const TriU N = tri_get(V, ni);
        const int j = (V.hh[N.v[0]] & (int)HID) == y ? 0 : ((V.hh[N.v[1]] & (int)HID) == y ? 1 : 2);
        push_fix(D, fix, nid, j, self);
        return nid;
    }
    if (y < s) return -1;  // y's side resolves this face
    const int nid = owned_tet_id(D, base, y, m, a, b);
    if (nid >= 0) push_fix(D, fix, nid, 3, self);
    return nid;
}

// tetrahedra owned by star s (a warp)
template <class C>
__device__ __forceinline__ void write_star(const Dev& D, const int* base, g4d_tet* tets, const int* sorted_to_input,
                                           int4* face, int s, int ntri, const int* ids, const typename C::Tri* gt,
                                           uint16_t* rank, int lane) {
    int pre = 0;
    for (int b0 = 0; b0 < ntri; b0 += 32) {
        const int t = b0 + lane;
        const bool kept = t < ntri && C::kept(gt[t]);
        const unsigned m = __ballot_sync(0xffffffffu, kept);
        if (t < ntri) rank[t] = (uint16_t)(pre + __popc(m & ((1u << lane) - 1u)));
        pre += __popc(m);
    }
    __syncwarp();
    for (int t = lane; t < ntri; t += 32) {
        const typename C::Tri T = gt[t];
        if (!C::kept(T)) continue;
        const int sl[3] = {C::tv(T, 0), C::tv(T, 1), C::tv(T, 2)};
        const int v[3] = {ids[sl[0]] & (int)HID, ids[sl[1]] & (int)HID, ids[sl[2]] & (int)HID};
        g4d_tet out;
        // neighbours across the faces that contain s: adjacent link triangles
        for (int i = 0; i < 3; ++i) {
            const int oi = C::to(T, i);
            const typename C::Tri N = gt[oi];
            const int e1 = sl[(i + 1) % 3], e2 = sl[(i + 2) % 3];
            int xs = C::tv(N, 0);
            for (int k = 0; k < 3; ++k)
                if (C::tv(N, k) != e1 && C::tv(N, k) != e2) xs = C::tv(N, k);
            const int x = ids[xs] & (int)HID;
            // a neighbour owned by x < s is linked by x's side
            out.opp[i] = (x > s && C::kept(N)) ? base[s] + rank[oi] : -1;
        }
        out.opp[3] = -1;  // k_tet_face3
        face[base[s] + rank[t]] = make_int4(s, v[0], v[1], v[2]);
        if (sorted_to_input) {
            out.v[0] = sorted_to_input[v[0]];
            out.v[1] = sorted_to_input[v[1]];
            out.v[2] = sorted_to_input[v[2]];
            out.v[3] = sorted_to_input[s];
        } else {
            out.v[0] = v[0]; out.v[1] = v[1]; out.v[2] = v[2]; out.v[3] = s;
        }
        tets[base[s] + rank[t]] = out;
    }
}

// tetrahedra owned by small star s (a warp), one neighbour per lane: the kept
// triangles are listed by rank, then lane k finds the neighbour across face
// k%3 of kept triangle k/3 (the faces that contain the owner; the face
// opposite it is k_tet_face3's), then each lane writes whole tetrahedra.
// buf: 128 B ranks, 128 B kept list, 3 ints per kept triangle.
__device__ __forceinline__ void write_star_small(const Dev& D, const int* base, g4d_tet* tets,
                                                 const int* sorted_to_input, int4* face, int s, int ntri,
                                                 const int* ids, const uint2* gt, uint8_t* buf, int lane) {
    uint8_t* rank = buf;
    uint8_t* kt = buf + 128;
    int* opp = reinterpret_cast<int*>(buf + 256);
    int nk = 0;
    for (int b0 = 0; b0 < ntri; b0 += 32) {
        const int t = b0 + lane;
        const bool kept = t < ntri && SmallStar::kept(gt[t]);
        const unsigned m = __ballot_sync(0xffffffffu, kept);
        const int r = nk + __popc(m & ((1u << lane) - 1u));
        if (t < ntri) rank[t] = (uint8_t)r;
        if (kept) kt[r] = (uint8_t)t;
        nk += __popc(m);
    }
    __syncwarp();
    const int bs = base[s];
    for (int k = lane; k < 3 * nk; k += 32) {
        const int r3 = k / 3, f = k - 3 * r3;
        const uint2 T = gt[kt[r3]];
        const int s0 = SmallStar::tv(T, 0), s1 = SmallStar::tv(T, 1), s2 = SmallStar::tv(T, 2);
        // across the face (s, v[f+1], v[f+2]): the adjacent link triangle
        const int oi = SmallStar::to(T, f);
        const uint2 N = gt[oi];
        const int e1 = f == 0 ? s1 : (f == 1 ? s2 : s0), e2 = f == 0 ? s2 : (f == 1 ? s0 : s1);
        const int n0 = SmallStar::tv(N, 0), n1 = SmallStar::tv(N, 1), n2 = SmallStar::tv(N, 2);
        const int xs = (n2 != e1 && n2 != e2) ? n2 : ((n1 != e1 && n1 != e2) ? n1 : n0);
        const int x = ids[xs] & (int)HID;
        // a neighbour owned by x < s is linked by x's side
        opp[k] = (x > s && SmallStar::kept(N)) ? bs + rank[oi] : -1;
    }
    __syncwarp();
    for (int r = lane; r < nk; r += 32) {
        const uint2 T = gt[kt[r]];
        const int v0 = ids[SmallStar::tv(T, 0)] & (int)HID, v1 = ids[SmallStar::tv(T, 1)] & (int)HID,
                  v2 = ids[SmallStar::tv(T, 2)] & (int)HID;
        g4d_tet out;
        if (sorted_to_input) {
            out.v[0] = sorted_to_input[v0];
            out.v[1] = sorted_to_input[v1];
            out.v[2] = sorted_to_input[v2];
            out.v[3] = sorted_to_input[s];
        } else {
            out.v[0] = v0; out.v[1] = v1; out.v[2] = v2; out.v[3] = s;
        }
        out.opp[0] = opp[3 * r];
        out.opp[1] = opp[3 * r + 1];
        out.opp[2] = opp[3 * r + 2];
        out.opp[3] = -1;  // k_tet_face3
        tets[bs + r] = out;
        face[bs + r] = make_int4(s, v0, v1, v2);
    }
}

__global__ void __launch_bounds__(32 * WARPS_PER_BLOCK) k_tet_write(Dev D, const int* base, g4d_tet* tets,
                                                                    const int* sorted_to_input, int4* face) {
    // large stars: triangle ranks; small stars: write_star_small's buffer
    __shared__ __align__(16) uint16_t srank[WARPS_PER_BLOCK][LTSTRIDE];
    static_assert(256 + 4 * TMAX * sizeof(int) <= LTSTRIDE * sizeof(uint16_t), "small-star output buffer");
    const int lane = threadIdx.x & 31;
    uint16_t* rank = srank[threadIdx.x >> 5];
    const int warps = gridDim.x * WARPS_PER_BLOCK;
    for (int s = blockIdx.x * WARPS_PER_BLOCK + (threadIdx.x >> 5); s < D.n; s += warps) {
        __syncwarp();  // the previous star's shared-memory reads are done
        const StarHdr h = D.hdr[s];
        const StarView V = star_view(D, s);
        const int* ids = V.hh;  // the link vertices' ids straight from the history hash
        if (!V.large)
            write_star_small(D, base, tets, sorted_to_input, face, s, h.ntri, ids, static_cast<const uint2*>(V.tri),
                             reinterpret_cast<uint8_t*>(rank), lane);
        else
            write_star<LargeStar>(D, base, tets, sorted_to_input, face, s, h.ntri, ids,
                                  static_cast<const uint4*>(V.tri), rank, lane);
    }
}

// the link across the face opposite the owner, one tetrahedron per thread
// (item: owner s and the other three vertices, written by k_tet_write); every
// lane does a remote lookup, so they overlap
__global__ void k_tet_face3(Dev D, const int* __restrict__ base, g4d_tet* tets, const int4* __restrict__ face,
                            int ntet, int2* fix) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        const int4 it = face[t];
        const int o = face_neighbor(D, base, fix, t, it.x, it.y, it.z, it.w);
        if (o >= 0) tets[t].opp[3] = o;
    }
}

// neighbour links queued by the other side (after every record is written)
__global__ void k_tet_fix(Dev D, g4d_tet* tets, const int2* __restrict__ fix) {
    const int n = *(volatile int*)&D.ctr->fix_next;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int2 f = fix[i];
        tets[f.x >> 2].opp[f.x & 3] = f.y;
    }
}

// training labels of the learned proposal: (s, v) is an edge of the final
// triangulation when v is in the final link of s
__global__ void k_ring_labels(Dev D, const int2* __restrict__ pair, const int* __restrict__ rows, int cap,
                              float* __restrict__ y) {
    const int n = min(*rows, cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        y[i] = hist_state(D, pair[i].x, pair[i].y) == 2 ? 1.f : 0.f;
}

#ifndef G4D_HOST_EMULATION
void launch_ring_labels(const Launch& L, const Dev& D, const int2* pair, const int* rows, int cap, float* y) {
    int b = (cap + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    k_ring_labels<<<b < 1 ? 1 : b, 256, 0, L.stream>>>(D, pair, rows, cap, y);
    ++*L.launches;
}

// --------------------------------------------------------------------------
// diagnostic predicate evaluation
// --------------------------------------------------------------------------

__global__ void k_eval_pred(int kind, const double* pts, const int* idx, int count, int8_t* out, unsigned* errw) {
    PredSink err;
    err.err = errw;
    err.dbg_set = nullptr;
    err.dbg_pts = nullptr;
    err.dbg_ids = nullptr;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        if (kind == 0) {
            const double* p = pts + 12 * (size_t)i;
            out[i] = (int8_t)orient3d(make_double3(p[0], p[1], p[2]), make_double3(p[3], p[4], p[5]),
                                      make_double3(p[6], p[7], p[8]), make_double3(p[9], p[10], p[11]), err);
        } else {
            const double* p = pts + 15 * (size_t)i;
            double3 q[5];
            for (int k = 0; k < 5; ++k) q[k] = make_double3(p[3 * k], p[3 * k + 1], p[3 * k + 2]);
            if (kind == 1) {
                const int* id = idx + 5 * (size_t)i;
                out[i] = (int8_t)orient4(q[0], q[1], q[2], q[3], q[4], id[0], id[1], id[2], id[3], id[4], err,
                                         nullptr);
            } else {
                int f = orient4_filter(q[0], q[1], q[2], q[3], q[4]);
                if (!f) {
                    IntPts<2> P;
                    if (to_int_points<2>(q, 5, P)) f = orient4_int<2>(P);
                    else {
                        IntPts<4> P4;
                        if (to_int_points<4>(q, 5, P4)) f = orient4_int<4>(P4);
                        else atomicOr(errw, PRED_ERR_PRECISION);
                    }
                }
                out[i] = (int8_t)f;
            }
        }
    }
}

void launch_eval_pred(const Launch& L, int kind, const double* pts, const int* idx, int count, int8_t* out,
                      unsigned* err) {
    int b = (count + 127) / 128;
    if (b > 148 * 8) b = 148 * 8;
    k_eval_pred<<<b < 1 ? 1 : b, 128, 0, L.stream>>>(kind, pts, idx, count, out, err);
    ++*L.launches;
}

// --------------------------------------------------------------------------

static int star_blocks(int items, int warps_per_block = WARPS_PER_BLOCK, int per_sm = 8) {
    int b = (items + warps_per_block - 1) / warps_per_block;
    const int cap = 148 * per_sm;
    if (b > cap) b = cap;
    return b < 1 ? 1 : b;
}

template <class C, bool EXACT, class K>
static void launch_star(const Launch& L, K kernel, const Dev& D, const int* list, int count) {
    const size_t sm = sizeof(WS<C>) * C::WARPS;
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    const int per_sm = C::LARGE ? 1 : 8;
    kernel<<<star_blocks(count, C::WARPS, per_sm), 32 * C::WARPS, sm, L.stream>>>(D, list, count);
    ++*L.launches;
}

void launch_star_build(const Launch& L, const Dev& D, const int* list, int count, bool exact) {
    const int c = list ? count : D.n;
    if (exact) launch_star<SmallStar, true>(L, k_star_build<SmallStar, true>, D, list, c);
    else launch_star<SmallStar, false>(L, k_star_build<SmallStar, false>, D, list, c);
}

void launch_star_build_large(const Launch& L, const Dev& D, const int* list, int count) {
    launch_star<LargeStar, true>(L, k_star_build<LargeStar, true>, D, list, count);
}

void launch_star_insert(const Launch& L, const Dev& D, const int* list, int count, bool exact) {
    if (exact) launch_star<SmallStar, true>(L, k_star_insert<SmallStar, true>, D, list, count);
    else launch_star<SmallStar, false>(L, k_star_insert<SmallStar, false>, D, list, count);
}

void launch_star_insert_large(const Launch& L, const Dev& D, const int* list, int count) {
    launch_star<LargeStar, true>(L, k_star_insert<LargeStar, true>, D, list, count);
}

void launch_promote(const Launch& L, const Dev& D, int count) {
    k_promote<<<star_blocks(count), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, count);
    ++*L.launches;
}

void launch_requeue(const Launch& L, const Dev& D, int count) {
    int b = (count + 127) / 128;
    if (b > 148 * 8) b = 148 * 8;
    k_requeue<<<b < 1 ? 1 : b, 128, 0, L.stream>>>(D, count);
    ++*L.launches;
}

void launch_emit(const Launch& L, const Dev& D, int count) {
    k_emit<<<star_blocks(count, WARPS_PER_BLOCK, 16), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, count);
    ++*L.launches;
}

void launch_reroute(const Launch& L, const Dev& D, int count) {
    int blocks = (count + 255) / 256;
    if (blocks > 148 * 4) blocks = 148 * 4;
    k_reroute<<<blocks, 256, 0, L.stream>>>(D, count);
    ++*L.launches;
}

void launch_proof(const Launch& L, const Dev& D, int count) {
    // the items that need a proof into the next round's drowned list (free
    // until the insertion kernels refill it), then the filter-only pass over
    // them, then the exact pass over what it left (counts read on the device,
    // so no host round trip), then the queue is emptied for the star kernels
    int* nneed = &D.ctr->proof_next;
    cudaMemsetAsync(nneed, 0, sizeof(int), L.stream);
    int b = (count + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    k_proof_need<<<b < 1 ? 1 : b, 256, 0, L.stream>>>(D, D.drown, count, D.drownNext, nneed);
    const int upper = count / 4 + 1;  // grid of the proof kernels (grid-stride over the device count)
    k_proof<false><<<star_blocks(upper), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, D.drownNext, nneed);
    k_proof<true><<<star_blocks(upper, WARPS_PER_BLOCK, 4), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, D.drownNext, nneed);
    cudaMemsetAsync(&D.ctr->exact_next, 0, sizeof(int), L.stream);
    *L.launches += 3;
}

void launch_check(const Launch& L, const Dev& D, unsigned long long* bad) {
    k_check<<<star_blocks(D.n), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, bad);
    ++*L.launches;
}

void launch_tet_count(const Launch& L, const Dev& D, int* cnt) {
    // filter-only pass, then the exact pass over the stars it left (count read
    // on the device), then the queue is emptied
    cudaMemsetAsync(&D.ctr->exact_next, 0, sizeof(int), L.stream);
    k_tet_count<false><<<star_blocks(D.n), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, cnt);
    k_tet_count<true><<<star_blocks(D.n, WARPS_PER_BLOCK, 2), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, cnt);
    cudaMemsetAsync(&D.ctr->exact_next, 0, sizeof(int), L.stream);
    *L.launches += 2;
}

void launch_tet_write(const Launch& L, const Dev& D, const int* base, g4d_tet* tets, const int* sorted_to_input,
                      int4* face, int ntet, int2* fix) {
    cudaMemsetAsync(&D.ctr->fix_next, 0, sizeof(int), L.stream);
    k_tet_write<<<star_blocks(D.n, WARPS_PER_BLOCK, 10), 32 * WARPS_PER_BLOCK, 0, L.stream>>>(D, base, tets, sorted_to_input, face);
    int blocks = (ntet + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    if (blocks < 1) blocks = 1;
    k_tet_face3<<<blocks, 256, 0, L.stream>>>(D, base, tets, face, ntet, fix);
    *L.launches += 2;
}

void launch_tet_fix(const Launch& L, const Dev& D, g4d_tet* tets, const int2* fix) {
    k_tet_fix<<<148 * 8, 256, 0, L.stream>>>(D, tets, fix);
    ++*L.launches;
}
#endif  // G4D_HOST_EMULATION

}  // namespace g4d
