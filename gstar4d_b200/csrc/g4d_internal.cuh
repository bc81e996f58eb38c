// Internal layouts and launch declarations of the B200 gStar4D pipeline.
//
// HBM layout (n points, G^3 grid):
//   P        double4[n]     points in Morton order (x,y,z,0): one 32-byte sector each
//   vox      uint32[n]      voxel of each point, packed x | y<<10 | z<<20
//   grid A   uint32[G^3]    digital Voronoi sites, packed voxel coords, x fastest
//   grid B   uint32[G^3]    scratch of the envelope passes, then the voxel ->
//                           leader-id map of the pair scan
//   hh       int32[n*256]   per-star history hash: every point ever inserted in the
//                           star (bit 31 = currently in the link), open addressing
//   tri      uint2[n*128]   per-star link triangles, 8 bytes each (packing below)
//   lhh/ltri                the same for the few stars promoted to the large class
//                           (4096 hash slots, 2048 triangles of 16 bytes)
//   hdr      StarHdr[n]     triangle count, history count, pass number, flags
//   bucket   int32[n*64]    initial candidate worksets (Voronoi pairs + missing)
//   inbox    int32[n*64]    insertion requests for the next splaying round
#pragma once

#ifndef G4D_HOST_EMULATION
#include <cuda_runtime.h>
#endif

#include <cstdint>

#include "gstar4d.h"

// Dynamic shared memory declaration (a host build of the warp kernels for
// unit testing supplies its own definition).
#ifndef G4D_DYN_SMEM
#define G4D_DYN_SMEM(name) extern __shared__ unsigned char name[]
#endif
// Error-site tracing hook (empty on the device; the host build prints).
#ifndef G4D_TRACE
#define G4D_TRACE(...) ((void)0)
#endif

namespace g4d {

constexpr uint32_t MARKER = 0xffffffffu;  // voxel without a site
// Two star storage classes. Every star starts in the small class; a star whose
// history or link outgrows it (points next to a dense sheet of points, e.g. a
// sampled sphere) moves to the large class between kernels.
constexpr int HSLOTS = 256;               // small: history hash slots per star
constexpr int HMAX = 127;                 // small: max history entries (hash load <= 1/2)
constexpr int TMAX = 124;                 // small: max link triangles (a link of 64 points)
constexpr int TSTRIDE = 128;              // small: triangle slots per star in HBM
constexpr int LHSLOTS = 4096;             // large: history hash slots
constexpr int LHMAX = 2047;               // large: max history entries
constexpr int LTMAX = 2044;               // large: max link triangles
constexpr int LTSTRIDE = 2048;            // large: triangle slots in HBM
constexpr int BUCKET_CAP = 64;            // initial candidates kept per star
constexpr int INBOX_CAP = 64;             // insertion requests per star per round
constexpr int MIN_WORKSET = 8;            // GDelCommon.h:49
constexpr int BLOCK_K_DEFAULT = 16;       // voxel-block workset pairs per point
constexpr uint32_t HEMPTY = 0x7fffffffu;
constexpr uint32_t HLINK = 0x80000000u;
constexpr uint32_t HID = 0x7fffffffu;

// error bits (device error word)
enum : unsigned {
    ERR_PRECISION = 1u,
    ERR_CAPACITY = 2u,
    ERR_TOPOLOGY = 4u,   // a hole that is not a disk, or every triangle beneath
    ERR_PROOF = 8u,      // no containment proof found
    ERR_DROWNCAP = 16u,  // drowned list full
    ERR_OVFCAP = 32u,    // overflow request list full (the host grows it and repeats the emission phase)
};

// star header flags
enum : uint8_t { HDR_BUILT = 2 };

struct __align__(8) StarHdr {
    uint16_t ntri, nhist;
    uint8_t pass, flags;
    uint16_t spare;
};

// device counters (one struct in HBM, read by the host once per round)
struct Counters {
    int ins_count;        // small stars queued for insertion
    int emit_next;        // stars queued for emission next round
    int drown_next;       // drowned items for next round
    int ins_count_large;  // large stars queued for insertion
    int promote_count;    // small stars that outgrew their class this round
    int exact_next;       // stars the filter-only kernel left for the exact kernel
    int build_big;        // initial stars too large for the small class
    int large_next;       // large-class slots handed out so far
    int ovf_next;         // insertion requests that found a full inbox (next round)
    int overflow;         // inbox overflow happened
    unsigned err;         // ERR_* bits
    unsigned exact;       // exact predicate evaluations
    unsigned long long insertions;
    unsigned long long drowned_total;
    unsigned long long proofs_total;
    int tet_count;
    int proposed;         // candidate pairs the learned proposal added
    int dbg_set;          // first failing exact-predicate input recorded below
    double dbg_pts[15];
    int dbg_ids[5];
    int fix_next;         // tetra output: neighbour links written by the other side
    int block_pairs;      // workset pairs added from voxel blocks
    int proof_next;       // drowned items of this round that need a proof
    unsigned long long cand_total;  // initial star insertions at most (sum over the worksets)
};

__host__ __device__ inline uint32_t enc_vox(uint32_t x, uint32_t y, uint32_t z) { return x | (y << 10) | (z << 20); }
__host__ __device__ inline uint32_t vx(uint32_t e) { return e & 1023u; }
__host__ __device__ inline uint32_t vy(uint32_t e) { return (e >> 10) & 1023u; }
__host__ __device__ inline uint32_t vz(uint32_t e) { return (e >> 20) & 1023u; }

// first probe of id v in a history hash of 2^LOG2 slots (multiplicative hashing)
template <int LOG2>
__device__ __forceinline__ uint32_t hslot0(int v) { return ((uint32_t)v * 2654435761u) >> (32 - LOG2); }

// Small-class triangle packing in HBM (8 bytes):
//   x = v0 | v1<<9 | v2<<18 | gen<<27 | kept<<31
//   y = o0 | o1<<8 | o2<<16 | j0<<24 | j1<<26 | j2<<28
// v* are history slots (9 bits); o* the adjacent triangle across the edge
// opposite v*; j* the position of the shared edge inside that neighbour;
// gen = creation pass (4 bits, 1..15); kept = lower-hull tetra at extraction.
constexpr uint32_t TRI_KEPT = 0x80000000u;
__device__ __forceinline__ int tri_v(uint2 T, int i) { return (int)((T.x >> (9 * i)) & 511u); }
__device__ __forceinline__ int tri_gen(uint2 T) { return (int)((T.x >> 27) & 15u); }
__device__ __forceinline__ int tri_o(uint2 T, int i) { return (int)((T.y >> (8 * i)) & 255u); }
__device__ __forceinline__ int tri_j(uint2 T, int i) { return (int)((T.y >> (24 + 2 * i)) & 3u); }
__device__ __forceinline__ uint2 tri_pack(int v0, int v1, int v2, int gen, int o0, int o1, int o2, int j0, int j1,
                                          int j2) {
    uint2 T;
    T.x = (uint32_t)v0 | ((uint32_t)v1 << 9) | ((uint32_t)v2 << 18) | ((uint32_t)(gen & 15) << 27);
    T.y = (uint32_t)o0 | ((uint32_t)o1 << 8) | ((uint32_t)o2 << 16) | ((uint32_t)j0 << 24) | ((uint32_t)j1 << 26) |
          ((uint32_t)j2 << 28);
    return T;
}

struct Dev {
    int n, G;
    const double4* P;
    const uint32_t* vox;
    const uint32_t* mkey;  // Morton keys, sorted
    const uint32_t* ckey;  // column-sorted voxel keys ((y*G+x)<<10 | z)
    const int* cid;        // column-sorted point ids
    const int* colStart;   // [G*G]
    const int* colEnd;     // [G*G]
    int* hh;
    uint2* tri;
    StarHdr* hdr;
    int* bucket;
    int* bucketCount;
    int* inbox;
    int* inboxCount;
    int* wlIns;
    int* wlEmit;
    int* wlEmitNext;
    int2* drown;
    int2* drownNext;
    int drownCap;
    Counters* ctr;
    // large star class: lidx[s] = slot in lhh/ltri, or -1 while s is small
    int* lidx;
    int* lhh;              // [largeCap * LHSLOTS]
    uint4* ltri;           // [largeCap * LTSTRIDE], packing in g4d_star.cu
    int largeCap;
    int* wlInsL;           // large stars with inbox requests
    int* wlPromote;        // small stars to move to the large class
    int* wlExact;          // stars that need the exact-predicate kernel
    int* wlBig;            // initial stars to build in the large class
    int anyLarge;          // some star is in the large class (else lidx is not read)
    uint32_t* keptMask;    // small stars: kept-triangle bits (TSTRIDE / 32 words each)
    // requests (star, point) that found the star's inbox full: re-sent next round
    int2* ovf;
    int2* ovfNext;
    int ovfCap;
    // batches: point ranges of the clouds (sorted order), nclouds + 1 offsets;
    // nclouds == 0 means one cloud [0, n)
    const int* cloudOff;
    int nclouds;
};

// column-sorted sites of one grid of a stack
template <class KeyT>
struct Cols {
    const KeyT* key;   // (column << 10) | z, sorted
    const int* cid;    // point id of each key
    const int* start;  // first key of each column of this grid
    const int* end;
    int G;
    const int* map;    // leader id at every occupied voxel of this grid, or null
};

// site (packed voxel) -> point id of the voxel's leader (smallest Morton index):
// one load from the voxel map when there is one, else a walk of its column
template <class KeyT>
__device__ __forceinline__ int site_to_id(const Cols<KeyT>& C, uint32_t e) {
    if (C.map) return C.map[((size_t)vz(e) * C.G + vy(e)) * C.G + vx(e)];
    const int c = (int)(vy(e) * (uint32_t)C.G + vx(e));
    const uint32_t z = vz(e);
    for (int j = C.start[c], je = C.end[c]; j < je; ++j)
        if ((uint32_t)(C.key[j] & 1023u) == z) return C.cid[j];
    return -1;
}

// Initial workset entry b of point a. Worksets are symmetric (b in a's <=> a in
// b's), which splaying relies on; an entry that finds a's workset full becomes
// an insertion request sent after the initial stars are built.
// entry b of a's workset at position pos (taken from bucketCount[a])
__device__ __forceinline__ void bucket_put(const Dev& D, int a, int b, int pos) {
    if (pos < BUCKET_CAP) {
        D.bucket[(size_t)a * BUCKET_CAP + pos] = b;
        return;
    }
    const int q = atomicAdd(&D.ctr->ovf_next, 1);
    if (q < D.ovfCap) D.ovfNext[q] = make_int2(a, b);
    else atomicOr(&D.ctr->err, ERR_OVFCAP);
}
__device__ __forceinline__ void bucket_push(const Dev& D, int a, int b) {
    bucket_put(D, a, b, atomicAdd(&D.bucketCount[a], 1));
}

// ---- launchers (host) --------------------------------------------------------
struct Launch {
    cudaStream_t stream;
    long long* launches;  // incremented per kernel launch
};

// order
void launch_minmax(const Launch& L, const double* xyz, int n, unsigned long long* mm);
void launch_scale_morton(const Launch& L, const double* xyz, const double* scaled_in, int n, int G,
                         const unsigned long long* mm, uint32_t* keys, int* vals, uint32_t* vox_in, unsigned* err);
void launch_gather(const Launch& L, const double* xyz, const uint32_t* vox_in, const int* order, int n,
                   double4* P, uint32_t* vox, int* sorted_to_input);
void launch_colkeys(const Launch& L, const uint32_t* vox, int n, int G, uint32_t* ckey, int* cid);
void launch_colranges(const Launch& L, const uint32_t* ckey, int n, int G, int* colStart, int* colEnd);
void launch_f32_to_f64(const Launch& L, const float* in, size_t count, double* out);

// batches (see g4d_order.cu)
void launch_b_order(const Launch& L, const double* xyz, int nslots, const long long* slotIn, const int* slotW,
                    const int* slotG, unsigned long long* mm, unsigned long long* keys, int* vals, uint32_t* vox_in,
                    long long* gidx, unsigned* err);
void launch_b_gather(const Launch& L, const double* xyz, const long long* gidx, const uint32_t* vox_in,
                     const int* order, const unsigned long long* skey, const int* slotW, int n, double4* P,
                     uint32_t* vox, int* local);
void launch_b_colkeys(const Launch& L, const uint32_t* vox, const unsigned long long* skey, const int* slotG,
                      const long long* slotCol, int n, unsigned long long* ckey, int* cid);
void launch_colranges_u64(const Launch& L, const unsigned long long* ckey, int n, int* colStart, int* colEnd);
void launch_b_occupancy(const Launch& L, const double* xyz, const long long* offs, int nclouds, int* occ);
void launch_b_slot_tets(const Launch& L, const int* base, const int* slotW, int nslots, int* tc);
void launch_b_localize(const Launch& L, const g4d_tet* in, int ntet, const unsigned long long* skey,
                       const int* local, const int* base, const int* slotW, const long long* dst, g4d_tet* out);

// pba
// Forms of the y and x passes (g4d_pba.cu): one thread per line, or lines
// staged in shared memory in tiles (4 lines per warp in both passes, 4 warps
// per block; or 2 lines per warp in the x pass, 2 warps per block). Their
// outputs are equally exact; which is fastest depends on the grid width, so
// contexts time them on the first grid of each width (g4d_api.cu).
enum PbaForm : int { PBA_LINES = 0, PBA_TILES_4 = 1, PBA_TILES_2 = 2, PBA_FORMS = 3 };
int pba_default_form(int G);
bool pba_form_ok(int form, int G);
void launch_pba_z(const Launch& L, const Dev& D, uint32_t* out);
// `in` is scratch (the line form keeps its stacks in it); form -1: the default
void launch_pba_y(const Launch& L, int G, uint32_t* in, uint32_t* out, int form = -1);
void launch_pba_x(const Launch& L, int G, uint32_t* in, uint32_t* out, int form = -1);
void launch_pairs(const Launch& L, const Dev& D, const uint32_t* grid, int* map);
void launch_site_map(const Launch& L, const Dev& D, int* map);
void launch_b_site_map(const Launch& L, const uint32_t* vox, const unsigned long long* skey, const int* slotG,
                       const long long* slotVox, int n, int* map);
void launch_missing(const Launch& L, const Dev& D);
// stacks of K grids of width G (batches; 64-bit column keys)
void launch_pba_z_stack(const Launch& L, int G, int K, const unsigned long long* ckey, const int* cs, const int* ce,
                        uint32_t* out);
void launch_pba_y_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out, int form = -1);
void launch_pba_x_stack(const Launch& L, int G, int K, uint32_t* in, uint32_t* out, int form = -1);
void launch_pairs_stack(const Launch& L, const Dev& D, const uint32_t* stack, int* map, int G, int K,
                        const unsigned long long* ckey, const int* cid, const int* cs, const int* ce);
void launch_missing_u64(const Launch& L, const Dev& D, const unsigned long long* mkey);
// workset pairs of each point with its k_sel nearest points of the 3x3x3 voxel
// block (single clouds; the insertion-request arrays serve as scratch)
void launch_block_pairs(const Launch& L, const Dev& D, const uint32_t* grid, const int* map, int k_sel);
// the same over a batch pass: point i of slot k = skey >> 30 in the grid at
// slotVox[k] (width slotG[k]) of the stacked grids and maps
void launch_block_pairs_batch(const Launch& L, const Dev& D, const uint32_t* grids, const int* maps,
                              const unsigned long long* skey, const int* slotG, const long long* slotVox, int k_sel);
// ctr->cand_total = sum over stars of the initial insertions they can make
// (the workset, pumped up to MIN_WORKSET): the initial build's drowned points
void launch_workset_total(const Launch& L, const Dev& D);

// stars
// Star kernels run first filter-only (exact = false: FP64 filter, no exact
// arithmetic in the kernel, more resident warps); a star that meets an
// undecided predicate is left untouched and listed in wlExact for the same
// kernel with exact predicates (exact = true).
void launch_star_build(const Launch& L, const Dev& D, const int* list, int count, bool exact);
void launch_star_build_large(const Launch& L, const Dev& D, const int* list, int count);
void launch_star_insert(const Launch& L, const Dev& D, const int* list, int count, bool exact);
void launch_star_insert_large(const Launch& L, const Dev& D, const int* list, int count);
void launch_promote(const Launch& L, const Dev& D, int count);
void launch_requeue(const Launch& L, const Dev& D, int count);
void launch_emit(const Launch& L, const Dev& D, int count);
void launch_proof(const Launch& L, const Dev& D, int count);
void launch_reroute(const Launch& L, const Dev& D, int count);
void launch_check(const Launch& L, const Dev& D, unsigned long long* bad);
void launch_tet_count(const Launch& L, const Dev& D, int* cnt);
void launch_tet_write(const Launch& L, const Dev& D, const int* base, g4d_tet* tets, const int* sorted_to_input,
                      int4* face, int ntet, int2* fix);
void launch_tet_fix(const Launch& L, const Dev& D, g4d_tet* tets, const int2* fix);
// learned star proposal (g4d_mlp.cu, g4d_proposal.cu)
constexpr int MLP_NPARAMS = 9473;
size_t mlp_infer_smem();
size_t mlp_train_smem();
void launch_mlp_infer(const Launch& L, const float* P, const uint16_t* X, int M, float* logits, unsigned* err);
void launch_mlp_train(const Launch& L, const float* P, const uint16_t* X, const float* Y, int M, const int* tiles,
                      int ntiles, float inv_batch, float* G, float* loss, unsigned* err);
void launch_adam(const Launch& L, float* P, float* G, float* m1, float* m2, int step, float lr);
void launch_mlp_wait_probe(const Launch& L, int limit, unsigned* err);
struct Ring {
    const uint32_t* grid;  // Voronoi sites of the cloud's grid
    Cols<uint32_t> cols;
    double scale;          // grid units per coordinate unit
    int cap;               // rows available
    int* rows;             // row counter
    int2* pair;            // [cap] (star, candidate)
    uint16_t* x;           // [cap * 16] BF16 features
    float* y;              // [cap] labels (final Delaunay edge), or null
};
void launch_ring(const Launch& L, const Dev& D, const Ring& R);
void launch_ring_labels(const Launch& L, const Dev& D, const int2* pair, const int* rows, int cap, float* y);
void launch_prop_merge(const Launch& L, const Dev& D, const int2* pair, const float* logits, const int* rows,
                       int cap, float threshold);
// mesh validator (g4d_check.cu)
size_t check_scratch_bytes(int ntet, int n);
cudaError_t run_mesh_check(cudaStream_t st, long long* launches, const double4* P, const int* order,
                           const g4d_tet* tets, int ntet, int n, void* scratch, unsigned long long* out,
                           unsigned* err);
void launch_eval_pred(const Launch& L, int kind, const double* pts, const int* idx, int count, int8_t* out,
                      unsigned* err);

}  // namespace g4d
