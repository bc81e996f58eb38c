/*
 * gStar4D-B200: C ABI of the B200-native 3D Delaunay triangulator.
 *
 * Point cloud in (FP64 x,y,z), tetrahedra with adjacency out. The entry points
 * below replace the reference's C++ facade (GDelaunay/GDelaunay.h:39-42,
 * GDelaunay/GDelaunay.cpp:47-104) with plain C types: status codes instead of
 * exit(-1), caller buffers never mutated unless the reference mutates them too,
 * one context per host thread instead of process-wide globals.
 *
 * Semantics shared with the reference:
 *  - Point indices in the output are either input indices (default) or the
 *    Morton-sorted order the reference reports (GDelData.cu:91-134).
 *  - Tetrahedron layout equals the reference's Tetrahedron (Common/Geometry.h:
 *    147-150): v[0..2] = owner link triangle, v[3] = owner star (the smallest
 *    vertex), orient3d(v0,v1,v2,v3) < 0 (GDelPredKernels.cu:628-665), opp[i] =
 *    index of the tetrahedron across the face opposite v[i], -1 if there is none.
 *  - The tetrahedra are the Delaunay tetrahedra under the reference's
 *    Simulation of Simplicity by Morton index (GDelPredDevice.h:142-698);
 *    zero-volume tetrahedra are dropped as in the reference.
 */
#ifndef GSTAR4D_H
#define GSTAR4D_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define G4D_API __attribute__((visibility("default")))
#else
#define G4D_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    G4D_OK = 0,
    G4D_ERR_ARG = 1,        /* invalid argument (sizes, grid, NULL pointers, duplicate points) */
    G4D_ERR_NOMEM = 2,      /* device or host allocation failed */
    G4D_ERR_TIMEOUT = 3,    /* an iteration cap was reached (splaying did not converge) */
    G4D_ERR_INTERNAL = 4,   /* an internal consistency check failed */
    G4D_ERR_CUDA = 5,       /* a CUDA runtime call failed */
    G4D_ERR_CAPACITY = 6,   /* a star outgrew the largest supported star size */
    G4D_ERR_PRECISION = 7,  /* coordinates span too wide a binary exponent range */
    G4D_ERR_NODEVICE = 8    /* no CUDA device, or the device is not sm_100 */
} g4d_status;

/* Mirrors the reference's Config (Common/Config.h:59-79) plus the B200 options. */
typedef struct {
    int seed;            /* -s   (CLI point generation) */
    int run_num;         /* -r */
    int grid_size;       /* -g   PBA grid width G: power of two, 32..1024; 0 = the reference's
                            density (about 134 voxels per point); -1 = autotuned (batches time
                            sample waves per size bucket and distribution; single clouds reuse
                            a width tuned on the same context) */
    int point_num;       /* -n */
    int dist;            /* -d   0 uniform, 1 gaussian, 2 ball, 3 sphere, 4 grid */
    int facet_max;       /* -f   kept for flag compatibility (no effect: no per-loop bound) */
    int log_verbose;     /* -verbose */
    int log_stats;       /* -stats */
    int log_timing;      /* -timing */
    int do_check;        /* -check: device star-consistency check after splaying */
    int pred_thread_num; /* -predThreadNum (kept for flag compatibility) */
    int pred_block_num;  /* -predBlockNum  (kept for flag compatibility) */
    int do_sorting;      /* -sort (always on: Morton order defines the SoS ranks) */
    int device;          /* CUDA device ordinal */
    int index_space;     /* 0: output indices are input indices; 1: Morton-sorted indices */
    int proposal;        /* 0: plain PBA stars; 1: learned star proposal (needs a model) */
    int max_splay_loops; /* cap on splaying loops before G4D_ERR_TIMEOUT; 0 = 4000. The
                            reference loops until the stars agree (GDelHost.cu:1393-1446) */
} g4d_config;

/* == Tetrahedron of Common/Geometry.h:147-150 */
typedef struct {
    int v[4];
    int opp[4];
} g4d_tet;

typedef struct {
    double t_init_ms, t_pba_ms, t_star_ms, t_splay_ms, t_out_ms, t_total_ms;
    long long star_insertions;   /* initial worksets inserted (LogStarInsNum) */
    long long splay_insertions;  /* insertions during splaying (LogSplayInsNum) */
    long long drowned, proofs, exact_predicates;
    int loops;                   /* splaying loops (LogLoopNum) */
    int missing;                 /* points absent from the digital Voronoi diagram */
    int grid_size;               /* grid actually used */
    int tets;
    long long gpu_launches;      /* kernels launched by this call */
    int large_stars;             /* stars that outgrew the small storage class */
    int proposed;                /* candidate pairs the learned proposal added */
    int pba_form;                /* form of the y and x passes used: 0 one thread per line,
                                    1 and 2 lines staged in shared memory (tile shapes) */
    int block_pairs;             /* workset pairs added from 3x3x3 voxel blocks */
} g4d_stats;

typedef struct g4d_ctx g4d_ctx;

/* Defaults: grid 0 (autotune), index_space 0, device 0, sorting on. */
G4D_API void g4d_default_config(g4d_config* cfg);

/* Replaces the reference's process-wide state set up by gdelInit/starsInit
 * (GDelHost.cu:136-234): one context owns a device, a stream and workspace. */
G4D_API g4d_status g4d_create(g4d_ctx** ctx, const g4d_config* cfg);
G4D_API void g4d_destroy(g4d_ctx* ctx);
G4D_API const char* g4d_last_error(const g4d_ctx* ctx);
G4D_API const char* g4d_status_string(g4d_status s);

/* One triangulation from host memory (gdelInit + gdelCompute + getTetraFromGpu,
 * GDelaunay.cpp:47-96, with Application::_scalePoint scaling, Application.cpp:
 * 589-603, of the FP64 points into grid units). xyz: n*3 doubles, input order,
 * not modified. *tets is allocated by the library (free with g4d_free).
 * sorted_to_input (optional, n ints): Morton position -> input index. */
G4D_API g4d_status g4d_triangulate(g4d_ctx* ctx, const double* xyz, int n, g4d_tet** tets, int* ntet,
                           int* sorted_to_input, g4d_stats* stats);

/* Same as g4d_triangulate but into a caller buffer (e.g. pinned host memory):
 * out may be NULL to query *ntet; returns G4D_ERR_ARG with *ntet set when cap
 * is too small. */
G4D_API g4d_status g4d_triangulate_to(g4d_ctx* ctx, const double* xyz, int n, g4d_tet* out, int cap, int* ntet,
                              int* sorted_to_input, g4d_stats* stats);

/* The same for float coordinates (the reference's default RealType =
 * float, Common/Geometry.h:53-57; Point3 = float[3]): the points are widened
 * to double on the device (exact), so the result is the triangulation of the
 * same values. The predicates stay exact, like the reference's float build;
 * for degenerate inputs the SoS ranks follow this library's double scaling. */
G4D_API g4d_status g4d_triangulate_to_f32(g4d_ctx* ctx, const float* xyz, int n, g4d_tet* out, int cap,
                                          int* ntet, int* sorted_to_input, g4d_stats* stats);

/* Same on device memory (inputs already resident in HBM, output left there).
 * d_xyz: n*3 doubles on ctx's device. The tetrahedra stay in a context-owned
 * device buffer returned through *d_tets (valid until the next call). */
G4D_API g4d_status g4d_triangulate_device(g4d_ctx* ctx, const double* d_xyz, int n, const g4d_tet** d_tets,
                                  int* ntet, g4d_stats* stats);

/* Reference-shaped entry points (GDelaunay.h:39-42).
 * g4d_gdel_init: points (n*3) are the predicate coordinates; scaled (n*3 grid
 * units in [1, G-2], or NULL when points are already in grid units) feeds the
 * grid and the Morton order. Like gdelInit (GDelData.cu:125-130) both arrays
 * are overwritten with the Morton-sorted order. */
G4D_API g4d_status g4d_gdel_init(g4d_ctx* ctx, double* points, double* scaled, int n);
/* gdelCompute: stage times in milliseconds (PBA, initial stars, splaying, output). */
G4D_API g4d_status g4d_gdel_compute(g4d_ctx* ctx, double* t_pba, double* t_star, double* t_splay, double* t_out);
/* getTetraFromGpu: tetrahedra in Morton-sorted indices; pointer valid until the
 * next compute or deinit. */
G4D_API g4d_status g4d_get_tetra(g4d_ctx* ctx, const g4d_tet** tets, int* ntet);
G4D_API g4d_status g4d_gdel_deinit(g4d_ctx* ctx);
/* Statistics of the context's last triangulation (the counters the reference
 * prints with -stats / -timing, GDelHost.cu:101-113). */
G4D_API g4d_status g4d_get_stats(const g4d_ctx* ctx, g4d_stats* stats);

/* Batched triangulation of many clouds. The reference is one cloud per process
 * with global state (GDelHost.cu:57-113), so this has no counterpart there; each
 * cloud's result is the one g4d_triangulate gives at the same grid width.
 * xyz holds all clouds back to back; cloud c spans points
 * [cloud_offsets[c], cloud_offsets[c+1]), cloud_offsets[0] = 0, at least 5
 * points each. Clouds are processed in passes of up to 8M points: one radix
 * sort over all clouds of a pass, one launch per distinct grid width for the
 * Voronoi kernels (the grids of a width are stacked), one star and splaying
 * pipeline over all of the pass's points. Tetrahedra of cloud c are
 * tets[tet_offsets[c] .. tet_offsets[c+1]) with cloud-local input indices.
 * *tets and *tet_offsets are library-allocated (g4d_free). */
G4D_API g4d_status g4d_triangulate_batch(g4d_ctx* ctx, const double* xyz, const int64_t* cloud_offsets, int nclouds,
                                 g4d_tet** tets, int64_t** tet_offsets, g4d_stats* stats);

/* The same into a caller buffer `out` of `cap` tetrahedra (pinned host memory
 * makes the copies run at full speed): each pass's tetrahedra are copied while
 * the next pass computes. tet_offsets (nclouds + 1 entries) and *ntet are set
 * in any case; when the batch has more than cap tetrahedra the call returns
 * G4D_ERR_ARG and out is incomplete. */
G4D_API g4d_status g4d_triangulate_batch_to(g4d_ctx* ctx, const double* xyz, const int64_t* cloud_offsets,
                                            int nclouds, g4d_tet* out, int64_t cap, int64_t* tet_offsets,
                                            int64_t* ntet, g4d_stats* stats);

/* The same with the points already on ctx's device (d_xyz, 3 doubles per
 * point); cloud_offsets stays on the host. The tetrahedra stay in a
 * context-owned device buffer (*d_tets) and *tet_offsets points to
 * context-owned host offsets; both stay valid until the next batch call. */
G4D_API g4d_status g4d_triangulate_batch_device(g4d_ctx* ctx, const double* d_xyz, const int64_t* cloud_offsets,
                                                int nclouds, const g4d_tet** d_tets, const int64_t** tet_offsets,
                                                g4d_stats* stats);

/* Diagnostic: evaluates the device predicates on `count` point sets (host
 * arrays). kind 0: orient3d sign of 4 points (12 doubles per set);
 * kind 1: lifted orient4 sign with Simulation of Simplicity (15 doubles and 5
 * indices per set); kind 2: orient4 without SoS (0 when degenerate). */
G4D_API g4d_status g4d_eval_predicates(g4d_ctx* ctx, int kind, const double* pts, const int* idx, int count,
                                       int8_t* out);

/* Diagnostic: the digital Voronoi diagram the star construction starts from
 * (PBA output, PBA/Pba.cu:105-122 doPba). xyz as in g4d_triangulate; sites
 * receives grid^3 values, voxel (x,y,z) at ((z*grid)+y)*grid+x, each the packed
 * voxel x | y<<10 | z<<20 of its nearest site (0xffffffff if none). */
G4D_API g4d_status g4d_voronoi(g4d_ctx* ctx, const double* xyz, int n, int grid, uint32_t* sites);

/* No counterpart in the reference. g4d_voronoi without any device allocation,
 * for callers that cannot allocate GPU memory (device memory owned by a host
 * framework's pool, or loops where cudaMalloc/cudaFree and their implicit
 * synchronization are not allowed). d_xyz (n*3 doubles) and d_sites (grid^3
 * values, layout as g4d_voronoi) are DEVICE pointers owned by the caller;
 * stream is a cudaStream_t (NULL: the legacy default stream). The work is
 * enqueued on that stream and the call returns without synchronizing.
 * Scratch is one fixed device array in the library (about 9.4 MB per device),
 * so n is at most 262144 and grid at most 128; larger sizes return
 * G4D_ERR_CAPACITY (with a message on stderr) and enqueue nothing. Every call
 * shares that array: calls that overlap on the GPU (other streams or threads)
 * race and must be serialized by the caller. The first call in each CUDA
 * context looks up the array's address (cached with the context's id, so a
 * cudaDeviceReset or another current context makes the next call look it up
 * again); make that first call outside any stream capture. The call does not
 * synchronize, so errors the device finds in the inputs (NaN or infinite
 * coordinates, all coordinates equal) are not reported: such points are
 * clamped into the grid and the result is meaningless. g4d_voronoi reports
 * them as G4D_ERR_ARG. */
G4D_API g4d_status g4d_voronoi_noalloc(const double* d_xyz, int n, int grid, uint32_t* d_sites, void* stream);

/* Learned star proposal (no counterpart in the reference). A BF16 MLP scores
 * candidate pairs (s, v) from the 5x5x5 block of the digital Voronoi grid around
 * each point; with config.proposal = 1 the accepted pairs join the initial
 * worksets. Splaying with exact predicates still decides every star, so the
 * tetrahedra do not change; only the splaying work does.
 * g4d_proposal_train: triangulates xyz with the plain method, labels every
 * candidate pair by whether it is an edge of the result, and trains the model
 * on the device for `epochs` passes (Adam, learning rate lr; a new context starts
 * from a fixed-seed initialisation, later calls continue). *loss receives the
 * last pass's mean binary cross-entropy. */
G4D_API g4d_status g4d_proposal_train(g4d_ctx* ctx, const double* xyz, int n, int epochs, float lr, float* loss);
/* Read (set = 0) or replace (set = 1) the 9473 FP32 model parameters:
 * W1[64][16], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4. */
G4D_API g4d_status g4d_proposal_weights(g4d_ctx* ctx, float* w, int count, int set);
/* Diagnostics of the tensor-core kernels on given rows (x: m rows of 16 BF16
 * features as uint16, y: labels): gradients of the mean loss with respect to
 * `params` (one training-kernel pass, no update), and logits. */
G4D_API g4d_status g4d_mlp_grad(g4d_ctx* ctx, const uint16_t* x, const float* y, int m, const float* params,
                                float* grads, float* loss);
G4D_API g4d_status g4d_mlp_infer(g4d_ctx* ctx, const uint16_t* x, int m, const float* params, float* logits);
/* Diagnostic of the bounded waits in the tensor-core kernels: one block sets
 * up tensor memory and an mbarrier like the MLP kernels, then waits with
 * `limit` polls on a phase that nothing completes. The wait runs out, the
 * kernel frees its tensor memory and returns: G4D_ERR_TIMEOUT, and the
 * context stays usable (the path a real timeout of an MLP kernel takes). */
G4D_API g4d_status g4d_mlp_wait_probe(g4d_ctx* ctx, int limit);

/* Counts of the mesh validator (TetraMesh::check, Common/Geometry.cu:200-393). */
typedef struct {
    long long vertices, edges, triangles, tets;  /* distinct V, E, F; T */
    long long euler;                             /* V - E + F - T: 1 for a triangulated ball */
    long long orient_fail;                       /* tetrahedra with orient3d(v0, v1, v2, v3) > 0 */
    long long insphere_fail;                     /* interior faces with insphere(tet, opposite vertex) < 0 */
    long long adjacency_fail;                    /* opp links out of range or not reciprocated */
} g4d_check_report;

/* The -check validator on the device: the reference's Euler, orientation and
 * in-sphere checks (Common/Geometry.cu:200-393) over the tetrahedra of the
 * context's last single-cloud triangulation (g4d_triangulate*, or
 * g4d_gdel_compute), with exact orient3d and insphere signs and no Simulation
 * of Simplicity, as the reference's validator computes them. Fills *report;
 * a valid Delaunay mesh has euler == 1 and every failure count 0. */
G4D_API g4d_status g4d_check_mesh(g4d_ctx* ctx, g4d_check_report* report);
/* The same validator on a caller's mesh: xyz (n*3 doubles, host) and tets
 * (ntet tetrahedra indexing xyz, host). Vertex and neighbour indices out of
 * range are counted, never followed. */
G4D_API g4d_status g4d_check_tets(g4d_ctx* ctx, const double* xyz, int n, const g4d_tet* tets, int ntet,
                                  g4d_check_report* report);

/* The command line's point generator: Application::makePoints
 * (Main/Application.cpp:316-473) with its KISS random numbers (DtRandom,
 * Common/DtRandom.cpp:44-109, unsigned long = 64 bits as on Linux). Writes n
 * distinct points (xyz: n*3) in grid units [1, grid-2] for distribution dist
 * (0 uniform, 1 gaussian, 2 ball, 3 sphere, 4 grid) and seed: the float values
 * the reference generates for -n n -g grid -d dist -s seed, held as doubles.
 * Host code only; needs no device. */
G4D_API g4d_status g4d_make_points(int n, int dist, int grid, int seed, double* xyz);

/* The context's CUDA stream (a cudaStream_t), for callers that time or order
 * their own work against the library's launches. */
G4D_API void* g4d_stream(g4d_ctx* ctx);

G4D_API void g4d_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
