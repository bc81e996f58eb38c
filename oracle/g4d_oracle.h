/*
 * CPU oracle for the gStar4D hot path (point cloud -> 3D Delaunay tetrahedra
 * with adjacency). TEST INFRASTRUCTURE ONLY: the product never links this.
 * It is the checker for the CUDA path and the timed CPU baseline.
 *
 * It restates the reference pipeline stage by stage:
 *   input scaling       Main/Application.cpp:589-603 (_scalePoint)
 *   Morton order        GDelaunay/GDelData.cu:51-134 (GetMortonNumber, stable sort)
 *   digital Voronoi     PBA/pba3DHost.cu:200-295, PBA/pba3DKernel.h:80-579
 *   missing points      GDelaunay/GDelHost.cu:259-287, GDelKernels.cu:109-135
 *   Voronoi pairs       GDelaunay/GDelHost.cu:289-350, GDelKernels.cu:137-299
 *   worksets + pumping  GDelaunay/GDelHost.cu:352-529, GDelKernels.cu:301-477
 *   initial cones       GDelaunay/GDelPredKernels.cu:45-158
 *   star insertion      GDelaunay/GDelKernels.cu:518-783, GDelPredKernels.cu:233-420
 *   star splaying       GDelaunay/GDelHost.cu:812-1470
 *   containment proof   GDelaunay/GDelPredKernels.cu:427-538
 *   tet extraction      GDelaunay/GDelHost.cu:1520-1607, GDelPredKernels.cu:628-665
 *   CPU validator       Common/Geometry.cu:200-393
 */
#ifndef G4D_ORACLE_H
#define G4D_ORACLE_H

#include "exact.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int v[4];   /* v[0..2] = owner triangle, v[3] = owner star (as the reference) */
    int opp[4]; /* tet across the face opposite v[i], -1 if none */
} ora_tet;

typedef struct {
    int points, grid, missing, loops, max_link;
    long long voronoi_pairs, workset_total, star_insertions, splay_insertions;
    long long drowned, proofs, exact_calls, consistency_repairs;
    double t_order, t_pba, t_star, t_splay, t_out, t_total;
    int max_hist;
} ora_stats;

/* Status codes (same meaning as the product's G4D_* codes). */
enum { ORA_OK = 0, ORA_ERR_ARG = 1, ORA_ERR_NOMEM = 2, ORA_ERR_TIMEOUT = 3, ORA_ERR_INTERNAL = 4 };

/* Scales points into grid units exactly as the reference's _scalePoint (min and
 * max over all coordinates, in double) and returns the stable Morton order:
 * sorted_to_input[i] = input index of sorted position i; voxel[3*i..] = the
 * voxel of sorted point i. */
int ora_morton_order(const double* xyz, int n, int grid, int* sorted_to_input, int* voxel);

/* Exact digital Voronoi diagram: site[((z*G)+y)*G+x] = sorted index of the
 * nearest site (voxel leader = smallest sorted index in the voxel). */
int ora_edt(const int* voxel, int n, int grid, int* site);

/* Distance check used by tests: for every voxel, squared distance to its site. */
long long ora_site_dist2(const int* voxel, int grid, const int* site, long long vox_index);

/* Full triangulation. Output tets use input indices when input_order != 0,
 * otherwise the Morton-sorted indices (the reference's index space). */
int ora_triangulate(const double* xyz, int n, int grid, int nthreads, int input_order,
                    ora_tet** tets, int* ntet, int* sorted_to_input, ora_stats* st);

/* Validator. report[0..9]: euler, orientation failures, insphere failures
 * (the reference's check), adjacency asymmetries, SoS local-Delaunay failures,
 * V, E, F, T, hull faces. rank: SoS rank of each vertex id used in tets. */
int ora_validate(const double* xyz, int n, const int* rank, const ora_tet* tets, int ntet,
                 long long* report);

void ora_free(void* p);

#ifdef __cplusplus
}
#endif
#endif
