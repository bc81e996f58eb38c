/*
 * Exact geometric predicates of the CPU oracle (test infrastructure only).
 *
 * Every predicate here returns the exact sign of a determinant over FP64 input
 * coordinates. Signs are obtained by a floating-point filter and, when the
 * filter cannot decide, by exact big-integer arithmetic on the coordinates
 * rescaled to a common binary exponent. This is a restatement of what the
 * reference computes with Shewchuk's adaptive expansions
 * (GDelaunay/GDelShewchukDevice.h:198-1421, Common/predicates.c) and of its
 * Simulation of Simplicity for the lifted 5x5 determinant
 * (GDelaunay/GDelPredDevice.h:142-698); the method differs, the signs must not.
 */
#ifndef G4D_ORACLE_EXACT_H
#define G4D_ORACLE_EXACT_H

#ifdef __cplusplus
extern "C" {
#endif

/* sign of det3(a-d, b-d, c-d): Shewchuk's orient3d sign convention. */
int ora_orient3d(const double* a, const double* b, const double* c, const double* d);

/* sign of the lifted 5x5 determinant | p  |p|^2  1 | over rows a..e, which is
 * Shewchuk's insphere(a,b,c,d,e). No symbolic perturbation. */
int ora_insphere(const double* a, const double* b, const double* c,
                 const double* d, const double* e);

/* insphere with Simulation of Simplicity by point index (never zero).
 * p: 5 points x 3 doubles; idx: their point indices. */
int ora_orient4_sos(const double* p, const int* idx);

/* SoS decision alone (the sign the perturbation gives when the determinant
 * is exactly zero). Exposed for tests. Returns the depth through *depth. */
int ora_sos_only(const double* p, const int* idx, int* depth);

/* Sign of the minor of M = [x y z w 1] (w = x^2+y^2+z^2) over the given rows of
 * the 5-point set p and the given coordinate columns (0..3) plus the ones
 * column; nrows == ncols + 1. Exposed for tests. */
int ora_minor_sign(const double* p, const int* rows, int nrows, const int* cols, int ncols);

/* Counters (not thread-safe; informational only). */
long long ora_exact_calls(void);

#ifdef __cplusplus
}
#endif
#endif
