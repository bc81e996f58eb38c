/*
 * C entry points over the reference's device predicates compiled for the host.
 *
 * Test infrastructure only (built into oracle/_ref/, never linked by the
 * product). Each function calls the reference's own routine:
 *   ref_insphere_fast   -> insphere()            GDelShewchukDevice.h:1052-1144
 *   ref_insphere_exact  -> insphereexact()       GDelShewchukDevice.h:884-1050
 *   ref_orient3d        -> shewchukOrient3D()    GDelPredDevice.h:56-74
 *   ref_orient4_sos     -> orientation4SoS()     GDelPredDevice.h:671-698
 *                          (_orientation4SoS     GDelPredDevice.h:142-669)
 */
#include "refpred_shim.h"
#include "GDelPredDevice.h"

#include <vector>

namespace {
std::vector<RealType> g_consts;
std::vector<RealType> g_scratch;
PredicateInfo g_info;

void ensure_init() {
    if (!g_consts.empty()) return;
    g_consts.assign(DPredicateBoundNum, 0.0);
    g_scratch.assign(PredicateTotalSize, 0.0);
    kerInitPredicate(g_consts.data());
    g_info._consts = g_consts.data();
    g_info._data = g_scratch.data();
}
}  // namespace

extern "C" {

double ref_insphere_fast(const double* p) {
    ensure_init();
    return insphere(g_info, p, p + 3, p + 6, p + 9, p + 12);
}

double ref_insphere_exact(const double* p) {
    ensure_init();
    return insphereexact(g_info, p, p + 3, p + 6, p + 9, p + 12);
}

int ref_orient3d(const double* p) {
    ensure_init();
    return (int)shewchukOrient3D(g_info._consts, p, p + 3, p + 6, p + 9);
}

/* p: 5 points x 3 doubles; idx: their 5 point indices (SoS ranks). */
int ref_orient4_sos(const double* p, const int* idx) {
    ensure_init();
    const double det = insphereexact(g_info, p, p + 3, p + 6, p + 9, p + 12);
    if (det > 0) return 1;
    if (det < 0) return -1;
    return (int)_orientation4SoS(g_info, p, p + 3, p + 6, p + 9, p + 12,
                                 idx[0], idx[1], idx[2], idx[3], idx[4]);
}

/* Same as ref_orient4_sos but skips the exact determinant and reports the
 * SoS decision alone (only meaningful when the determinant is zero). */
int ref_sos_only(const double* p, const int* idx) {
    ensure_init();
    return (int)_orientation4SoS(g_info, p, p + 3, p + 6, p + 9, p + 12,
                                 idx[0], idx[1], idx[2], idx[3], idx[4]);
}

}  // extern "C"
