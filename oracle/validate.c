/*
 * CPU validator (TEST INFRASTRUCTURE ONLY). Restates the reference's -check
 * (Common/Geometry.cu:200-393): Euler characteristic V-E+F-T == 1 (211-317),
 * tetra orientation orient3d <= 0 (319-344) and the in-sphere test across every
 * shared face (346-393). Adds two checks of its own: adjacency symmetry, and the
 * local Delaunay test under the reference's Simulation of Simplicity, which
 * together with a valid triangulation certifies the unique SoS Delaunay
 * triangulation.
 */
#include "g4d_oracle.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int cmp_u64(const void* x, const void* y) {
    const unsigned long long a = *(const unsigned long long*)x, b = *(const unsigned long long*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

typedef struct { int v[3]; } tri3;
static int cmp_tri3(const void* x, const void* y) {
    const tri3* a = (const tri3*)x;
    const tri3* b = (const tri3*)y;
    for (int i = 0; i < 3; ++i)
        if (a->v[i] != b->v[i]) return a->v[i] < b->v[i] ? -1 : 1;
    return 0;
}

static long long count_unique_u64(unsigned long long* a, long long n) {
    if (n == 0) return 0;
    qsort(a, n, sizeof(unsigned long long), cmp_u64);
    long long k = 1;
    for (long long i = 1; i < n; ++i) if (a[i] != a[i - 1]) ++k;
    return k;
}

int ora_validate(const double* xyz, int n, const int* rank, const ora_tet* T, int nt,
                 long long* rep) {
    (void)n;
    memset(rep, 0, sizeof(long long) * 10);
    /* Euler */
    unsigned long long* vv = (unsigned long long*)malloc(sizeof(unsigned long long) * 4 * (size_t)(nt > 0 ? nt : 1));
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < 4; ++k) vv[4 * (size_t)t + k] = (unsigned)T[t].v[k];
    const long long V = count_unique_u64(vv, 4LL * nt);
    free(vv);
    unsigned long long* ee = (unsigned long long*)malloc(sizeof(unsigned long long) * 6 * (size_t)(nt ? nt : 1));
    long long ne = 0;
    for (int t = 0; t < nt; ++t)
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) {
                unsigned a = (unsigned)T[t].v[i], b = (unsigned)T[t].v[j];
                if (a > b) { unsigned x = a; a = b; b = x; }
                ee[ne++] = ((unsigned long long)a << 32) | b;
            }
    const long long E = count_unique_u64(ee, ne);
    free(ee);
    tri3* ff = (tri3*)malloc(sizeof(tri3) * 4 * (size_t)(nt ? nt : 1));
    long long nf = 0;
    for (int t = 0; t < nt; ++t)
        for (int f = 0; f < 4; ++f) {
            tri3 x;
            int m = 0;
            for (int j = 0; j < 4; ++j) if (j != f) x.v[m++] = T[t].v[j];
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b)
                    if (x.v[a] > x.v[b]) { int s = x.v[a]; x.v[a] = x.v[b]; x.v[b] = s; }
            ff[nf++] = x;
        }
    qsort(ff, nf, sizeof(tri3), cmp_tri3);
    long long F = nf ? 1 : 0;
    for (long long i = 1; i < nf; ++i) if (cmp_tri3(&ff[i], &ff[i - 1])) ++F;
    free(ff);
    rep[0] = V - E + F - nt;
    rep[5] = V; rep[6] = E; rep[7] = F; rep[8] = nt;

    long long orient_fail = 0, insph_fail = 0, asym = 0, sos_fail = 0, hull = 0;
#pragma omp parallel for schedule(static) reduction(+ : orient_fail, insph_fail, asym, sos_fail, hull)
    for (int t = 0; t < nt; ++t) {
        const ora_tet* a = &T[t];
        const double* p[4];
        for (int k = 0; k < 4; ++k) p[k] = xyz + 3 * (size_t)a->v[k];
        if (ora_orient3d(p[0], p[1], p[2], p[3]) > 0) ++orient_fail;
        for (int f = 0; f < 4; ++f) {
            const int o = a->opp[f];
            if (o < 0) { ++hull; continue; }
            if (o >= nt) { ++asym; continue; }
            const ora_tet* b = &T[o];
            int back = -1;
            for (int g = 0; g < 4; ++g) if (b->opp[g] == t) back = g;
            if (back < 0) { ++asym; continue; }
            /* shared face must match */
            int shared = 0;
            for (int i = 0; i < 4; ++i) {
                if (i == f) continue;
                for (int j = 0; j < 4; ++j) if (j != back && b->v[j] == a->v[i]) ++shared;
            }
            if (shared != 3) { ++asym; continue; }
            if (t > o) continue;
            const int w = b->v[back];
            const double* q = xyz + 3 * (size_t)w;
            if (ora_insphere(p[0], p[1], p[2], p[3], q) < 0) ++insph_fail;
            /* SoS: w must lie strictly outside the (perturbed) circumsphere of a;
             * with a negatively oriented, outside means orient4 > 0. */
            double buf[15];
            int id[5];
            for (int k = 0; k < 4; ++k) {
                for (int c = 0; c < 3; ++c) buf[3 * k + c] = p[k][c];
                id[k] = rank ? rank[a->v[k]] : a->v[k];
            }
            for (int c = 0; c < 3; ++c) buf[12 + c] = q[c];
            id[4] = rank ? rank[w] : w;
            if (ora_orient4_sos(buf, id) < 0) ++sos_fail;
        }
    }
    rep[1] = orient_fail;
    rep[2] = insph_fail;
    rep[3] = asym;
    rep[4] = sos_fail;
    rep[9] = hull;
    return 0;
}
