/*
 * CPU oracle: exact predicates (TEST INFRASTRUCTURE ONLY — never linked by the
 * product; the product's predicates live in gstar4d_b200/csrc).
 *
 * Restates the signs computed by the reference's predicates:
 *   orient3d      GDelaunay/GDelPredDevice.h:56-74 (shewchukOrient3D),
 *                 Common/predicates.c:2057 (host orient3d)
 *   insphere      GDelaunay/GDelShewchukDevice.h:884-1144 (insphereexact / filter),
 *                 Common/predicates.c:3919 (host insphere)
 *   orient4 SoS   GDelaunay/GDelPredDevice.h:142-698 (_orientation4SoS, 49 depths)
 *
 * Method (own design): a floating-point filter with a conservative error bound
 * decides most signs; otherwise all coordinates involved are rescaled exactly
 * to integers sharing one binary exponent and the determinant is evaluated in
 * sign-magnitude big-integer arithmetic. The Simulation-of-Simplicity term
 * sequence is generated at load time from the Edelsbrunner-Mucke expansion of
 * the perturbed 5x5 determinant [x y z w 1] (perturbation eps^(2^(4r+3-c)) on
 * row r, coordinate column c): all partial matchings ordered by exponent, cut
 * at the first constant term, keeping the first occurrence of every distinct
 * minor. That yields the same 49-term sequence the reference hard-codes.
 */
#include "exact.h"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Sign-magnitude big integers                                               */
/* ------------------------------------------------------------------------- */

#define BN_MAX 112 /* 3584 bits */

typedef struct {
    int n;   /* used limbs; 0 means zero */
    int neg; /* 1 if negative */
    uint32_t d[BN_MAX];
} bn;

static void bn_norm(bn* a) {
    while (a->n > 0 && a->d[a->n - 1] == 0) a->n--;
    if (a->n == 0) a->neg = 0;
}

static int mag_cmp(const bn* a, const bn* b) {
    if (a->n != b->n) return a->n < b->n ? -1 : 1;
    for (int i = a->n - 1; i >= 0; --i)
        if (a->d[i] != b->d[i]) return a->d[i] < b->d[i] ? -1 : 1;
    return 0;
}

static void mag_add(bn* r, const bn* a, const bn* b) {
    const int n = a->n > b->n ? a->n : b->n;
    uint64_t c = 0;
    for (int i = 0; i < n; ++i) {
        const uint64_t s = c + (uint64_t)(i < a->n ? a->d[i] : 0) + (uint64_t)(i < b->n ? b->d[i] : 0);
        r->d[i] = (uint32_t)s;
        c = s >> 32;
    }
    r->n = n;
    if (c) {
        if (n >= BN_MAX) { fprintf(stderr, "oracle bn overflow\n"); abort(); }
        r->d[r->n++] = (uint32_t)c;
    }
}

/* |r| = |a| - |b|, requires |a| >= |b| */
static void mag_sub(bn* r, const bn* a, const bn* b) {
    int64_t borrow = 0;
    const int n = a->n;
    for (int i = 0; i < n; ++i) {
        int64_t s = (int64_t)a->d[i] - (int64_t)(i < b->n ? b->d[i] : 0) - borrow;
        if (s < 0) { s += ((int64_t)1 << 32); borrow = 1; } else borrow = 0;
        r->d[i] = (uint32_t)s;
    }
    r->n = n;
}

static void bn_add(bn* r, const bn* a, const bn* b) {
    if (a->neg == b->neg) {
        const int neg = a->neg;
        mag_add(r, a, b);
        r->neg = neg;
    } else if (mag_cmp(a, b) >= 0) {
        const int neg = a->neg;
        mag_sub(r, a, b);
        r->neg = neg;
    } else {
        const int neg = b->neg;
        mag_sub(r, b, a);
        r->neg = neg;
    }
    bn_norm(r);
}

static void bn_sub(bn* r, const bn* a, const bn* b) {
    bn nb = *b;
    if (nb.n) nb.neg = !nb.neg;
    bn_add(r, a, &nb);
}

static void bn_mul(bn* r, const bn* a, const bn* b) {
    if (a->n == 0 || b->n == 0) { r->n = 0; r->neg = 0; return; }
    const int n = a->n + b->n;
    if (n > BN_MAX) { fprintf(stderr, "oracle bn overflow (mul)\n"); abort(); }
    uint32_t t[BN_MAX];
    memset(t, 0, sizeof(uint32_t) * n);
    for (int i = 0; i < a->n; ++i) {
        uint64_t c = 0;
        for (int j = 0; j < b->n; ++j) {
            const uint64_t s = (uint64_t)a->d[i] * b->d[j] + t[i + j] + c;
            t[i + j] = (uint32_t)s;
            c = s >> 32;
        }
        t[i + b->n] = (uint32_t)c;
    }
    memcpy(r->d, t, sizeof(uint32_t) * n);
    r->n = n;
    r->neg = a->neg ^ b->neg;
    bn_norm(r);
}

/* r = m * 2^shift with m a signed 64-bit integer (|m| < 2^63) */
static void bn_from_shifted(bn* r, int64_t m, int shift) {
    r->n = 0;
    r->neg = 0;
    if (m == 0) return;
    uint64_t u = m < 0 ? (uint64_t)(-m) : (uint64_t)m;
    const int limb = shift / 32, bit = shift % 32;
    if (limb + 4 > BN_MAX) { fprintf(stderr, "oracle: coordinate exponent range too wide\n"); abort(); }
    memset(r->d, 0, sizeof(uint32_t) * (limb + 4));
    /* place u << bit starting at limb */
    const uint64_t lo = u << bit;
    const uint64_t hi = bit ? (u >> (64 - bit)) : 0;
    r->d[limb] = (uint32_t)lo;
    r->d[limb + 1] = (uint32_t)(lo >> 32);
    r->d[limb + 2] = (uint32_t)hi;
    r->d[limb + 3] = (uint32_t)(hi >> 32);
    r->n = limb + 4;
    r->neg = m < 0;
    bn_norm(r);
}

static int bn_sign(const bn* a) { return a->n == 0 ? 0 : (a->neg ? -1 : 1); }

/* ------------------------------------------------------------------------- */
/* Exact minors of M = [x y z w 1] over up to 5 points                       */
/* ------------------------------------------------------------------------- */

static long long g_exact_calls = 0;
long long ora_exact_calls(void) { return g_exact_calls; }

/* Converts npts points to integers at a common binary exponent. Fills
 * X[i][0..2] and W[i] = X^2+Y^2+Z^2. */
static void to_integers(const double* const* pts, int npts, bn X[][3], bn* W) {
    int64_t mant[5][3];
    int ex[5][3];
    int emin = 1 << 30;
    for (int i = 0; i < npts; ++i)
        for (int c = 0; c < 3; ++c) {
            const double v = pts[i][c];
            if (v == 0.0) { mant[i][c] = 0; ex[i][c] = 0; continue; }
            int e;
            const double m = frexp(v, &e);            /* v = m * 2^e, 0.5 <= |m| < 1 */
            int64_t M = (int64_t)ldexp(m, 53);        /* exact */
            int ee = e - 53;
            while ((M & 1) == 0) { M /= 2; ++ee; }    /* strip trailing zeros */
            mant[i][c] = M;
            ex[i][c] = ee;
            if (ee < emin) emin = ee;
        }
    for (int i = 0; i < npts; ++i) {
        for (int c = 0; c < 3; ++c) {
            if (mant[i][c] == 0) { X[i][c].n = 0; X[i][c].neg = 0; continue; }
            const int sh = ex[i][c] - emin;
            if (sh > 2000) { fprintf(stderr, "oracle: coordinate exponent range too wide\n"); abort(); }
            bn_from_shifted(&X[i][c], mant[i][c], sh);
        }
        bn t, acc;
        bn_mul(&acc, &X[i][0], &X[i][0]);
        bn_mul(&t, &X[i][1], &X[i][1]);
        bn_add(&acc, &acc, &t);
        bn_mul(&t, &X[i][2], &X[i][2]);
        bn_add(&W[i], &acc, &t);
    }
}

static void bn_det(bn* out, bn m[4][4], int n) {
    if (n == 1) { *out = m[0][0]; return; }
    if (n == 2) {
        bn a, b;
        bn_mul(&a, &m[0][0], &m[1][1]);
        bn_mul(&b, &m[0][1], &m[1][0]);
        bn_sub(out, &a, &b);
        return;
    }
    bn acc;
    acc.n = 0; acc.neg = 0;
    for (int j = 0; j < n; ++j) {
        if (m[0][j].n == 0) continue;
        bn sub[4][4];
        for (int r = 1; r < n; ++r) {
            int cc = 0;
            for (int c = 0; c < n; ++c)
                if (c != j) sub[r - 1][cc++] = m[r][c];
        }
        bn d, p;
        bn_det(&d, sub, n - 1);
        bn_mul(&p, &m[0][j], &d);
        if (j & 1) bn_sub(&acc, &acc, &p); else bn_add(&acc, &acc, &p);
    }
    *out = acc;
}

/* Sign of det of the matrix with rows `rows` (indices into pts) and columns
 * `cols` (0..3 = x,y,z,w) followed by a ones column. nrows == ncols + 1. */
static int exact_minor(const double* const* pts, int npts, const int* rows, int nrows,
                       const int* cols, int ncols) {
    ++g_exact_calls;
    if (ncols == 0) return 1; /* det [1] */
    static __thread bn X[5][3];
    static __thread bn W[5];
    to_integers(pts, npts, X, W);
    const int last = rows[nrows - 1];
    bn m[4][4];
    for (int i = 0; i < ncols; ++i)
        for (int j = 0; j < ncols; ++j) {
            const int c = cols[j];
            const bn* a = c < 3 ? &X[rows[i]][c] : &W[rows[i]];
            const bn* b = c < 3 ? &X[last][c] : &W[last];
            bn_sub(&m[i][j], a, b);
        }
    bn d;
    bn_det(&d, m, ncols);
    return bn_sign(&d);
}

int ora_minor_sign(const double* p, const int* rows, int nrows, const int* cols, int ncols) {
    const double* pts[5] = {p, p + 3, p + 6, p + 9, p + 12};
    return exact_minor(pts, 5, rows, nrows, cols, ncols);
}

/* ------------------------------------------------------------------------- */
/* Floating-point filters (conservative bounds; no FMA contraction)          */
/* ------------------------------------------------------------------------- */

#define ORA_EPS 1.1102230246251565e-16 /* 2^-53 */

static int orient3d_filter(const double* a, const double* b, const double* c, const double* d) {
    const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
    const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
    const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
    const double p1 = bdx * cdy, p2 = cdx * bdy;
    const double p3 = cdx * ady, p4 = adx * cdy;
    const double p5 = adx * bdy, p6 = bdx * ady;
    const double det = adz * (p1 - p2) + bdz * (p3 - p4) + cdz * (p5 - p6);
    const double perm = (fabs(p1) + fabs(p2)) * fabs(adz) + (fabs(p3) + fabs(p4)) * fabs(bdz) +
                        (fabs(p5) + fabs(p6)) * fabs(cdz);
    const double bound = 16.0 * ORA_EPS * perm;
    if (perm < 1e-280) return 0;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return 0;
}

static int insphere_filter(const double* pa, const double* pb, const double* pc,
                           const double* pd, const double* pe) {
    const double aex = pa[0] - pe[0], bex = pb[0] - pe[0], cex = pc[0] - pe[0], dex = pd[0] - pe[0];
    const double aey = pa[1] - pe[1], bey = pb[1] - pe[1], cey = pc[1] - pe[1], dey = pd[1] - pe[1];
    const double aez = pa[2] - pe[2], bez = pb[2] - pe[2], cez = pc[2] - pe[2], dez = pd[2] - pe[2];
    const double aexbey = aex * bey, bexaey = bex * aey;
    const double bexcey = bex * cey, cexbey = cex * bey;
    const double cexdey = cex * dey, dexcey = dex * cey;
    const double dexaey = dex * aey, aexdey = aex * dey;
    const double aexcey = aex * cey, cexaey = cex * aey;
    const double bexdey = bex * dey, dexbey = dex * bey;
    const double ab = aexbey - bexaey, bc = bexcey - cexbey, cd = cexdey - dexcey;
    const double da = dexaey - aexdey, ac = aexcey - cexaey, bd = bexdey - dexbey;
    const double abP = fabs(aexbey) + fabs(bexaey), bcP = fabs(bexcey) + fabs(cexbey);
    const double cdP = fabs(cexdey) + fabs(dexcey), daP = fabs(dexaey) + fabs(aexdey);
    const double acP = fabs(aexcey) + fabs(cexaey), bdP = fabs(bexdey) + fabs(dexbey);
    const double abc = aez * bc - bez * ac + cez * ab;
    const double bcd = bez * cd - cez * bd + dez * bc;
    const double cda = cez * da + dez * ac + aez * cd;
    const double dab = dez * ab + aez * bd + bez * da;
    const double abcP = fabs(aez) * bcP + fabs(bez) * acP + fabs(cez) * abP;
    const double bcdP = fabs(bez) * cdP + fabs(cez) * bdP + fabs(dez) * bcP;
    const double cdaP = fabs(cez) * daP + fabs(dez) * acP + fabs(aez) * cdP;
    const double dabP = fabs(dez) * abP + fabs(aez) * bdP + fabs(bez) * daP;
    const double alift = aex * aex + aey * aey + aez * aez;
    const double blift = bex * bex + bey * bey + bez * bez;
    const double clift = cex * cex + cey * cey + cez * cez;
    const double dlift = dex * dex + dey * dey + dez * dez;
    const double det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
    const double perm = (dlift * abcP + clift * dabP) + (blift * cdaP + alift * bcdP);
    const double bound = 32.0 * ORA_EPS * perm;
    if (perm < 1e-250) return 0;
    if (det > bound) return 1;
    if (-det > bound) return -1;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Public predicates                                                         */
/* ------------------------------------------------------------------------- */

int ora_orient3d(const double* a, const double* b, const double* c, const double* d) {
    const int s = orient3d_filter(a, b, c, d);
    if (s) return s;
    const double* pts[4] = {a, b, c, d};
    const int rows[4] = {0, 1, 2, 3};
    const int cols[3] = {0, 1, 2};
    return exact_minor(pts, 4, rows, 4, cols, 3);
}

static int insphere_exact(const double* const* pts) {
    const int rows[5] = {0, 1, 2, 3, 4};
    const int cols[4] = {0, 1, 2, 3};
    return exact_minor(pts, 5, rows, 5, cols, 4);
}

int ora_insphere(const double* a, const double* b, const double* c, const double* d,
                 const double* e) {
    const int s = insphere_filter(a, b, c, d, e);
    if (s) return s;
    const double* pts[5] = {a, b, c, d, e};
    return insphere_exact(pts);
}

/* ---- Simulation of Simplicity term table, generated at load time -------- */

typedef struct {
    int nrows, ncols;
    int rows[5];
    int cols[4];
    int coef;
} sos_term;

static sos_term g_sos[64];
static int g_sos_n = 0;

static int perm_parity(const int* p, int n) {
    int s = 1;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (p[i] > p[j]) s = -s;
    return s;
}

typedef struct { unsigned mask; int size; int r[4]; int c[4]; } sos_cand;

static int cand_cmp(const void* x, const void* y) {
    const sos_cand* a = (const sos_cand*)x;
    const sos_cand* b = (const sos_cand*)y;
    return a->mask < b->mask ? -1 : (a->mask > b->mask ? 1 : 0);
}

__attribute__((constructor)) static void build_sos_table(void) {
    /* enumerate partial matchings of rows {0..4} x coordinate columns {0..3} */
    static sos_cand cand[4096];
    int nc = 0;
    for (int size = 1; size <= 4; ++size) {
        int R[4];
        /* row combinations */
        for (int rmask = 0; rmask < 32; ++rmask) {
            if (__builtin_popcount(rmask) != size) continue;
            int k = 0;
            for (int r = 0; r < 5; ++r) if (rmask & (1 << r)) R[k++] = r;
            /* column permutations of size `size` from 4 */
            int C[4];
            for (int c0 = 0; c0 < 4; ++c0)
                for (int c1 = 0; c1 < 4; ++c1)
                    for (int c2 = 0; c2 < 4; ++c2)
                        for (int c3 = 0; c3 < 4; ++c3) {
                            C[0] = c0; C[1] = c1; C[2] = c2; C[3] = c3;
                            int ok = 1;
                            for (int i = 0; i < size && ok; ++i)
                                for (int j = i + 1; j < size; ++j)
                                    if (C[i] == C[j]) { ok = 0; break; }
                            /* only enumerate each permutation once: unused slots 0 */
                            for (int i = size; i < 4 && ok; ++i) if (C[i] != 0) ok = 0;
                            if (!ok) continue;
                            sos_cand* s = &cand[nc++];
                            s->size = size;
                            s->mask = 0;
                            for (int i = 0; i < size; ++i) {
                                s->r[i] = R[i];
                                s->c[i] = C[i];
                                s->mask |= 1u << (4 * R[i] + (3 - C[i]));
                            }
                        }
        }
    }
    qsort(cand, nc, sizeof(sos_cand), cand_cmp);
    /* the first constant term: rows 0..3 matched to columns x,y,z,w */
    const unsigned stop = (1u << 3) | (1u << 6) | (1u << 9) | (1u << 12);
    g_sos_n = 0;
    for (int i = 0; i < nc && cand[i].mask <= stop; ++i) {
        const sos_cand* s = &cand[i];
        sos_term t;
        t.nrows = 0;
        t.ncols = 0;
        for (int r = 0; r < 5; ++r) {
            int used = 0;
            for (int j = 0; j < s->size; ++j) if (s->r[j] == r) used = 1;
            if (!used) t.rows[t.nrows++] = r;
        }
        for (int c = 0; c < 4; ++c) {
            int used = 0;
            for (int j = 0; j < s->size; ++j) if (s->c[j] == c) used = 1;
            if (!used) t.cols[t.ncols++] = c;
        }
        int sumrc = 0;
        for (int j = 0; j < s->size; ++j) sumrc += s->r[j] + s->c[j];
        t.coef = ((sumrc & 1) ? -1 : 1) * perm_parity(s->c, s->size);
        /* keep first occurrence of each distinct minor */
        int dup = 0;
        for (int k = 0; k < g_sos_n && !dup; ++k) {
            if (g_sos[k].nrows != t.nrows || g_sos[k].ncols != t.ncols) continue;
            if (memcmp(g_sos[k].rows, t.rows, sizeof(int) * t.nrows) == 0 &&
                memcmp(g_sos[k].cols, t.cols, sizeof(int) * t.ncols) == 0)
                dup = 1;
        }
        if (!dup) g_sos[g_sos_n++] = t;
    }
}

int ora_sos_only(const double* p, const int* idx, int* depth) {
    int order[5] = {0, 1, 2, 3, 4};
    int key[5];
    for (int i = 0; i < 5; ++i) key[i] = idx[i];
    int parity = 1;
    for (int i = 0; i < 4; ++i)
        for (int j = 4; j > i; --j)
            if (key[j] < key[j - 1]) {
                int t = key[j]; key[j] = key[j - 1]; key[j - 1] = t;
                t = order[j]; order[j] = order[j - 1]; order[j - 1] = t;
                parity = -parity;
            }
    const double* pts[5];
    for (int i = 0; i < 5; ++i) pts[i] = p + 3 * order[i];
    for (int k = 0; k < g_sos_n; ++k) {
        const sos_term* t = &g_sos[k];
        const int s = exact_minor(pts, 5, t->rows, t->nrows, t->cols, t->ncols);
        if (s) {
            if (depth) *depth = k + 1;
            return parity * t->coef * s;
        }
    }
    fprintf(stderr, "oracle: SoS table exhausted\n");
    abort();
}

int ora_orient4_sos(const double* p, const int* idx) {
    const int s = insphere_filter(p, p + 3, p + 6, p + 9, p + 12);
    if (s) return s;
    const double* pts[5] = {p, p + 3, p + 6, p + 9, p + 12};
    const int e = insphere_exact(pts);
    if (e) return e;
    return ora_sos_only(p, idx, NULL);
}

int ora_sos_table_size(void) { return g_sos_n; }
