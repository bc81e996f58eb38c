/*
 * CPU oracle pipeline (TEST INFRASTRUCTURE ONLY; see g4d_oracle.h for the map
 * of reference functions each stage restates). Round-based star splaying with
 * OpenMP over stars; deterministic result (the Delaunay triangulation under the
 * reference's Simulation of Simplicity is unique for given coordinates and
 * Morton index order).
 */
#define _GNU_SOURCE
#include "g4d_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define MIN_WORKSET 8 /* GDelCommon.h:49 */

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void ora_free(void* p) { free(p); }

/* ------------------------------------------------------------------------- */
/* growable int vector                                                       */
/* ------------------------------------------------------------------------- */
typedef struct { int* a; int n, cap; } ivec;
static void iv_push(ivec* v, int x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 16;
        v->a = (int*)realloc(v->a, sizeof(int) * v->cap);
    }
    v->a[v->n++] = x;
}
static int iv_has(const ivec* v, int x) {
    for (int i = 0; i < v->n; ++i) if (v->a[i] == x) return 1;
    return 0;
}

typedef struct { long long* a; long long n, cap; } lvec;
static void lv_push(lvec* v, long long x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? 2 * v->cap : 1024;
        v->a = (long long*)realloc(v->a, sizeof(long long) * v->cap);
    }
    v->a[v->n++] = x;
}
static int cmp_ll(const void* x, const void* y) {
    const long long a = *(const long long*)x, b = *(const long long*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}
static int cmp_int(const void* x, const void* y) {
    const int a = *(const int*)x, b = *(const int*)y;
    return a < b ? -1 : (a > b ? 1 : 0);
}

/* ------------------------------------------------------------------------- */
/* Scaling and Morton order (Application.cpp:589-603, GDelData.cu:51-134)    */
/* ------------------------------------------------------------------------- */

static int spread10(int v) {
    v = (v | (v << 16)) & 0x030000FF;
    v = (v | (v << 8)) & 0x0300F00F;
    v = (v | (v << 4)) & 0x030C30C3;
    v = (v | (v << 2)) & 0x09249249;
    return v;
}

int ora_morton_order(const double* xyz, int n, int grid, int* sorted_to_input, int* voxel) {
    if (n < 5 || grid < 32 || grid > 1024 || (grid & (grid - 1))) return ORA_ERR_ARG;
    double mn = xyz[0], mx = xyz[0];
    for (long long i = 0; i < 3LL * n; ++i) {
        if (xyz[i] < mn) mn = xyz[i];
        if (xyz[i] > mx) mx = xyz[i];
    }
    const double rng = mx - mn;
    if (!(rng > 0)) return ORA_ERR_ARG;
    long long* key = (long long*)malloc(sizeof(long long) * n);
    int* vin = (int*)malloc(sizeof(int) * 3 * (size_t)n);
    if (!key || !vin) { free(key); free(vin); return ORA_ERR_NOMEM; }
    for (int i = 0; i < n; ++i) {
        int m = 0;
        for (int c = 0; c < 3; ++c) {
            double t = xyz[3 * (size_t)i + c] - mn;
            t = (double)(grid - 3) * t;
            t = t / rng;
            t = t + 1.0;
            const int q = (int)t;
            vin[3 * (size_t)i + c] = q;
            m |= spread10(q) << c;
        }
        key[i] = ((long long)m << 32) | (long long)i; /* ties keep input order */
    }
    qsort(key, n, sizeof(long long), cmp_ll);
    for (int i = 0; i < n; ++i) {
        const int src = (int)(key[i] & 0xffffffffLL);
        sorted_to_input[i] = src;
        if (voxel) for (int c = 0; c < 3; ++c) voxel[3 * (size_t)i + c] = vin[3 * (size_t)src + c];
    }
    free(key);
    free(vin);
    return ORA_OK;
}

/* ------------------------------------------------------------------------- */
/* Exact digital Voronoi diagram: separable lower envelopes                  */
/* (Felzenszwalb-Huttenlocher), restating what PBA's three phases compute   */
/* (pba3DHost.cu:200-245): nearest site per voxel under squared distance.    */
/* ------------------------------------------------------------------------- */

#define GI(G, x, y, z) ((((size_t)(z)) * (G) + (y)) * (size_t)(G) + (x))

static void envelope(int len, const long long* f, const int* cand, int* out, int* v, double* zb) {
    /* f[q] = height (INT64_MAX if none), cand[q] = site at q */
    int k = -1;
    for (int q = 0; q < len; ++q) {
        if (f[q] == INT64_MAX) continue;
        if (k < 0) { k = 0; v[0] = q; zb[0] = -1e300; zb[1] = 1e300; continue; }
        for (;;) {
            const int p = v[k];
            const double s = ((double)(f[q] + (long long)q * q) - (double)(f[p] + (long long)p * p)) /
                             (2.0 * (q - p));
            if (s <= zb[k]) {
                if (k == 0) { v[0] = q; zb[0] = -1e300; zb[1] = 1e300; break; }
                --k;
                continue;
            }
            ++k;
            v[k] = q;
            zb[k] = s;
            zb[k + 1] = 1e300;
            break;
        }
    }
    if (k < 0) { for (int q = 0; q < len; ++q) out[q] = -1; return; }
    int j = 0;
    for (int q = 0; q < len; ++q) {
        while (zb[j + 1] < q) ++j;
        out[q] = cand[v[j]];
    }
}

int ora_edt(const int* voxel, int n, int G, int* site) {
    const size_t G3 = (size_t)G * G * G;
    for (size_t i = 0; i < G3; ++i) site[i] = -1;
    for (int i = 0; i < n; ++i) {
        const size_t gi = GI(G, voxel[3 * (size_t)i], voxel[3 * (size_t)i + 1], voxel[3 * (size_t)i + 2]);
        if (site[gi] < 0) site[gi] = i; /* leader: smallest sorted index */
    }
    int* tmp = (int*)malloc(sizeof(int) * G3);
    if (!tmp) return ORA_ERR_NOMEM;
    /* pass Z: site -> tmp */
#pragma omp parallel
    {
        long long* f = (long long*)malloc(sizeof(long long) * G);
        int* cand = (int*)malloc(sizeof(int) * G);
        int* out = (int*)malloc(sizeof(int) * G);
        int* v = (int*)malloc(sizeof(int) * (G + 1));
        double* zb = (double*)malloc(sizeof(double) * (G + 2));
#pragma omp for schedule(static)
        for (int yx = 0; yx < G * G; ++yx) {
            const int x = yx % G, y = yx / G;
            for (int z = 0; z < G; ++z) {
                const int s = site[GI(G, x, y, z)];
                f[z] = s >= 0 ? 0 : INT64_MAX;
                cand[z] = s;
            }
            envelope(G, f, cand, out, v, zb);
            for (int z = 0; z < G; ++z) tmp[GI(G, x, y, z)] = out[z];
        }
        /* pass Y: tmp -> site */
#pragma omp for schedule(static)
        for (int zx = 0; zx < G * G; ++zx) {
            const int x = zx % G, z = zx / G;
            for (int y = 0; y < G; ++y) {
                const int s = tmp[GI(G, x, y, z)];
                cand[y] = s;
                if (s < 0) { f[y] = INT64_MAX; continue; }
                const long long dz = voxel[3 * (size_t)s + 2] - z;
                f[y] = dz * dz;
            }
            envelope(G, f, cand, out, v, zb);
            for (int y = 0; y < G; ++y) site[GI(G, x, y, z)] = out[y];
        }
        /* pass X: site -> tmp */
#pragma omp for schedule(static)
        for (int zy = 0; zy < G * G; ++zy) {
            const int y = zy % G, z = zy / G;
            for (int x = 0; x < G; ++x) {
                const int s = site[GI(G, x, y, z)];
                cand[x] = s;
                if (s < 0) { f[x] = INT64_MAX; continue; }
                const long long dy = voxel[3 * (size_t)s + 1] - y, dz = voxel[3 * (size_t)s + 2] - z;
                f[x] = dy * dy + dz * dz;
            }
            envelope(G, f, cand, out, v, zb);
            for (int x = 0; x < G; ++x) tmp[GI(G, x, y, z)] = out[x];
        }
        free(f); free(cand); free(out); free(v); free(zb);
    }
    memcpy(site, tmp, sizeof(int) * G3);
    free(tmp);
    return ORA_OK;
}

long long ora_site_dist2(const int* voxel, int G, const int* site, long long vi) {
    const int s = site[vi];
    if (s < 0) return -1;
    const int x = (int)(vi % G), y = (int)((vi / G) % G), z = (int)(vi / ((long long)G * G));
    const long long dx = voxel[3 * (size_t)s] - x, dy = voxel[3 * (size_t)s + 1] - y,
                    dz = voxel[3 * (size_t)s + 2] - z;
    return dx * dx + dy * dy + dz * dz;
}

/* ------------------------------------------------------------------------- */
/* Stars                                                                     */
/* ------------------------------------------------------------------------- */

typedef struct { int v[3]; unsigned char alive, fresh; } otri;

typedef struct {
    otri* t;
    int nt, ct;
    ivec hist;     /* every point ever inserted (symmetric relation) */
    ivec pend;     /* insertions for the next round */
    ivec changed;  /* candidates for drowned detection after a round */
} ostar;

typedef struct {
    const double* P; /* sorted points, original coordinates */
    int n;
    ostar* S;
    int fail;
} octx;

static int o4(const double* P, int a, int b, int c, int d, int e) {
    double buf[15];
    const int id[5] = {a, b, c, d, e};
    for (int i = 0; i < 5; ++i) memcpy(buf + 3 * i, P + 3 * (size_t)id[i], sizeof(double) * 3);
    return ora_orient4_sos(buf, id);
}

static otri* new_tri(ostar* s) {
    for (int i = 0; i < s->nt; ++i)
        if (!s->t[i].alive) return &s->t[i];
    if (s->nt == s->ct) {
        s->ct = s->ct ? 2 * s->ct : 32;
        s->t = (otri*)realloc(s->t, sizeof(otri) * s->ct);
    }
    return &s->t[s->nt++];
}

static void compact_tris(ostar* s) {
    int k = 0;
    for (int i = 0; i < s->nt; ++i) if (s->t[i].alive) s->t[k++] = s->t[i];
    s->nt = k;
}

static int in_link(const ostar* s, int v) {
    for (int i = 0; i < s->nt; ++i) {
        const otri* t = &s->t[i];
        if (t->alive && (t->v[0] == v || t->v[1] == v || t->v[2] == v)) return 1;
    }
    return 0;
}

static void link_set(const ostar* s, ivec* out) {
    out->n = 0;
    for (int i = 0; i < s->nt; ++i) {
        const otri* t = &s->t[i];
        if (!t->alive) continue;
        for (int k = 0; k < 3; ++k) if (!iv_has(out, t->v[k])) iv_push(out, t->v[k]);
    }
}

/* Initial 4-simplex cone (GDelPredKernels.cu:45-158): link triangles of the
 * pentachoron (l0,l1,l2,l3,star), oriented so that orient4(tri, star, q) > 0
 * for the opposite link vertex q. */
static void make_cone(const double* P, ostar* s, int star, int l0, int l1, int l2, int l3) {
    int l[4] = {l0, l1, l2, l3};
    if (o4(P, l[0], l[1], l[2], l[3], star) < 0) { int t = l[0]; l[0] = l[1]; l[1] = t; }
    static const int F[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
    s->nt = 0;
    for (int f = 0; f < 4; ++f) {
        otri* t = new_tri(s);
        for (int k = 0; k < 3; ++k) t->v[k] = l[F[f][k]];
        t->alive = 1;
        t->fresh = 1;
    }
}

/* Insert point p into star(star): beneath triangles (orient4 < 0) are removed
 * and the hole boundary is fanned to p (GDelKernels.cu:622-783). Returns 0 if
 * p is beneath no triangle (p lies inside the cone: drowned). */
static int star_insert(const double* P, ostar* s, int star, int p) {
    int nb = 0;
    int* bl = (int*)alloca(sizeof(int) * (s->nt + 1));
    for (int i = 0; i < s->nt; ++i) {
        otri* t = &s->t[i];
        if (!t->alive) continue;
        if (o4(P, t->v[0], t->v[1], t->v[2], star, p) < 0) bl[nb++] = i;
    }
    if (!nb) return 0;
    int* eu = (int*)alloca(sizeof(int) * 3 * nb);
    int* ev = (int*)alloca(sizeof(int) * 3 * nb);
    for (int i = 0; i < nb; ++i) {
        const otri* t = &s->t[bl[i]];
        for (int k = 0; k < 3; ++k) { eu[3 * i + k] = t->v[k]; ev[3 * i + k] = t->v[(k + 1) % 3]; }
    }
    for (int i = 0; i < nb; ++i) s->t[bl[i]].alive = 0;
    for (int e = 0; e < 3 * nb; ++e) {
        int interior = 0;
        for (int f = 0; f < 3 * nb; ++f)
            if (eu[f] == ev[e] && ev[f] == eu[e]) { interior = 1; break; }
        if (interior) continue;
        otri* t = new_tri(s);
        t->v[0] = eu[e];
        t->v[1] = ev[e];
        t->v[2] = p;
        t->alive = 1;
        t->fresh = 1;
    }
    return 1;
}

/* Containment proof (GDelPredKernels.cu:427-538): 4 link vertices of star
 * `star` that enclose `inv`: exVert (first vertex of the first live triangle)
 * plus a live triangle not containing exVert whose three consecutive vertex
 * pairs all give the same orient4(star, inv, exVert, v_i, v_{i+1}). */
static int find_proof(const double* P, const ostar* s, int star, int inv, int* proof) {
    int i0 = 0;
    while (i0 < s->nt && !s->t[i0].alive) ++i0;
    if (i0 >= s->nt) return 0;
    const int ex = s->t[i0].v[0];
    for (int i = i0; i < s->nt; ++i) {
        const otri* t = &s->t[i];
        if (!t->alive) continue;
        if (t->v[0] == ex || t->v[1] == ex || t->v[2] == ex) continue;
        int prev = 0, vi;
        for (vi = 0; vi < 3; ++vi) {
            const int o = o4(P, star, inv, ex, t->v[vi], t->v[(vi + 1) % 3]);
            if (vi > 0 && o != prev) break;
            prev = o;
        }
        if (vi >= 3) {
            proof[0] = ex; proof[1] = t->v[0]; proof[2] = t->v[1]; proof[3] = t->v[2];
            return 1;
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Pairs from the digital Voronoi diagram                                    */
/* ------------------------------------------------------------------------- */

/* Candidate Delaunay edges: every two distinct sites of a 2x2x2 voxel cube in
 * which at least three sites meet (a digital Voronoi edge or vertex). The
 * reference reads the same cubes and emits around digital Voronoi vertices
 * (GDelKernels.cu:137-299). */
static void grid_pairs(const int* site, int G, lvec* out) {
    const int nt = omp_get_max_threads();
    lvec* per = (lvec*)calloc(nt, sizeof(lvec));
#pragma omp parallel
    {
        const int tid = omp_get_thread_num();
        lvec* pv = &per[tid];
        const int CACHE = 1 << 14;
        long long* cache = (long long*)malloc(sizeof(long long) * CACHE);
        for (int i = 0; i < CACHE; ++i) cache[i] = -1;
#pragma omp for schedule(dynamic, 4)
        for (int zy = 0; zy < (G - 1) * (G - 1); ++zy) {
            const int y = zy % (G - 1), z = zy / (G - 1);
            for (int x = 0; x < G - 1; ++x) {
                int s[8], ns = 0;
                for (int dz = 0; dz < 2; ++dz)
                    for (int dy = 0; dy < 2; ++dy)
                        for (int dx = 0; dx < 2; ++dx) {
                            const int v = site[GI(G, x + dx, y + dy, z + dz)];
                            int dup = 0;
                            for (int k = 0; k < ns; ++k) if (s[k] == v) { dup = 1; break; }
                            if (!dup) s[ns++] = v;
                        }
                if (ns < 3) continue; /* only digital Voronoi edges and vertices */
                for (int a = 0; a < ns; ++a)
                    for (int b = a + 1; b < ns; ++b) {
                        const int lo = s[a] < s[b] ? s[a] : s[b], hi = s[a] < s[b] ? s[b] : s[a];
                        const long long key = ((long long)lo << 32) | (unsigned)hi;
                        const unsigned h = (unsigned)((key * 0x9E3779B97F4A7C15ULL) >> 50) & (CACHE - 1);
                        if (cache[h] == key) continue;
                        cache[h] = key;
                        lv_push(pv, key);
                    }
            }
        }
        free(cache);
    }
    out->n = 0;
    for (int t = 0; t < nt; ++t) {
        for (long long i = 0; i < per[t].n; ++i) lv_push(out, per[t].a[i]);
        free(per[t].a);
    }
    free(per);
    qsort(out->a, out->n, sizeof(long long), cmp_ll);
    long long k = 0;
    for (long long i = 0; i < out->n; ++i)
        if (k == 0 || out->a[i] != out->a[k - 1]) out->a[k++] = out->a[i];
    out->n = k;
}

/* ------------------------------------------------------------------------- */
/* Splaying                                                                  */
/* ------------------------------------------------------------------------- */

/* Collect (star, vert) insertion requests, keep those not yet in the star's
 * history, add the reciprocal request, and append to the stars' pending lists.
 * Returns the number of new insertions. */
static long long dispatch_pairs(octx* C, lvec* pairs) {
    qsort(pairs->a, pairs->n, sizeof(long long), cmp_ll);
    long long k = 0;
    for (long long i = 0; i < pairs->n; ++i)
        if (k == 0 || pairs->a[i] != pairs->a[k - 1]) pairs->a[k++] = pairs->a[i];
    pairs->n = k;
    long long added = 0;
    for (long long i = 0; i < pairs->n; ++i) {
        const int s = (int)(pairs->a[i] >> 32), v = (int)(pairs->a[i] & 0xffffffffLL);
        if (s == v) continue;
        ostar* S = &C->S[s];
        if (iv_has(&S->hist, v) || iv_has(&S->pend, v)) continue;
        iv_push(&S->pend, v);
        ++added;
        ostar* V = &C->S[v];
        if (!iv_has(&V->hist, s) && !iv_has(&V->pend, s)) { iv_push(&V->pend, s); ++added; }
    }
    return added;
}

static void insert_pending(octx* C, long long* ins_count) {
    long long cnt = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : cnt)
    for (int s = 0; s < C->n; ++s) {
        ostar* S = &C->S[s];
        if (!S->pend.n) continue;
        qsort(S->pend.a, S->pend.n, sizeof(int), cmp_int);
        ivec before = {0};
        link_set(S, &before);
        S->changed.n = 0;
        for (int i = 0; i < before.n; ++i) iv_push(&S->changed, before.a[i]);
        for (int i = 0; i < S->pend.n; ++i) {
            const int p = S->pend.a[i];
            iv_push(&S->hist, p);
            iv_push(&S->changed, p);
            star_insert(C->P, S, s, p);
            ++cnt;
        }
        S->pend.n = 0;
        compact_tris(S);
        free(before.a);
    }
    *ins_count += cnt;
}

/* Drowned points (inserted or previously linked, no longer in the link) whose
 * own star still links back get a containment proof. */
static void drowned_proofs(octx* C, lvec* out, long long* drowned, long long* proofs) {
    const int nt = omp_get_max_threads();
    lvec* per = (lvec*)calloc(nt, sizeof(lvec));
    long long dn = 0, pn = 0;
    int fail = 0;
#pragma omp parallel reduction(+ : dn, pn) reduction(| : fail)
    {
        lvec* pv = &per[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 64)
        for (int s = 0; s < C->n; ++s) {
            ostar* S = &C->S[s];
            for (int i = 0; i < S->changed.n; ++i) {
                const int p = S->changed.a[i];
                if (in_link(S, p)) continue;
                if (!in_link(&C->S[p], s)) continue;
                ++dn;
                int proof[4];
                if (!find_proof(C->P, S, s, p, proof)) { fail = 1; continue; }
                for (int k = 0; k < 4; ++k) {
                    if (proof[k] == p) continue;
                    lv_push(pv, ((long long)p << 32) | (unsigned)proof[k]);
                    ++pn;
                }
            }
        }
    }
    for (int t = 0; t < nt; ++t) {
        for (long long i = 0; i < per[t].n; ++i) lv_push(out, per[t].a[i]);
        free(per[t].a);
    }
    free(per);
    for (int s = 0; s < C->n; ++s) C->S[s].changed.n = 0;
    if (fail) C->fail = 1;
    *drowned += dn;
    *proofs += pn;
}

/* Consistency requests from fresh triangles (GDelKernels.cu:818-939): every
 * link edge (u,v), u<v, asks that u and v know each other. */
static void fresh_requests(octx* C, lvec* out, int all) {
    const int nt = omp_get_max_threads();
    lvec* per = (lvec*)calloc(nt, sizeof(lvec));
#pragma omp parallel
    {
        lvec* pv = &per[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 64)
        for (int s = 0; s < C->n; ++s) {
            ostar* S = &C->S[s];
            for (int i = 0; i < S->nt; ++i) {
                otri* t = &S->t[i];
                if (!t->alive || (!t->fresh && !all)) continue;
                t->fresh = 0;
                for (int k = 0; k < 3; ++k) {
                    const int u = t->v[k], v = t->v[(k + 1) % 3];
                    if (u > v) continue;
                    if (iv_has(&C->S[u].hist, v)) continue;
                    lv_push(pv, ((long long)u << 32) | (unsigned)v);
                }
            }
        }
    }
    for (int t = 0; t < nt; ++t) {
        for (long long i = 0; i < per[t].n; ++i) lv_push(out, per[t].a[i]);
        free(per[t].a);
    }
    free(per);
}

/* Star consistency (GDelKernels.cu:1193-1271): triangle (a,b,c) of star s must
 * appear as (b,s,c) (up to rotation) in star a, and likewise for b and c. */
static long long count_inconsistent(octx* C) {
    long long bad = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : bad)
    for (int s = 0; s < C->n; ++s) {
        const ostar* S = &C->S[s];
        for (int i = 0; i < S->nt; ++i) {
            const otri* t = &S->t[i];
            if (!t->alive) continue;
            for (int k = 0; k < 3; ++k) {
                const int a = t->v[k], b = t->v[(k + 1) % 3], c = t->v[(k + 2) % 3];
                /* expected in star a: cyclic (b, s, c) */
                const ostar* A = &C->S[a];
                int found = 0;
                for (int j = 0; j < A->nt && !found; ++j) {
                    const otri* u = &A->t[j];
                    if (!u->alive) continue;
                    for (int r = 0; r < 3; ++r)
                        if (u->v[r] == b && u->v[(r + 1) % 3] == s && u->v[(r + 2) % 3] == c) {
                            found = 1;
                            break;
                        }
                }
                if (!found) ++bad;
            }
        }
    }
    return bad;
}

/* ------------------------------------------------------------------------- */
/* Face hashing for adjacency                                                */
/* ------------------------------------------------------------------------- */

typedef struct { int a, b, c; int tet; int fi; } fent;

static void sort3(int* x) {
    int t;
    if (x[0] > x[1]) { t = x[0]; x[0] = x[1]; x[1] = t; }
    if (x[1] > x[2]) { t = x[1]; x[1] = x[2]; x[2] = t; }
    if (x[0] > x[1]) { t = x[0]; x[0] = x[1]; x[1] = t; }
}

static int link_adjacency(ora_tet* tets, int ntet) {
    const size_t cap = 1;
    size_t H = cap;
    while (H < (size_t)ntet * 8) H <<= 1;
    fent* tab = (fent*)malloc(sizeof(fent) * H);
    if (!tab) return ORA_ERR_NOMEM;
    for (size_t i = 0; i < H; ++i) tab[i].tet = -1;
    for (int t = 0; t < ntet; ++t)
        for (int f = 0; f < 4; ++f) tets[t].opp[f] = -1;
    for (int t = 0; t < ntet; ++t)
        for (int f = 0; f < 4; ++f) {
            int k[3], m = 0;
            for (int j = 0; j < 4; ++j) if (j != f) k[m++] = tets[t].v[j];
            sort3(k);
            unsigned long long h = ((unsigned long long)(unsigned)k[0] * 0x9E3779B97F4A7C15ULL) ^
                                   ((unsigned long long)(unsigned)k[1] * 0xC2B2AE3D27D4EB4FULL) ^
                                   ((unsigned long long)(unsigned)k[2] * 0x165667B19E3779F9ULL);
            size_t i = (size_t)(h >> 7) & (H - 1);
            for (;;) {
                fent* e = &tab[i];
                if (e->tet < 0) { e->a = k[0]; e->b = k[1]; e->c = k[2]; e->tet = t; e->fi = f; break; }
                if (e->a == k[0] && e->b == k[1] && e->c == k[2]) {
                    tets[t].opp[f] = e->tet;
                    tets[e->tet].opp[e->fi] = t;
                    break;
                }
                i = (i + 1) & (H - 1);
            }
        }
    free(tab);
    return ORA_OK;
}

/* ------------------------------------------------------------------------- */
/* Full pipeline                                                             */
/* ------------------------------------------------------------------------- */

int ora_triangulate(const double* xyz, int n, int G, int nthreads, int input_order,
                    ora_tet** tets_out, int* ntet_out, int* sorted_to_input, ora_stats* st) {
    ora_stats local;
    if (!st) st = &local;
    memset(st, 0, sizeof(*st));
    st->points = n;
    st->grid = G;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const double t0 = now_s();
    const long long ex0 = ora_exact_calls();

    int* order = (int*)malloc(sizeof(int) * n);
    int* vox = (int*)malloc(sizeof(int) * 3 * (size_t)n);
    double* P = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    if (!order || !vox || !P) return ORA_ERR_NOMEM;
    int rc = ora_morton_order(xyz, n, G, order, vox);
    if (rc) { free(order); free(vox); free(P); return rc; }
    for (int i = 0; i < n; ++i) memcpy(P + 3 * (size_t)i, xyz + 3 * (size_t)order[i], sizeof(double) * 3);
    const double t1 = now_s();
    st->t_order = t1 - t0;

    /* digital Voronoi diagram */
    const size_t G3 = (size_t)G * G * G;
    int* site = (int*)malloc(sizeof(int) * G3);
    if (!site) return ORA_ERR_NOMEM;
    rc = ora_edt(vox, n, G, site);
    if (rc) return rc;
    const double t2 = now_s();
    st->t_pba = t2 - t1;

    /* worksets: Voronoi pairs + missing points, reciprocated */
    octx C;
    C.P = P;
    C.n = n;
    C.fail = 0;
    C.S = (ostar*)calloc(n, sizeof(ostar));
    lvec pairs = {0};
    grid_pairs(site, G, &pairs);
    st->voronoi_pairs = pairs.n;
    for (long long i = 0; i < pairs.n; ++i) {
        const int a = (int)(pairs.a[i] >> 32), b = (int)(pairs.a[i] & 0xffffffffLL);
        iv_push(&C.S[a].hist, b);
        iv_push(&C.S[b].hist, a);
    }
    for (int i = 0; i < n; ++i) {
        const int leader = site[GI(G, vox[3 * (size_t)i], vox[3 * (size_t)i + 1], vox[3 * (size_t)i + 2])];
        if (leader != i) {
            ++st->missing;
            if (!iv_has(&C.S[i].hist, leader)) iv_push(&C.S[i].hist, leader);
            if (!iv_has(&C.S[leader].hist, i)) iv_push(&C.S[leader].hist, i);
        }
    }
    free(site);
    /* pumping (GDelKernels.cu:370-477): stars with fewer than 8 candidates
     * borrow from their candidates' worksets, then from 0,1,2,... */
    {
        int** add = (int**)calloc(n, sizeof(int*));
        int* addn = (int*)calloc(n, sizeof(int));
        for (int s = 0; s < n; ++s) {
            ostar* S = &C.S[s];
            const int need = S->hist.n < MIN_WORKSET ? MIN_WORKSET - S->hist.n : 0;
            if (!need) continue;
            add[s] = (int*)malloc(sizeof(int) * need);
            for (int i = 0; i < S->hist.n && addn[s] < need; ++i) {
                const ostar* N = &C.S[S->hist.a[i]];
                for (int j = 0; j < N->hist.n && addn[s] < need; ++j) {
                    const int c = N->hist.a[j];
                    if (c == s || iv_has(&S->hist, c)) continue;
                    int dup = 0;
                    for (int k = 0; k < addn[s]; ++k) if (add[s][k] == c) dup = 1;
                    if (!dup) add[s][addn[s]++] = c;
                }
            }
            for (int c = 0; c < n && addn[s] < need; ++c) {
                if (c == s || iv_has(&S->hist, c)) continue;
                int dup = 0;
                for (int k = 0; k < addn[s]; ++k) if (add[s][k] == c) dup = 1;
                if (!dup) add[s][addn[s]++] = c;
            }
        }
        for (int s = 0; s < n; ++s) {
            for (int k = 0; k < addn[s]; ++k) {
                const int c = add[s][k];
                if (!iv_has(&C.S[s].hist, c)) iv_push(&C.S[s].hist, c);
                if (!iv_has(&C.S[c].hist, s)) iv_push(&C.S[c].hist, s);
            }
            free(add[s]);
        }
        free(add);
        free(addn);
    }
    free(pairs.a);
    pairs.a = NULL;
    pairs.n = pairs.cap = 0;

    /* initial stars: cone from the 4 first candidates, then insert the rest */
    long long wtotal = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : wtotal)
    for (int s = 0; s < n; ++s) {
        ostar* S = &C.S[s];
        qsort(S->hist.a, S->hist.n, sizeof(int), cmp_int);
        wtotal += S->hist.n;
        make_cone(P, S, s, S->hist.a[0], S->hist.a[1], S->hist.a[2], S->hist.a[3]);
        for (int i = 4; i < S->hist.n; ++i) star_insert(P, S, s, S->hist.a[i]);
        compact_tris(S);
        for (int i = 0; i < S->hist.n; ++i) iv_push(&S->changed, S->hist.a[i]);
    }
    st->workset_total = wtotal;
    st->star_insertions = wtotal;
    const double t3 = now_s();
    st->t_star = t3 - t2;

    /* splaying rounds (GDelHost.cu:1389-1470) */
    int repairs = 0;
    for (int loop = 0;; ++loop) {
        if (loop > 100000) { C.fail = 2; break; }
        lvec req = {0};
        drowned_proofs(&C, &req, &st->drowned, &st->proofs);
        fresh_requests(&C, &req, 0);
        const long long added = dispatch_pairs(&C, &req);
        free(req.a);
        if (C.fail) break;
        if (added == 0) {
            const long long bad = count_inconsistent(&C);
            if (bad == 0) { st->loops = loop; break; }
            if (++repairs > 3) { C.fail = 3; break; }
            ++st->consistency_repairs;
            lvec r2 = {0};
            fresh_requests(&C, &r2, 1);
            const long long a2 = dispatch_pairs(&C, &r2);
            free(r2.a);
            if (a2 == 0) { C.fail = 3; break; }
        }
        insert_pending(&C, &st->splay_insertions);
    }
    const double t4 = now_s();
    st->t_splay = t4 - t3;
    if (C.fail) {
        for (int s = 0; s < n; ++s) { free(C.S[s].t); free(C.S[s].hist.a); free(C.S[s].pend.a); free(C.S[s].changed.a); }
        free(C.S); free(P); free(vox); free(order);
        return C.fail == 2 ? ORA_ERR_TIMEOUT : ORA_ERR_INTERNAL;
    }

    /* extraction: owner triangles on the lower hull (GDelHost.cu:1520-1607) */
    int* base = (int*)malloc(sizeof(int) * (n + 1));
    base[0] = 0;
    int maxl = 0;
    for (int s = 0; s < n; ++s) {
        const ostar* S = &C.S[s];
        int c = 0;
        for (int i = 0; i < S->nt; ++i) {
            const otri* t = &S->t[i];
            if (t->alive && s < t->v[0] && s < t->v[1] && s < t->v[2]) ++c;
        }
        base[s + 1] = base[s] + c;
        if (S->nt > maxl) maxl = S->nt;
    }
    st->max_link = (maxl + 4) / 2;
    for (int s = 0; s < n; ++s)
        if (C.S[s].hist.n > st->max_hist) st->max_hist = C.S[s].hist.n;
    const int nown = base[n];
    ora_tet* tets = (ora_tet*)malloc(sizeof(ora_tet) * (nown ? nown : 1));
    unsigned char* keep = (unsigned char*)calloc(nown ? nown : 1, 1);
#pragma omp parallel for schedule(dynamic, 64)
    for (int s = 0; s < n; ++s) {
        const ostar* S = &C.S[s];
        int k = base[s];
        for (int i = 0; i < S->nt; ++i) {
            const otri* t = &S->t[i];
            if (!(t->alive && s < t->v[0] && s < t->v[1] && s < t->v[2])) continue;
            ora_tet* T = &tets[k];
            T->v[0] = t->v[0]; T->v[1] = t->v[1]; T->v[2] = t->v[2]; T->v[3] = s;
            keep[k] = ora_orient3d(P + 3 * (size_t)t->v[0], P + 3 * (size_t)t->v[1],
                                   P + 3 * (size_t)t->v[2], P + 3 * (size_t)s) < 0;
            ++k;
        }
    }
    int nt = 0;
    for (int i = 0; i < nown; ++i) if (keep[i]) tets[nt++] = tets[i];
    free(keep);
    free(base);
    rc = link_adjacency(tets, nt);
    if (input_order)
        for (int i = 0; i < nt; ++i)
            for (int k = 0; k < 4; ++k) tets[i].v[k] = order[tets[i].v[k]];
    if (sorted_to_input) memcpy(sorted_to_input, order, sizeof(int) * n);
    const double t5 = now_s();
    st->t_out = t5 - t4;
    st->t_total = t5 - t0;
    st->exact_calls = ora_exact_calls() - ex0;
    for (int s = 0; s < n; ++s) { free(C.S[s].t); free(C.S[s].hist.a); free(C.S[s].pend.a); free(C.S[s].changed.a); }
    free(C.S);
    free(P);
    free(vox);
    free(order);
    *tets_out = tets;
    *ntet_out = nt;
    return rc;
}
