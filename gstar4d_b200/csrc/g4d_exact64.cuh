// Exact sign of the lifted 5x5 determinant for integer points below 2^61 in
// magnitude, in 64-bit limbs with every width bounded by its operands:
//   D  = P[r] - P[4]                         |D|   < 2^62        int64
//   m2 = Dx_i Dy_j - Dx_j Dy_i               |m2|  < 2^125       2 limbs, two's complement
//   m3 = Dz_i m2_jk - Dz_j m2_ik + Dz_k m2_ij |m3| < 3 2^187     3 limbs, two's complement
//   L  = Dx^2 + Dy^2 + Dz^2                  L     < 3 2^124     2 limbs, unsigned
//   det = -L0 m3_0 + L1 m3_1 - L2 m3_2 + L3 m3_3, |det| < 2^317  5 limbs, two's complement
// This is the same expansion, term for term, as the general multi-limb
// routine (orient4_int), which stays the path for wider coordinates; it is
// plain C++ on the host as well, so the host tests compare it with
// arbitrary-precision integers.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define G4D_HD __host__ __device__ __forceinline__
#else
#define G4D_HD inline
#endif

namespace g4d {
namespace x64 {

G4D_HD void umul(uint64_t a, uint64_t b, uint64_t* lo, uint64_t* hi) {
#ifdef __CUDA_ARCH__
    *lo = a * b;
    *hi = __umul64hi(a, b);
#else
    const unsigned __int128 p = (unsigned __int128)a * b;
    *lo = (uint64_t)p;
    *hi = (uint64_t)(p >> 64);
#endif
}

// two's complement negation of n limbs
G4D_HD void neg(uint64_t* a, int n) {
    uint64_t c = 1;
    for (int i = 0; i < n; ++i) {
        const uint64_t t = ~a[i] + c;
        c = (c && t == 0) ? 1 : 0;
        a[i] = t;
    }
}

// acc (N limbs, two's complement) += mag or -= mag (n <= N limbs, unsigned)
template <int N>
G4D_HD void addsub(uint64_t* acc, const uint64_t* mag, int n, bool sub) {
    uint64_t carry = sub ? 1 : 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        uint64_t m = i < n ? mag[i] : 0;
        if (sub) m = ~m;
        const uint64_t s = acc[i] + m;
        uint64_t c = s < m ? 1 : 0;
        const uint64_t s2 = s + carry;
        c += s2 < carry ? 1 : 0;
        acc[i] = s2;
        carry = c;
    }
}

// r[0..na+nb) = a * b, unsigned
template <int NA, int NB>
G4D_HD void mulmag(const uint64_t* a, const uint64_t* b, uint64_t* r) {
#pragma unroll
    for (int k = 0; k < NA + NB; ++k) r[k] = 0;
#pragma unroll
    for (int i = 0; i < NA; ++i) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            uint64_t lo, hi;
            umul(a[i], b[j], &lo, &hi);
            const uint64_t t = r[i + j] + lo;
            uint64_t c = t < lo ? 1 : 0;
            const uint64_t t2 = t + carry;
            c += t2 < carry ? 1 : 0;
            r[i + j] = t2;
            carry = hi + c;  // the 128-bit total fits, so this cannot wrap
        }
        r[i + NB] = carry;
    }
}

G4D_HD uint64_t absu(int64_t v) { return v < 0 ? (uint64_t)0 - (uint64_t)v : (uint64_t)v; }

// signed 64 x 64 -> 128 (two limbs, two's complement)
G4D_HD void smul(int64_t a, int64_t b, uint64_t* r) {
    uint64_t lo, hi;
    umul(absu(a), absu(b), &lo, &hi);
    r[0] = lo;
    r[1] = hi;
    if ((a < 0) != (b < 0)) neg(r, 2);
}

// true when every coordinate is below 2^61 in magnitude
G4D_HD bool fits61(const int64_t (*X)[3]) {
    uint64_t o = 0;
    for (int i = 0; i < 5; ++i)
        for (int c = 0; c < 3; ++c) o |= absu(X[i][c]);
    return o < (1ull << 61);
}

// sign of the lifted determinant over points X[0..4] (translated by X[4]);
// requires fits61(X)
G4D_HD int orient4_sign(const int64_t (*X)[3]) {
    int64_t D[4][3];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 3; ++c) D[r][c] = X[r][c] - X[4][c];
    uint64_t m2[4][4][2];
#pragma unroll 1
    for (int i = 0; i < 4; ++i)
#pragma unroll 1
        for (int j = i + 1; j < 4; ++j) {
            uint64_t p[2], q[2];
            smul(D[i][0], D[j][1], p);
            smul(D[j][0], D[i][1], q);
            neg(q, 2);
            const uint64_t lo = p[0] + q[0];
            m2[i][j][0] = lo;
            m2[i][j][1] = p[1] + q[1] + (lo < p[0] ? 1 : 0);
        }
    const int tri[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
    uint64_t det[5] = {0, 0, 0, 0, 0};
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        const int i = tri[r][0], j = tri[r][1], k = tri[r][2];
        // m3 = Dz_i m2[j][k] - Dz_j m2[i][k] + Dz_k m2[i][j]
        uint64_t m3[3] = {0, 0, 0};
        const int rows[3] = {i, j, k};
        const int pr[3][2] = {{j, k}, {i, k}, {i, j}};
#pragma unroll 1
        for (int t = 0; t < 3; ++t) {
            const int64_t z = D[rows[t]][2];
            uint64_t m[2] = {m2[pr[t][0]][pr[t][1]][0], m2[pr[t][0]][pr[t][1]][1]};
            bool sub = t == 1;
            if ((int64_t)m[1] < 0) {
                neg(m, 2);
                sub = !sub;
            }
            if (z < 0) sub = !sub;
            const uint64_t az = absu(z);
            uint64_t prod[3];
            mulmag<1, 2>(&az, m, prod);
            addsub<3>(m3, prod, 3, sub);
        }
        // L = Dx^2 + Dy^2 + Dz^2
        uint64_t L[2] = {0, 0};
#pragma unroll 1
        for (int c = 0; c < 3; ++c) {
            const uint64_t a = absu(D[r][c]);
            uint64_t sq[2];
            umul(a, a, &sq[0], &sq[1]);
            addsub<2>(L, sq, 2, false);
        }
        bool sub = (r & 1) == 0;  // det = -L0 m3_0 + L1 m3_1 - L2 m3_2 + L3 m3_3
        if ((int64_t)m3[2] < 0) {
            neg(m3, 3);
            sub = !sub;
        }
        uint64_t term[5];
        mulmag<2, 3>(L, m3, term);
        addsub<5>(det, term, 5, sub);
    }
    if ((int64_t)det[4] < 0) return -1;
    return (det[0] | det[1] | det[2] | det[3] | det[4]) ? 1 : 0;
}

}  // namespace x64
}  // namespace g4d
