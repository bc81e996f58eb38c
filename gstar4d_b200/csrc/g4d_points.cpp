// The command line's point generator (host code, no device needed).
//
// Restates Application::makePoints (Main/Application.cpp:316-473) and its
// random numbers, DtRandom (Common/DtRandom.cpp:44-109): Marsaglia's KISS
// combination of a multiply-with-carry pair, a 3-shift register and a
// congruential generator. The reference keeps the generator state in
// `unsigned long`, which is 64 bits on the LP64 systems this library runs on,
// so every state update below is 64-bit unsigned arithmetic (the sequences
// differ from a Windows build of the reference, where the type has 32 bits).
// Coordinates are float values in grid units [1, G-2]; a point equal to an
// earlier one is drawn again. The float/double evaluation follows the
// reference's expressions: float arithmetic where its operands are float, the
// logarithm and square root of the Gaussian transform in double (the C
// library's log and sqrt, which the reference's unqualified calls resolve to).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_set>

#include "gstar4d.h"

namespace {

class Kiss {
public:
    Kiss(int seed, int lo, int hi)
        : z_((uint64_t)(int64_t)seed), w_((uint64_t)(int64_t)seed), jsr_((uint64_t)(int64_t)seed),
          jcong_((uint64_t)(int64_t)seed), lo_((float)lo), hi_((float)hi) {}

    // uniform in [lo, hi] (the top end is reached when the integer rounds up
    // to 2^64 in float)
    float next() { return lo_ + (hi_ - lo_) * unit(); }

    // three coordinates from a 3D Marsaglia polar draw, truncated to
    // [-3, 3) standard deviations and mapped onto [lo, hi]
    void gaussian(float& x, float& y, float& z) {
        float a, b, c, tx, ty, tz;
        for (;;) {
            float s;
            do {
                a = 2.0f * unit() - 1.0f;
                b = 2.0f * unit() - 1.0f;
                c = 2.0f * unit() - 1.0f;
                s = a * a + b * b + c * c;
            } while ((double)s >= 1.0);
            const float f = (float)std::sqrt((-2.0 * std::log((double)s)) / (double)s);
            tx = a * f;
            ty = b * f;
            tz = c * f;
            if (!(tx < -3.0f || tx >= 3.0f || ty < -3.0f || ty >= 3.0f || tz < -3.0f || tz >= 3.0f)) break;
        }
        x = lo_ + (hi_ - lo_) * ((tx + 3.0f) / 6.0f);
        y = lo_ + (hi_ - lo_) * ((ty + 3.0f) / 6.0f);
        z = lo_ + (hi_ - lo_) * ((tz + 3.0f) / 6.0f);
    }

private:
    uint64_t bits() {
        z_ = 36969u * (z_ & 0xffffu) + (z_ >> 16);
        w_ = 18000u * (w_ & 0xffffu) + (w_ >> 16);
        const uint64_t mwc = (z_ << 16) + w_;
        jcong_ = 69069u * jcong_ + 1234567u;
        jsr_ ^= jsr_ << 17;
        jsr_ ^= jsr_ >> 13;
        jsr_ ^= jsr_ << 5;
        return (mwc ^ jcong_) + jsr_;
    }
    // the 64-bit integer rounded to float, over 2^64 (float(ULONG_MAX) + 1)
    float unit() { return (float)bits() / ((float)UINT64_MAX + 1.0f); }

    uint64_t z_, w_, jsr_, jcong_;
    float lo_, hi_;
};

struct Key {
    uint32_t a, b, c;
    bool operator==(const Key& o) const { return a == o.a && b == o.b && c == o.c; }
};
struct KeyHash {
    size_t operator()(const Key& k) const {
        uint64_t h = ((uint64_t)k.a << 32 | k.b) * 0x9E3779B97F4A7C15ull;
        return (size_t)(h ^ ((uint64_t)k.c * 0xC2B2AE3D27D4EB4Full) ^ (h >> 29));
    }
};

uint32_t fbits(float v) {
    uint32_t u;
    std::memcpy(&u, &v, sizeof(u));
    return u;
}

}  // namespace

// Coordinates are positive (at least 1 for the cube distributions, at least
// 0.05 (G-2) for the ball and the sphere), so equal values have equal bits and
// the set can key on the bit patterns.
extern "C" G4D_API g4d_status g4d_make_points(int n, int dist, int grid, int seed, double* xyz) {
    if (n < 0 || !xyz || dist < 0 || dist > 4 || grid < 8) return G4D_ERR_ARG;
    const int lo = 1, hi = grid - 2;
    const bool unit_cube = dist == 2 || dist == 3;  // ball and sphere draw in [0, 1] and scale
    Kiss rng(seed, unit_cube ? 0 : lo, unit_cube ? 1 : hi);
    std::unordered_set<Key, KeyHash> seen;
    seen.reserve((size_t)n * 2);
    const float r_out = 0.45f * 0.45f, r_in = 0.4f * 0.4f;
    for (int i = 0; i < n;) {
        float x = 0.f, y = 0.f, z = 0.f;
        switch (dist) {
            case 0:
                x = rng.next();
                y = rng.next();
                z = rng.next();
                break;
            case 1:
                rng.gaussian(x, y, z);
                break;
            case 2:
            case 3: {
                float d;
                do {
                    x = rng.next() - 0.5f;
                    y = rng.next() - 0.5f;
                    z = rng.next() - 0.5f;
                    d = x * x + y * y + z * z;
                } while (d > r_out || (dist == 3 && d < r_in));
                x = (x + 0.5f) * (float)hi;
                y = (y + 0.5f) * (float)hi;
                z = (z + 0.5f) * (float)hi;
                break;
            }
            default: {
                float v[3];
                for (int k = 0; k < 3; ++k) {
                    const float val = rng.next();
                    const float frac = (float)((double)val - std::floor((double)val));
                    v[k] = (float)(frac < 0.5f ? std::floor((double)val) : std::ceil((double)val));
                }
                x = v[0];
                y = v[1];
                z = v[2];
            }
        }
        // a coordinate that reached the top cell moves one cell down
        if (std::floor((double)x) >= hi) x -= 1.0f;
        if (std::floor((double)y) >= hi) y -= 1.0f;
        if (std::floor((double)z) >= hi) z -= 1.0f;
        if (!seen.insert(Key{fbits(x), fbits(y), fbits(z)}).second) continue;
        xyz[3 * (size_t)i] = x;
        xyz[3 * (size_t)i + 1] = y;
        xyz[3 * (size_t)i + 2] = z;
        ++i;
    }
    return G4D_OK;
}
