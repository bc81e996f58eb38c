// Input scaling, Morton keys and the sorted point layout.
//
// Restates Application::_scalePoint (Main/Application.cpp:589-603: one min and
// max over all coordinates, p -> 1 + (G-3)(p-min)/(max-min)) and the Morton
// order of PointData::init (GDelaunay/GDelData.cu:51-134: 10 bits per axis,
// x in bit 0, stable sort). The Morton positions are the Simulation-of-
// Simplicity ranks, so the arithmetic here is IEEE round-to-nearest with no
// contraction, identical to the reference's host-side double evaluation.
#include "g4d_internal.cuh"

namespace g4d {

__device__ __forceinline__ unsigned long long dkey(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
    const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__global__ void k_minmax(const double* __restrict__ xyz, long long m, unsigned long long* mm) {
    unsigned long long lo = ~0ull, hi = 0ull;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const unsigned long long k = dkey(xyz[i]);
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// mode: mm != nullptr -> scale xyz with the global min/max; else grid_src holds
// grid coordinates (the reference's scaled points, or points already in grid units).
__global__ void k_scale_morton(const double* __restrict__ xyz, const double* __restrict__ grid_src, int n, int G,
                               const unsigned long long* __restrict__ mm, uint32_t* __restrict__ keys,
                               int* __restrict__ vals, uint32_t* __restrict__ vox_in, unsigned* err) {
    double mn = 0.0, rng = 1.0;
    if (mm) {
        mn = dkey_inv(mm[0]);
        rng = __dsub_rn(dkey_inv(mm[1]), mn);
    }
    const double g3 = (double)(G - 3);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t q[3];
        for (int c = 0; c < 3; ++c) {
            double t;
            if (mm) {
                t = __dsub_rn(xyz[3 * (size_t)i + c], mn);
                t = __dmul_rn(g3, t);
                t = __ddiv_rn(t, rng);
                t = __dadd_rn(t, 1.0);
            } else {
                t = grid_src[3 * (size_t)i + c];
            }
            int v = (int)t;
            if (!(t >= 1.0) || v > G - 2) {
                atomicOr(err, 0x100u);  // coordinates outside [1, G-2]
                v = v < 1 ? 1 : (v > G - 2 ? G - 2 : v);
            }
            q[c] = (uint32_t)v;
        }
        // keys and vals feed the Morton sort; callers without one pass null
        if (keys) keys[i] = spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
        if (vals) vals[i] = i;
        vox_in[i] = enc_vox(q[0], q[1], q[2]);
    }
}

__global__ void k_gather(const double* __restrict__ xyz, const uint32_t* __restrict__ vox_in,
                         const int* __restrict__ order, int n, double4* __restrict__ P, uint32_t* __restrict__ vox,
                         int* __restrict__ sorted_to_input) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = order[i];
        P[i] = make_double4(xyz[3 * (size_t)s], xyz[3 * (size_t)s + 1], xyz[3 * (size_t)s + 2], 0.0);
        vox[i] = vox_in[s];
        if (sorted_to_input) sorted_to_input[i] = s;
    }
}

__global__ void k_colkeys(const uint32_t* __restrict__ vox, int n, int G, uint32_t* __restrict__ ckey,
                          int* __restrict__ cid) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = vox[i];
        ckey[i] = ((vy(e) * (uint32_t)G + vx(e)) << 10) | vz(e);
        cid[i] = i;
    }
}

template <class KeyT>
__global__ void k_colranges(const KeyT* __restrict__ ckey, int n, int* __restrict__ cs, int* __restrict__ ce) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const KeyT c = ckey[i] >> 10;
        if (i == 0 || (ckey[i - 1] >> 10) != c) cs[c] = i;
        if (i == n - 1 || (ckey[i + 1] >> 10) != c) ce[c] = i + 1;
    }
}

static int blocks_for(long long work, int threads) {
    long long b = (work + threads - 1) / threads;
    const long long cap = 148LL * 16;
    if (b > cap) b = cap;
    return (int)(b < 1 ? 1 : b);
}

void launch_minmax(const Launch& L, const double* xyz, int n, unsigned long long* mm) {
    k_minmax<<<blocks_for(3LL * n, 256), 256, 0, L.stream>>>(xyz, 3LL * n, mm);
    ++*L.launches;
}

void launch_scale_morton(const Launch& L, const double* xyz, const double* grid_src, int n, int G,
                         const unsigned long long* mm, uint32_t* keys, int* vals, uint32_t* vox_in, unsigned* err) {
    k_scale_morton<<<blocks_for(n, 256), 256, 0, L.stream>>>(xyz, grid_src, n, G, mm, keys, vals, vox_in, err);
    ++*L.launches;
}

void launch_gather(const Launch& L, const double* xyz, const uint32_t* vox_in, const int* order, int n, double4* P,
                   uint32_t* vox, int* sorted_to_input) {
    k_gather<<<blocks_for(n, 256), 256, 0, L.stream>>>(xyz, vox_in, order, n, P, vox, sorted_to_input);
    ++*L.launches;
}

void launch_colkeys(const Launch& L, const uint32_t* vox, int n, int G, uint32_t* ckey, int* cid) {
    k_colkeys<<<blocks_for(n, 256), 256, 0, L.stream>>>(vox, n, G, ckey, cid);
    ++*L.launches;
}

void launch_colranges(const Launch& L, const uint32_t* ckey, int n, int G, int* colStart, int* colEnd) {
    (void)G;
    k_colranges<<<blocks_for(n, 256), 256, 0, L.stream>>>(ckey, n, colStart, colEnd);
    ++*L.launches;
}


// ---------------------------------------------------------------------------
// Batches. The clouds of one pass ("slots", grouped by grid width) are sorted
// together under 64-bit keys slot << 30 | Morton, so every cloud's points stay
// contiguous and in its own Morton order; slotW[k] is the first sorted position
// of slot k (and the first position of its points in the pass's input order).
// ---------------------------------------------------------------------------

// per-slot min and max over all coordinates of the cloud (one block per slot)
__global__ void k_b_minmax(const double* __restrict__ xyz, const long long* __restrict__ slotIn,
                           const int* __restrict__ slotW, unsigned long long* __restrict__ mm) {
    __shared__ unsigned long long slo[32], shi[32];
    const int k = blockIdx.x;
    const long long m = 3LL * (slotW[k + 1] - slotW[k]);
    const double* p = xyz + 3 * slotIn[k];
    unsigned long long lo = ~0ull, hi = 0ull;
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        const unsigned long long v = dkey(p[i]);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) { slo[threadIdx.x >> 5] = lo; shi[threadIdx.x >> 5] = hi; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            lo = slo[w] < lo ? slo[w] : lo;
            hi = shi[w] > hi ? shi[w] : hi;
        }
        mm[2 * k] = lo;
        mm[2 * k + 1] = hi;
    }
}

// per-slot scaling (the same arithmetic as k_scale_morton), 64-bit sort keys
__global__ void k_b_scale(const double* __restrict__ xyz, const long long* __restrict__ slotIn,
                          const int* __restrict__ slotW, const int* __restrict__ slotG,
                          const unsigned long long* __restrict__ mm, unsigned long long* __restrict__ keys,
                          int* __restrict__ vals, uint32_t* __restrict__ vox_in, long long* __restrict__ gidx,
                          unsigned* err) {
    const int k = blockIdx.x;
    const int w0 = slotW[k], n = slotW[k + 1] - w0, G = slotG[k];
    const long long in0 = slotIn[k];
    const double mn = dkey_inv(mm[2 * k]);
    const double rng = __dsub_rn(dkey_inv(mm[2 * k + 1]), mn);
    const double g3 = (double)(G - 3);
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const long long i = in0 + j;
        uint32_t q[3];
        for (int c = 0; c < 3; ++c) {
            double t = __dsub_rn(xyz[3 * i + c], mn);
            t = __dmul_rn(g3, t);
            t = __ddiv_rn(t, rng);
            t = __dadd_rn(t, 1.0);
            int v = (int)t;
            if (!(t >= 1.0) || v > G - 2) {
                atomicOr(err, 0x100u);
                v = v < 1 ? 1 : (v > G - 2 ? G - 2 : v);
            }
            q[c] = (uint32_t)v;
        }
        const int w = w0 + j;
        keys[w] = ((unsigned long long)k << 30) | spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2);
        vals[w] = w;
        vox_in[w] = enc_vox(q[0], q[1], q[2]);
        gidx[w] = i;
    }
}

// sorted layout: coordinates, voxels, cloud-local input index of every point
__global__ void k_b_gather(const double* __restrict__ xyz, const long long* __restrict__ gidx,
                           const uint32_t* __restrict__ vox_in, const int* __restrict__ order,
                           const unsigned long long* __restrict__ skey, const int* __restrict__ slotW, int n,
                           double4* __restrict__ P, uint32_t* __restrict__ vox, int* __restrict__ local) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int w = order[i];
        const long long g = gidx[w];
        P[i] = make_double4(xyz[3 * g], xyz[3 * g + 1], xyz[3 * g + 2], 0.0);
        vox[i] = vox_in[w];
        local[i] = w - slotW[(int)(skey[i] >> 30)];
    }
}

// column keys: (column of the slot's grid in the stacked column index) << 10 | z
__global__ void k_b_colkeys(const uint32_t* __restrict__ vox, const unsigned long long* __restrict__ skey,
                            const int* __restrict__ slotG, const long long* __restrict__ slotCol, int n,
                            unsigned long long* __restrict__ ckey, int* __restrict__ cid) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int k = (int)(skey[i] >> 30);
        const uint32_t e = vox[i];
        const unsigned long long col = (unsigned long long)slotCol[k] + (unsigned long long)vy(e) * slotG[k] + vx(e);
        ckey[i] = (col << 10) | vz(e);
        cid[i] = i;
    }
}

// float coordinates widened to double (exact: every float is a double)
__global__ void k_f32_to_f64(const float* __restrict__ in, size_t count, double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

void launch_f32_to_f64(const Launch& L, const float* in, size_t count, double* out) {
    size_t blocks = (count + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_f32_to_f64<<<(int)(blocks < 1 ? 1 : blocks), 256, 0, L.stream>>>(in, count, out);
    ++*L.launches;
}

// tetrahedra per slot
__global__ void k_b_slot_tets(const int* __restrict__ base, const int* __restrict__ slotW, int nslots,
                              int* __restrict__ tc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nslots; k += gridDim.x * blockDim.x)
        tc[k] = base[slotW[k + 1]] - base[slotW[k]];
}

// cloud-local tetrahedra: point ids -> the cloud's input indices, neighbour ids
// -> the cloud's own tetrahedron numbering, written at the cloud's output offset
__global__ void k_b_localize(const g4d_tet* __restrict__ in, int ntet, const unsigned long long* __restrict__ skey,
                             const int* __restrict__ local, const int* __restrict__ base,
                             const int* __restrict__ slotW, const long long* __restrict__ dst,
                             g4d_tet* __restrict__ out) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        g4d_tet T = in[t];
        const int k = (int)(skey[T.v[3]] >> 30);
        const int tb = base[slotW[k]];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T.v[i] = local[T.v[i]];
            T.opp[i] = T.opp[i] >= 0 ? T.opp[i] - tb : -1;
        }
        out[dst[k] + (t - tb)] = T;
    }
}

// Distribution class input: occupancy of an 8^3 histogram of a strided sample
// of up to 4096 points of each cloud (one block per cloud). The host function
// occupancy() in g4d_api.cu does the same arithmetic in the same order.
__global__ void k_b_occupancy(const double* __restrict__ xyz, const long long* __restrict__ offs, int* __restrict__ occ) {
    __shared__ unsigned long long slo[8], shi[8];
    __shared__ unsigned bits[16];
    const int c = blockIdx.x;
    const long long n = offs[c + 1] - offs[c];
    const long long m = n < 4096 ? n : 4096;
    const long long step = n / m > 1 ? n / m : 1;
    const double* p = xyz + 3 * offs[c];
    unsigned long long lo = ~0ull, hi = 0ull;
    for (long long k = threadIdx.x; k < 3 * m; k += blockDim.x) {
        const unsigned long long v = dkey(p[3 * ((k / 3) * step) + k % 3]);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if (threadIdx.x < 16) bits[threadIdx.x] = 0;
    if ((threadIdx.x & 31) == 0) { slo[threadIdx.x >> 5] = lo; shi[threadIdx.x >> 5] = hi; }
    __syncthreads();
    lo = slo[0];
    hi = shi[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
        lo = slo[w] < lo ? slo[w] : lo;
        hi = shi[w] > hi ? shi[w] : hi;
    }
    const double dlo = dkey_inv(lo), dhi = dkey_inv(hi);
    const double span = dhi > dlo ? __dsub_rn(dhi, dlo) : 1.0;
    for (long long i = threadIdx.x; i < m; i += blockDim.x) {
        int q[3];
        for (int k = 0; k < 3; ++k) {
            const int b = (int)__ddiv_rn(__dmul_rn(8.0, __dsub_rn(p[3 * (i * step) + k], dlo)), span);
            q[k] = b < 7 ? b : 7;
        }
        const int cell = (q[2] * 8 + q[1]) * 8 + q[0];
        atomicOr(&bits[cell >> 5], 1u << (cell & 31));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int f = 0;
        for (int w = 0; w < 16; ++w) f += __popc(bits[w]);
        occ[c] = f;
    }
}

void launch_b_occupancy(const Launch& L, const double* xyz, const long long* offs, int nclouds, int* occ) {
    k_b_occupancy<<<nclouds, 256, 0, L.stream>>>(xyz, offs, occ);
    ++*L.launches;
}

void launch_b_order(const Launch& L, const double* xyz, int nslots, const long long* slotIn, const int* slotW,
                    const int* slotG, unsigned long long* mm, unsigned long long* keys, int* vals, uint32_t* vox_in,
                    long long* gidx, unsigned* err) {
    k_b_minmax<<<nslots, 256, 0, L.stream>>>(xyz, slotIn, slotW, mm);
    k_b_scale<<<nslots, 256, 0, L.stream>>>(xyz, slotIn, slotW, slotG, mm, keys, vals, vox_in, gidx, err);
    *L.launches += 2;
}

void launch_b_gather(const Launch& L, const double* xyz, const long long* gidx, const uint32_t* vox_in,
                     const int* order, const unsigned long long* skey, const int* slotW, int n, double4* P,
                     uint32_t* vox, int* local) {
    k_b_gather<<<blocks_for(n, 256), 256, 0, L.stream>>>(xyz, gidx, vox_in, order, skey, slotW, n, P, vox, local);
    ++*L.launches;
}

void launch_b_colkeys(const Launch& L, const uint32_t* vox, const unsigned long long* skey, const int* slotG,
                      const long long* slotCol, int n, unsigned long long* ckey, int* cid) {
    k_b_colkeys<<<blocks_for(n, 256), 256, 0, L.stream>>>(vox, skey, slotG, slotCol, n, ckey, cid);
    ++*L.launches;
}

void launch_colranges_u64(const Launch& L, const unsigned long long* ckey, int n, int* colStart, int* colEnd) {
    k_colranges<<<blocks_for(n, 256), 256, 0, L.stream>>>(ckey, n, colStart, colEnd);
    ++*L.launches;
}

void launch_b_slot_tets(const Launch& L, const int* base, const int* slotW, int nslots, int* tc) {
    k_b_slot_tets<<<blocks_for(nslots, 256), 256, 0, L.stream>>>(base, slotW, nslots, tc);
    ++*L.launches;
}

void launch_b_localize(const Launch& L, const g4d_tet* in, int ntet, const unsigned long long* skey,
                       const int* local, const int* base, const int* slotW, const long long* dst, g4d_tet* out) {
    k_b_localize<<<blocks_for(ntet, 256), 256, 0, L.stream>>>(in, ntet, skey, local, base, slotW, dst, out);
    ++*L.launches;
}

}  // namespace g4d
