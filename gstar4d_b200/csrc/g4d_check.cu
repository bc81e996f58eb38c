// Device validator of a tetrahedral mesh: the checks of the reference's
// TetraMesh::check (Common/Geometry.cu:200-393), run on the GPU so that the
// -check flag stays fast at millions of points.
//
//  - Euler characteristic V - E + F - T (1 for a triangulated ball), with V, E
//    and F counted as distinct vertices, edges and triangles of the tetrahedron
//    list (the reference sorts and uniques on the host; here CUB radix sorts:
//    edges as one 64-bit key, triangles by a two-pass least-significant-digit
//    sort, third vertex first, then the first two);
//  - orientation: a tetrahedron fails when orient3d(v0, v1, v2, v3) > 0;
//  - in-sphere: for every interior face, taken once from its tetrahedron of
//    smaller index, the vertex of the neighbour opposite the face fails when
//    insphere(v0, v1, v2, v3, opposite) < 0.
// orient3d and insphere are the exact signs of Shewchuk's predicates (the
// filter and exact stages of g4d_predicates.cuh, no Simulation of Simplicity,
// as in the reference's validator). A neighbour index out of range, or a
// neighbour that does not link back (checked from both sides), counts as an
// adjacency failure (the reference asserts on it).
#include <cub/cub.cuh>

#include "g4d_internal.cuh"
#include "g4d_predicates.cuh"

namespace g4d {

namespace {

__device__ __forceinline__ int remap(const int* inv, int v) { return inv ? inv[v] : v; }

__device__ __forceinline__ double3 pt(const double4* P, const int* inv, int v) {
    const double4 q = P[remap(inv, v)];
    return make_double3(q.x, q.y, q.z);
}

// sorted vertex ids of face f (the face opposite v[f])
__device__ __forceinline__ void face_ids(const g4d_tet& t, int f, int& a, int& b, int& c) {
    int w[3], k = 0;
    for (int i = 0; i < 4; ++i)
        if (i != f) w[k++] = t.v[i];
    a = min(w[0], min(w[1], w[2]));
    c = max(w[0], max(w[1], w[2]));
    b = w[0] + w[1] + w[2] - a - c;
}

// Shewchuk's insphere sign: the lifted orientation without SoS (0 when the
// five points are cospherical)
__device__ __noinline__ int insphere_sign(const double3* q, unsigned* err) {
    int f = orient4_filter(q[0], q[1], q[2], q[3], q[4]);
    if (f) return f;
    IntPts<2> P;
    if (to_int_points<2>(q, 5, P)) return orient4_int<2>(P);
    IntPts<4> P4;
    if (to_int_points<4>(q, 5, P4)) return orient4_int<4>(P4);
    atomicOr(err, PRED_ERR_PRECISION);
    return 0;
}

}  // namespace

__global__ void k_chk_inverse(const int* __restrict__ order, int n, int* __restrict__ inv) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) inv[order[i]] = i;
}

// vertex marks and the 6 edge keys of every tetrahedron
__global__ void k_chk_edges(const g4d_tet* __restrict__ tets, int ntet, int n, int* __restrict__ mark,
                            unsigned long long* __restrict__ ekey, unsigned* err) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        const g4d_tet T = tets[t];
        bool ok = true;
        for (int i = 0; i < 4; ++i) ok = ok && T.v[i] >= 0 && T.v[i] < n;
        if (!ok) atomicOr(err, 0x200u);  // a vertex id out of range
        int e = 0;
        for (int i = 0; i < 4; ++i) {
            if (ok) mark[T.v[i]] = 1;
            for (int j = i + 1; j < 4; ++j) {
                const unsigned long long a = (unsigned)min(T.v[i], T.v[j]), b = (unsigned)max(T.v[i], T.v[j]);
                ekey[6 * (size_t)t + e++] = (a << 32) | b;
            }
        }
    }
}

// the third (largest) vertex of each of the 4 triangles, and the triangle's
// index 4 t + f
__global__ void k_chk_tris(const g4d_tet* __restrict__ tets, int ntet, uint32_t* __restrict__ tkey_c,
                           uint32_t* __restrict__ tidx) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        const g4d_tet T = tets[t];
        for (int f = 0; f < 4; ++f) {
            int a, b, c;
            face_ids(T, f, a, b, c);
            tkey_c[4 * (size_t)t + f] = (uint32_t)c;
            tidx[4 * (size_t)t + f] = 4u * (uint32_t)t + f;
        }
    }
}

// the (a, b) key of each triangle in the order of the first sort pass
__global__ void k_chk_tri_ab(const g4d_tet* __restrict__ tets, const uint32_t* __restrict__ tidx, size_t m,
                             unsigned long long* __restrict__ ab) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t k = tidx[i];
        int a, b, c;
        face_ids(tets[k >> 2], (int)(k & 3u), a, b, c);
        ab[i] = ((unsigned long long)(unsigned)a << 32) | (unsigned)b;
    }
}

// distinct values of a sorted key array
__global__ void k_chk_distinct_u64(const unsigned long long* __restrict__ k, size_t m, unsigned long long* count) {
    unsigned long long c = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x)
        c += (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// distinct triangles: sorted by (a, b) and, among equal (a, b), by c
__global__ void k_chk_distinct_tri(const g4d_tet* __restrict__ tets, const unsigned long long* __restrict__ ab,
                                   const uint32_t* __restrict__ tidx, size_t m, unsigned long long* count) {
    unsigned long long cnt = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < m; i += (size_t)gridDim.x * blockDim.x) {
        bool fresh = i == 0 || ab[i] != ab[i - 1];
        if (!fresh) {
            int a, b, c0, c1;
            face_ids(tets[tidx[i] >> 2], (int)(tidx[i] & 3u), a, b, c0);
            face_ids(tets[tidx[i - 1] >> 2], (int)(tidx[i - 1] & 3u), a, b, c1);
            fresh = c0 != c1;
        }
        cnt += fresh ? 1 : 0;
    }
    for (int o = 16; o; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(count, cnt);
}

// counts[0]: orientation failures, counts[1]: in-sphere failures,
// counts[2]: adjacency failures
__global__ void k_chk_geometry(const double4* __restrict__ P, const int* __restrict__ inv,
                               const g4d_tet* __restrict__ tets, int ntet, int n, unsigned long long* counts,
                               unsigned* err) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntet; t += gridDim.x * blockDim.x) {
        const g4d_tet T = tets[t];
        bool ok = true;
        for (int i = 0; i < 4; ++i) ok = ok && T.v[i] >= 0 && T.v[i] < n;
        if (!ok) continue;  // reported by k_chk_edges
        double3 q[5];
        for (int i = 0; i < 4; ++i) q[i] = pt(P, inv, T.v[i]);
        PredSink sink{err, nullptr, nullptr, nullptr};
        if (orient3d(q[0], q[1], q[2], q[3], sink) > 0) atomicAdd(&counts[0], 1ull);
        for (int f = 0; f < 4; ++f) {
            const int o = T.opp[f];
            if (o == -1) continue;
            if (o < 0 || o >= ntet) {
                atomicAdd(&counts[2], 1ull);
                continue;
            }
            // every link must come back; the in-sphere test runs once per
            // pair, from the smaller index
            const g4d_tet U = tets[o];
            int k = -1;
            for (int j = 0; j < 4; ++j)
                if (U.opp[j] == t) k = j;
            if (k < 0 || U.v[k] < 0 || U.v[k] >= n) {
                atomicAdd(&counts[2], 1ull);
                continue;
            }
            if (t > o) continue;
            q[4] = pt(P, inv, U.v[k]);
            if (insphere_sign(q, err) < 0) atomicAdd(&counts[1], 1ull);
        }
    }
}

static int grid_for(size_t work) {
    size_t b = (work + 255) / 256;
    if (b > 148 * 8) b = 148 * 8;
    return (int)(b < 1 ? 1 : b);
}

// Scratch: the edge phase needs 2 x 8 B per edge key (6 per tetrahedron),
// the triangle phase 2 x (4 + 4 + 8) B per triangle key (4 per tetrahedron);
// the phases follow each other and share one area, followed by CUB's
// temporary storage and two n-int arrays.
static size_t cub_bytes(size_t m6, size_t m4) {
    size_t s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, s1, (unsigned long long*)nullptr, (unsigned long long*)nullptr, m6);
    cub::DeviceRadixSort::SortPairs(nullptr, s2, (uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, m4);
    cub::DeviceRadixSort::SortPairs(nullptr, s3, (unsigned long long*)nullptr, (unsigned long long*)nullptr,
                                    (uint32_t*)nullptr, (uint32_t*)nullptr, m4);
    cub::DeviceReduce::Sum(nullptr, s4, (int*)nullptr, (int*)nullptr, 1 << 30);
    size_t b = s1 > s2 ? s1 : s2;
    b = b > s3 ? b : s3;
    return b > s4 ? b : s4;
}

static size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t check_scratch_bytes(int ntet, int n) {
    const size_t m6 = 6 * (size_t)ntet, m4 = 4 * (size_t)ntet;
    const size_t edges = 2 * round256(8 * m6);
    const size_t tris = 4 * round256(4 * m4) + 2 * round256(8 * m4);
    return (edges > tris ? edges : tris) + round256(cub_bytes(m6, m4)) + 2 * round256(sizeof(int) * (size_t)n) + 256;
}

// scratch: check_scratch_bytes(ntet, n) bytes, 256-byte aligned; order:
// Morton position -> input index when the tetrahedra use input indices (else
// null); out[0..5] = V, E, F, orientation, in-sphere and adjacency failures.
cudaError_t run_mesh_check(cudaStream_t st, long long* launches, const double4* P, const int* order,
                           const g4d_tet* tets, int ntet, int n, void* scratch, unsigned long long* out,
                           unsigned* err) {
    const size_t m6 = 6 * (size_t)ntet, m4 = 4 * (size_t)ntet;
    unsigned char* s = static_cast<unsigned char*>(scratch);
    auto take = [&](size_t bytes) {
        unsigned char* p = s;
        s += round256(bytes);
        return p;
    };
    int* inv = reinterpret_cast<int*>(take(sizeof(int) * (size_t)n));
    int* mark = reinterpret_cast<int*>(take(sizeof(int) * (size_t)n));
    const size_t cubb = round256(cub_bytes(m6, m4));
    void* cub_tmp = take(cubb);
    unsigned char* area = s;
    // edge phase
    unsigned long long* e0 = reinterpret_cast<unsigned long long*>(area);
    unsigned long long* e1 = reinterpret_cast<unsigned long long*>(area + round256(8 * m6));
    // triangle phase (same area)
    uint32_t* c0 = reinterpret_cast<uint32_t*>(area);
    uint32_t* c1 = reinterpret_cast<uint32_t*>(area + round256(4 * m4));
    uint32_t* i0 = reinterpret_cast<uint32_t*>(area + 2 * round256(4 * m4));
    uint32_t* i1 = reinterpret_cast<uint32_t*>(area + 3 * round256(4 * m4));
    unsigned long long* ab0 = reinterpret_cast<unsigned long long*>(area + 4 * round256(4 * m4));
    unsigned long long* ab1 = reinterpret_cast<unsigned long long*>(area + 4 * round256(4 * m4) + round256(8 * m4));
    cudaError_t e;
    if ((e = cudaMemsetAsync(out, 0, 6 * sizeof(unsigned long long), st))) return e;
    if ((e = cudaMemsetAsync(mark, 0, sizeof(int) * (size_t)n, st))) return e;
    if (order) {
        k_chk_inverse<<<grid_for(n), 256, 0, st>>>(order, n, inv);
        ++*launches;
    }
    size_t tmp = cubb;
    // vertices and edges
    k_chk_edges<<<grid_for(ntet), 256, 0, st>>>(tets, ntet, n, mark, e0, err);
    ++*launches;
    if ((e = cub::DeviceRadixSort::SortKeys(cub_tmp, tmp, e0, e1, m6, 0, 64, st))) return e;
    ++*launches;
    k_chk_distinct_u64<<<grid_for(m6), 256, 0, st>>>(e1, m6, &out[1]);
    ++*launches;
    tmp = cubb;
    if ((e = cub::DeviceReduce::Sum(cub_tmp, tmp, mark, reinterpret_cast<int*>(e0), n, st))) return e;
    ++*launches;
    if ((e = cudaMemcpyAsync(&out[0], e0, sizeof(int), cudaMemcpyDeviceToDevice, st))) return e;
    // triangles: sorted by c, then stably by (a, b)
    k_chk_tris<<<grid_for(ntet), 256, 0, st>>>(tets, ntet, c0, i0);
    ++*launches;
    tmp = cubb;
    if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, tmp, c0, c1, i0, i1, m4, 0, 32, st))) return e;
    ++*launches;
    k_chk_tri_ab<<<grid_for(m4), 256, 0, st>>>(tets, i1, m4, ab0);
    ++*launches;
    tmp = cubb;
    if ((e = cub::DeviceRadixSort::SortPairs(cub_tmp, tmp, ab0, ab1, i1, i0, m4, 0, 64, st))) return e;
    ++*launches;
    k_chk_distinct_tri<<<grid_for(m4), 256, 0, st>>>(tets, ab1, i0, m4, &out[2]);
    ++*launches;
    // orientation, in-sphere, adjacency
    k_chk_geometry<<<grid_for(ntet), 256, 0, st>>>(P, order ? inv : nullptr, tets, ntet, n, out + 3, err);
    ++*launches;
    return cudaGetLastError();
}

}  // namespace g4d
