// Digital Voronoi diagram without any device allocation.
//
// Some callers cannot allocate GPU memory: code whose device memory belongs to
// a host framework's pool that must not be bypassed, or a time-critical loop
// where cudaMalloc/cudaFree (which can synchronize the whole device) are not
// allowed. For them g4d_voronoi_noalloc computes the same grid as
// g4d_voronoi (scaling, seeding, the three nearest-site passes) on buffers the
// caller owns, and takes its scratch from the fixed array below instead of
// allocating.
//
// The array is a file-scope __device__ object: every GPU that loads this
// library holds it (about 9 MB) until the process exits. Host code sees only a
// stand-in for it, so the device address is looked up with
// cudaGetSymbolAddress, with the device current, and that address is what the
// kernels receive. The address belongs to one CUDA context: the lookup is
// cached per device together with the id of the context it was made in
// (cuCtxGetId), and made again when the current context is another one (after
// cudaDeviceReset, or under a context the caller created with the driver API).
// All calls share the array and it keeps the previous call's contents, so
// calls that overlap on the GPU (different streams, or several host threads)
// race; callers must serialize them.
//
// The first call in each context does the set-up (the address lookup, which
// may also load this library's kernels into that context); make that first
// call outside any stream capture.
#include <cuda.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "g4d_internal.cuh"

namespace g4d {

constexpr int NA_MAX_POINTS = 1 << 18;  // 262,144 points
constexpr int NA_MAX_GRID = 128;        // 128^3 voxels

// scratch layout (byte offsets, each region 256-byte aligned); no Morton
// sort runs here, so the scaling writes only the voxel of each point
constexpr size_t NA_OFF_MINMAX = 0;                                               // 2 x u64
constexpr size_t NA_OFF_ERR = 256;                                                // u32
constexpr size_t NA_OFF_VOX = 512;                                                // u32[NA_MAX_POINTS]
constexpr size_t NA_OFF_GRID = NA_OFF_VOX + 4 * (size_t)NA_MAX_POINTS;            // u32[NA_MAX_GRID^3]
constexpr size_t NA_BYTES = NA_OFF_GRID + 4 * (size_t)NA_MAX_GRID * NA_MAX_GRID * NA_MAX_GRID;

static __device__ __align__(256) unsigned char g_na_scratch[NA_BYTES];

__global__ void k_na_fill(uint32_t* __restrict__ g, size_t count, uint32_t v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        g[i] = v;
}

// every point marks its voxel with the voxel's own packed coordinates
__global__ void k_na_seed(const uint32_t* __restrict__ vox, int n, int G, uint32_t* __restrict__ g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t e = vox[i];
        g[((size_t)vz(e) * G + vy(e)) * G + vx(e)] = e;
    }
}

// z flood from the seeded grid: prev = nearest seed at or below z (written to
// `tmp`), then a downward sweep picks prev or the nearest seed above, ties to
// the lower one (the same rule as k_pba_z).
__global__ void k_na_zflood(int G, uint32_t* __restrict__ g, uint32_t* __restrict__ tmp) {
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 4 + threadIdx.y;
    if (x >= G || y >= G) return;
    const size_t plane = (size_t)G * G;
    uint32_t* col = g + (size_t)y * G + x;
    uint32_t* pcol = tmp + (size_t)y * G + x;
    int prev = -(1 << 20);
    for (int z = 0; z < G; ++z) {
        if (col[z * plane] != MARKER) prev = z;
        pcol[z * plane] = (uint32_t)(prev + (1 << 20));
    }
    int next = 1 << 20;
    bool any = prev >= 0;
    for (int z = G - 1; z >= 0; --z) {
        const int pz = (int)pcol[z * plane] - (1 << 20);
        int zs;
        if (!any) {
            col[z * plane] = MARKER;
            continue;
        }
        zs = (z - pz <= next - z) ? pz : next;
        if (col[z * plane] != MARKER) next = z;  // seeds at z count as "above" for z-1
        col[z * plane] = enc_vox(x, y, zs);
    }
}

// Address of the scratch array, looked up once per (device, context).
struct NaAddr {
    unsigned long long ctx_id;  // cuCtxGetId of the context the lookup was made in (0: none yet)
    void* addr;
};
static std::mutex g_na_mutex;
static NaAddr g_na_addr[64];

// Id of the calling thread's current context (0 when there is none yet).
// The driver entry points come through the runtime, so the library needs no
// link against libcuda.
static unsigned long long na_current_ctx_id() {
    typedef CUresult (*GetCurrent)(CUcontext*);
    typedef CUresult (*GetId)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
            qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b)
            return 0;
        get_current = reinterpret_cast<GetCurrent>(a);
        get_id = reinterpret_cast<GetId>(b);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch array in the current context, or null.
static void* na_scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_na_mutex);
    NaAddr& e = g_na_addr[dev];
    const unsigned long long id = na_current_ctx_id();
    if (e.addr && id != 0 && e.ctx_id == id) return e.addr;
    void* p = nullptr;
    // makes the device's primary context current when none is yet
    if (cudaGetSymbolAddress(&p, g_na_scratch) != cudaSuccess || !p) {
        (void)cudaGetLastError();
        return nullptr;
    }
    e.addr = p;
    e.ctx_id = na_current_ctx_id();  // 0 (unknown) forces a new lookup next time
    return p;
}

}  // namespace g4d

using namespace g4d;

// Launches: scaling bounds, scaling, fill, seed, z flood, y pass, x pass, all
// on `stream`; returns without synchronizing.
extern "C" g4d_status g4d_voronoi_noalloc(const double* d_xyz, int n, int grid, uint32_t* d_sites, void* stream) {
    if (!d_xyz || !d_sites || n < 1 || grid < 32 || (grid & (grid - 1))) return G4D_ERR_ARG;
    if (n > NA_MAX_POINTS || grid > NA_MAX_GRID) {
        std::fprintf(stderr,
                     "g4d_voronoi_noalloc: n=%d grid=%d is beyond the fixed scratch (at most %d points, grid %d)\n",
                     n, grid, NA_MAX_POINTS, NA_MAX_GRID);
        return G4D_ERR_CAPACITY;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return G4D_ERR_NODEVICE;
    // first call in this context: look up the array's device address
    void* base = na_scratch_address(dev);
    if (!base) return G4D_ERR_CUDA;
    unsigned char* s = static_cast<unsigned char*>(base);
    unsigned long long* mm = reinterpret_cast<unsigned long long*>(s + NA_OFF_MINMAX);
    unsigned* err = reinterpret_cast<unsigned*>(s + NA_OFF_ERR);
    uint32_t* vox = reinterpret_cast<uint32_t*>(s + NA_OFF_VOX);
    uint32_t* tmp = reinterpret_cast<uint32_t*>(s + NA_OFF_GRID);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    long long launches = 0;
    Launch L{st, &launches};
    // the array keeps the previous call's contents: reset what must start fresh
    if (cudaMemsetAsync(mm, 0xff, 8, st) != cudaSuccess || cudaMemsetAsync(mm + 1, 0, 8, st) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(unsigned), st) != cudaSuccess)
        return G4D_ERR_CUDA;
    launch_minmax(L, d_xyz, n, mm);
    launch_scale_morton(L, d_xyz, nullptr, n, grid, mm, nullptr, nullptr, vox, err);
    const size_t G3 = (size_t)grid * grid * grid;
    k_na_fill<<<148 * 4, 256, 0, st>>>(d_sites, G3, MARKER);
    k_na_seed<<<(n + 255) / 256, 256, 0, st>>>(vox, n, grid, d_sites);
    k_na_zflood<<<dim3(grid / 32, grid / 4), dim3(32, 4), 0, st>>>(grid, d_sites, tmp);
    launch_pba_y(L, grid, d_sites, tmp);
    launch_pba_x(L, grid, tmp, d_sites);
    return cudaGetLastError() == cudaSuccess ? G4D_OK : G4D_ERR_CUDA;
}
