// Learned star proposal: a small BF16 MLP on the 5th-generation tensor cores.
//
// Model (9,473 FP32 master parameters, BF16 copies feed the tensor cores):
//   z1 = x W1^T + b1 (16 -> 64), a1 = relu(z1)
//   z2 = a1 W2^T + b2 (64 -> 64), a2 = relu(z2)
//   z3 = a2 W3^T + b3 (64 -> 64), a3 = relu(z3)
//   logit = a3 . w4 + b4
// x holds 6 features of a candidate pair padded with zeros to 16 (one MMA K
// step). Every GEMM is a tcgen05.mma (kind::f16, BF16 operands from shared
// memory, FP32 accumulators in tensor memory, M = 128 rows per tile):
//   forward:  z1, z2, z3                       (N = 64)
//   backward: da2 = dz3 W3, da1 = dz2 W2       (N = 64, transposed weights)
//             [dW3; dW2] = [dz3^T; dz2^T] [a2^T; a1^T]^T   (one M=128, N=128,
//             K=128 GEMM whose two diagonal 64x64 blocks are the gradients)
//             dW1 = [dz1^T; 0] x                (M=128, N=16, K=128)
// The weight-gradient GEMMs accumulate in tensor memory across all tiles a CTA
// processes; each CTA adds its sums to the global gradients once at the end.
// Activations and output gradients are rounded to BF16 where they enter a GEMM
// (the CPU restatement used to check the gradients rounds at the same points).
//
// Shared-memory operands use the canonical K-major layout without swizzle: an
// R x K BF16 matrix is stored as 8x8 core matrices (8 rows of 16 bytes), core
// (r/8, k/8) at byte ((k/8) * (R/8) + r/8) * 128, so the descriptor's stride
// byte offset (between 8-row groups) is 128 and its leading byte offset
// (between the two 8-column halves of one K=16 step) is 16 R.
#include <cuda_bf16.h>

#include <cstdint>

#include "g4d_internal.cuh"

namespace g4d {

constexpr int MLP_K0 = 16, MLP_H = 64;
// parameter vector layout (FP32)
constexpr int P_W1 = 0;                        // [64][16]
constexpr int P_B1 = P_W1 + MLP_H * MLP_K0;    // [64]
constexpr int P_W2 = P_B1 + MLP_H;             // [64][64]
constexpr int P_B2 = P_W2 + MLP_H * MLP_H;     // [64]
constexpr int P_W3 = P_B2 + MLP_H;             // [64][64]
constexpr int P_B3 = P_W3 + MLP_H * MLP_H;     // [64]
constexpr int P_W4 = P_B3 + MLP_H;             // [64]
constexpr int P_B4 = P_W4 + MLP_H;             // [1]
constexpr int MLP_PARAMS = P_B4 + 1;           // 9473
static_assert(MLP_PARAMS == 9473, "parameter layout");

constexpr uint32_t MLP_ERR_TIMEOUT = 0x1000u;  // an mbarrier wait ran out

// ---------------------------------------------------------------------------
// tcgen05 / mbarrier helpers (inline PTX)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R x K BF16 matrix in the K-major layout
__device__ __forceinline__ uint32_t kmaj(int r, int k, int R) {
    return ((uint32_t)((k >> 3) * (R >> 3) + (r >> 3)) << 7) + ((uint32_t)(r & 7) << 4) + ((uint32_t)(k & 7) << 1);
}

// shared-memory matrix descriptor: no swizzle, version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: FP32 accumulate, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// D[128 x N] (+)= A[128 x K] B[N x K]^T, K a multiple of 16; a, b: shared
// addresses of the K-major operands (rows 128 and N)
__device__ __forceinline__ void gemm(uint32_t d_tmem, uint32_t a, uint32_t b, int N, int K, bool accumulate) {
    const uint32_t la = 16u * 128u, lb = 16u * (uint32_t)N;
    const uint32_t id = idesc_bf16(128, N);
    for (int ks = 0; ks < K / 16; ++ks)
        umma(d_tmem, sdesc(a + 2u * la * ks, la, 128u), sdesc(b + 2u * lb * ks, lb, 128u), id,
             (accumulate || ks > 0) ? 1u : 0u);
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// bounded wait for the phase with the given parity; false after `limit` polls
// (the default is about a second)
constexpr int MBAR_LIMIT = 1 << 20;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = MBAR_LIMIT) {
    for (int i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// 16 FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16*>(base + off) = __float2bfloat16_rn(v);
}

// weights as K-major B operands: W [N x K] as stored (rows = outputs), or its
// transpose (rows = inputs) for the backward GEMMs
__device__ void load_weight(unsigned char* dst, const float* W, int N, int K, bool transpose) {
    for (int e = threadIdx.x; e < N * K; e += blockDim.x) {
        const int n = e / K, k = e % K;
        const float v = transpose ? W[k * N + n] : W[n * K + k];
        st_bf16(dst, kmaj(n, k, N), v);
    }
}

// ---------------------------------------------------------------------------
// inference: logits of M candidate rows
// ---------------------------------------------------------------------------

// About 40 KB: layer 2's activations overwrite layer 1's in `a` (the MMA
// that read them has completed), so four CTAs share an SM, each with 128
// tensor-memory columns (z1 and z3 in columns 0..63, z2 in 64..127).
struct InferSmem {
    unsigned char w1[64 * 16 * 2], w2[64 * 64 * 2], w3[64 * 64 * 2];
    unsigned char x[128 * 16 * 2], a[128 * 64 * 2];
    float b[3 * 64 + 64 + 1];
    uint64_t bar;
    uint32_t tmem;
};

// relu(z + bias) of 16 accumulator columns, as BF16 (round to nearest even)
// into columns c .. c + 15 of row t of a K-major A operand: two 16-byte stores
__device__ __forceinline__ void store_act16(unsigned char* dst, int t, int c, const float* z, const float* bias) {
    uint32_t pk[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const __nv_bfloat162 h =
            __floats2bfloat162_rn(fmaxf(z[2 * i] + bias[2 * i], 0.f), fmaxf(z[2 * i + 1] + bias[2 * i + 1], 0.f));
        pk[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    *reinterpret_cast<uint4*>(dst + kmaj(t, c, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(dst + kmaj(t, c + 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
}

// 128 threads; thread t owns row t of every tile (tensor-memory lane t)
__global__ void __launch_bounds__(128, 4) k_mlp_infer(const float* __restrict__ P, const uint16_t* __restrict__ X,
                                                      int M, float* __restrict__ logits, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw_mlp[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw_mlp);
    const int t = threadIdx.x, warp = t >> 5;
    load_weight(S.w1, P + P_W1, 64, 16, false);
    load_weight(S.w2, P + P_W2, 64, 64, false);
    load_weight(S.w3, P + P_W3, 64, 64, false);
    for (int i = t; i < 3 * 64 + 65; i += 128) {
        const int layer = i / 64, j = i % 64;
        S.b[i] = layer == 0 ? P[P_B1 + j] : layer == 1 ? P[P_B2 + j] : layer == 2 ? P[P_B3 + j]
               : (i < 4 * 64 ? P[P_W4 + j] : P[P_B4]);
    }
    if (t == 0) mbar_init(&S.bar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(smem_u32(&S.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tb = S.tmem;
    const uint32_t lane_addr = tb + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0, failed_phase = 0;
    bool ok = true;  // the same in every thread of the block
    const int ntiles = (M + 127) / 128;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int row = tile * 128 + t;
        // x: 16 BF16 features of this row
        const uint4* xs = reinterpret_cast<const uint4*>(X + (size_t)row * MLP_K0);
        uint4 q0 = make_uint4(0, 0, 0, 0), q1 = q0;
        if (row < M) { q0 = xs[0]; q1 = xs[1]; }
        *reinterpret_cast<uint4*>(S.x + kmaj(t, 0, 128)) = q0;
        *reinterpret_cast<uint4*>(S.x + kmaj(t, 8, 128)) = q1;
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
        float z[16];
        for (int layer = 0; layer < 3 && ok; ++layer) {
            const uint32_t col = layer == 1 ? 64u : 0u;
            if (t == 0) {
                const uint32_t a = smem_u32(layer == 0 ? S.x : S.a);
                const uint32_t b = smem_u32(layer == 0 ? S.w1 : (layer == 1 ? S.w2 : S.w3));
                gemm(tb + col, a, b, 64, layer == 0 ? 16 : 64, false);
                umma_commit(&S.bar);
            }
            // a wait that ran out in any thread stops the whole block; the
            // MMAs it waited for are drained before the tensor memory is freed
            ok = __syncthreads_and(mbar_wait(&S.bar, phase));
            if (!ok) {
                failed_phase = phase;
                break;
            }
            phase ^= 1u;
            tc_after_sync();
            float acc = 0.f;
            for (int c = 0; c < 64; c += 16) {
                tmem_ld16(lane_addr + col + c, z);
                if (layer < 2) {
                    store_act16(S.a, t, c, z, S.b + 64 * layer + c);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) acc = fmaf(fmaxf(z[i] + S.b[128 + c + i], 0.f), S.b[192 + c + i], acc);
                }
            }
            if (layer == 2 && row < M) logits[row] = acc + S.b[256];
            fence_async_smem();
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
        }
    }
    if (!ok && t == 0) {
        atomicOr(err, MLP_ERR_TIMEOUT);
        mbar_wait(&S.bar, failed_phase, 4 * MBAR_LIMIT);  // the MMAs still in flight
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tb));
}

// ---------------------------------------------------------------------------
// training: forward, loss, backward; gradients summed into G (FP32)
// ---------------------------------------------------------------------------

struct TrainSmem {
    unsigned char w1[64 * 16 * 2], w2[64 * 64 * 2], w3[64 * 64 * 2];   // B operands, forward
    unsigned char w2t[64 * 64 * 2], w3t[64 * 64 * 2];                   // B operands, backward
    unsigned char x[128 * 16 * 2];      // A: x            [128 x 16]
    unsigned char xt[16 * 128 * 2];     // B: x^T          [16 x 128]
    unsigned char a1[128 * 64 * 2];     // A: a1           [128 x 64]
    unsigned char a2[128 * 64 * 2];     // A: a2
    unsigned char dz3[128 * 64 * 2];    // A: dz3
    unsigned char dz2[128 * 64 * 2];    // A: dz2
    unsigned char bcat[128 * 128 * 2];  // B: [a2^T; a1^T] [128 x 128]
    unsigned char acat[128 * 128 * 2];  // A: [dz3^T; dz2^T] [128 x 128]
    unsigned char adw1[128 * 128 * 2];  // A: [dz1^T; 0]   [128 x 128]
    float b[3 * 64 + 64 + 1];
    float gb[3 * 64 + 64 + 1];          // bias, w4, b4 gradient sums of this CTA
    float loss;
    uint64_t bar;
    uint32_t tmem;
};

// tensor-memory columns
constexpr uint32_t TC_Z1 = 0, TC_Z2 = 64, TC_Z3 = 128, TC_DA2 = 192, TC_DA1 = 256, TC_DW = 320, TC_DW1 = 448;

__device__ __forceinline__ float warp_sum(float v) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// tiles[0..ntiles) (or 0..ntiles-1 when tiles is null) of 128 rows each; rows
// at or beyond M count as padding (no loss, no gradient)
__global__ void __launch_bounds__(128, 1) k_mlp_train(const float* __restrict__ P, const uint16_t* __restrict__ X,
                                                      const float* __restrict__ Y, int M, const int* __restrict__ tiles,
                                                      int ntiles, float inv_batch, float* __restrict__ G,
                                                      float* __restrict__ loss_out, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw_mlp[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw_mlp);
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    load_weight(S.w1, P + P_W1, 64, 16, false);
    load_weight(S.w2, P + P_W2, 64, 64, false);
    load_weight(S.w3, P + P_W3, 64, 64, false);
    load_weight(S.w2t, P + P_W2, 64, 64, true);
    load_weight(S.w3t, P + P_W3, 64, 64, true);
    for (int i = t; i < 3 * 64 + 65; i += 128) {
        const int layer = i / 64, j = i % 64;
        S.b[i] = layer == 0 ? P[P_B1 + j] : layer == 1 ? P[P_B2 + j] : layer == 2 ? P[P_B3 + j]
               : (i < 4 * 64 ? P[P_W4 + j] : P[P_B4]);
        S.gb[i] = 0.f;
    }
    // the lower half of [dz1^T; 0] stays zero
    for (int e = t; e < 64 * 128; e += 128) st_bf16(S.adw1, kmaj(64 + e / 128, e % 128, 128), 0.f);
    if (t == 0) { S.loss = 0.f; mbar_init(&S.bar); }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&S.tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tb = S.tmem;
    const uint32_t lane_addr = tb + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0, failed_phase = 0;
    bool ok = true, any = false;  // ok: the same in every thread of the block
    float lsum = 0.f;
    // wait for the MMAs committed last. A wait that ran out in any thread
    // clears ok in all of them: no further MMA is issued, the rest of the tile
    // runs on stale tensor memory and is discarded, and the MMAs of the failed
    // phase are drained before the tensor memory is freed.
    auto sync_mma = [&]() {
        if (ok) {
            ok = __syncthreads_and(mbar_wait(&S.bar, phase));
            if (!ok) failed_phase = phase;
        }
        phase ^= 1u;
        tc_after_sync();
    };
    auto sync_smem = [&]() {  // operands written by threads -> visible to the MMAs
        fence_async_smem();
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
    };
    for (int it = blockIdx.x; it < ntiles && ok; it += gridDim.x) {
        const int tile = tiles ? tiles[it] : it;
        const int row = tile * 128 + t;
        const bool valid = row < M;
        // x and x^T
        uint4 q0 = make_uint4(0, 0, 0, 0), q1 = q0;
        if (valid) {
            const uint4* xs = reinterpret_cast<const uint4*>(X + (size_t)row * MLP_K0);
            q0 = xs[0];
            q1 = xs[1];
        }
        *reinterpret_cast<uint4*>(S.x + kmaj(t, 0, 128)) = q0;
        *reinterpret_cast<uint4*>(S.x + kmaj(t, 8, 128)) = q1;
        {
            const uint16_t* h0 = reinterpret_cast<const uint16_t*>(&q0);
            const uint16_t* h1 = reinterpret_cast<const uint16_t*>(&q1);
            for (int f = 0; f < 8; ++f) {
                *reinterpret_cast<uint16_t*>(S.xt + kmaj(f, t, 16)) = h0[f];
                *reinterpret_cast<uint16_t*>(S.xt + kmaj(8 + f, t, 16)) = h1[f];
            }
        }
        sync_smem();
        // forward, layers 1 and 2: a = relu(z + b) into the A operand and [a2^T; a1^T]
        uint32_t mask[3][2] = {{0, 0}, {0, 0}, {0, 0}};
        float z[16];
        for (int layer = 0; layer < 2; ++layer) {
            if (t == 0 && ok) {
                gemm(tb + (layer == 0 ? TC_Z1 : TC_Z2), smem_u32(layer == 0 ? S.x : S.a1),
                     smem_u32(layer == 0 ? S.w1 : S.w2), 64, layer == 0 ? 16 : 64, false);
                umma_commit(&S.bar);
            }
            sync_mma();
            unsigned char* aop = layer == 0 ? S.a1 : S.a2;
            const int brow = layer == 0 ? 64 : 0;  // a1^T in rows 64..127, a2^T in rows 0..63
            for (int c = 0; c < 64; c += 16) {
                tmem_ld16(lane_addr + (layer == 0 ? TC_Z1 : TC_Z2) + c, z);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float zz = z[i] + S.b[64 * layer + c + i];
                    const float a = fmaxf(zz, 0.f);
                    if (zz > 0.f) mask[layer][(c + i) >> 5] |= 1u << ((c + i) & 31);
                    st_bf16(aop, kmaj(t, c + i, 128), a);
                    st_bf16(S.bcat, kmaj(brow + c + i, t, 128), a);
                }
            }
            sync_smem();
        }
        // layer 3, the logit, the loss and dz3
        if (t == 0 && ok) {
            gemm(tb + TC_Z3, smem_u32(S.a2), smem_u32(S.w3), 64, 64, false);
            umma_commit(&S.bar);
        }
        sync_mma();
        float a3[64];
        float logit = S.b[256];
        for (int c = 0; c < 64; c += 16) {
            tmem_ld16(lane_addr + TC_Z3 + c, z);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float zz = z[i] + S.b[128 + c + i];
                a3[c + i] = fmaxf(zz, 0.f);
                if (zz > 0.f) mask[2][(c + i) >> 5] |= 1u << ((c + i) & 31);
                logit = fmaf(a3[c + i], S.b[192 + c + i], logit);
            }
        }
        float dl = 0.f;
        if (valid) {
            const float y = Y[row];
            // binary cross-entropy with logits: max(l,0) - l y + log(1 + exp(-|l|))
            lsum += fmaxf(logit, 0.f) - logit * y + log1pf(__expf(-fabsf(logit)));
            dl = (1.f / (1.f + __expf(-logit)) - y) * inv_batch;
        }
        // w4, b4, b3 gradients (sums over the tile's rows) and dz3
        {
            const float s4 = warp_sum(dl);
            if (lane == 0) atomicAdd(&S.gb[256], s4);
        }
        for (int j = 0; j < 64; ++j) {
            const float gw = warp_sum(dl * a3[j]);
            const float dz = ((mask[2][j >> 5] >> (j & 31)) & 1u) ? dl * S.b[192 + j] : 0.f;
            const float gbj = warp_sum(dz);
            if (lane == 0) { atomicAdd(&S.gb[192 + j], gw); atomicAdd(&S.gb[128 + j], gbj); }
            st_bf16(S.dz3, kmaj(t, j, 128), dz);
            st_bf16(S.acat, kmaj(j, t, 128), dz);
        }
        sync_smem();
        // da2 = dz3 W3 -> dz2
        if (t == 0 && ok) {
            gemm(tb + TC_DA2, smem_u32(S.dz3), smem_u32(S.w3t), 64, 64, false);
            umma_commit(&S.bar);
        }
        sync_mma();
        for (int c = 0; c < 64; c += 16) {
            tmem_ld16(lane_addr + TC_DA2 + c, z);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int j = c + i;
                const float dz = ((mask[1][j >> 5] >> (j & 31)) & 1u) ? z[i] : 0.f;
                st_bf16(S.dz2, kmaj(t, j, 128), dz);
                st_bf16(S.acat, kmaj(64 + j, t, 128), dz);
                z[i] = dz;
            }
            for (int i = 0; i < 16; ++i) {
                const float g = warp_sum(z[i]);
                if (lane == 0) atomicAdd(&S.gb[64 + c + i], g);
            }
        }
        sync_smem();
        // da1 = dz2 W2, and [dW3; dW2] += [dz3^T; dz2^T] [a2^T; a1^T]^T
        if (t == 0 && ok) {
            gemm(tb + TC_DA1, smem_u32(S.dz2), smem_u32(S.w2t), 64, 64, false);
            gemm(tb + TC_DW, smem_u32(S.acat), smem_u32(S.bcat), 128, 128, any);
            umma_commit(&S.bar);
        }
        sync_mma();
        for (int c = 0; c < 64; c += 16) {
            tmem_ld16(lane_addr + TC_DA1 + c, z);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int j = c + i;
                const float dz = ((mask[0][j >> 5] >> (j & 31)) & 1u) ? z[i] : 0.f;
                st_bf16(S.adw1, kmaj(j, t, 128), dz);
                z[i] = dz;
            }
            for (int i = 0; i < 16; ++i) {
                const float g = warp_sum(z[i]);
                if (lane == 0) atomicAdd(&S.gb[c + i], g);
            }
        }
        sync_smem();
        // dW1 += [dz1^T; 0] x
        if (t == 0 && ok) {
            gemm(tb + TC_DW1, smem_u32(S.adw1), smem_u32(S.xt), 16, 128, any);
            umma_commit(&S.bar);
        }
        sync_mma();  // the next tile overwrites the operands
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
        any = true;
    }
    // this CTA's sums into the global gradients
    if (ok && any) {
        float v[16];
        // rows 0..63 (warps 0, 1): dW3 = columns 0..63; rows 64..127 (warps 2, 3): dW2 = columns 64..127
        const int j = t & 63;
        const int base = t < 64 ? P_W3 : P_W2;
        const uint32_t col0 = TC_DW + (t < 64 ? 0u : 64u);
        for (int c = 0; c < 64; c += 16) {
            tmem_ld16(lane_addr + col0 + c, v);
            for (int i = 0; i < 16; ++i) atomicAdd(&G[base + j * 64 + c + i], v[i]);
        }
        tmem_ld16(lane_addr + TC_DW1, v);
        if (t < 64)
            for (int i = 0; i < 16; ++i) atomicAdd(&G[P_W1 + j * 16 + i], v[i]);
    }
    const float ls = warp_sum(lsum);
    if (lane == 0) atomicAdd(&S.loss, ls);
    __syncthreads();
    if (ok && any) {
        for (int i = t; i < 3 * 64 + 65; i += 128) {
            const int layer = i / 64, j = i % 64;
            const int dst = layer == 0 ? P_B1 + j : layer == 1 ? P_B2 + j : layer == 2 ? P_B3 + j
                          : (i < 4 * 64 ? P_W4 + j : P_B4);
            atomicAdd(&G[dst], S.gb[i]);
        }
        if (t == 0) atomicAdd(loss_out, S.loss);
    }
    if (!ok && t == 0) {
        atomicOr(err, MLP_ERR_TIMEOUT);
        mbar_wait(&S.bar, failed_phase, 4 * MBAR_LIMIT);  // the MMAs still in flight
    }
    tc_before_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tb));
}

// The waits above end after a bounded number of polls. This kernel runs the
// same set-up (tensor memory, an mbarrier) and then waits on a phase that
// nothing completes, with `limit` polls: the wait runs out, the kernel records
// MLP_ERR_TIMEOUT, frees its tensor memory and returns, and the context stays
// usable. Tests use it to exercise the timeout path without a fault.
__global__ void __launch_bounds__(128) k_mlp_wait_probe(int limit, unsigned* err) {
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem;
    const int t = threadIdx.x, warp = t >> 5;
    if (t == 0) mbar_init(&bar);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;" ::"r"(smem_u32(&tmem)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tb = tmem;
    const bool ok = __syncthreads_and(mbar_wait(&bar, 0, limit));  // no arrival is ever made
    if (!ok && t == 0) atomicOr(err, MLP_ERR_TIMEOUT);             // nothing in flight to drain
    tc_before_sync();
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;" ::"r"(tb));
}

// Adam step on the FP32 master parameters
__global__ void k_adam(float* __restrict__ P, float* __restrict__ G, float* __restrict__ m1, float* __restrict__ m2,
                       int n, float lr, float beta1, float beta2, float c1, float c2, float eps) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float g = G[i];
        const float a = beta1 * m1[i] + (1.f - beta1) * g;
        const float b = beta2 * m2[i] + (1.f - beta2) * g * g;
        m1[i] = a;
        m2[i] = b;
        P[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
        G[i] = 0.f;
    }
}

// ---------------------------------------------------------------------------

size_t mlp_infer_smem() { return sizeof(InferSmem) + 1024; }
size_t mlp_train_smem() { return sizeof(TrainSmem) + 1024; }

void launch_mlp_infer(const Launch& L, const float* P, const uint16_t* X, int M, float* logits, unsigned* err) {
    const int ntiles = (M + 127) / 128;
    const size_t sm = sizeof(InferSmem);
    cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    // four CTAs per SM: 128 tensor-memory columns and about 40 KB of shared memory each
    int blocks = ntiles < 4 * 148 ? ntiles : 4 * 148;
    k_mlp_infer<<<blocks < 1 ? 1 : blocks, 128, sm, L.stream>>>(P, X, M, logits, err);
    ++*L.launches;
}

void launch_mlp_train(const Launch& L, const float* P, const uint16_t* X, const float* Y, int M, const int* tiles,
                      int ntiles, float inv_batch, float* G, float* loss, unsigned* err) {
    const size_t sm = sizeof(TrainSmem);
    cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    // one CTA per SM: 512 tensor-memory columns
    int blocks = ntiles < 148 ? ntiles : 148;
    k_mlp_train<<<blocks < 1 ? 1 : blocks, 128, sm, L.stream>>>(P, X, Y, M, tiles, ntiles, inv_batch, G, loss, err);
    ++*L.launches;
}

void launch_mlp_wait_probe(const Launch& L, int limit, unsigned* err) {
    k_mlp_wait_probe<<<1, 128, 0, L.stream>>>(limit, err);
    ++*L.launches;
}

void launch_adam(const Launch& L, float* P, float* G, float* m1, float* m2, int step, float lr) {
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f, c2 = 1.f;
    for (int i = 0; i < step; ++i) { c1 *= b1; c2 *= b2; }
    k_adam<<<(MLP_PARAMS + 255) / 256, 256, 0, L.stream>>>(P, G, m1, m2, MLP_PARAMS, lr, b1, b2, 1.f - c1, 1.f - c2,
                                                            1e-8f);
    ++*L.launches;
}

}  // namespace g4d
