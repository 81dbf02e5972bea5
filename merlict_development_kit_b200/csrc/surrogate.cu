// surrogate.cu -- kernels of the learned surrogate (merlict_b200_surrogate.h).
//
// The hidden and output layers are BF16 GEMMs on the fifth-generation tensor
// cores: C = A B^T with A (M x K) and B (N x K) both K-major in "tile
// images" (every 128-row x 64-column tile one contiguous, 128-byte-swizzled
// block), so that one bulk copy (cp.async.bulk, the TMA engine) moves a tile
// from global into shared memory with no tensor map.  Per CTA: one M = 128
// row tile times one N tile, FP32 accumulators in tensor memory; warp 0
// issues the bulk copies into a 4-stage ring, one thread of warp 1 issues
// tcgen05.mma (K = 16 per instruction) and commits each stage back to the
// producer, warps 2..5 run the epilogue (tcgen05.ld, bias, SiLU or its
// derivative, BF16 tile images of the result and of its transpose for the
// next GEMM).  Every wait is bounded: on a timeout the kernel records an
// error (mlgpu_sg_sync_errors), skips the rest of its work, frees its tensor
// memory and returns.
//
// Layer 0 (5 inputs), the loss, the optimiser, weight packing and the
// sampling of the mixture run on the CUDA cores in FP32.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "merlict_b200_philox.h"
#include "merlict_b200_surrogate.h"
#include "mlgpu_internal.h"
#include "paired_f32.cuh"

namespace mlgpu {
namespace sg {
namespace {

constexpr int kH = MLGPU_SG_HIDDEN;          // 256
constexpr int kOut = MLGPU_SG_OUTPUTS;       // 73
constexpr int kOutPad = MLGPU_SG_OUTPUTS_PADDED;   // 80
constexpr int kOutK = 128;                   // the output width as a K dimension (64-multiple)
constexpr int kIn = MLGPU_SG_INPUTS;         // 5
constexpr int kInLd = 8;                     // floats per input row
constexpr int kFreq = MLGPU_SG_OCTAVES;      // octaves of the sin/cos encoding
constexpr int kEnc = MLGPU_SG_ENCODED;       // encoded input width (128)
constexpr int kStages = 4;
constexpr int kThreads = 192;                // warp 0 copies, warp 1 MMA, warps 2..5 epilogue
constexpr int kPersThreads = 320;            // persistent GEMM: warps 2..9 epilogue

// parameter offsets (floats): layer l = W[out][in] then b[out]
constexpr uint64_t kW0 = 0, kB0 = kW0 + (uint64_t)kH*kEnc;
constexpr uint64_t kW1 = kB0 + kH, kB1 = kW1 + (uint64_t)kH*kH;
constexpr uint64_t kW2 = kB1 + kH, kB2 = kW2 + (uint64_t)kH*kH;
constexpr uint64_t kW3 = kB2 + kH, kB3 = kW3 + (uint64_t)kH*kH;
constexpr uint64_t kW4 = kB3 + kH, kB4 = kW4 + (uint64_t)kOut*kH;
constexpr uint64_t kParams = kB4 + kOut;
__host__ __device__ constexpr uint64_t w_off(int l) {
    return l == 0 ? kW0 : l == 1 ? kW1 : l == 2 ? kW2 : l == 3 ? kW3 : kW4;
}
__host__ __device__ constexpr uint64_t b_off(int l) {
    return l == 0 ? kB0 : l == 1 ? kB1 : l == 2 ? kB2 : l == 3 ? kB3 : kB4;
}

// weight images (bytes): layers 1..3 forward (256 x 256) and transposed
// (256 x 256); layer 4 forward (80 x 256) and transposed (256 x 128);
// layer 0 forward (256 x 128)
constexpr uint64_t kImgHH = (uint64_t)kH*kH*2;
constexpr uint64_t kImgW4 = (uint64_t)kOutPad*kH*2;
constexpr uint64_t kImgW4T = (uint64_t)kH*kOutK*2;
constexpr uint64_t kImgW0 = (uint64_t)kH*kEnc*2;
constexpr uint64_t kImgBytes = 6*kImgHH + kImgW4 + kImgW4T + kImgW0;
__host__ __device__ constexpr uint64_t img_w(int l) { return (uint64_t)(l - 1)*2*kImgHH; }        // l = 1..3
__host__ __device__ constexpr uint64_t img_wt(int l) { return (uint64_t)(l - 1)*2*kImgHH + kImgHH; }
constexpr uint64_t kImgW4Off = 6*kImgHH, kImgW4TOff = 6*kImgHH + kImgW4;
constexpr uint64_t kImgW0Off = kImgW4TOff + kImgW4T;

__device__ unsigned int g_error;   // first device error (a timed-out wait)

__host__ __device__ __forceinline__ uint64_t img_off(uint32_t rows, uint32_t r, uint32_t k) {
    return ((uint64_t)(k >> 6)*(rows >> 3) + (r >> 3))*1024u + (r & 7u)*128u +
           ((((k & 63u) >> 3) ^ (r & 7u)) << 4) + ((k & 7u) << 1);
}

// ---- PTX wrappers -----------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.b32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Waits for the phase with `parity` to complete; false after about a second.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > (1ll << 31)) return false;
    return true;
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Shared-memory descriptor of a K-major operand in the 128-byte swizzled
// layout: rows of 128 bytes, 8-row atoms 1024 bytes apart (SBO), leading
// offset unused (1), version 1 (sm_100), layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B,
// both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 :: "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate),
                    "r"(z), "r"(z), "r"(z), "r"(z));
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                   "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                   "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ float ex2_ftz(float a) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}
__device__ __forceinline__ float rcp_ftz(float a) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a));
    return r;
}

constexpr float kLog2e = 1.4426950408889634f;
// SiLU z / (1 + 2^(-z log2 e)) with the hardware's approximate base-2
// exponential and reciprocal (relative error about 2^-22 each; for
// z -> -inf the exponential overflows to inf and the result is -0).
// silu_pair does the same on two values with paired instructions, to the
// same bits.
__device__ __forceinline__ float silu(float z) {
    return __fmul_rn(z, rcp_ftz(__fadd_rn(1.0f, ex2_ftz(__fmul_rn(z, -kLog2e)))));
}
__device__ __forceinline__ uint64_t silu_pair(uint64_t z) {
    float u0, u1, d0, d1;
    f2_split(mul2(z, f2(-kLog2e, -kLog2e)), &u0, &u1);
    f2_split(add2(f2(ex2_ftz(u0), ex2_ftz(u1)), f2(1.0f, 1.0f)), &d0, &d1);
    return mul2(z, f2(rcp_ftz(d0), rcp_ftz(d1)));
}
__device__ __forceinline__ float dsilu(float z) {
    const float s = __fdividef(1.0f, 1.0f + __expf(-z));
    return s*(1.0f + z*(1.0f - s));
}
__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);   // .x = a (low half)
    return *reinterpret_cast<const uint32_t*>(&h);
}
// Stores 8 consecutive k values of row r of an image.
__device__ __forceinline__ void img_store8(uint8_t* img, uint32_t rows, uint32_t r, uint32_t k,
                                           const float* v) {
    uint4 q;
    q.x = pack_bf16x2(v[0], v[1]); q.y = pack_bf16x2(v[2], v[3]);
    q.z = pack_bf16x2(v[4], v[5]); q.w = pack_bf16x2(v[6], v[7]);
    *reinterpret_cast<uint4*>(img + img_off(rows, r, k)) = q;
}
__device__ __forceinline__ void img_store1(uint8_t* img, uint32_t rows, uint32_t r, uint32_t k,
                                           float v) {
    *reinterpret_cast<__nv_bfloat16*>(img + img_off(rows, r, k)) = __float2bfloat16_rn(v);
}

// ---- the GEMM ------------------------------------------------------------------

enum { kEpiF32 = 0, kEpiSilu = 1, kEpiDSilu = 2 };

struct GemmArgs {
    const uint8_t* a; uint32_t a_rows;     // A image (M x K)
    const uint8_t* b; uint32_t b_rows;     // B image (N x K)
    uint32_t k_chunks;                     // 64-wide K chunks per CTA (gridDim.z splits K)
    const float* bias;                     // [bias_n] or null
    uint32_t bias_n;                       // columns that have a bias
    float* out; uint32_t ld; uint64_t split_stride; uint32_t n_store;   // FP32 C
    uint8_t* img; uint32_t img_rows;       // image of the result (rows = M, K = N)
    uint8_t* img_t; uint32_t img_t_rows;   // image of its transpose (rows = N, K = M)
    float* z; uint32_t z_ld;               // pre-activations: written (SiLU) or read (dSiLU)
    float* col_sum;                        // [N] column sums of the result (dSiLU)
};

template <int kN>
__host__ __device__ constexpr uint32_t stage_bytes() { return 128u*128u + (uint32_t)kN*128u; }
template <int kN>
__host__ __device__ constexpr uint32_t gemm_smem_bytes() { return kStages*stage_bytes<kN>() + 1024u + 256u; }
template <int kN>
__host__ __device__ constexpr uint32_t tmem_cols() {
    return kN <= 32 ? 32u : kN <= 64 ? 64u : kN <= 128 ? 128u : 256u;
}

template <int kN, int kEpi>
__global__ void __launch_bounds__(kThreads, 1)
umma_gemm_kernel(const GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~(uintptr_t)1023);
    constexpr uint32_t kBytesA = 128u*128u, kBytesB = (uint32_t)kN*128u;
    constexpr uint32_t kStage = kBytesA + kBytesB;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages*kStage);
    uint64_t* empty = full + kStages;
    uint64_t* done = empty + kStages;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
    __shared__ int s_failed;
    __shared__ uint32_t s_issued, s_consumed;   // K chunks copied in / taken by the MMAs
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t m0 = blockIdx.x*128u, n0 = blockIdx.y*(uint32_t)kN;
    const uint32_t kc0 = blockIdx.z*g.k_chunks;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(done, 1);
        s_failed = 0;
        s_issued = 0;
        s_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(tmem_cols<kN>()));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            for (uint32_t kc = 0; kc < g.k_chunks; kc++) {
                const uint32_t s = kc % kStages;
                if (kc >= (uint32_t)kStages && !mbar_wait(&empty[s], ((kc/kStages) - 1) & 1)) {
                    s_failed = 1;
                    break;
                }
                uint8_t* dst = smem + s*kStage;
                const uint64_t kk = kc0 + kc;
                mbar_expect_tx(&full[s], kStage);
                bulk_g2s(dst, g.a + (kk*(g.a_rows >> 3) + (m0 >> 3))*1024u, kBytesA, &full[s]);
                bulk_g2s(dst + kBytesA, g.b + (kk*(g.b_rows >> 3) + (n0 >> 3))*1024u, kBytesB,
                         &full[s]);
                s_issued = kc + 1;
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, kN);
            uint32_t issued = 0;
            for (uint32_t kc = 0; kc < g.k_chunks; kc++) {
                const uint32_t s = kc % kStages;
                if (!mbar_wait(&full[s], (kc/kStages) & 1)) { s_failed = 1; break; }
                s_consumed = kc + 1;
                tc_fence_after();
                const uint32_t a_addr = smem_u32(smem + s*kStage);
                const uint32_t b_addr = a_addr + kBytesA;
#pragma unroll
                for (uint32_t ks = 0; ks < 4; ks++)
                    umma_bf16(tmem, sw128_desc(a_addr + ks*32u), sw128_desc(b_addr + ks*32u), idesc,
                              (kc | ks) != 0u ? 1u : 0u);
                umma_commit(&empty[s]);
                issued++;
            }
            // arrives when every MMA issued above has completed
            umma_commit(done);
            (void)issued;
        }
    } else {
        // epilogue: warp w reads tensor-memory lanes 32 (w % 4) .. + 31
        const bool ok = __all_sync(0xffffffffu, mbar_wait(done, 0));   // warp-uniform
        tc_fence_after();
        if (!ok) s_failed = 1;
        const uint32_t q = (uint32_t)warp & 3u;
        const uint32_t row = m0 + q*32u + (uint32_t)lane;
        const uint32_t taddr = tmem + ((q*32u) << 16);
        for (uint32_t c0 = 0; ok && c0 < (uint32_t)kN; c0 += 32) {
            float v[32];
            tmem_ld32(taddr + c0, v);
            const uint32_t nb = n0 + c0;
            if (kEpi == kEpiF32) {
                if (g.bias) {
#pragma unroll
                    for (int j = 0; j < 32; j++) v[j] += (nb + j < g.bias_n) ? __ldg(g.bias + nb + j) : 0.0f;
                }
                float* o = g.out + (uint64_t)blockIdx.z*g.split_stride + (uint64_t)row*g.ld + nb;
                if (nb + 32 <= g.n_store && (g.ld & 3u) == 0) {
#pragma unroll
                    for (int j = 0; j < 32; j += 4)
                        *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                } else {
                    for (int j = 0; j < 32; j++) if (nb + j < g.n_store) o[j] = v[j];
                }
            } else if (kEpi == kEpiSilu) {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const float zz = v[j] + __ldg(g.bias + nb + j);
                    if (g.z) g.z[(uint64_t)row*g.z_ld + nb + j] = zz;
                    v[j] = silu(zz);
                }
#pragma unroll
                for (int j = 0; j < 32; j += 8) img_store8(g.img, g.img_rows, row, nb + j, v + j);
                if (g.img_t) {
#pragma unroll
                    for (int j = 0; j < 32; j++) img_store1(g.img_t, g.img_t_rows, nb + j, row, v[j]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32; j++)
                    v[j] *= dsilu(g.z[(uint64_t)row*g.z_ld + nb + j]);
                if (g.img) {
#pragma unroll
                    for (int j = 0; j < 32; j += 8) img_store8(g.img, g.img_rows, row, nb + j, v + j);
                }
                if (g.img_t) {
#pragma unroll
                    for (int j = 0; j < 32; j++) img_store1(g.img_t, g.img_t_rows, nb + j, row, v[j]);
                }
                if (g.out) {
                    float* o = g.out + (uint64_t)row*g.ld + nb;
#pragma unroll
                    for (int j = 0; j < 32; j += 4)
                        *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
                }
                if (g.col_sum) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        float t = v[j];
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                        if (lane == 0) atomicAdd(g.col_sum + nb + j, t);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && s_failed) {
        atomicCAS(&g_error, 0u, (unsigned)MLGPU_ERR_RUNTIME);
        // A CTA must not exit, nor free its tensor memory, with its own bulk
        // copies or MMAs still in flight: wait (again bounded) for the
        // copies no MMA consumed and for the MMAs' final commit.
        for (uint32_t kc = s_consumed; kc < s_issued; kc++)
            mbar_wait(&full[kc % kStages], (kc/kStages) & 1);
        mbar_wait(done, 0);
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(tmem_cols<kN>()));
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

// The epilogue of one 32-column slice of row `row` (shared by both GEMMs).
template <int kEpi>
__device__ __forceinline__ void epilogue32(const GemmArgs& g, uint32_t row, uint32_t nb,
                                           uint32_t split, float* v, int lane) {
    if (kEpi == kEpiF32) {
        if (g.bias) {
#pragma unroll
            for (int j = 0; j < 32; j++) v[j] += (nb + j < g.bias_n) ? __ldg(g.bias + nb + j) : 0.0f;
        }
        float* o = g.out + (uint64_t)split*g.split_stride + (uint64_t)row*g.ld + nb;
        if (nb + 32 <= g.n_store && (g.ld & 3u) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        } else {
            for (int j = 0; j < 32; j++) if (nb + j < g.n_store) o[j] = v[j];
        }
    } else if (kEpi == kEpiSilu) {
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const float zz = v[j] + __ldg(g.bias + nb + j);
            if (g.z) g.z[(uint64_t)row*g.z_ld + nb + j] = zz;
            v[j] = silu(zz);
        }
#pragma unroll
        for (int j = 0; j < 32; j += 8) img_store8(g.img, g.img_rows, row, nb + j, v + j);
        if (g.img_t) {
#pragma unroll
            for (int j = 0; j < 32; j++) img_store1(g.img_t, g.img_t_rows, nb + j, row, v[j]);
        }
    } else {
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] *= dsilu(g.z[(uint64_t)row*g.z_ld + nb + j]);
        if (g.img) {
#pragma unroll
            for (int j = 0; j < 32; j += 8) img_store8(g.img, g.img_rows, row, nb + j, v + j);
        }
        if (g.img_t) {
#pragma unroll
            for (int j = 0; j < 32; j++) img_store1(g.img_t, g.img_t_rows, nb + j, row, v[j]);
        }
        if (g.out) {
            float* o = g.out + (uint64_t)row*g.ld + nb;
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(o + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
        if (g.col_sum) {
#pragma unroll
            for (int j = 0; j < 32; j++) {
                float t = v[j];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (lane == 0) atomicAdd(g.col_sum + nb + j, t);
            }
        }
    }
}

// ---- the persistent, weight-resident GEMM ------------------------------------------
//
// For the layers whose B is a weight matrix (N x K, K = 64 kKChunks): each
// CTA loads B into shared memory once and then streams 128-row tiles of A
// (tile = blockIdx.x, + gridDim.x, ...) through a 4-chunk ring.  Two
// accumulators in tensor memory let the epilogue of one tile overlap the
// MMAs of the next: the MMA thread commits a tile to acc_full[t & 1], the
// eight epilogue warps drain it (two per tensor-memory lane quarter, each
// taking every other 32-column slice) and arrive on acc_empty[t & 1].

constexpr int kARing = 4;

template <int kN, int kKChunks>
__host__ __device__ constexpr uint32_t pers_smem_bytes() {
    return (uint32_t)kKChunks*(uint32_t)kN*128u + kARing*16384u + 1024u + 256u;
}

template <int kN, int kKChunks, int kEpi>
__global__ void __launch_bounds__(kPersThreads, 1)
umma_persistent_kernel(const GemmArgs g, uint32_t num_tiles) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~(uintptr_t)1023);
    constexpr uint32_t kBChunk = (uint32_t)kN*128u;
    constexpr uint32_t kBBytes = (uint32_t)kKChunks*kBChunk;
    constexpr uint32_t kCols = tmem_cols<kN>();
    uint8_t* sB = smem;
    uint8_t* sA = smem + kBBytes;                  // kARing chunks of 16 KB
    uint64_t* b_full = reinterpret_cast<uint64_t*>(sA + kARing*16384u);
    uint64_t* a_full = b_full + 1;
    uint64_t* a_empty = a_full + kARing;
    uint64_t* acc_full = a_empty + kARing;
    uint64_t* acc_empty = acc_full + 2;
    uint64_t* drained = acc_empty + 2;             // the MMA thread's last commit
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    __shared__ int s_failed;
    __shared__ uint32_t s_issued, s_consumed;   // A chunks copied in / taken by the MMAs
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        mbar_init(b_full, 1);
        for (int s = 0; s < kARing; s++) { mbar_init(&a_full[s], 1); mbar_init(&a_empty[s], 1); }
        for (int s = 0; s < 2; s++) { mbar_init(&acc_full[s], 1); mbar_init(&acc_empty[s], 8); }
        mbar_init(drained, 1);
        s_failed = 0;
        s_issued = 0;
        s_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(2u*kCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            mbar_expect_tx(b_full, kBBytes);
            for (uint32_t kc = 0; kc < (uint32_t)kKChunks; kc++)
                bulk_g2s(sB + kc*kBChunk, g.b + (uint64_t)kc*(g.b_rows >> 3)*1024u, kBChunk, b_full);
            uint32_t it = 0;
            bool ok = true;
            for (uint32_t tile = blockIdx.x; ok && tile < num_tiles; tile += gridDim.x) {
                for (uint32_t kc = 0; kc < (uint32_t)kKChunks; kc++, it++) {
                    const uint32_t s = it % kARing;
                    if (it >= (uint32_t)kARing && !mbar_wait(&a_empty[s], ((it/kARing) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&a_full[s], 16384u);
                    bulk_g2s(sA + s*16384u,
                             g.a + ((uint64_t)kc*(g.a_rows >> 3) + (uint64_t)tile*16u)*1024u,
                             16384u, &a_full[s]);
                    s_issued = it + 1;
                }
            }
            if (!ok) s_failed = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_bf16(128, kN);
            bool ok = mbar_wait(b_full, 0);
            uint32_t it = 0, t = 0;
            for (uint32_t tile = blockIdx.x; ok && tile < num_tiles; tile += gridDim.x, t++) {
                const uint32_t acc = t & 1u;
                if (t >= 2 && !mbar_wait(&acc_empty[acc], ((t >> 1) - 1) & 1)) { ok = false; break; }
                tc_fence_after();
                const uint32_t d = tmem + acc*kCols;
                for (uint32_t kc = 0; kc < (uint32_t)kKChunks; kc++, it++) {
                    const uint32_t s = it % kARing;
                    if (!mbar_wait(&a_full[s], (it/kARing) & 1)) { ok = false; break; }
                    s_consumed = it + 1;
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(sA + s*16384u);
                    const uint32_t b_addr = smem_u32(sB + kc*kBChunk);
#pragma unroll
                    for (uint32_t ks = 0; ks < 4; ks++)
                        umma_bf16(d, sw128_desc(a_addr + ks*32u), sw128_desc(b_addr + ks*32u), idesc,
                                  (kc | ks) != 0u ? 1u : 0u);
                    umma_commit(&a_empty[s]);
                }
                if (!ok) break;
                umma_commit(&acc_full[acc]);
            }
            if (!ok) s_failed = 1;
            // arrives when every MMA issued above has completed
            umma_commit(drained);
        }
    } else {
        // warp w reads tensor-memory lanes 32 (w % 4) .. + 31; warps 2..5
        // take the even 32-column slices, warps 6..9 the odd ones
        const uint32_t q = (uint32_t)warp & 3u;
        const uint32_t half = (uint32_t)(warp - 2) >> 2;
        uint32_t t = 0;
        for (uint32_t tile = blockIdx.x; tile < num_tiles; tile += gridDim.x, t++) {
            const uint32_t acc = t & 1u;
            const bool ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[acc], (t >> 1) & 1));
            tc_fence_after();
            if (!ok) { s_failed = 1; break; }
            const uint32_t row = tile*128u + q*32u + (uint32_t)lane;
            const uint32_t taddr = tmem + acc*kCols + ((q*32u) << 16);
            for (uint32_t c0 = half*32u; c0 < (uint32_t)kN; c0 += 64) {
                float v[32];
                tmem_ld32(taddr + c0, v);
                epilogue32<kEpi>(g, row, c0, 0, v, lane);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[acc]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && s_failed) {
        atomicCAS(&g_error, 0u, (unsigned)MLGPU_ERR_RUNTIME);
        // no exit, and no freeing of tensor memory, with this CTA's bulk
        // copies or MMAs in flight: wait (again bounded) for the weight
        // copies, the A chunks no MMA consumed and the MMAs' final commit
        mbar_wait(b_full, 0);
        for (uint32_t it = s_consumed; it < s_issued; it++)
            mbar_wait(&a_full[it % kARing], (it/kARing) & 1);
        mbar_wait(drained, 0);
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(2u*kCols));
    }
}

int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

// C = A W^T with W (N x 64 kKChunks) resident: m rows (a multiple of 128).
template <int kN, int kKChunks, int kEpi>
cudaError_t launch_persistent(const GemmArgs& g, uint32_t m, cudaStream_t s) {
    constexpr uint32_t smem = pers_smem_bytes<kN, kKChunks>();
    static bool attr = false;
    if (!attr) {
        const cudaError_t e = cudaFuncSetAttribute(umma_persistent_kernel<kN, kKChunks, kEpi>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const uint32_t tiles = m/128u;
    const uint32_t per_sm = smem <= 110u*1024u ? 2u : 1u;
    const uint32_t grid = tiles < per_sm*(uint32_t)sm_count() ? tiles : per_sm*(uint32_t)sm_count();
    umma_persistent_kernel<kN, kKChunks, kEpi><<<grid, kPersThreads, smem, s>>>(g, tiles);
    return cudaGetLastError();
}

template <int kN, int kEpi>
cudaError_t launch_gemm(const GemmArgs& g, uint32_t m, uint32_t n, uint32_t splits, cudaStream_t s) {
    constexpr uint32_t smem = gemm_smem_bytes<kN>();
    static bool attr = false;
    if (!attr) {
        const cudaError_t e = cudaFuncSetAttribute(umma_gemm_kernel<kN, kEpi>,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const dim3 grid(m/128u, n/(uint32_t)kN, splits);
    umma_gemm_kernel<kN, kEpi><<<grid, kThreads, smem, s>>>(g);
    return cudaGetLastError();
}

// ---- CUDA-core kernels -------------------------------------------------------------

// Tile images of the tensor-core layers' weights from the FP32 masters.
__global__ void pack_weights_kernel(const float* __restrict__ p, uint8_t* __restrict__ img) {
    // work items: 8-element chunks of the 8 images
    const uint32_t per_hh = kH*kH/8;                 // chunks of a 256 x 256 image
    const uint32_t per_w4 = kOutPad*kH/8, per_w4t = kH*kOutK/8, per_w0 = kH*kEnc/8;
    const uint32_t total = 6*per_hh + per_w4 + per_w4t + per_w0;
    for (uint32_t t = blockIdx.x*blockDim.x + threadIdx.x; t < total; t += gridDim.x*blockDim.x) {
        float v[8];
        uint8_t* dst;
        uint32_t rows, r, k;
        if (t < 6*per_hh) {
            const int l = 1 + (int)(t/(2*per_hh));
            const bool tr = ((t/per_hh) & 1u) != 0;
            const uint32_t c = t % per_hh;
            r = c/(kH/8); k = (c % (kH/8))*8;
            rows = kH;
            dst = img + (tr ? img_wt(l) : img_w(l));
            const float* W = p + w_off(l);
            for (int j = 0; j < 8; j++) v[j] = tr ? W[(uint64_t)(k + j)*kH + r] : W[(uint64_t)r*kH + k + j];
        } else if (t < 6*per_hh + per_w4) {
            const uint32_t c = t - 6*per_hh;
            r = c/(kH/8); k = (c % (kH/8))*8;
            rows = kOutPad;
            dst = img + kImgW4Off;
            const float* W = p + kW4;
            for (int j = 0; j < 8; j++) v[j] = r < (uint32_t)kOut ? W[(uint64_t)r*kH + k + j] : 0.0f;
        } else if (t < 6*per_hh + per_w4 + per_w4t) {
            const uint32_t c = t - 6*per_hh - per_w4;
            r = c/(kOutK/8); k = (c % (kOutK/8))*8;
            rows = kH;
            dst = img + kImgW4TOff;
            const float* W = p + kW4;
            for (int j = 0; j < 8; j++) v[j] = (k + j) < (uint32_t)kOut ? W[(uint64_t)(k + j)*kH + r] : 0.0f;
        } else {
            const uint32_t c = t - 6*per_hh - per_w4 - per_w4t;
            r = c/(kEnc/8); k = (c % (kEnc/8))*8;
            rows = kH;
            dst = img + kImgW0Off;
            const float* W = p + kW0;
            for (int j = 0; j < 8; j++) v[j] = W[(uint64_t)r*kEnc + k + j];
        }
        img_store8(dst, rows, r, k, v);
    }
}

// The fixed encoding of the 5 normalised inputs into kEnc features: the
// inputs themselves, then sin(pi 2^l x_j) and cos(pi 2^l x_j) for j = 0..4
// and l = 0..kFreq-1 (feature 5 + 2 (kFreq j + l) + c), then zeros.  The
// argument 2^l x_j (a product by a power of two) is exact in FP32 and
// sincospif reduces it exactly.
__device__ __forceinline__ float encoded(const float* xi, int f) {
    if (f < kIn) return xi[f];
    const int g = f - kIn;
    if (g >= 2*kFreq*kIn) return 0.0f;
    const int j = g/(2*kFreq), l = (g % (2*kFreq)) >> 1;
    float sn, cs;
    sincospif(__fmul_rn(xi[j], (float)(1 << l)), &sn, &cs);
    return (g & 1) ? cs : sn;
}

// One thread per (row, 8 features): the encoded inputs as a tile image
// (rows = batch, K = kEnc) and, when training, its transpose's image.
__global__ void __launch_bounds__(256)
encode_kernel(const float* __restrict__ x, uint32_t batch, uint8_t* __restrict__ img,
              uint8_t* __restrict__ img_t) {
    const uint64_t t = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x;
    const uint32_t row = (uint32_t)(t/(kEnc/8));
    const int f0 = (int)(t % (kEnc/8))*8;
    if (row >= batch) return;
    float xi[kIn];
#pragma unroll
    for (int j = 0; j < kIn; j++) xi[j] = __ldg(x + (uint64_t)row*kInLd + j);
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = encoded(xi, f0 + k);
    img_store8(img, batch, row, (uint32_t)f0, v);
    if (img_t) {
#pragma unroll
        for (int k = 0; k < 8; k++) img_store1(img_t, kEnc, (uint32_t)(f0 + k), row, v[k]);
    }
}

// ---- the fused inference forward ----------------------------------------------------
//
// All five layers of 128-row tiles in one persistent kernel, the
// activations never leaving the SM.  Each CTA keeps two tiles in flight, in
// slots 0 and 1: a slot holds its tile's activation in shared memory as a
// 128-row image (4 chunks of 64 columns, 16 KB each) and its accumulator in
// tensor memory (256 columns).  The layers' weights stream through a ring
// of 32 KB stages (one 64-wide K chunk of one layer per stage; they stay in
// L2).  The two slots take turns: while the tensor cores run layer l of one
// slot, the epilogue warps drain layer l - 1 of the other into its
// activation image (bias, SiLU, BF16), so the MMAs and the epilogue overlap
// across tiles.  Steps run in the order (pair, layer, slot); the epilogue
// of a step releases the slot's four activation chunks on four barriers
// (after the last of them the accumulator is free as well), and the MMAs of
// the slot's next step wait for all four.  At the last layer the epilogue
// warps first encode the slot's next tile into chunks 0 and 1, then write
// the 80 FP32 outputs, then release chunks 2 and 3.
//
// The arithmetic is that of the layer-by-layer path (same encoding, K
// order, bias addition, SiLU and BF16 rounding), so both give the same bits.
//
// Roles: warp 0 lane 0 copies weight chunks, warp 1 lane 0 issues the MMAs,
// warps 2..17 encode and drain: warp w reads tensor-memory lane quarter
// w % 4 (rows 32 (w % 4) ..) and takes 16 of each 64-column chunk's
// columns (16 ((w - 2) / 4) ..), so that every scheduler has four such
// warps to hide the latency of the epilogue's dependent arithmetic.  Every
// wait is bounded; after a timeout every role leaves its loop, the kernel
// records the error and waits (bounded) for its own copies and MMAs before
// freeing tensor memory.

constexpr int kFusedThreads = 576;
constexpr int kEpiWarps = 16;
constexpr int kWRing = 3;                       // weight stages
constexpr uint32_t kWStage = 32768u;            // 256 rows x 64 K x 2 bytes
constexpr uint32_t kActChunk = 16384u;          // 128 rows x 64 K x 2 bytes
constexpr uint32_t kSlotBytes = 4u*kActChunk;   // one tile's activation image
constexpr uint32_t kFusedBarOff = 2u*kSlotBytes + kWRing*kWStage;

__host__ __device__ constexpr uint32_t fused_smem_bytes() {
    return kFusedBarOff + 24u*8u + 1024u;
}

// K chunk kc of layer l's weight image: its offset in the images and its
// bytes (layer 0: 256 x 128, 2 chunks; 1..3: 256 x 256; 4: 80 x 256).
__device__ __forceinline__ void weight_chunk(uint32_t l, uint32_t kc, uint64_t* off,
                                             uint32_t* bytes) {
    if (l == 0) {
        *off = kImgW0Off + (uint64_t)kc*kWStage; *bytes = kWStage;
    } else if (l < 4) {
        *off = img_w((int)l) + (uint64_t)kc*kWStage; *bytes = kWStage;
    } else {
        *off = kImgW4Off + (uint64_t)kc*(kOutPad*128u); *bytes = kOutPad*128u;
    }
}

// The steps of a CTA that owns `n` tiles, in order: step i is (pair, layer,
// slot) = (i / 10, (i / 2) % 5, i % 2), skipped when its tile (local index
// 2 pair + slot) does not exist.
struct StepIter {
    uint32_t n, i;
    __device__ __forceinline__ bool next(uint32_t* k, uint32_t* l, uint32_t* s) {
        for (;; i++) {
            const uint32_t kk = 2u*(i/10u) + (i & 1u);
            if (2u*(i/10u) >= n) return false;
            if (kk < n) {
                *k = kk; *l = (i >> 1) % 5u; *s = i & 1u;
                i++;
                return true;
            }
        }
    }
};

// Encodes features [64 p + 16 h, + 16) of row r of a tile (inputs xi) into
// chunk p of the activation image: the values of encoded(), one sincospif
// per (input, octave) for its sine and cosine features.  f0 is the same
// for the whole warp, so the branches do not diverge.
__device__ __forceinline__ void encode_part(uint8_t* act, uint32_t r, uint32_t p, uint32_t h,
                                            const float* xi) {
    const int f0 = (int)(p*64u + h*16u);
    float v[16];
    int pair = -1;
    float sn = 0.0f, cs = 0.0f;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int f = f0 + k;
        if (f < kIn) {
            v[k] = xi[f];
        } else if (f - kIn >= 2*kFreq*kIn) {
            v[k] = 0.0f;
        } else {
            const int g = f - kIn;
            if ((g >> 1) != pair) {
                pair = g >> 1;
                const int j = g/(2*kFreq), l = (g % (2*kFreq)) >> 1;
                sincospif(__fmul_rn(xi[j], (float)(1 << l)), &sn, &cs);
            }
            v[k] = (g & 1) ? cs : sn;
        }
    }
    uint8_t* rowp = act + p*kActChunk + r*128u;
#pragma unroll
    for (uint32_t u = 0; u < 2; u++) {
        uint4 q;
        q.x = pack_bf16x2(v[8*u], v[8*u + 1]); q.y = pack_bf16x2(v[8*u + 2], v[8*u + 3]);
        q.z = pack_bf16x2(v[8*u + 4], v[8*u + 5]); q.w = pack_bf16x2(v[8*u + 6], v[8*u + 7]);
        *reinterpret_cast<uint4*>(rowp + (((h*2u + u) ^ (r & 7u)) << 4)) = q;
    }
}

// Makes this warp's shared-memory writes visible to the tensor cores and
// arrives (once per warp) on `bar`.
__device__ __forceinline__ void release_chunk(uint64_t* bar, int lane) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(bar);
}

__global__ void __launch_bounds__(kFusedThreads, 1)
fused_forward_kernel(const float* __restrict__ p, const uint8_t* __restrict__ img,
                     const float* __restrict__ x, uint32_t num_tiles, float* __restrict__ y) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                               ~(uintptr_t)1023);
    uint8_t* ring = smem + 2u*kSlotBytes;                       // kWRing x 32 KB
    uint64_t* w_full = reinterpret_cast<uint64_t*>(smem + kFusedBarOff);
    uint64_t* w_empty = w_full + kWRing;
    uint64_t* act_ready = w_empty + kWRing;                     // [slot][chunk], one arrival per epilogue warp
    uint64_t* acc_full = act_ready + 8;                         // [slot]
    uint64_t* drained = acc_full + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drained + 1);
    __shared__ int s_failed;
    __shared__ uint32_t s_issued, s_consumed;   // weight chunks copied in / taken by the MMAs
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // this CTA's tiles: blockIdx.x + k gridDim.x, k < n
    const uint32_t n = blockIdx.x < num_tiles ? (num_tiles - blockIdx.x + gridDim.x - 1)/gridDim.x : 0u;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kWRing; s++) { mbar_init(&w_full[s], 1); mbar_init(&w_empty[s], 1); }
        for (int c = 0; c < 8; c++) mbar_init(&act_ready[c], kEpiWarps);
        for (int a = 0; a < 2; a++) mbar_init(&acc_full[a], 1);
        mbar_init(drained, 1);
        s_failed = 0;
        s_issued = 0;
        s_consumed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tmem_slot)), "r"(512u));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t it = 0, k, l, sl;
            bool ok = true;
            StepIter st{n, 0};
            while (ok && st.next(&k, &l, &sl)) {
                const uint32_t chunks = l == 0 ? (uint32_t)(kEnc/64) : (uint32_t)(kH/64);
                for (uint32_t kc = 0; kc < chunks; kc++, it++) {
                    const uint32_t s = it % kWRing;
                    if (it >= (uint32_t)kWRing && !mbar_wait(&w_empty[s], ((it/kWRing) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    uint32_t bytes;
                    uint64_t off;
                    weight_chunk(l, kc, &off, &bytes);
                    mbar_expect_tx(&w_full[s], bytes);
                    bulk_g2s(ring + s*kWStage, img + off, bytes, &w_full[s]);
                    s_issued = it + 1;
                }
            }
            if (!ok) s_failed = 1;
        }
    } else if (warp == 1) {
        if (lane == 0) {
            uint32_t it = 0, k, l, sl;
            uint32_t ready = 0;   // bit 4 slot + chunk: parity of the next act_ready phase
            bool ok = true;
            StepIter st{n, 0};
            while (ok && st.next(&k, &l, &sl)) {
                // the slot's activation chunks written and its accumulator drained
                for (uint32_t c = 0; ok && c < 4; c++) {
                    const uint32_t b = sl*4u + c;
                    ok = mbar_wait(&act_ready[b], (ready >> b) & 1u);
                    ready ^= 1u << b;
                }
                if (!ok) break;
                tc_fence_after();
                const uint32_t idesc = l == 4 ? idesc_bf16(128, kOutPad) : idesc_bf16(128, kH);
                const uint32_t d = tmem + sl*256u;
                const uint32_t chunks = l == 0 ? (uint32_t)(kEnc/64) : (uint32_t)(kH/64);
                for (uint32_t kc = 0; kc < chunks; kc++, it++) {
                    const uint32_t s = it % kWRing;
                    if (!mbar_wait(&w_full[s], (it/kWRing) & 1)) { ok = false; break; }
                    s_consumed = it + 1;
                    tc_fence_after();
                    const uint32_t a_addr = smem_u32(smem + sl*kSlotBytes + kc*kActChunk);
                    const uint32_t b_addr = smem_u32(ring + s*kWStage);
#pragma unroll
                    for (uint32_t ks = 0; ks < 4; ks++)
                        umma_bf16(d, sw128_desc(a_addr + ks*32u), sw128_desc(b_addr + ks*32u),
                                  idesc, (kc | ks) != 0u ? 1u : 0u);
                    umma_commit(&w_empty[s]);
                }
                if (ok) umma_commit(&acc_full[sl]);
            }
            if (!ok) s_failed = 1;
            // arrives when every MMA issued above has completed
            umma_commit(drained);
        }
    } else {
        const uint32_t q = (uint32_t)warp & 3u;
        const uint32_t h = (uint32_t)(warp - 2) >> 2;          // 16-column slice 0..3
        const uint32_t r = q*32u + (uint32_t)lane;             // row within the tile
        const uint32_t lane_base = (q*32u) << 16;
        float xi[kIn];
        // the first tile of each slot: its inputs encoded, its accumulator free
        for (uint32_t sl = 0; sl < 2u && sl < n; sl++) {
            const uint64_t row = (uint64_t)(blockIdx.x + sl*gridDim.x)*128u + r;
#pragma unroll
            for (int j = 0; j < kIn; j++) xi[j] = __ldg(x + row*kInLd + j);
            uint8_t* act = smem + sl*kSlotBytes;
            encode_part(act, r, 0, h, xi);
            release_chunk(&act_ready[sl*4u + 0u], lane);
            encode_part(act, r, 1, h, xi);
            release_chunk(&act_ready[sl*4u + 1u], lane);
            release_chunk(&act_ready[sl*4u + 2u], lane);
            release_chunk(&act_ready[sl*4u + 3u], lane);
        }
        uint32_t accp = 0, k, l, sl;   // accp bit s: parity of acc_full[s]'s next phase
        bool ok = true;
        StepIter st{n, 0};
        while (st.next(&k, &l, &sl)) {
            ok = __all_sync(0xffffffffu, mbar_wait(&acc_full[sl], (accp >> sl) & 1u));
            accp ^= 1u << sl;
            tc_fence_after();
            if (!ok) break;
            uint8_t* act = smem + sl*kSlotBytes;
            uint64_t* ready = act_ready + sl*4u;
            const uint32_t taddr = tmem + sl*256u + lane_base;
            if (l < 4) {
                const float* bl = p + b_off((int)l);
                for (uint32_t kc = 0; kc < 4; kc++) {
                    const uint32_t c = kc*64u + h*16u;
                    float v[16];
                    tmem_ld16(taddr + c, v);
                    uint32_t pk[8];
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        const float4 b = __ldg(reinterpret_cast<const float4*>(bl + c + j));
                        float a0, a1, a2, a3;
                        f2_split(silu_pair(add2(f2(v[j], v[j + 1]), f2(b.x, b.y))), &a0, &a1);
                        f2_split(silu_pair(add2(f2(v[j + 2], v[j + 3]), f2(b.z, b.w))), &a2, &a3);
                        pk[j/2] = pack_bf16x2(a0, a1);
                        pk[j/2 + 1] = pack_bf16x2(a2, a3);
                    }
                    uint8_t* rowp = act + kc*kActChunk + r*128u;
#pragma unroll
                    for (uint32_t u = 0; u < 2; u++)
                        *reinterpret_cast<uint4*>(rowp + (((h*2u + u) ^ (r & 7u)) << 4)) =
                            make_uint4(pk[4*u], pk[4*u + 1], pk[4*u + 2], pk[4*u + 3]);
                    release_chunk(&ready[kc], lane);
                }
            } else {
                // the slot's next tile first: its layer 0 can start once the
                // outputs below are out of tensor memory
                const uint32_t next = k + 2u;
                if (next < n) {
                    const uint64_t row = (uint64_t)(blockIdx.x + next*gridDim.x)*128u + r;
#pragma unroll
                    for (int j = 0; j < kIn; j++) xi[j] = __ldg(x + row*kInLd + j);
                    encode_part(act, r, 0, h, xi);
                    release_chunk(&ready[0], lane);
                    encode_part(act, r, 1, h, xi);
                    release_chunk(&ready[1], lane);
                }
                float* orow = y + ((uint64_t)(blockIdx.x + k*gridDim.x)*128u + r)*kOutPad;
                for (uint32_t c = h*16u; c < (uint32_t)kOutPad; c += 64u) {
                    float v[16];
                    tmem_ld16(taddr + c, v);
#pragma unroll
                    for (int j = 0; j < 16; j += 4) {
                        float o[4];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            const uint32_t col = c + (uint32_t)(j + u);
                            o[u] = v[j + u] + (col < (uint32_t)kOut ? __ldg(p + kB4 + col) : 0.0f);
                        }
                        *reinterpret_cast<float4*>(orow + c + j) = make_float4(o[0], o[1], o[2], o[3]);
                    }
                }
                if (next < n) {
                    release_chunk(&ready[2], lane);
                    release_chunk(&ready[3], lane);
                }
            }
        }
        if (!ok) s_failed = 1;
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0) {
        if (s_failed) {
            atomicCAS(&g_error, 0u, (unsigned)MLGPU_ERR_RUNTIME);
            // the weight chunks no MMA consumed
            for (uint32_t it = s_consumed; it < s_issued; it++)
                mbar_wait(&w_full[it % kWRing], (it/kWRing) & 1);
        }
        // the MMAs' final commit (also on success: no arrive left pending)
        mbar_wait(drained, 0);
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(512u));
    }
}

// The loss of one photon and its gradient with respect to the 73 outputs
// (scaled by 1/batch).  Outputs y: reach logit, then per component k:
// weight logit, 4 means, 4 log-sigmas (clamped to [-9, 3]).
__device__ float photon_loss(const float* y, const float* t, bool reached, float* dy) {
    const float l = y[0];
    const float sig = 1.0f/(1.0f + __expf(-l));
    // softplus(l) - r l, computed stably
    float loss = fmaxf(l, 0.0f) + log1pf(__expf(-fabsf(l))) - (reached ? l : 0.0f);
    dy[0] = sig - (reached ? 1.0f : 0.0f);
    for (int j = 1; j < kOut; j++) dy[j] = 0.0f;
    if (!reached) return loss;
    constexpr int K = MLGPU_SG_COMPONENTS, D = MLGPU_SG_DIMS;
    float amax = -INFINITY;
    for (int k = 0; k < K; k++) amax = fmaxf(amax, y[1 + 9*k]);
    float asum = 0.0f;
    for (int k = 0; k < K; k++) asum += __expf(y[1 + 9*k] - amax);
    const float log_norm = amax + __logf(asum);
    float ell[K];
    float lmax = -INFINITY;
    for (int k = 0; k < K; k++) {
        const float* c = y + 1 + 9*k;
        float e = c[0] - log_norm;
        for (int d = 0; d < D; d++) {
            const float ls = fminf(fmaxf(c[5 + d], -9.0f), 3.0f);
            const float u = (t[d] - c[1 + d])*__expf(-ls);
            e += -0.5f*u*u - ls - 0.91893853320467274f;   // log sqrt(2 pi)
        }
        ell[k] = e;
        lmax = fmaxf(lmax, e);
    }
    float esum = 0.0f;
    for (int k = 0; k < K; k++) esum += __expf(ell[k] - lmax);
    loss += -(lmax + __logf(esum));
    for (int k = 0; k < K; k++) {
        const float* c = y + 1 + 9*k;
        float* dc = dy + 1 + 9*k;
        const float gam = __expf(ell[k] - lmax)/esum;
        const float pi = __expf(c[0] - log_norm);
        dc[0] = pi - gam;
        for (int d = 0; d < D; d++) {
            const float raw = c[5 + d];
            const float ls = fminf(fmaxf(raw, -9.0f), 3.0f);
            const float inv = __expf(-ls);
            const float u = (t[d] - c[1 + d])*inv;
            dc[1 + d] = -gam*u*inv;
            dc[5 + d] = (raw >= -9.0f && raw <= 3.0f) ? gam*(1.0f - u*u) : 0.0f;
        }
    }
    return loss;
}

// One thread per photon: loss, dY images (rows = batch, K = 128) and
// (rows = 128, K = batch), output-bias gradient, loss sum.
__global__ void __launch_bounds__(256)
loss_kernel(const float* __restrict__ y, const float* __restrict__ targets,
            const uint8_t* __restrict__ reached, uint32_t batch, uint8_t* __restrict__ dy_img,
            uint8_t* __restrict__ dyt_img, float* __restrict__ grad_b4, float* __restrict__ loss_sum) {
    const uint32_t row = blockIdx.x*blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    float dy[kOutK];
    float loss = 0.0f;
    if (row < batch) {
        float yy[kOut], t[4];
        for (int j = 0; j < kOut; j++) yy[j] = y[(uint64_t)row*kOutPad + j];
        for (int d = 0; d < 4; d++) t[d] = targets[(uint64_t)row*4 + d];
        loss = photon_loss(yy, t, reached[row] != 0, dy);
        const float inv_b = 1.0f/(float)batch;
        loss *= inv_b;
        for (int j = 0; j < kOut; j++) dy[j] *= inv_b;
    } else {
        for (int j = 0; j < kOut; j++) dy[j] = 0.0f;
    }
    for (int j = kOut; j < kOutK; j++) dy[j] = 0.0f;
    if (row < batch) {
        for (int j = 0; j < kOutK; j += 8) img_store8(dy_img, batch, row, j, dy + j);
        for (int j = 0; j < kOutK; j++) img_store1(dyt_img, kOutK, j, row, dy[j]);
    }
    for (int j = 0; j < kOut; j++) {
        float s = dy[j];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicAdd(grad_b4 + j, s);
    }
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
    if (lane == 0) atomicAdd(loss_sum, loss);
}

// Sums the split-K partials of a weight gradient into the gradient buffer
// (rows < out_rows of a [rows][256] partial).
__global__ void reduce_dw_kernel(const float* __restrict__ ws, uint32_t splits, uint64_t stride,
                                 uint32_t out_rows, uint32_t cols, float* __restrict__ grad) {
    const uint32_t n = out_rows*cols;
    for (uint32_t i = blockIdx.x*blockDim.x + threadIdx.x; i < n; i += gridDim.x*blockDim.x) {
        float s = 0.0f;
        for (uint32_t k = 0; k < splits; k++) s += ws[k*stride + i];
        grad[i] = s;
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, uint64_t n, float lr, float c1, float c2) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        const float gi = g[i];
        const float mi = 0.9f*m[i] + 0.1f*gi;
        const float vi = 0.999f*v[i] + 0.001f*gi*gi;
        m[i] = mi;
        v[i] = vi;
        if (lr != 0.0f) p[i] -= lr*(mi*c1)/(sqrtf(vi*c2) + 1e-8f);
    }
}

// ---- sampling and the exact sensor lookup ---------------------------------------

struct Grid {
    uint32_t num_sensors;
    const float* center; const float* rotation; const float* inner; const int32_t* sensor_id;
    float x0, y0, inv_cell;
    uint32_t nx, ny;
    const uint32_t* cell_start; const uint32_t* cell_items;
    float hu[2], hv[2], hw[2];
};

// The sensor whose hexagon (HexagonalPrismZ.cpp:18-29, strict bounds)
// contains (x, y), or -1.
__device__ int32_t lookup_sensor(const Grid& g, float x, float y) {
    const float fx = (x - g.x0)*g.inv_cell, fy = (y - g.y0)*g.inv_cell;
    if (!(fx >= 0.0f && fy >= 0.0f && fx < (float)g.nx && fy < (float)g.ny)) return -1;
    const uint32_t cell = (uint32_t)fy*g.nx + (uint32_t)fx;
    for (uint32_t i = __ldg(g.cell_start + cell); i < __ldg(g.cell_start + cell + 1); i++) {
        const uint32_t s = __ldg(g.cell_items + i);
        const float dx = x - __ldg(g.center + 2*s), dy = y - __ldg(g.center + 2*s + 1);
        const float c = __ldg(g.rotation + 2*s), sn = __ldg(g.rotation + 2*s + 1);
        const float lx = c*dx + sn*dy, ly = -sn*dx + c*dy;   // into the sensor frame
        const float in = __ldg(g.inner + s);
        if (fabsf(g.hu[0]*lx + g.hu[1]*ly) < in && fabsf(g.hv[0]*lx + g.hv[1]*ly) < in &&
            fabsf(g.hw[0]*lx + g.hw[1]*ly) < in)
            return __ldg(g.sensor_id + s);
    }
    return -1;
}

__global__ void __launch_bounds__(256)
sample_kernel(const float* __restrict__ out, const float* __restrict__ x, uint32_t n,
              const float* __restrict__ linear, const float* __restrict__ scale, float in_limit,
              float sigma_limit, uint64_t seed, uint64_t offset, const Grid grid,
              int32_t* __restrict__ sensor, float* __restrict__ px, float* __restrict__ py,
              float* __restrict__ pcx, float* __restrict__ pcy, uint8_t* __restrict__ fallback) {
    const uint32_t i = blockIdx.x*blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* y = out + (uint64_t)i*kOutPad;
    float xi[kIn];
    bool outside = false;
    for (int j = 0; j < kIn; j++) {
        xi[j] = x[(uint64_t)i*kInLd + j];
        outside |= !(fabsf(xi[j]) <= in_limit);
    }
    const uint64_t stream = offset + i;
    int32_t sid = -1;
    float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    uint8_t fb = outside ? 1 : 0;
    if (!fb) {
        const double u0 = mlgpu_philox_uniform(seed, stream, 0);
        const float reach = 1.0f/(1.0f + __expf(-y[0]));
        if ((float)u0 < reach) {
            // the component, by its weight
            constexpr int K = MLGPU_SG_COMPONENTS;
            float amax = -INFINITY;
            for (int k = 0; k < K; k++) amax = fmaxf(amax, y[1 + 9*k]);
            float w[K], ws = 0.0f;
            for (int k = 0; k < K; k++) { w[k] = __expf(y[1 + 9*k] - amax); ws += w[k]; }
            const float u1 = (float)mlgpu_philox_uniform(seed, stream, 1)*ws;
            int kc = K - 1;
            float acc = 0.0f;
            for (int k = 0; k < K; k++) { acc += w[k]; if (u1 < acc) { kc = k; break; } }
            const float* c = y + 1 + 9*kc;
            // two Box-Muller pairs
            float nrm[4];
            for (int h = 0; h < 2; h++) {
                const double a = mlgpu_philox_uniform(seed, stream, 2 + 2*h);
                const double b = mlgpu_philox_uniform(seed, stream, 3 + 2*h);
                const float r = sqrtf(-2.0f*__logf(fmaxf((float)a, 1e-30f)));
                float sn, cs;
                __sincosf(6.283185307179586f*(float)b, &sn, &cs);
                nrm[2*h] = r*cs; nrm[2*h + 1] = r*sn;
            }
            float sig_pos = 0.0f;
            for (int d = 0; d < 4; d++) {
                const float ls = fminf(fmaxf(c[5 + d], -9.0f), 3.0f);
                const float s = __expf(ls);
                const float tn = c[1 + d] + s*nrm[d];
                float base = linear[d*6 + 5];
                for (int j = 0; j < kIn; j++) base += linear[d*6 + j]*xi[j];
                t[d] = base + scale[d]*tn;
                if (d < 2) sig_pos = fmaxf(sig_pos, s*scale[d]);
            }
            if (sig_pos > sigma_limit) fb = 1;
            else sid = grid.nx ? lookup_sensor(grid, t[0], t[1]) : -2;   // -2: reached the plane
        }
    }
    sensor[i] = fb ? -1 : sid;
    if (px) px[i] = t[0];
    if (py) py[i] = t[1];
    if (pcx) pcx[i] = t[2];
    if (pcy) pcy[i] = t[3];
    fallback[i] = fb;
}

// ---- workspace layout ------------------------------------------------------------

struct Work {
    uint8_t* enc_img;     // encoded inputs (rows = batch, K = 128)
    uint8_t* enc_imgt;    // and transposed (rows = 128, K = batch), training
    uint8_t* h_img[4];    // layer outputs h0..h3 (rows = batch, K = 256)
    uint8_t* h_imgt[4];   // their transposes (rows = 256, K = batch), training
    float* z[4];          // pre-activations z0..z3, training
    float* y;             // [batch][80]
    uint8_t* dy_img;      // [batch x 128]
    uint8_t* dyt_img;     // [128 x batch]
    uint8_t* dz_img[2];   // ping-pong dZ images (rows = batch, K = 256)
    uint8_t* dz_imgt[2];  // and transposes
    float* ws;            // split-K partials
    float* grads;         // [params]
    float* loss;          // [1]
};

constexpr uint32_t kSplits = 64;

uint64_t up256(uint64_t x) { return (x + 255) & ~uint64_t(255); }

uint64_t carve(uint8_t* base, uint32_t batch, bool training, Work* w) {
    uint64_t off = 0;
    auto take = [&](uint64_t bytes) { uint8_t* p = base ? base + off : nullptr; off += up256(bytes); return p; };
    const uint64_t himg = (uint64_t)batch*kH*2;
    w->enc_img = take((uint64_t)batch*kEnc*2);
    for (int l = 0; l < 4; l++) w->h_img[l] = take(himg);
    w->y = reinterpret_cast<float*>(take((uint64_t)batch*kOutPad*4));
    if (training) {
        w->enc_imgt = take((uint64_t)batch*kEnc*2);
        for (int l = 0; l < 4; l++) w->h_imgt[l] = take(himg);
        for (int l = 0; l < 4; l++) w->z[l] = reinterpret_cast<float*>(take((uint64_t)batch*kH*4));
        w->dy_img = take((uint64_t)batch*kOutK*2);
        w->dyt_img = take((uint64_t)batch*kOutK*2);
        for (int k = 0; k < 2; k++) { w->dz_img[k] = take(himg); w->dz_imgt[k] = take(himg); }
        w->ws = reinterpret_cast<float*>(take((uint64_t)kSplits*kH*kH*4));
        w->grads = reinterpret_cast<float*>(take(kParams*4));
        w->loss = reinterpret_cast<float*>(take(256));
    } else {
        w->enc_imgt = nullptr;
        for (int l = 0; l < 4; l++) w->h_imgt[l] = nullptr;
        for (int l = 0; l < 4; l++) w->z[l] = nullptr;
    }
    return off;
}

GemmArgs gemm_args(const uint8_t* a, uint32_t a_rows, const uint8_t* b, uint32_t b_rows,
                   uint32_t k_chunks) {
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.a = a; g.a_rows = a_rows; g.b = b; g.b_rows = b_rows; g.k_chunks = k_chunks;
    return g;
}

// The forward pass (training: also transposed images and pre-activations).
cudaError_t forward(const float* p, const uint8_t* img, const float* x, uint32_t batch,
                    const Work& w, float* y, bool training, cudaStream_t s) {
    encode_kernel<<<(uint32_t)(((uint64_t)batch*(kEnc/8) + 255)/256), 256, 0, s>>>(
        x, batch, w.enc_img, training ? w.enc_imgt : nullptr);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) {
        GemmArgs g = gemm_args(w.enc_img, batch, img + kImgW0Off, kH, kEnc/64);
        g.bias = p + kB0; g.bias_n = kH;
        g.img = w.h_img[0]; g.img_rows = batch;
        g.img_t = training ? w.h_imgt[0] : nullptr; g.img_t_rows = kH;
        g.z = training ? w.z[0] : nullptr; g.z_ld = kH;
        e = launch_persistent<256, kEnc/64, kEpiSilu>(g, batch, s);
    }
    for (int l = 1; l <= 3 && e == cudaSuccess; l++) {
        GemmArgs g = gemm_args(w.h_img[l - 1], batch, img + img_w(l), kH, kH/64);
        g.bias = p + b_off(l); g.bias_n = kH;
        g.img = w.h_img[l]; g.img_rows = batch;
        g.img_t = training ? w.h_imgt[l] : nullptr; g.img_t_rows = kH;
        g.z = training ? w.z[l] : nullptr; g.z_ld = kH;
        e = launch_persistent<256, 4, kEpiSilu>(g, batch, s);
    }
    if (e == cudaSuccess) {
        GemmArgs g = gemm_args(w.h_img[3], batch, img + kImgW4Off, kOutPad, kH/64);
        g.bias = p + kB4; g.bias_n = kOut;
        g.out = y; g.ld = kOutPad; g.n_store = kOutPad;
        e = launch_persistent<kOutPad, 4, kEpiF32>(g, batch, s);
    }
    return e;
}

// The inference forward pass in one launch (fused_forward_kernel).
cudaError_t forward_fused(const float* p, const uint8_t* img, const float* x, uint32_t batch,
                          float* y, cudaStream_t s) {
    constexpr uint32_t smem = fused_smem_bytes();
    static bool attr = false;
    if (!attr) {
        const cudaError_t e = cudaFuncSetAttribute(fused_forward_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const uint32_t tiles = batch/128u;
    const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
    fused_forward_kernel<<<grid, kFusedThreads, smem, s>>>(p, img, x, tiles, y);
    return cudaGetLastError();
}

cudaError_t train_step(float* p, uint8_t* img, float* m, float* v, const float* x,
                       const float* targets, const uint8_t* reached, uint32_t batch,
                       uint32_t step, float lr, float* loss_out, float* grads_out, const Work& w,
                       cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(w.grads, 0, kParams*4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w.loss, 0, 4, s);
    if (e == cudaSuccess) e = forward(p, img, x, batch, w, w.y, true, s);
    if (e != cudaSuccess) return e;
    loss_kernel<<<(batch + 255)/256, 256, 0, s>>>(w.y, targets, reached, batch, w.dy_img,
                                                   w.dyt_img, w.grads + kB4, w.loss);
    e = cudaGetLastError();
    const uint32_t kchunks = batch/64;
    uint32_t splits = kSplits;
    while (splits > 1 && kchunks % splits) splits >>= 1;
    const uint64_t ws_stride = (uint64_t)kH*kH;
    // output layer: dW4 = dY^T h3 (rows = 128 padded outputs), dH3 = dY W4
    if (e == cudaSuccess) {
        GemmArgs g = gemm_args(w.dyt_img, kOutK, w.h_imgt[3], kH, kchunks/splits);
        g.out = w.ws; g.ld = kH; g.split_stride = ws_stride; g.n_store = kH;
        e = launch_gemm<256, kEpiF32>(g, kOutK, kH, splits, s);
    }
    if (e == cudaSuccess) {
        reduce_dw_kernel<<<148, 256, 0, s>>>(w.ws, splits, ws_stride, kOut, kH, w.grads + kW4);
        e = cudaGetLastError();
    }
    int cur = 0;
    if (e == cudaSuccess) {
        GemmArgs g = gemm_args(w.dy_img, batch, img + kImgW4TOff, kH, kOutK/64);
        g.z = w.z[3]; g.z_ld = kH;
        g.img = w.dz_img[cur]; g.img_rows = batch;
        g.img_t = w.dz_imgt[cur]; g.img_t_rows = kH;
        g.col_sum = w.grads + kB3;
        e = launch_persistent<256, 2, kEpiDSilu>(g, batch, s);
    }
    // hidden layers l = 3, 2, 1: dW_l = dZ_l^T h_{l-1}, dZ_{l-1} = (dZ_l W_l) * SiLU'(z_{l-1})
    for (int l = 3; l >= 1 && e == cudaSuccess; l--) {
        GemmArgs g = gemm_args(w.dz_imgt[cur], kH, w.h_imgt[l - 1], kH, kchunks/splits);
        g.out = w.ws; g.ld = kH; g.split_stride = ws_stride; g.n_store = kH;
        e = launch_gemm<256, kEpiF32>(g, kH, kH, splits, s);
        if (e != cudaSuccess) break;
        reduce_dw_kernel<<<148, 256, 0, s>>>(w.ws, splits, ws_stride, kH, kH, w.grads + w_off(l));
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        GemmArgs d = gemm_args(w.dz_img[cur], batch, img + img_wt(l), kH, kH/64);
        d.z = w.z[l - 1]; d.z_ld = kH;
        d.col_sum = w.grads + b_off(l - 1);
        d.img = w.dz_img[cur ^ 1]; d.img_rows = batch;
        d.img_t = w.dz_imgt[cur ^ 1]; d.img_t_rows = kH;
        e = launch_persistent<256, 4, kEpiDSilu>(d, batch, s);
        cur ^= 1;
    }
    // layer 0: dW0 = dZ0^T enc (dZ0's images are at `cur` now)
    if (e == cudaSuccess) {
        GemmArgs g = gemm_args(w.dz_imgt[cur], kH, w.enc_imgt, kEnc, kchunks/splits);
        g.out = w.ws; g.ld = kEnc; g.split_stride = ws_stride; g.n_store = kEnc;
        e = launch_gemm<kEnc, kEpiF32>(g, kH, kEnc, splits, s);
    }
    if (e == cudaSuccess) {
        reduce_dw_kernel<<<148, 256, 0, s>>>(w.ws, splits, ws_stride, kH, kEnc, w.grads + kW0);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && grads_out)
        e = cudaMemcpyAsync(grads_out, w.grads, kParams*4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && loss_out)
        e = cudaMemcpyAsync(loss_out, w.loss, 4, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) {
        const double c1 = 1.0/(1.0 - std::pow(0.9, (double)step));
        const double c2 = 1.0/(1.0 - std::pow(0.999, (double)step));
        adam_kernel<<<148, 256, 0, s>>>(p, w.grads, m, v, kParams, lr, (float)c1, (float)c2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        pack_weights_kernel<<<148, 256, 0, s>>>(p, img);
        e = cudaGetLastError();
    }
    return e;
}

}  // namespace
}  // namespace sg
}  // namespace mlgpu

using namespace mlgpu;
using namespace mlgpu::sg;

extern "C" {

size_t mlgpu_sg_image_offset(uint32_t rows, uint32_t r, uint32_t k) { return (size_t)img_off(rows, r, k); }

uint64_t mlgpu_sg_param_count(void) { return kParams; }
uint64_t mlgpu_sg_image_bytes(void) { return kImgBytes; }

uint64_t mlgpu_sg_workspace_bytes(uint32_t batch, int training) {
    Work w;
    return carve(nullptr, batch, training != 0, &w);
}

int mlgpu_sg_gemm_f32(const void* a_img, uint32_t a_rows, const void* b_img, uint32_t b_rows,
                      uint32_t m, uint32_t n, uint32_t k_chunks, const float* bias, float* c,
                      void* cuda_stream) {
    if (!a_img || !b_img || !c) return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (m == 0 || m % 128 || a_rows < m || a_rows % 128 || k_chunks == 0 || b_rows < n ||
        b_rows % 8)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT,
                            "m must be a positive multiple of 128 within a_rows (a multiple of 128)");
    GemmArgs g = gemm_args(static_cast<const uint8_t*>(a_img), a_rows,
                           static_cast<const uint8_t*>(b_img), b_rows, k_chunks);
    g.bias = bias; g.bias_n = n; g.out = c; g.ld = n; g.n_store = n;
    const cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    cudaError_t e;
    if (n % 256 == 0 && b_rows % 256 == 0) e = launch_gemm<256, kEpiF32>(g, m, n, 1, s);
    else if (n % 128 == 0 && b_rows % 128 == 0) e = launch_gemm<128, kEpiF32>(g, m, n, 1, s);
    else if (n == 80 && b_rows == 80) e = launch_gemm<80, kEpiF32>(g, m, n, 1, s);
    else return report_error(MLGPU_ERR_INVALID_ARGUMENT, "n must be 80 or a multiple of 128");
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_pack_weights(const float* params, void* images, void* cuda_stream) {
    if (!params || !images) return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    pack_weights_kernel<<<148, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
        params, static_cast<uint8_t*>(images));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_forward(const float* params, const void* images, const float* inputs,
                     uint32_t batch, float* outputs, void* workspace, void* cuda_stream) {
    (void)workspace;   // the fused pass keeps its activations on chip
    if (!params || !images || !inputs || !outputs)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (batch == 0 || batch % 128)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "batch must be a positive multiple of 128");
    const cudaError_t e = forward_fused(params, static_cast<const uint8_t*>(images), inputs, batch,
                                        outputs, static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_forward_layered(const float* params, const void* images, const float* inputs,
                             uint32_t batch, float* outputs, void* workspace, void* cuda_stream) {
    if (!params || !images || !inputs || !outputs || !workspace)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (batch == 0 || batch % 128)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "batch must be a positive multiple of 128");
    Work w;
    carve(static_cast<uint8_t*>(workspace), batch, false, &w);
    const cudaError_t e = forward(params, static_cast<const uint8_t*>(images), inputs, batch, w,
                                  outputs, false, static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_train_step(float* params, void* images, float* adam_m, float* adam_v,
                        const float* inputs, const float* targets, const uint8_t* reached,
                        uint32_t batch, uint32_t step, float lr, float* loss, float* grads,
                        void* workspace, void* cuda_stream) {
    if (!params || !images || !adam_m || !adam_v || !inputs || !targets || !reached || !workspace)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (batch == 0 || batch % 128)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "batch must be a positive multiple of 128");
    if (step == 0) return report_error(MLGPU_ERR_INVALID_ARGUMENT, "step is 1-based");
    Work w;
    carve(static_cast<uint8_t*>(workspace), batch, true, &w);
    const cudaError_t e = train_step(params, static_cast<uint8_t*>(images), adam_m, adam_v, inputs,
                                     targets, reached, batch, step, lr, loss, grads, w,
                                     static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_sample(const float* outputs, const float* inputs, uint32_t n, const float* linear,
                    const float* scale, float in_limit, float sigma_limit, uint64_t seed,
                    uint64_t photon_offset, const mlgpu_sg_sensor_grid* grid, int32_t* sensor,
                    float* x, float* y, float* cx, float* cy, uint8_t* fallback,
                    void* cuda_stream) {
    if (!outputs || !inputs || !linear || !scale || !sensor || !fallback)
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (grid && (!grid->center || !grid->rotation || !grid->inner || !grid->sensor_id ||
                 !grid->cell_start || !grid->cell_items || !(grid->cell > 0.0) ||
                 grid->nx == 0 || grid->ny == 0))
        return report_error(MLGPU_ERR_INVALID_ARGUMENT, "incomplete sensor grid");
    if (n == 0) return MLGPU_OK;
    Grid g;
    memset(&g, 0, sizeof(g));
    if (grid) {
    g.num_sensors = grid->num_sensors;
    g.center = grid->center; g.rotation = grid->rotation; g.inner = grid->inner;
    g.sensor_id = grid->sensor_id;
    g.x0 = (float)grid->x0; g.y0 = (float)grid->y0; g.inv_cell = (float)(1.0/grid->cell);
    g.nx = grid->nx; g.ny = grid->ny;
    g.cell_start = grid->cell_start; g.cell_items = grid->cell_items;
    for (int k = 0; k < 2; k++) {
        g.hu[k] = (float)grid->hex_u[k]; g.hv[k] = (float)grid->hex_v[k]; g.hw[k] = (float)grid->hex_w[k];
    }
    }
    sample_kernel<<<(n + 255)/256, 256, 0, static_cast<cudaStream_t>(cuda_stream)>>>(
        outputs, inputs, n, linear, scale, in_limit, sigma_limit, seed, photon_offset, g, sensor,
        x, y, cx, cy, fallback);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}

int mlgpu_sg_sync_errors(void* cuda_stream) {
    cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    unsigned int code = 0;
    e = cudaMemcpyFromSymbol(&code, g_error, sizeof(code));
    if (e != cudaSuccess) return report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    if (code) {
        const unsigned int zero = 0;
        cudaMemcpyToSymbol(g_error, &zero, sizeof(zero));
        return report_error((int)code, "a tensor-core kernel timed out waiting for its operands");
    }
    return MLGPU_OK;
}

}  // extern "C"
