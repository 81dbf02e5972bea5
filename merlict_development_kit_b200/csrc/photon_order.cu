// photon_order.cu -- the order in which the wavefront tracers take photons
// into their pool.
//
// Photons of a batch arrive in random order, so neighbouring ray slots
// would walk unrelated parts of the scene and gather unrelated leaf records.
// Before tracing, the batch is put into the order of a 4-D Morton key over
// (support x, support y, direction x, direction y), each quantised to
// kBitsPerDim bits over the batch's own range: photons close in that order
// start close together and travel in nearly the same direction, so they
// tend to hit the same facets, lenses and lixels step after step.  The sort
// is a counting sort: a histogram of the keys, an exclusive scan, and a
// scatter of photon indices.  The order within a key is whatever the
// atomics give; it changes nothing in the results, since every photon keeps
// its own index, random stream and result slot.
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

constexpr int kBitsPerDim = 5;
constexpr uint32_t kCells = 1u << (4*kBitsPerDim);
constexpr int kScanBlock = 1024;

// Total order of floats as unsigned ints (for atomic min/max).
__device__ __forceinline__ uint32_t order_bits(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_order_bits(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

template <typename In>
__device__ __forceinline__ void key_coords(const DevPhotons& p, uint64_t i, float* v) {
    v[0] = (float)__ldg(static_cast<const In*>(p.sx) + i);
    v[1] = (float)__ldg(static_cast<const In*>(p.sy) + i);
    v[2] = (float)__ldg(static_cast<const In*>(p.dx) + i);
    v[3] = (float)__ldg(static_cast<const In*>(p.dy) + i);
}

// range[2k] = min, range[2k + 1] = max of coordinate k (order bits); NaNs
// are left out.
template <typename In>
__global__ void __launch_bounds__(256)
order_range_kernel(const DevPhotons p, uint64_t n, uint32_t* range) {
    float lo[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
    float hi[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        float v[4];
        key_coords<In>(p, i, v);
#pragma unroll
        for (int k = 0; k < 4; k++) {
            lo[k] = fminf(lo[k], v[k]);   // fminf/fmaxf drop a NaN operand
            hi[k] = fmaxf(hi[k], v[k]);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            atomicMin(&range[2*k], order_bits(lo[k]));
            atomicMax(&range[2*k + 1], order_bits(hi[k]));
        }
    }
}

__device__ __forceinline__ uint32_t spread4(uint32_t x) {
    // bit b of x goes to bit 4b
    uint32_t r = 0;
#pragma unroll
    for (int b = 0; b < kBitsPerDim; b++) r |= ((x >> b) & 1u) << (4*b);
    return r;
}

template <typename In>
__global__ void __launch_bounds__(256)
order_key_kernel(const DevPhotons p, uint64_t n, const uint32_t* range, uint32_t* key,
                 uint32_t* hist) {
    float lo[4], scale[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        lo[k] = from_order_bits(range[2*k]);
        const float ext = from_order_bits(range[2*k + 1]) - lo[k];
        scale[k] = ext > 0.0f ? (float)(1 << kBitsPerDim)/ext : 0.0f;
    }
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        float v[4];
        key_coords<In>(p, i, v);
        uint32_t k4 = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            // clamp into [0, 2^bits - 1]; a NaN becomes 0
            const float q = fminf(fmaxf((v[k] - lo[k])*scale[k], 0.0f),
                                  (float)((1 << kBitsPerDim) - 1));
            k4 |= spread4((uint32_t)q) << k;
        }
        key[i] = k4;
        atomicAdd(&hist[k4], 1u);
    }
}

// Exclusive scan of kCells counts: per-block scans, then the block sums.
__global__ void __launch_bounds__(kScanBlock)
order_scan_blocks_kernel(uint32_t* hist, uint32_t* block_sum) {
    __shared__ uint32_t warp_sum[kScanBlock/32];
    const uint32_t i = blockIdx.x*kScanBlock + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t v = hist[i];
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = warp_sum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;   // inclusive
    }
    __syncthreads();
    const uint32_t before = wid > 0 ? warp_sum[wid - 1] : 0u;
    hist[i] = before + x - v;   // exclusive within the block
    if (threadIdx.x == kScanBlock - 1) block_sum[blockIdx.x] = before + x;
}

__global__ void __launch_bounds__(kScanBlock)
order_scan_sums_kernel(uint32_t* block_sum, int blocks) {
    __shared__ uint32_t warp_sum[kScanBlock/32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t v = (int)threadIdx.x < blocks ? block_sum[threadIdx.x] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = warp_sum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;
    }
    __syncthreads();
    const uint32_t before = wid > 0 ? warp_sum[wid - 1] : 0u;
    if ((int)threadIdx.x < blocks) block_sum[threadIdx.x] = before + x - v;
}

__global__ void __launch_bounds__(kScanBlock)
order_scan_add_kernel(uint32_t* hist, const uint32_t* block_sum) {
    hist[blockIdx.x*kScanBlock + threadIdx.x] += block_sum[blockIdx.x];
}

__global__ void __launch_bounds__(256)
order_scatter_kernel(uint64_t n, const uint32_t* key, uint32_t* next, uint32_t* order) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x)
        order[atomicAdd(&next[key[i]], 1u)] = (uint32_t)i;
}

// The photons themselves into their place in the order: one 64-byte record
// each, (sx, sy), (sz, dx), (dy, dz), (wavelength, index_base + i), the values as
// the tracers read them (a float input widened to double, which is exact).
// The input planes are read in order and the record stored whole, so that
// the intake reads the records sequentially instead of gathering seven
// planes through a permutation.
template <typename In>
__global__ void __launch_bounds__(256)
order_scatter_records_kernel(const DevPhotons p, uint64_t n, const uint32_t* key, uint32_t* next,
                             double2* sorted, uint64_t index_base) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        auto ld = [i](const void* plane) { return (double)__ldg(static_cast<const In*>(plane) + i); };
        const double sx = ld(p.sx), sy = ld(p.sy), sz = ld(p.sz);
        const double dx = ld(p.dx), dy = ld(p.dy), dz = ld(p.dz), wl = ld(p.wavelength);
        double2* r = sorted + 4*(uint64_t)atomicAdd(&next[key[i]], 1u);
        r[0] = make_double2(sx, sy);
        r[1] = make_double2(sz, dx);
        r[2] = make_double2(dy, dz);
        r[3] = make_double2(wl, __longlong_as_double((long long)(index_base + i)));
    }
}

}  // namespace

size_t photon_order_scratch_bytes(uint64_t n) {
    return (size_t)n*sizeof(uint32_t) + ((size_t)kCells + kCells/kScanBlock + 8)*sizeof(uint32_t);
}

cudaError_t launch_photon_order(const DevPhotons& p, int in_dtype, uint64_t n, uint32_t* order,
                                double2* sorted, uint64_t index_base, void* scratch, int grid,
                                cudaStream_t s) {
    uint32_t* key = static_cast<uint32_t*>(scratch);
    uint32_t* hist = key + n;
    uint32_t* block_sum = hist + kCells;
    uint32_t* range = block_sum + kCells/kScanBlock;
    static_assert(kCells/kScanBlock <= kScanBlock, "block sums must fit one scan block");
    cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)kCells*sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    const uint32_t init[8] = {~0u, 0u, ~0u, 0u, ~0u, 0u, ~0u, 0u};
    for (int k = 0; k < 8; k++) {
        e = cudaMemsetAsync(range + k, init[k] ? 0xff : 0x00, sizeof(uint32_t), s);
        if (e != cudaSuccess) return e;
    }
    if (in_dtype == MLGPU_F64) {
        order_range_kernel<double><<<grid, 256, 0, s>>>(p, n, range);
        order_key_kernel<double><<<grid, 256, 0, s>>>(p, n, range, key, hist);
    } else {
        order_range_kernel<float><<<grid, 256, 0, s>>>(p, n, range);
        order_key_kernel<float><<<grid, 256, 0, s>>>(p, n, range, key, hist);
    }
    order_scan_blocks_kernel<<<kCells/kScanBlock, kScanBlock, 0, s>>>(hist, block_sum);
    order_scan_sums_kernel<<<1, kScanBlock, 0, s>>>(block_sum, (int)(kCells/kScanBlock));
    order_scan_add_kernel<<<kCells/kScanBlock, kScanBlock, 0, s>>>(hist, block_sum);
    if (!sorted)
        order_scatter_kernel<<<grid, 256, 0, s>>>(n, key, hist, order);
    else if (in_dtype == MLGPU_F64)
        order_scatter_records_kernel<double><<<grid, 256, 0, s>>>(p, n, key, hist, sorted,
                                                                  index_base);
    else
        order_scatter_records_kernel<float><<<grid, 256, 0, s>>>(p, n, key, hist, sorted,
                                                                 index_base);
    return cudaGetLastError();
}

}  // namespace mlgpu
