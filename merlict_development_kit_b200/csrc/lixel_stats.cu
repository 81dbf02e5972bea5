// lixel_stats.cu -- per-sensor calibration statistics on the device:
// plenoscope::calibration::LixelStatisticsFiller
// (merlict_portal_plenoscope/calibration/LixelStatisticsFiller.cpp:20-62)
// with its OnlineStatistics (OnlineStatistics.cpp:15-50).
//
// The photons that reached a sensor are put into sensor order by a stable
// radix sort (so each sensor sees its photons in their original order), then
// one thread per sensor runs merlict's online update (n += 1; delta = x -
// mean; mean += delta/n; m2 += delta (x - mean); sum += x) over them, in
// the same order and arithmetic (--fmad=false), and writes the
// LixelStatistic fields as merlict computes them.
#include <cmath>
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

struct Online {
    double n = 0.0, sum = 0.0, mean = 0.0, m2 = 0.0;
    __device__ void add(double x) {
        n += 1.0;
        const double delta = x - mean;
        mean += delta/n;
        m2 += delta*(x - mean);
        sum += x;
    }
    __device__ float mean_out() const { return (float)(sum/n); }
    __device__ float std_out() const {
        return n < 2.0 ? __int_as_float(0x7fc00000) : (float)sqrt(m2/n);
    }
};

__global__ void __launch_bounds__(256)
stats_keys_kernel(const int32_t* __restrict__ sensor, uint64_t n, uint32_t* __restrict__ key,
                  uint32_t* __restrict__ idx) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        const int32_t s = sensor[i];
        key[i] = s >= 0 ? (uint32_t)s : 0xffffffffu;   // photons without a sensor sort last
        idx[i] = (uint32_t)i;
    }
}

__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* a, uint64_t n, uint32_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (a[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// One thread per sensor: count and the online statistics of its photons.
__global__ void __launch_bounds__(128)
stats_reduce_kernel(const uint32_t* __restrict__ key, const uint32_t* __restrict__ idx, uint64_t n,
                    uint32_t num_sensors, const float* __restrict__ cx, const float* __restrict__ cy,
                    const float* __restrict__ x, const float* __restrict__ y,
                    const float* __restrict__ t, double emitted, float* __restrict__ out) {
    const uint32_t s = blockIdx.x*blockDim.x + threadIdx.x;
    if (s >= num_sensors) return;
    const uint64_t b = lower_bound_u32(key, n, s), e = lower_bound_u32(key, n, s + 1);
    Online ocx, ocy, ox, oy, ot;
    for (uint64_t k = b; k < e; k++) {
        const uint32_t i = __ldg(idx + k);
        ocx.add((double)__ldg(cx + i));
        ocy.add((double)__ldg(cy + i));
        ox.add((double)__ldg(x + i));
        oy.add((double)__ldg(y + i));
        ot.add((double)__ldg(t + i));
    }
    const unsigned int count = (unsigned int)(e - b);
    // LixelStatisticsFiller::get_lixel_statistics, LixelStatisticsFiller.cpp:43-62
    float* o = out + (uint64_t)s*12;
    o[0] = (float)((double)count/emitted);
    o[1] = (float)((double)sqrtf((float)count)/emitted);
    o[2] = ocx.mean_out(); o[3] = ocx.std_out();
    o[4] = ocy.mean_out(); o[5] = ocy.std_out();
    o[6] = ox.mean_out(); o[7] = ox.std_out();
    o[8] = oy.mean_out(); o[9] = oy.std_out();
    o[10] = ot.mean_out(); o[11] = ot.std_out();
}

}  // namespace

size_t lixel_stats_scratch_bytes(uint64_t n) {
    return 6*((n*4 + 255) & ~uint64_t(255)) + radix_sort_temp_bytes(n) + 256;
}

cudaError_t launch_lixel_stats(const int32_t* sensor, const float* const* values, uint64_t n,
                               uint32_t num_sensors, double emitted, float* out, void* scratch,
                               size_t scratch_bytes, int grid, cudaStream_t s) {
    const uint64_t a = (n*4 + 255) & ~uint64_t(255);
    char* p = static_cast<char*>(scratch);
    uint32_t* key_in = reinterpret_cast<uint32_t*>(p);
    uint32_t* idx_in = reinterpret_cast<uint32_t*>(p + a);
    uint32_t* key_out = reinterpret_cast<uint32_t*>(p + 2*a);
    uint32_t* idx_out = reinterpret_cast<uint32_t*>(p + 3*a);
    uint32_t* key_tmp = reinterpret_cast<uint32_t*>(p + 4*a);
    uint32_t* idx_tmp = reinterpret_cast<uint32_t*>(p + 5*a);
    void* temp = p + 6*a;
    stats_keys_kernel<<<grid, 256, 0, s>>>(sensor, n, key_in, idx_in);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // stable: photons of one sensor keep their order (device_sort.cu)
    e = radix_sort_pairs(key_in, idx_in, key_out, idx_out, key_tmp, idx_tmp, n, 32, temp, s);
    if (e != cudaSuccess) return e;
    stats_reduce_kernel<<<(num_sensors + 127)/128, 128, 0, s>>>(
        key_out, idx_out, n, num_sensors, values[0], values[1], values[2], values[3], values[4],
        emitted, out);
    return cudaGetLastError();
}

}  // namespace mlgpu
