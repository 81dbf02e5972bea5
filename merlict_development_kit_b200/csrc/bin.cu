// bin.cu -- per-sensor arrival counts and time histograms without atomics.
//
// The statistics a caller of merlict's Sensors::assign_photons
// (merlict/sensor/Sensors.cpp:79-81) derives from the arrival lists:
// photons per sensor and, optionally, their arrival-time histogram.
//
// Key space: key = sensor * (B + 1) + time bin, the extra bin B holding the
// arrivals outside [t_min, t_max).  The grid is (key tiles) x (photon
// slices).  A CTA scans its photon slice, keeps the keys of its tile, and
// every warp adds into its own private shared-memory histogram: lanes that
// share a key are merged with __match_any_sync and only the lowest such lane
// writes, so no two threads ever update the same word concurrently.  The
// CTA then sums its warps' histograms and stores the tile with plain stores
// into the slice's partial histogram; a second kernel sums the slices.
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

constexpr int kBinWarps = 8;
constexpr int kBinTile = 4096;   // keys per CTA tile: 8 warps x 16 KiB of shared memory

__device__ __forceinline__ int32_t arrival_key(int32_t s, const double* time, uint64_t i,
                                               uint32_t B, double t_min, double t_max) {
    if (s < 0) return -1;
    if (B == 0) return s;
    const double f = (time[i] - t_min) / (t_max - t_min) * (double)B;
    const uint32_t tb = (f >= 0.0 && f < (double)B) ? (uint32_t)f : B;
    return s*(int32_t)(B + 1) + (int32_t)tb;
}

__global__ void __launch_bounds__(kBinWarps*32)
bin_tiles_kernel(const int32_t* __restrict__ sensor, const double* __restrict__ time,
                 uint64_t n, uint32_t B, double t_min, double t_max, int32_t num_keys,
                 uint32_t* __restrict__ partial, uint64_t slice_len) {
    extern __shared__ uint32_t hist[];   // [kBinWarps][kBinTile]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t tile0 = blockIdx.x*kBinTile;
    const int32_t tile_len = min(kBinTile, num_keys - tile0);
    for (int k = threadIdx.x; k < kBinWarps*kBinTile; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    uint32_t* mine = hist + warp*kBinTile;
    const uint64_t begin = (uint64_t)blockIdx.y*slice_len;
    const uint64_t end = min(n, begin + slice_len);
    for (uint64_t base = begin + (uint64_t)warp*32; base < end; base += kBinWarps*32) {
        const uint64_t i = base + lane;
        int32_t key = -1;
        if (i < end) key = arrival_key(__ldg(sensor + i), time, i, B, t_min, t_max);
        const bool in = key >= tile0 && key < tile0 + tile_len;
        const unsigned valid = __ballot_sync(0xffffffffu, in);
        if (in) {
            const unsigned same = __match_any_sync(valid, key);
            if (lane == __ffs(same) - 1) mine[key - tile0] += __popc(same);
        }
        __syncwarp();
    }
    __syncthreads();
    uint32_t* out = partial + (uint64_t)blockIdx.y*num_keys + tile0;
    for (int k = threadIdx.x; k < tile_len; k += blockDim.x) {
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kBinWarps; w++) sum += hist[w*kBinTile + k];
        out[k] = sum;
    }
}

__global__ void bin_reduce_kernel(const uint32_t* __restrict__ partial, uint32_t slices,
                                  int32_t num_sensors, uint32_t B, int32_t num_keys,
                                  uint32_t* __restrict__ counts, uint32_t* __restrict__ time_hist) {
    const int32_t s = blockIdx.x*blockDim.x + threadIdx.x;
    if (s >= num_sensors) return;
    uint32_t total = 0;
    for (uint32_t b = 0; b <= B; b++) {
        const int32_t key = s*(int32_t)(B + 1) + (int32_t)b;
        uint32_t v = 0;
        for (uint32_t j = 0; j < slices; j++) v += partial[(uint64_t)j*num_keys + key];
        total += v;
        if (time_hist && b < B) time_hist[(uint64_t)s*B + b] = v;
    }
    counts[s] = total;
}

}  // namespace

cudaError_t launch_bin_arrivals(const DevScene& sc, const int32_t* sensor, const double* time,
                                uint64_t n, uint32_t* counts, uint32_t* time_hist,
                                uint32_t num_bins, double t_min, double t_max,
                                uint32_t* scratch, size_t scratch_words, cudaStream_t s) {
    const int32_t num_sensors = sc.num_sensors;
    if (num_sensors <= 0) return cudaSuccess;
    const uint32_t B = time_hist ? num_bins : 0;
    const int32_t num_keys = num_sensors*(int32_t)(B + 1);
    const int32_t tiles = (num_keys + kBinTile - 1)/kBinTile;
    // enough CTAs to fill the GPU twice, limited by the scratch size
    uint32_t slices = (uint32_t)((2*148 + tiles - 1)/tiles);
    if (slices < 1) slices = 1;
    if (slices > 32) slices = 32;
    while (slices > 1 && (uint64_t)slices*num_keys > scratch_words) slices--;
    if ((uint64_t)slices*num_keys > scratch_words) return cudaErrorInvalidValue;
    if (n == 0) slices = 1;
    const uint64_t slice_len = n == 0 ? 1 : (n + slices - 1)/slices;
    const size_t smem = sizeof(uint32_t)*kBinWarps*kBinTile;
    cudaError_t e = cudaFuncSetAttribute(bin_tiles_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    bin_tiles_kernel<<<dim3(tiles, slices), kBinWarps*32, smem, s>>>(
        sensor, time, n, B, t_min, t_max, num_keys, scratch, slice_len);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bin_reduce_kernel<<<(num_sensors + 255)/256, 256, 0, s>>>(
        scratch, slices, num_sensors, B, num_keys, counts, time_hist);
    return cudaGetLastError();
}

}  // namespace mlgpu
