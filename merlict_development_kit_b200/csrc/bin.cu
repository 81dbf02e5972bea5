// bin.cu -- per-sensor arrival counts and time histograms without atomics.
//
// The statistics a caller of merlict's Sensors::assign_photons
// (merlict/sensor/Sensors.cpp:79-81) derives from the arrival lists:
// photons per sensor and, optionally, their arrival-time histogram.
//
// Key space: key = sensor * (B + 1) + time bin, the extra bin B holding the
// arrivals outside [t_min, t_max).  The grid is (key tiles) x (photon
// slices).  A CTA scans its photon slice, keeps the keys of its tile, and
// every warp adds into its own private shared-memory histogram (16-bit
// counters, twice the keys per tile, when no warp can count past 65,535 in
// one slice; 32-bit otherwise): lanes that
// share a key are merged with __match_any_sync and only the lowest such lane
// writes, so no two threads ever update the same word concurrently.  The
// CTA then sums its warps' histograms and stores the tile with plain stores
// into the slice's partial histogram; a second kernel sums the slices.
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

constexpr int kBinWarps = 8;
constexpr int kBinWarpBytes = 16384;   // each warp's private histogram: 16 KiB of shared memory

// Keys per CTA tile with counters of type Count: 4096 (32-bit) or 8192
// (16-bit, used only when no warp can count more than 65,535 photons).
template <typename Count>
__host__ __device__ constexpr int bin_tile() { return kBinWarpBytes/(int)sizeof(Count); }

__device__ __forceinline__ int32_t arrival_key(int32_t s, const double* time, uint64_t i,
                                               uint32_t B, double t_min, double t_max) {
    if (s < 0) return -1;
    if (B == 0) return s;
    const double f = (time[i] - t_min) / (t_max - t_min) * (double)B;
    const uint32_t tb = (f >= 0.0 && f < (double)B) ? (uint32_t)f : B;
    return s*(int32_t)(B + 1) + (int32_t)tb;
}

template <typename Count>
__global__ void __launch_bounds__(kBinWarps*32)
bin_tiles_kernel(const int32_t* __restrict__ sensor, const double* __restrict__ time,
                 uint64_t n, uint32_t B, double t_min, double t_max, int32_t num_keys,
                 uint32_t* __restrict__ partial, uint64_t slice_len) {
    constexpr int kBinTile = bin_tile<Count>();
    extern __shared__ uint32_t hist_words[];   // [kBinWarps][kBinTile] counters
    Count* hist = reinterpret_cast<Count*>(hist_words);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t tile0 = blockIdx.x*kBinTile;
    const int32_t tile_len = min(kBinTile, num_keys - tile0);
    for (int k = threadIdx.x; k < kBinWarps*kBinWarpBytes/4; k += blockDim.x) hist_words[k] = 0;
    __syncthreads();
    Count* mine = hist + warp*kBinTile;
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
            if (lane == __ffs(same) - 1) mine[key - tile0] += (Count)__popc(same);
        }
        __syncwarp();
    }
    __syncthreads();
    uint32_t* out = partial + (uint64_t)blockIdx.y*num_keys + tile0;
    for (int k = threadIdx.x; k < tile_len; k += blockDim.x) {
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kBinWarps; w++) sum += (uint32_t)hist[w*kBinTile + k];
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
    // whole waves: one CTA of this kernel fits an SM (its shared memory),
    // so tiles x slices is kept at or just under twice the SM count -- a
    // few CTAs over a wave would run alone as a third wave
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms < 1) sms = 1;
    auto plan = [&](int tile, uint32_t* slices_out) -> bool {
        const int32_t tiles = (num_keys + tile - 1)/tile;
        uint32_t slices = (uint32_t)((2*sms)/tiles);
        if (slices < 1) slices = 1;
        if (slices > 64) slices = 64;
        while (slices > 1 && (uint64_t)slices*num_keys > scratch_words) slices--;
        if ((uint64_t)slices*num_keys > scratch_words) return false;
        *slices_out = n == 0 ? 1u : slices;
        return true;
    };
    uint32_t slices = 1;
    // 16-bit counters when no warp's share of a slice can reach 65,536
    // photons (a warp takes every eighth group of 32 photons of its slice)
    bool narrow = plan(bin_tile<uint16_t>(), &slices);
    const uint64_t per_warp = n == 0 ? 0 : ((n + slices - 1)/slices + kBinWarps*32 - 1)/(kBinWarps*32)*32;
    if (narrow && per_warp > 65535) narrow = false;
    if (!narrow && !plan(bin_tile<uint32_t>(), &slices)) return cudaErrorInvalidValue;
    const int32_t tile = narrow ? bin_tile<uint16_t>() : bin_tile<uint32_t>();
    const int32_t tiles = (num_keys + tile - 1)/tile;
    const uint64_t slice_len = n == 0 ? 1 : (n + slices - 1)/slices;
    const size_t smem = (size_t)kBinWarps*kBinWarpBytes;
    cudaError_t e;
    if (narrow) {
        e = cudaFuncSetAttribute(bin_tiles_kernel<uint16_t>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        bin_tiles_kernel<uint16_t><<<dim3(tiles, slices), kBinWarps*32, smem, s>>>(
            sensor, time, n, B, t_min, t_max, num_keys, scratch, slice_len);
    } else {
        e = cudaFuncSetAttribute(bin_tiles_kernel<uint32_t>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        bin_tiles_kernel<uint32_t><<<dim3(tiles, slices), kBinWarps*32, smem, s>>>(
            sensor, time, n, B, t_min, t_max, num_keys, scratch, slice_len);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    bin_reduce_kernel<<<(num_sensors + 255)/256, 256, 0, s>>>(
        scratch, slices, num_sensors, B, num_keys, counts, time_hist);
    return cudaGetLastError();
}

}  // namespace mlgpu
