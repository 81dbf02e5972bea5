// device_sort.cu -- the sorts and scans of the calibration and signal-chain
// rows: a stable LSD radix sort of (32-bit key, 32-bit value) pairs, a
// counting sort by a small key, a sort of the long runs of a segmented
// array by (64-bit key, value) (one block per run), and exclusive sums
// into 64-bit offsets.
//
// Radix sort, 8-bit digits, one pass per digit (as many as the key bits
// need), each pass three launches over tiles of kSortTile elements:
//   count    per tile, how many of its keys have each digit, stored
//            digit-major (digit * tiles + tile) so that
//   scan     one exclusive sum over all of them gives, for every (digit,
//            tile), where the tile's keys with that digit start;
//   scatter  each tile again, in rounds of one element per thread: a key's
//            place is its (digit, tile) start + the keys of its digit in
//            the earlier rounds + those in lower warps of this round + its
//            rank among the lanes of its warp with that digit
//            (__match_any_sync) -- the order of equal digits is the input
//            order, so the sort is stable.
// The long-run sort applies the same stable rounds inside one block, over
// the run's keys in global memory (ping-pong between the two halves the
// caller provides).
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads/32;
constexpr int kSortItems = 8;
constexpr uint32_t kSortTile = kSortThreads*kSortItems;   // 2048 keys per tile
constexpr int kDigits = 256;
constexpr int kScanThreads = 1024;
constexpr uint32_t kScanTile = kScanThreads*4;              // 4096 values per block

template <typename Key>
__device__ __forceinline__ uint32_t digit_of(Key k, int shift) {
    return (uint32_t)(k >> shift) & (kDigits - 1);
}

__global__ void __launch_bounds__(kSortThreads)
sort_count_kernel(const uint32_t* __restrict__ key, uint64_t n, int shift, uint32_t tiles,
                  uint32_t* __restrict__ counts) {
    __shared__ uint32_t hist[kDigits];
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < kDigits; d += blockDim.x) hist[d] = 0;
        __syncthreads();
        const uint64_t b = (uint64_t)tile*kSortTile;
        const uint64_t e = b + kSortTile < n ? b + kSortTile : n;
        for (uint64_t i = b + threadIdx.x; i < e; i += blockDim.x)
            atomicAdd(&hist[digit_of(__ldg(key + i), shift)], 1u);
        __syncthreads();
        for (int d = threadIdx.x; d < kDigits; d += blockDim.x)
            counts[(uint64_t)d*tiles + tile] = hist[d];
        __syncthreads();
    }
}

// The stable placement of one round of up to blockDim.x keys (one per
// thread, in thread order): returns this thread's place among the round's
// keys of its digit, and leaves each warp's count of every digit in
// `warp_count` ([kSortWarps][kDigits] of shared memory).
__device__ __forceinline__ uint32_t stable_rank(bool valid, uint32_t digit,
                                                uint32_t (*warp_count)[kDigits]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = threadIdx.x; k < kSortWarps*kDigits; k += blockDim.x)
        (&warp_count[0][0])[k] = 0;
    __syncthreads();
    const unsigned live = __ballot_sync(0xffffffffu, valid);
    uint32_t rank = 0;
    if (valid) {
        const unsigned peers = __match_any_sync(live, digit);
        rank = (uint32_t)__popc(peers & ((1u << lane) - 1u));
        if (lane == __ffs(peers) - 1) warp_count[warp][digit] = (uint32_t)__popc(peers);
    }
    __syncthreads();
    if (valid)
        for (int w = 0; w < warp; w++) rank += warp_count[w][digit];
    return rank;
}

__global__ void __launch_bounds__(kSortThreads)
sort_scatter_kernel(const uint32_t* __restrict__ key_in, const uint32_t* __restrict__ val_in,
                    uint64_t n, int shift, uint32_t tiles, const uint64_t* __restrict__ start,
                    uint32_t* __restrict__ key_out, uint32_t* __restrict__ val_out) {
    __shared__ uint32_t warp_count[kSortWarps][kDigits];
    __shared__ uint64_t base[kDigits];
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < kDigits; d += blockDim.x)
            base[d] = start[(uint64_t)d*tiles + tile];
        __syncthreads();
        const uint64_t b = (uint64_t)tile*kSortTile;
        for (int r = 0; r < kSortItems; r++) {
            const uint64_t i = b + (uint64_t)r*blockDim.x + threadIdx.x;
            const bool valid = i < n;
            uint32_t k = 0, v = 0, d = 0;
            if (valid) {
                k = __ldg(key_in + i);
                v = __ldg(val_in + i);
                d = digit_of(k, shift);
            }
            const uint32_t rank = stable_rank(valid, d, warp_count);
            if (valid) {
                const uint64_t o = base[d] + rank;
                key_out[o] = k;
                val_out[o] = v;
            }
            __syncthreads();
            // the round's keys of each digit move that digit's base on
            for (int dd = threadIdx.x; dd < kDigits; dd += blockDim.x) {
                uint32_t c = 0;
                for (int w = 0; w < kSortWarps; w++) c += warp_count[w][dd];
                base[dd] += c;
            }
            __syncthreads();
        }
    }
}

// ---- exclusive sums into 64-bit offsets ------------------------------------

template <typename In>
__device__ __forceinline__ uint64_t block_exclusive(const In* in, uint64_t n, uint64_t b,
                                                   uint64_t v[4], uint64_t* total) {
    __shared__ uint64_t warp_sum[kScanThreads/32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t local = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t i = b + 4*(uint64_t)threadIdx.x + j;
        v[j] = i < n ? (uint64_t)in[i] : 0ull;
        local += v[j];
    }
    uint64_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint64_t s = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;
    }
    __syncthreads();
    const uint64_t before = (warp > 0 ? warp_sum[warp - 1] : 0ull) + x - local;
    *total = warp_sum[kScanThreads/32 - 1];
    __syncthreads();
    return before;
}

// Per block of kScanTile values: their exclusive sums within the block,
// and the block's total into sums[block].  `in` and `out` may be the same
// array (every value is read before the block's barrier, written after).
template <typename In>
__global__ void __launch_bounds__(kScanThreads)
scan_tiles_kernel(const In* in, uint64_t n, uint64_t* out, uint64_t* __restrict__ sums) {
    const uint64_t b = (uint64_t)blockIdx.x*kScanTile;
    uint64_t v[4], total;
    uint64_t run = block_exclusive(in, n, b, v, &total);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const uint64_t i = b + 4*(uint64_t)threadIdx.x + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads)
scan_add_kernel(uint64_t* __restrict__ out, uint64_t n, const uint64_t* __restrict__ sums) {
    const uint64_t add = sums[blockIdx.x];
    const uint64_t b = (uint64_t)blockIdx.x*kScanTile;
    for (uint64_t i = b + threadIdx.x; i < b + kScanTile && i < n; i += blockDim.x) out[i] += add;
}

uint64_t scan_levels_words(uint64_t n) {
    uint64_t words = 0;
    while (n > 1) {
        n = (n + kScanTile - 1)/kScanTile;
        words += n + 1;
    }
    return words;
}

template <typename In>
cudaError_t exclusive_sum(const In* in, uint64_t* out, uint64_t n, uint64_t* temp,
                          cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint64_t blocks = (n + kScanTile - 1)/kScanTile;
    scan_tiles_kernel<In><<<(unsigned)blocks, kScanThreads, 0, s>>>(in, n, out, temp);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || blocks == 1) return e;
    // the block totals, summed the same way, then added back
    e = exclusive_sum<uint64_t>(temp, temp, blocks, temp + blocks + 1, s);
    if (e != cudaSuccess) return e;
    scan_add_kernel<<<(unsigned)blocks, kScanThreads, 0, s>>>(out, n, temp);
    return cudaGetLastError();
}

// ---- the long runs of a segmented array, one block per run -------------------

// Run t of the list: [begin[t], end[t]) of the keys (64-bit) and values;
// empty runs (begin == end) are skipped.  Each run is sorted by (key,
// value): four stable passes on the value's bytes, then eight on the
// key's.  The sorted run is written to key_out/val_out; key_in/val_in serve
// as the other ping-pong half and are overwritten.
__global__ void __launch_bounds__(kSortThreads)
segment_sort_kernel(uint64_t* __restrict__ key_in, uint32_t* __restrict__ val_in,
                    uint64_t* __restrict__ key_out, uint32_t* __restrict__ val_out,
                    const uint64_t* __restrict__ begin, const uint64_t* __restrict__ end,
                    uint32_t runs) {
    __shared__ uint32_t warp_count[kSortWarps][kDigits];
    __shared__ uint32_t hist[kDigits];
    __shared__ uint64_t base[kDigits];
    for (uint32_t t = blockIdx.x; t < runs; t += gridDim.x) {
        const uint64_t b = begin[t], m = end[t] - b;
        if (m == 0) continue;
        uint64_t* ki = key_in + b; uint32_t* vi = val_in + b;
        uint64_t* ko = key_out + b; uint32_t* vo = val_out + b;
        for (int pass = 0; pass < 12; pass++) {
            // passes 0-3: the value's bytes; 4-11: the key's
            const bool on_val = pass < 4;
            const int shift = on_val ? 8*pass : 8*(pass - 4);
            auto digit = [&](uint64_t i) {
                return on_val ? digit_of(vi[i], shift) : digit_of(ki[i], shift);
            };
            for (int d = threadIdx.x; d < kDigits; d += blockDim.x) hist[d] = 0;
            __syncthreads();
            for (uint64_t i = threadIdx.x; i < m; i += blockDim.x)
                atomicAdd(&hist[digit(i)], 1u);
            __syncthreads();
            if (threadIdx.x == 0) {
                uint64_t run = 0;
                for (int d = 0; d < kDigits; d++) { base[d] = run; run += hist[d]; }
            }
            __syncthreads();
            for (uint64_t r0 = 0; r0 < m; r0 += blockDim.x) {
                const uint64_t i = r0 + threadIdx.x;
                const bool valid = i < m;
                uint64_t k = 0;
                uint32_t v = 0, d = 0;
                if (valid) { k = ki[i]; v = vi[i]; d = digit(i); }
                const uint32_t rank = stable_rank(valid, d, warp_count);
                if (valid) {
                    ko[base[d] + rank] = k;
                    vo[base[d] + rank] = v;
                }
                __syncthreads();
                for (int dd = threadIdx.x; dd < kDigits; dd += blockDim.x) {
                    uint32_t c = 0;
                    for (int w = 0; w < kSortWarps; w++) c += warp_count[w][dd];
                    base[dd] += c;
                }
                __syncthreads();
            }
            uint64_t* kt = ki; ki = ko; ko = kt;
            uint32_t* vt = vi; vi = vo; vo = vt;
        }
        // twelve passes: the result is back in the input half; to the output
        for (uint64_t i = threadIdx.x; i < m; i += blockDim.x) {
            key_out[b + i] = key_in[b + i];
            val_out[b + i] = val_in[b + i];
        }
        __syncthreads();
    }
}

// ---- counting sort by a small key --------------------------------------------

// Photons with equal keys within a warp are merged (__match_any_sync): one
// atomic per key and warp.
__global__ void __launch_bounds__(256)
count_keys_kernel(const uint32_t* __restrict__ key, uint64_t n, uint32_t* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    for (uint64_t b = (uint64_t)blockIdx.x*blockDim.x + (threadIdx.x & ~31u); b < n;
         b += (uint64_t)gridDim.x*blockDim.x) {
        const uint64_t i = b + lane;
        const bool valid = i < n;
        const uint32_t k = valid ? __ldg(key + i) : 0u;
        const unsigned live = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned peers = __match_any_sync(live, k);
            if (lane == __ffs(peers) - 1) atomicAdd(count + k, (unsigned)__popc(peers));
        }
    }
}

__global__ void __launch_bounds__(256)
cursor_kernel(const uint64_t* __restrict__ offset, uint32_t keys, uint32_t* __restrict__ cursor) {
    for (uint32_t k = blockIdx.x*blockDim.x + threadIdx.x; k < keys; k += gridDim.x*blockDim.x)
        cursor[k] = (uint32_t)offset[k];
}

__global__ void __launch_bounds__(256)
place_keys_kernel(const uint32_t* __restrict__ key, uint64_t n, uint32_t* __restrict__ cursor,
                  uint32_t* __restrict__ index_out) {
    const int lane = threadIdx.x & 31;
    for (uint64_t b = (uint64_t)blockIdx.x*blockDim.x + (threadIdx.x & ~31u); b < n;
         b += (uint64_t)gridDim.x*blockDim.x) {
        const uint64_t i = b + lane;
        const bool valid = i < n;
        const uint32_t k = valid ? __ldg(key + i) : 0u;
        const unsigned live = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const unsigned peers = __match_any_sync(live, k);
            const int leader = __ffs(peers) - 1;
            uint32_t first = 0;
            if (lane == leader) first = atomicAdd(cursor + k, (unsigned)__popc(peers));
            first = __shfl_sync(peers, first, leader);
            index_out[first + __popc(peers & ((1u << lane) - 1u))] = (uint32_t)i;
        }
    }
}

}  // namespace

size_t counting_sort_temp_bytes(uint64_t n, uint32_t keys) {
    // counts and cursors (32-bit, each rounded up to 64 entries), the scan's levels
    return 2*(((uint64_t)keys + 1 + 63) & ~uint64_t(63))*sizeof(uint32_t) +
           exclusive_sum_temp_bytes((uint64_t)keys + 1) + 256;
}

cudaError_t counting_sort(const uint32_t* key, uint64_t n, uint32_t keys, uint32_t* index_out,
                          uint64_t* offset, void* temp, cudaStream_t s) {
    if (n >= (1ull << 32)) return cudaErrorInvalidValue;
    uint32_t* count = static_cast<uint32_t*>(temp);                       // keys + 1
    uint32_t* cursor = count + (((uint64_t)keys + 1 + 63) & ~uint64_t(63));
    uint64_t* scan_tmp = reinterpret_cast<uint64_t*>(
        cursor + (((uint64_t)keys + 1 + 63) & ~uint64_t(63)));
    cudaError_t e = cudaMemsetAsync(count, 0, ((uint64_t)keys + 1)*sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (n + 255)/256;
    const unsigned grid = (unsigned)(want < (uint64_t)(8*sms) ? (want ? want : 1) : 8*sms);
    count_keys_kernel<<<grid, 256, 0, s>>>(key, n, count);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = exclusive_sum<uint32_t>(count, offset, (uint64_t)keys + 1, scan_tmp, s);
    if (e != cudaSuccess) return e;
    cursor_kernel<<<(keys + 255)/256, 256, 0, s>>>(offset, keys, cursor);
    place_keys_kernel<<<grid, 256, 0, s>>>(key, n, cursor, index_out);
    return cudaGetLastError();
}

size_t radix_sort_temp_bytes(uint64_t n) {
    const uint64_t tiles = (n + kSortTile - 1)/kSortTile;
    const uint64_t counts = tiles*kDigits;
    return (size_t)(2*counts + scan_levels_words(counts) + 8)*sizeof(uint64_t);
}

cudaError_t radix_sort_pairs(const uint32_t* key_in, const uint32_t* val_in, uint32_t* key_out,
                             uint32_t* val_out, uint32_t* key_tmp, uint32_t* val_tmp, uint64_t n,
                             int key_bits, void* temp, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t tiles = (uint32_t)((n + kSortTile - 1)/kSortTile);
    const uint64_t counts = (uint64_t)tiles*kDigits;
    uint32_t* cnt = static_cast<uint32_t*>(temp);
    uint64_t* start = static_cast<uint64_t*>(temp) + counts;   // after the 32-bit counts
    uint64_t* scan_tmp = start + counts;
    const int passes = key_bits <= 0 ? 1 : (key_bits + 7)/8;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned)(tiles < (uint32_t)(8*sms) ? tiles : (uint32_t)(8*sms));
    // pass p reads `src` and writes `dst`; the last pass writes the outputs
    const uint32_t* ksrc = key_in;
    const uint32_t* vsrc = val_in;
    for (int p = 0; p < passes; p++) {
        // the destinations alternate so that the last pass lands in *_out
        const bool to_out = ((passes - 1 - p) & 1) == 0;
        uint32_t* kdst = to_out ? key_out : key_tmp;
        uint32_t* vdst = to_out ? val_out : val_tmp;
        sort_count_kernel<<<grid, kSortThreads, 0, s>>>(ksrc, n, 8*p, tiles, cnt);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = exclusive_sum<uint32_t>(cnt, start, counts, scan_tmp, s);
        if (e != cudaSuccess) return e;
        sort_scatter_kernel<<<grid, kSortThreads, 0, s>>>(ksrc, vsrc, n, 8*p, tiles, start, kdst,
                                                         vdst);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        ksrc = kdst;
        vsrc = vdst;
    }
    return cudaSuccess;
}

size_t exclusive_sum_temp_bytes(uint64_t n) {
    return (size_t)(scan_levels_words(n) + 8)*sizeof(uint64_t);
}

cudaError_t exclusive_sum_u64(const uint64_t* in, uint64_t* out, uint64_t n, void* temp,
                              cudaStream_t s) {
    return exclusive_sum<uint64_t>(in, out, n, static_cast<uint64_t*>(temp), s);
}

cudaError_t exclusive_sum_u32(const uint32_t* in, uint64_t* out, uint64_t n, void* temp,
                              cudaStream_t s) {
    return exclusive_sum<uint32_t>(in, out, n, static_cast<uint64_t*>(temp), s);
}

cudaError_t sort_long_runs(uint64_t* key_in, uint32_t* val_in, uint64_t* key_out,
                           uint32_t* val_out, const uint64_t* begin, const uint64_t* end,
                           uint32_t runs, cudaStream_t s) {
    if (runs == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = runs < (uint32_t)(4*sms) ? runs : (uint32_t)(4*sms);
    segment_sort_kernel<<<grid, kSortThreads, 0, s>>>(key_in, val_in, key_out, val_out, begin,
                                                      end, runs);
    return cudaGetLastError();
}

}  // namespace mlgpu
