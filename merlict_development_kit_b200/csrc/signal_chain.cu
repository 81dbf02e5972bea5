// signal_chain.cu -- the signal chain after binning for one event, on the
// device: photon pipelines (merlict_signal_processing/PipelinePhoton.cpp:
// 25-65), night-sky background (merlict_portal_plenoscope/
// night_sky_background/Injector.cpp:8-98), photo-electric conversion
// (merlict_signal_processing/PhotoElectricConverter.cpp:31-90) and
// single-pulse extraction (merlict_signal_processing/pulse_extraction.cpp:
// 9-35).
//
// Layout of the work:
//   1. photons sorted by (sensor, arrival time, input index): two stable
//      radix sorts (CUB), time keys first; each sensor's pipeline is then a
//      contiguous run, found by binary search;
//   2. the exposure window: min/max of the Cherenkov arrival times, their
//      histogram on 2 + sqrt(n) linearly spaced edges (block-private bins in
//      shared memory), the first fullest bin -> the window's start;
//   3. one thread per lixel walks its pipeline merged with its background
//      photons (drawn on the fly: the Poisson stream first, to know their
//      number, then their wavelengths), converts every photon to pulses and
//      extracts each pulse into a time slice -- twice: a counting pass, a
//      scan of the counts, and a writing pass with the same draws.
//
// Draws: stage s (1 background, 2 conversion, 3 extraction) of lixel i
// draws uniforms k = 0, 1, ... of the Philox stream ((0xF0 | s) << 56) |
// (offset + i) in the order merlict's code asks for them; a normal deviate
// is mean + std sqrt(-2 ln(1 - u1)) cos(2 pi u2) of two uniforms.
// Compiled with --fmad=false: the arithmetic is merlict's, in merlict's
// order, so only log and cos (CUDA's, not the C library's) can differ in
// the last bit.
#include <cmath>
#include <cstdint>
#include <cub/cub.cuh>

#include "merlict_b200_philox.h"
#include "mlgpu_internal.h"
#include "fp64_geometry.cuh"

namespace mlgpu {
namespace {

constexpr int32_t kNightSkyBackground = -100;      // simulation_truth.h:15-17
constexpr int32_t kAccidental = -201;
constexpr int32_t kCrosstalk = -202;
constexpr double kNumberTimeSlices = 100.0;         // pulse_extraction.h:13
constexpr uint32_t kMaxDraws = 0xFFFFFF00u;         // counter space of one stream
constexpr int kSmemBins = 12288;                    // block-private histogram limit

__device__ __forceinline__ uint64_t time_key(double t) {
    const uint64_t b = (uint64_t)__double_as_longlong(t);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

__device__ __forceinline__ double key_time(uint64_t k) {
    const uint64_t b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ uint64_t stage_stream(uint64_t stage, uint64_t offset, uint64_t lixel) {
    return ((0xF0ull | stage) << 56) | ((offset + lixel) & ((1ull << 56) - 1));
}

// Generator::expovariate (merlict/random/Generator.cpp:36-39)
__device__ __forceinline__ double expovariate(double u, double rate) {
    return -log(u)/rate;
}

__device__ __forceinline__ void raise_error(unsigned int* err, int code) {
    atomicCAS(err, 0u, (unsigned)code);
}

// ---- 1. pipelines ------------------------------------------------------------

__global__ void __launch_bounds__(256)
sc_time_keys_kernel(const double* __restrict__ time, uint64_t n, uint64_t* __restrict__ key,
                    uint32_t* __restrict__ idx) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        key[i] = time_key(__ldg(time + i));
        idx[i] = (uint32_t)i;
    }
}

__global__ void __launch_bounds__(256)
sc_sensor_keys_kernel(const int32_t* __restrict__ sensor, const uint32_t* __restrict__ idx,
                      uint64_t n, uint32_t num_sensors, uint32_t* __restrict__ key,
                      unsigned int* __restrict__ err) {
    for (uint64_t j = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x*blockDim.x) {
        const int32_t s = __ldg(sensor + __ldg(idx + j));
        if (s >= (int32_t)num_sensors) raise_error(err, MLGPU_ERR_INVALID_ARGUMENT);
        key[j] = (s >= 0 && s < (int32_t)num_sensors) ? (uint32_t)s : 0xffffffffu;
    }
}

__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* a, uint64_t n, uint32_t v) {
    uint64_t lo = 0, hi = n;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// pipeline offsets and the earliest / latest Cherenkov arrival
// (Injector.cpp:21-41: min over the pipelines' fronts from DBL_MAX, max over
// their backs from DBL_MIN)
__global__ void __launch_bounds__(128)
sc_pipelines_kernel(const uint32_t* __restrict__ skey, const uint32_t* __restrict__ idx,
                    const double* __restrict__ time, uint64_t n, uint32_t num_sensors,
                    uint64_t* __restrict__ pipe_off, unsigned long long* __restrict__ minmax) {
    const uint32_t s = blockIdx.x*blockDim.x + threadIdx.x;
    if (s > num_sensors) return;
    const uint64_t b = lower_bound_u32(skey, n, s);
    pipe_off[s] = b;
    if (s == num_sensors) return;
    const uint64_t e = lower_bound_u32(skey, n, s + 1);
    if (e > b) {
        atomicMin(minmax + 0, (unsigned long long)time_key(__ldg(time + __ldg(idx + b))));
        atomicMax(minmax + 1, (unsigned long long)time_key(__ldg(time + __ldg(idx + e - 1))));
    }
}

// ---- 2. the exposure window, Injector.cpp:43-59 -----------------------------------

struct Edges {
    double lo, step;
    uint32_t count;             // bin edges; count - 1 bins
    __device__ double at(uint32_t i) const { return lo + step*(double)i; }   // numeric::linspace
};

__device__ __forceinline__ Edges make_edges(const unsigned long long* minmax, uint64_t n) {
    Edges e;
    const double lo = key_time(minmax[0]), hi = key_time(minmax[1]);
    e.count = (uint32_t)(2.0 + sqrt((double)n));
    e.lo = lo;
    e.step = (hi - lo)/(double)(e.count - 1);
    return e;
}

// Histogram1::fill_in (Histogram1.cpp:29-44): std::upper_bound over the edges
__device__ __forceinline__ int64_t bin_of(const Edges& e, double t) {
    uint32_t first = 0, len = e.count;
    while (len > 0) {
        const uint32_t half = len >> 1, mid = first + half;
        if (t < e.at(mid)) { len = half; }
        else { first = mid + 1; len -= half + 1; }
    }
    if (first == 0 || first == e.count) return -1;     // under- or overflow
    return (int64_t)first - 1;
}

__global__ void __launch_bounds__(256)
sc_histogram_kernel(const uint32_t* __restrict__ idx, const double* __restrict__ time,
                    const uint64_t* __restrict__ pipe_off, uint32_t num_sensors,
                    const unsigned long long* __restrict__ minmax, uint32_t* __restrict__ bins,
                    int use_smem) {
    extern __shared__ uint32_t sbins[];
    const uint64_t n = pipe_off[num_sensors];
    if (n == 0) return;
    const Edges e = make_edges(minmax, n);
    const uint32_t nb = e.count - 1;
    if (use_smem) {
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) sbins[i] = 0;
        __syncthreads();
    }
    for (uint64_t j = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x*blockDim.x) {
        const int64_t b = bin_of(e, __ldg(time + __ldg(idx + j)));
        if (b >= 0) atomicAdd(use_smem ? sbins + b : bins + b, 1u);
    }
    if (use_smem) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x)
            if (sbins[i]) atomicAdd(bins + i, sbins[i]);
    }
}

// Histogram1::mode / arg_max (Histogram1.cpp:46-60): the first fullest bin
__global__ void __launch_bounds__(1024)
sc_window_kernel(const uint64_t* __restrict__ pipe_off, uint32_t num_sensors,
                 const unsigned long long* __restrict__ minmax, const uint32_t* __restrict__ bins,
                 double exposure_time, double* __restrict__ start) {
    __shared__ uint64_t best[32];
    const uint64_t n = pipe_off[num_sensors];
    double mode = 0.0;
    if (n > 0) {
        const Edges e = make_edges(minmax, n);
        const uint32_t nb = e.count - 1;
        // (count << 32) | (~index): the max is the fullest, then the first
        uint64_t v = 0;
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) {
            const uint64_t c = ((uint64_t)bins[i] << 32) | (uint64_t)(0xffffffffu - i);
            if (bins[i] > 0 && c > v) v = c;
        }
        for (int o = 16; o > 0; o >>= 1) {
            const uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if ((threadIdx.x & 31) == 0) best[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x < 32) {
            v = threadIdx.x < (blockDim.x >> 5) ? best[threadIdx.x] : 0;
            for (int o = 16; o > 0; o >>= 1) {
                const uint64_t w = __shfl_xor_sync(0xffffffffu, v, o);
                v = w > v ? w : v;
            }
        }
        const uint32_t arg = v ? 0xffffffffu - (uint32_t)v : 0u;
        mode = 0.5*(e.at(arg + 1) + e.at(arg));
    }
    if (threadIdx.x == 0) *start = mode - 0.5*exposure_time;
}

// ---- 3. one lixel ---------------------------------------------------------------

template <bool kWrite>
struct Extractor {
    const SignalChainParams& P;
    uint64_t seed, stream;
    uint32_t k = 0;
    uint32_t n = 0;
    uint8_t* slice;
    int32_t* truth;
    __device__ Extractor(const SignalChainParams& p, uint64_t sd, uint64_t s, uint8_t* sl,
                         int32_t* tr)
        : P(p), seed(sd), stream(s), slice(sl), truth(tr) {}
    // extract_pulses, pulse_extraction.cpp:17-30
    __device__ __forceinline__ void pulse(double t, int32_t id) {
        const double u1 = mlgpu_philox_uniform(seed, stream, k);
        const double u2 = mlgpu_philox_uniform(seed, stream, k + 1);
        k += 2;
        const double z = 0.0 + P.arrival_time_std*(sqrt(-2.0*log(1.0 - u1))*cos(2.0*M_PI*u2));
        const double r = round((t + z)/P.time_slice_duration);
        if (r >= 0.0 && r < kNumberTimeSlices) {
            if (kWrite) {
                slice[n] = (uint8_t)(int32_t)r;
                truth[n] = id;
            }
            n++;
        }
    }
};

template <bool kWrite>
__global__ void __launch_bounds__(128)
sc_lixel_kernel(SignalChainParams P, uint64_t seed, uint64_t offset,
                const uint64_t* __restrict__ pipe_off,
                const uint32_t* __restrict__ idx, const double* __restrict__ time,
                const double* __restrict__ wavelength, const int32_t* __restrict__ truth,
                const float* __restrict__ efficiency, uint32_t num_sensors,
                const double* __restrict__ start, uint64_t* __restrict__ count,
                int32_t* __restrict__ nsb_count, const uint64_t* __restrict__ out_off,
                uint8_t* __restrict__ out_slice, int32_t* __restrict__ out_truth,
                unsigned int* __restrict__ err) {
    const uint32_t l = blockIdx.x*blockDim.x + threadIdx.x;
    if (l >= num_sensors) return;
    const double S = *start;
    const double T = P.exposure_time;
    const uint64_t s_nsb = stage_stream(1, offset, l);
    const uint64_t s_pec = stage_stream(2, offset, l);
    int e = 0;
    // background photons: the Poisson stream first (Injector.cpp:62-72)
    const double rate = P.nsb_rate*(double)__ldg(efficiency + l)/P.num_lixel;
    const double e0 = expovariate(mlgpu_philox_uniform(seed, s_nsb, 0), rate);
    uint32_t nsb = 0;
    {
        double sum = e0;
        uint32_t kk = 1;
        while (sum < T) {
            if (kk >= kMaxDraws) { e = MLGPU_ERR_RUNTIME; break; }
            sum = sum + expovariate(mlgpu_philox_uniform(seed, s_nsb, kk++), rate);
            nsb++;
        }
    }
    if (!kWrite && nsb_count) nsb_count[l] = (int32_t)nsb;
    Extractor<kWrite> x(P, seed, stage_stream(3, offset, l),
                        kWrite ? out_slice + out_off[l] : nullptr,
                        kWrite ? out_truth + out_off[l] : nullptr);
    uint32_t kp = 0;           // conversion draws
    // the pipeline merged with the background photons, in time order
    // (Injector.cpp:73-97, Cherenkov photons first on equal times), each
    // converted (PhotoElectricConverter.cpp:35-50) and its pulses extracted
    uint64_t c = pipe_off[l];
    const uint64_t c_end = pipe_off[l + 1];
    uint32_t m = 0;
    double s_m = e0;           // the background photon m is at S + s_m
    while (!e && (c < c_end || m < nsb)) {
        double t, w;
        int32_t id;
        const uint32_t ci = c < c_end ? __ldg(idx + c) : 0u;
        const double tc = c < c_end ? __ldg(time + ci) : 0.0;
        const double tn = S + s_m;
        if (c < c_end && (m >= nsb || !(tn < tc))) {
            t = tc;
            w = __ldg(wavelength + ci);
            id = __ldg(truth + ci);
            c++;
        } else {
            t = tn;
            const double u = mlgpu_philox_uniform(seed, s_nsb, nsb + 1 + m);
            w = fp64::func_eval_points(P.cdf, P.num_cdf, u*P.total_integral, &e);   // SamplesFromDistribution::draw
            id = kNightSkyBackground;
            m++;
            if (m < nsb)
                s_m = s_m + expovariate(mlgpu_philox_uniform(seed, s_nsb, m), rate);
        }
        const double t_rel = t - S;
        const double q = fp64::func_eval_points(P.qe, P.num_qe, w, &e);
        if (e) break;
        if (kp >= kMaxDraws) { e = MLGPU_ERR_RUNTIME; break; }
        if (q >= mlgpu_philox_uniform(seed, s_pec, kp++)) {
            x.pulse(t_rel, id);
            // Converter::add_pulse: crosstalk while the draw allows it
            while (kp < kMaxDraws && P.second_puls >= mlgpu_philox_uniform(seed, s_pec, kp++))
                x.pulse(t_rel, kCrosstalk);
        }
    }
    // dark pulses (PhotoElectricConverter.cpp:70-88)
    if (!e) {
        double sum = expovariate(mlgpu_philox_uniform(seed, s_pec, kp++), P.dark_rate);
        while (sum < T) {
            if (kp >= kMaxDraws || x.k >= kMaxDraws) { e = MLGPU_ERR_RUNTIME; break; }
            const double next = expovariate(mlgpu_philox_uniform(seed, s_pec, kp++), P.dark_rate);
            x.pulse(sum, kAccidental);
            while (kp < kMaxDraws && P.second_puls >= mlgpu_philox_uniform(seed, s_pec, kp++))
                x.pulse(sum, kCrosstalk);
            sum = sum + next;
        }
    }
    if (e) raise_error(err, e);
    if (!kWrite) count[l] = e ? 0 : x.n;
}

struct ChainScratch {
    uint64_t *tkey_in, *tkey_out;
    uint32_t *idx_in, *idx_out, *skey_in, *skey_out;
    uint64_t *pipe_off, *counts;
    uint32_t* bins;
    uint64_t nbins;
    unsigned long long* minmax;
    double* start;
    void* temp;
    size_t temp_bytes;
};

inline uint64_t align256(uint64_t b) { return (b + 255) & ~uint64_t(255); }

size_t cub_temp_bytes(uint64_t n, uint32_t ns) {
    size_t cub64 = 0, cub32 = 0, scan = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub64, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n);
    cub::DeviceRadixSort::SortPairs(nullptr, cub32, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)n);
    cub::DeviceScan::ExclusiveSum(nullptr, scan, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                  (int)ns + 1);
    size_t t = cub64 > cub32 ? cub64 : cub32;
    return t > scan ? t : scan;
}

// fixed part of the scratch: sort buffers, pipelines, counts, bins, scalars
uint64_t fixed_bytes(uint64_t n, uint32_t ns, uint64_t* nbins) {
    *nbins = (uint64_t)(2.0 + sqrt((double)n)) + 1;
    return 2*align256(n*8) + 4*align256(n*4) + 2*align256((uint64_t)(ns + 1)*8) +
           align256(*nbins*4) + 256;
}

ChainScratch layout(uint64_t n, uint32_t ns, void* scratch, size_t bytes) {
    ChainScratch c;
    char* p = static_cast<char*>(scratch);
    c.tkey_in = reinterpret_cast<uint64_t*>(p); p += align256(n*8);
    c.tkey_out = reinterpret_cast<uint64_t*>(p); p += align256(n*8);
    c.idx_in = reinterpret_cast<uint32_t*>(p); p += align256(n*4);
    c.idx_out = reinterpret_cast<uint32_t*>(p); p += align256(n*4);
    c.skey_in = reinterpret_cast<uint32_t*>(p); p += align256(n*4);
    c.skey_out = reinterpret_cast<uint32_t*>(p); p += align256(n*4);
    c.pipe_off = reinterpret_cast<uint64_t*>(p); p += align256((uint64_t)(ns + 1)*8);
    c.counts = reinterpret_cast<uint64_t*>(p); p += align256((uint64_t)(ns + 1)*8);
    c.nbins = (uint64_t)(2.0 + sqrt((double)n)) + 1;
    c.bins = reinterpret_cast<uint32_t*>(p); p += align256(c.nbins*4);
    c.minmax = reinterpret_cast<unsigned long long*>(p);
    c.start = reinterpret_cast<double*>(p + 16);
    p += 256;
    c.temp = p;
    c.temp_bytes = bytes - (size_t)(p - static_cast<char*>(scratch));
    return c;
}

}  // namespace

size_t signal_chain_scratch_bytes(uint64_t n, uint32_t num_sensors) {
    uint64_t nbins = 0;
    return fixed_bytes(n, num_sensors, &nbins) + cub_temp_bytes(n, num_sensors) + 256;
}

// Steps 1-2 and the counting pass of step 3: the pulses per lixel, scanned
// into a.channel_offset (num_sensors + 1 entries, the last the total), and
// the window start at *start_dev (in the scratch).  The caller reads the
// total, checks its capacity and then calls launch_signal_chain_write.
cudaError_t launch_signal_chain_count(const SignalChainArgs& a, void* scratch, size_t scratch_bytes,
                                      int grid, cudaStream_t s, const double** start_dev) {
    const uint64_t n = a.num_photons;
    const uint32_t ns = a.num_sensors;
    if (n >= (1ull << 31)) return cudaErrorInvalidValue;
    const ChainScratch c = layout(n, ns, scratch, scratch_bytes);
    *start_dev = c.start;
    size_t temp_bytes = c.temp_bytes;
    // 1. sort by (sensor, time, index): time first, then a stable sort by sensor
    if (n > 0) {
        sc_time_keys_kernel<<<grid, 256, 0, s>>>(a.time, n, c.tkey_in, c.idx_in);
        cudaError_t e = cub::DeviceRadixSort::SortPairs(c.temp, temp_bytes, c.tkey_in, c.tkey_out,
                                                        c.idx_in, c.idx_out, (int)n, 0, 64, s);
        if (e != cudaSuccess) return e;
        sc_sensor_keys_kernel<<<grid, 256, 0, s>>>(a.sensor, c.idx_out, n, ns, c.skey_in, a.err);
        e = cub::DeviceRadixSort::SortPairs(c.temp, temp_bytes, c.skey_in, c.skey_out, c.idx_out,
                                            c.idx_in, (int)n, 0, 32, s);
        if (e != cudaSuccess) return e;
    }
    // c.idx_in: the photons by (sensor, time); c.skey_out: their sensors.
    // minmax starts at the time keys of DBL_MAX and DBL_MIN.
    static const unsigned long long init[2] = {0xffefffffffffffffull, 0x8010000000000000ull};
    cudaError_t e = cudaMemcpyAsync(c.minmax, init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    sc_pipelines_kernel<<<(ns + 1 + 127)/128, 128, 0, s>>>(c.skey_out, c.idx_in, a.time, n, ns,
                                                          c.pipe_off, c.minmax);
    // 2. the exposure window
    e = cudaMemsetAsync(c.bins, 0, c.nbins*4, s);
    if (e != cudaSuccess) return e;
    const int use_smem = c.nbins <= (uint64_t)kSmemBins;
    sc_histogram_kernel<<<grid, 256, use_smem ? c.nbins*4 : 0, s>>>(
        c.idx_in, a.time, c.pipe_off, ns, c.minmax, c.bins, use_smem);
    sc_window_kernel<<<1, 1024, 0, s>>>(c.pipe_off, ns, c.minmax, c.bins, a.params.exposure_time,
                                        c.start);
    // 3. the counting pass and the scan of the counts
    e = cudaMemsetAsync(c.counts, 0, (uint64_t)(ns + 1)*8, s);
    if (e != cudaSuccess) return e;
    if (ns > 0)
        sc_lixel_kernel<false><<<(ns + 127)/128, 128, 0, s>>>(
            a.params, a.seed, a.offset, c.pipe_off, c.idx_in, a.time, a.wavelength, a.truth,
            a.efficiency, ns, c.start, c.counts, a.nsb_count, nullptr, nullptr, nullptr, a.err);
    temp_bytes = c.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(c.temp, temp_bytes, c.counts, a.channel_offset, (int)ns + 1,
                                      s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// The writing pass: the same draws, each kept pulse at its channel's offset.
cudaError_t launch_signal_chain_write(const SignalChainArgs& a, void* scratch, size_t scratch_bytes,
                                      cudaStream_t s) {
    const ChainScratch c = layout(a.num_photons, a.num_sensors, scratch, scratch_bytes);
    if (a.num_sensors > 0)
        sc_lixel_kernel<true><<<(a.num_sensors + 127)/128, 128, 0, s>>>(
            a.params, a.seed, a.offset, c.pipe_off, c.idx_in, a.time, a.wavelength, a.truth,
            a.efficiency, a.num_sensors, c.start, nullptr, nullptr, a.channel_offset, a.slice,
            a.slice_truth, a.err);
    return cudaGetLastError();
}

}  // namespace mlgpu
