// signal_chain.cu -- the signal chain after binning for one event, on the
// device: photon pipelines (merlict_signal_processing/PipelinePhoton.cpp:
// 25-65), night-sky background (merlict_portal_plenoscope/
// night_sky_background/Injector.cpp:8-98), photo-electric conversion
// (merlict_signal_processing/PhotoElectricConverter.cpp:31-90) and
// single-pulse extraction (merlict_signal_processing/pulse_extraction.cpp:
// 9-35).
//
// Layout of the work:
//   1. pipelines: a counting sort by sensor (device_sort.cu; photons
//      without a sensor last; it also gives every pipeline's offset), then
//      every sensor's run by (arrival time, input index) -- ranks in shared
//      memory for runs of up to 4096 photons, a stable radix sort of each
//      longer run by one block (device_sort.cu) -- then the photons'
//      time, wavelength and truth id gathered into pipeline order,
//      contiguous per lixel;
//   2. the exposure window: min/max of the Cherenkov arrival times (one
//      atomic per warp), their histogram on 2 + sqrt(n) linearly spaced
//      edges (block-private bins in shared memory), the first fullest bin;
//   3. one thread per lixel walks its pipeline merged with its background
//      photons (the Poisson stream first, to know their number, then their
//      wavelengths) and converts every photon to electric pulses -- twice:
//      a counting pass, a scan of the counts (the host reads the total and
//      sizes the pulse buffer), a writing pass with the same draws;
//   4. extraction, one thread per pulse: pulse j of lixel i takes draws 2j
//      and 2j + 1 of its stream; the kept pulses are compacted (a scan of
//      the keep flags), which also gives each channel's offset.
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
sc_sensor_keys_kernel(const int32_t* __restrict__ sensor, uint64_t n, uint32_t num_sensors,
                      uint32_t* __restrict__ key, uint32_t* __restrict__ idx,
                      unsigned int* __restrict__ err) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        const int32_t s = __ldg(sensor + i);
        if (s >= (int32_t)num_sensors) raise_error(err, MLGPU_ERR_INVALID_ARGUMENT);
        key[i] = (s >= 0 && s < (int32_t)num_sensors) ? (uint32_t)s : num_sensors;
        idx[i] = (uint32_t)i;
    }
}

__global__ void __launch_bounds__(256)
sc_time_keys_kernel(const uint32_t* __restrict__ idx, const double* __restrict__ time,
                    const uint64_t* __restrict__ pipe_off, uint32_t num_sensors,
                    uint64_t* __restrict__ key) {
    const uint64_t n = pipe_off[num_sensors];
    for (uint64_t j = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x*blockDim.x)
        key[j] = time_key(__ldg(time + __ldg(idx + j)));
}

// Every sensor's run by (time key, input index), i.e. stable by time: runs
// of up to kWarpSegment photons by one warp in shared memory, up to
// kBlockSegment by one block (sc_segsort_block_kernel), longer ones by a
// radix sort of the run by (time key, index) by one block (sort_long_runs).
// Each element's place is its rank in the run, so the order the counting
// sort left within a sensor does not matter.
constexpr uint32_t kWarpSegment = 256;
constexpr uint32_t kBlockSegment = 4096;
constexpr int kSegWarps = 8;

__device__ __forceinline__ bool sorts_before(uint64_t ka, uint32_t va, uint64_t kb, uint32_t vb) {
    return ka < kb || (ka == kb && va < vb);
}

__global__ void __launch_bounds__(kSegWarps*32)
sc_segsort_warp_kernel(const uint64_t* __restrict__ key_in, const uint32_t* __restrict__ val_in,
                       const uint64_t* __restrict__ pipe_off, uint32_t num_sensors,
                       uint64_t* __restrict__ key_out, uint32_t* __restrict__ val_out,
                       uint32_t* __restrict__ medium, unsigned int* __restrict__ num_medium,
                       uint64_t* __restrict__ large_begin, uint64_t* __restrict__ large_end,
                       unsigned int* __restrict__ num_large) {
    __shared__ uint64_t sk[kSegWarps][kWarpSegment];
    __shared__ uint32_t sv[kSegWarps][kWarpSegment];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t l = blockIdx.x*kSegWarps + w;
    if (l >= num_sensors) return;
    const uint64_t b = pipe_off[l];
    const uint64_t m = pipe_off[l + 1] - b;
    if (m == 0) return;
    if (m > kWarpSegment) {
        if (lane == 0) {
            if (m <= kBlockSegment) {
                medium[atomicAdd(num_medium, 1u)] = l;
            } else {
                const unsigned int k = atomicAdd(num_large, 1u);
                large_begin[k] = b;
                large_end[k] = b + m;
            }
        }
        return;
    }
    const uint32_t mm = (uint32_t)m;
    for (uint32_t i = lane; i < mm; i += 32) {
        sk[w][i] = key_in[b + i];
        sv[w][i] = val_in[b + i];
    }
    __syncwarp();
    for (uint32_t i = lane; i < mm; i += 32) {
        const uint64_t ki = sk[w][i];
        const uint32_t vi = sv[w][i];
        uint32_t r = 0;
        for (uint32_t j = 0; j < mm; j++) r += sorts_before(sk[w][j], sv[w][j], ki, vi) ? 1u : 0u;
        key_out[b + r] = ki;
        val_out[b + r] = vi;
    }
}

__global__ void __launch_bounds__(512)
sc_segsort_block_kernel(const uint64_t* __restrict__ key_in, const uint32_t* __restrict__ val_in,
                        const uint64_t* __restrict__ pipe_off, const uint32_t* __restrict__ medium,
                        const unsigned int* __restrict__ num_medium, uint64_t* __restrict__ key_out,
                        uint32_t* __restrict__ val_out) {
    extern __shared__ uint64_t seg_smem[];
    uint64_t* sk = seg_smem;
    uint32_t* sv = reinterpret_cast<uint32_t*>(seg_smem + kBlockSegment);
    const unsigned int count = *num_medium;
    for (unsigned int t = blockIdx.x; t < count; t += gridDim.x) {
        const uint32_t l = medium[t];
        const uint64_t b = pipe_off[l];
        const uint32_t m = (uint32_t)(pipe_off[l + 1] - b);
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
            sk[i] = key_in[b + i];
            sv[i] = val_in[b + i];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
            const uint64_t ki = sk[i];
            const uint32_t vi = sv[i];
            uint32_t r = 0;
            for (uint32_t j = 0; j < m; j++) r += sorts_before(sk[j], sv[j], ki, vi) ? 1u : 0u;
            key_out[b + r] = ki;
            val_out[b + r] = vi;
        }
        __syncthreads();
    }
}

// the photons' fields in pipeline order
__global__ void __launch_bounds__(256)
sc_gather_kernel(const uint32_t* __restrict__ idx, const double* __restrict__ time,
                 const double* __restrict__ wavelength, const int32_t* __restrict__ truth,
                 const uint64_t* __restrict__ pipe_off, uint32_t num_sensors,
                 double* __restrict__ t_out, double* __restrict__ w_out,
                 int32_t* __restrict__ r_out) {
    const uint64_t n = pipe_off[num_sensors];
    for (uint64_t j = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; j < n;
         j += (uint64_t)gridDim.x*blockDim.x) {
        const uint32_t i = __ldg(idx + j);
        t_out[j] = __ldg(time + i);
        w_out[j] = __ldg(wavelength + i);
        r_out[j] = __ldg(truth + i);
    }
}

// The earliest and latest Cherenkov arrival (Injector.cpp:21-41: min over
// the pipelines' fronts from DBL_MAX, max over their backs from DBL_MIN);
// one atomic per warp.
__global__ void __launch_bounds__(128)
sc_minmax_kernel(const double* __restrict__ t, const uint64_t* __restrict__ pipe_off,
                 uint32_t num_sensors, unsigned long long* __restrict__ minmax) {
    const uint32_t s = blockIdx.x*blockDim.x + threadIdx.x;
    unsigned long long lo = 0xffffffffffffffffull, hi = 0ull;
    if (s < num_sensors) {
        const uint64_t b = pipe_off[s], e = pipe_off[s + 1];
        if (e > b) {
            lo = time_key(t[b]);
            hi = time_key(t[e - 1]);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long c = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = c > hi ? c : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        if (lo != 0xffffffffffffffffull) atomicMin(minmax + 0, lo);
        if (hi != 0ull) atomicMax(minmax + 1, hi);
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
sc_histogram_kernel(const double* __restrict__ t, const uint64_t* __restrict__ pipe_off,
                    uint32_t num_sensors, const unsigned long long* __restrict__ minmax,
                    uint32_t* __restrict__ bins, int use_smem) {
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
        const int64_t b = bin_of(e, t[j]);
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

// ---- 3. background and conversion, one lixel per thread ----------------------------

// The electric pulses of lixel l: counted (kWrite false) or written at
// e_off[l] (time relative to the window start, truth id, lixel).
template <bool kWrite>
__global__ void __launch_bounds__(128)
sc_lixel_kernel(SignalChainParams P, uint64_t seed, uint64_t offset,
                const uint64_t* __restrict__ pipe_off, const double* __restrict__ time,
                const double* __restrict__ wavelength, const int32_t* __restrict__ truth,
                const float* __restrict__ efficiency, uint32_t num_sensors,
                const double* __restrict__ start, uint64_t* __restrict__ count,
                int32_t* __restrict__ nsb_count, const uint64_t* __restrict__ e_off,
                double* __restrict__ e_time, int32_t* __restrict__ e_truth,
                uint32_t* __restrict__ e_lixel, unsigned int* __restrict__ err) {
    const uint32_t l = blockIdx.x*blockDim.x + threadIdx.x;
    if (l >= num_sensors) return;
    const double S = *start;
    const double T = P.exposure_time;
    const uint64_t s_nsb = stage_stream(1, offset, l);
    const uint64_t s_pec = stage_stream(2, offset, l);
    int e = 0;
    uint64_t out = kWrite ? e_off[l] : 0;
    uint32_t pulses = 0;
    auto pulse = [&](double t, int32_t id) {
        if (kWrite) {
            e_time[out] = t;
            e_truth[out] = id;
            e_lixel[out] = l;
            out++;
        }
        pulses++;
    };
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
    uint32_t kp = 0;           // conversion draws
    // the pipeline merged with the background photons, in time order
    // (Injector.cpp:73-97, Cherenkov photons first on equal times), each
    // converted (PhotoElectricConverter.cpp:35-50)
    uint64_t c = pipe_off[l];
    const uint64_t c_end = pipe_off[l + 1];
    uint32_t m = 0;
    double s_m = e0;           // the background photon m is at S + s_m
    while (!e && (c < c_end || m < nsb)) {
        double t, w;
        int32_t id;
        const double tc = c < c_end ? time[c] : 0.0;
        const double tn = S + s_m;
        if (c < c_end && (m >= nsb || !(tn < tc))) {
            t = tc;
            w = wavelength[c];
            id = truth[c];
            c++;
        } else {
            t = tn;
            const double u = mlgpu_philox_uniform(seed, s_nsb, nsb + 1 + m);
            // SamplesFromDistribution::draw
            w = fp64::func_eval_points(P.cdf, P.num_cdf, u*P.total_integral, &e);
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
            pulse(t_rel, id);
            // Converter::add_pulse: crosstalk while the draw allows it
            while (kp < kMaxDraws && P.second_puls >= mlgpu_philox_uniform(seed, s_pec, kp++))
                pulse(t_rel, kCrosstalk);
        }
    }
    // dark pulses (PhotoElectricConverter.cpp:70-88)
    if (!e) {
        double sum = expovariate(mlgpu_philox_uniform(seed, s_pec, kp++), P.dark_rate);
        while (sum < T) {
            if (kp >= kMaxDraws || pulses >= kMaxDraws/2) { e = MLGPU_ERR_RUNTIME; break; }
            const double next = expovariate(mlgpu_philox_uniform(seed, s_pec, kp++), P.dark_rate);
            pulse(sum, kAccidental);
            while (kp < kMaxDraws && P.second_puls >= mlgpu_philox_uniform(seed, s_pec, kp++))
                pulse(sum, kCrosstalk);
            sum = sum + next;
        }
    }
    if (e) raise_error(err, e);
    if (!kWrite) count[l] = e ? 0 : pulses;
}

// ---- 4. extraction, one pulse per thread (pulse_extraction.cpp:17-30) ---------------

__global__ void __launch_bounds__(256)
sc_extract_kernel(SignalChainParams P, uint64_t seed, uint64_t offset,
                  const uint64_t* __restrict__ e_off, const double* __restrict__ e_time,
                  const uint32_t* __restrict__ e_lixel, uint64_t num_pulses,
                  uint32_t num_sensors, uint8_t* __restrict__ slice,
                  uint32_t* __restrict__ keep) {
    for (uint64_t p = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; p < num_pulses;
         p += (uint64_t)gridDim.x*blockDim.x) {
        const uint32_t l = e_lixel[p];
        if (l >= num_sensors) {            // not written: the writing pass stopped early
            slice[p] = 0;
            keep[p] = 0u;
            continue;
        }
        const uint32_t j = (uint32_t)(p - e_off[l]);
        const uint64_t st = stage_stream(3, offset, l);
        const double u1 = mlgpu_philox_uniform(seed, st, 2*j);
        const double u2 = mlgpu_philox_uniform(seed, st, 2*j + 1);
        const double z = 0.0 + P.arrival_time_std*(sqrt(-2.0*log(1.0 - u1))*cos(2.0*M_PI*u2));
        const double r = round((e_time[p] + z)/P.time_slice_duration);
        const bool k = r >= 0.0 && r < kNumberTimeSlices;
        slice[p] = k ? (uint8_t)(int32_t)r : (uint8_t)0;
        keep[p] = k ? 1u : 0u;
    }
    // one more flag so that the scan also gives the total
    if (blockIdx.x == 0 && threadIdx.x == 0) keep[num_pulses] = 0u;
}

__global__ void __launch_bounds__(256)
sc_scatter_kernel(const uint8_t* __restrict__ slice, const int32_t* __restrict__ e_truth,
                  const uint32_t* __restrict__ keep, const uint64_t* __restrict__ pos,
                  uint64_t num_pulses, uint8_t* __restrict__ out_slice,
                  int32_t* __restrict__ out_truth) {
    for (uint64_t p = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; p < num_pulses;
         p += (uint64_t)gridDim.x*blockDim.x) {
        if (keep[p]) {
            const uint64_t q = pos[p];
            out_slice[q] = slice[p];
            out_truth[q] = e_truth[p];
        }
    }
}

// channel c's first kept pulse: the kept pulses before lixel c's first pulse
__global__ void __launch_bounds__(128)
sc_channel_offsets_kernel(const uint64_t* __restrict__ e_off, const uint64_t* __restrict__ pos,
                          uint32_t num_sensors, uint64_t* __restrict__ channel_offset) {
    const uint32_t s = blockIdx.x*blockDim.x + threadIdx.x;
    if (s <= num_sensors) channel_offset[s] = pos[e_off[s]];
}

// ---- scratch --------------------------------------------------------------------

inline uint64_t align256(uint64_t b) { return (b + 255) & ~uint64_t(255); }

// key bits for sensor indices 0..num_sensors (num_sensors: no sensor)
int sensor_key_bits(uint32_t num_sensors) {
    int b = 1;
    while (b < 32 && (num_sensors >> b)) b++;
    return b;
}

struct PhotonScratch {
    uint32_t *skey_in, *skey_out, *idx_in, *idx_out;
    uint64_t *tkey_in, *tkey_out;
    double *t, *w;
    int32_t* r;
    uint64_t *pipe_off, *counts, *e_off;
    uint32_t* medium;                 // sensors with kWarpSegment < photons <= kBlockSegment
    uint64_t *large_begin, *large_end;
    uint64_t large_slots;             // at most n / (kBlockSegment + 1) longer runs
    uint32_t* bins;
    uint64_t nbins;
    unsigned long long* minmax;
    unsigned int* seg_counts;         // [0] medium, [1] large
    double* start;
    void* temp;
    size_t temp_bytes;
};

uint64_t large_slots_for(uint64_t n) { return n/(kBlockSegment + 1) + 1; }

size_t photon_temp_bytes(uint64_t n, uint32_t ns) {
    const size_t a = counting_sort_temp_bytes(n, ns + 1);
    const size_t c = exclusive_sum_temp_bytes((uint64_t)ns + 1);
    return a > c ? a : c;
}

PhotonScratch photon_layout(uint64_t n, uint32_t ns, void* scratch, size_t bytes) {
    PhotonScratch c;
    char* p = static_cast<char*>(scratch);
    const uint64_t a4 = align256(n*4), a8 = align256(n*8), as = align256((uint64_t)(ns + 2)*8);
    c.skey_in = reinterpret_cast<uint32_t*>(p); p += a4;
    c.skey_out = reinterpret_cast<uint32_t*>(p); p += a4;
    c.idx_in = reinterpret_cast<uint32_t*>(p); p += a4;
    c.idx_out = reinterpret_cast<uint32_t*>(p); p += a4;
    c.tkey_in = reinterpret_cast<uint64_t*>(p); p += a8;
    c.tkey_out = reinterpret_cast<uint64_t*>(p); p += a8;
    c.t = reinterpret_cast<double*>(p); p += a8;
    c.w = reinterpret_cast<double*>(p); p += a8;
    c.r = reinterpret_cast<int32_t*>(p); p += a4;
    c.pipe_off = reinterpret_cast<uint64_t*>(p); p += as;
    c.counts = reinterpret_cast<uint64_t*>(p); p += as;
    c.e_off = reinterpret_cast<uint64_t*>(p); p += as;
    c.medium = reinterpret_cast<uint32_t*>(p); p += align256((uint64_t)(ns + 1)*4);
    c.large_slots = large_slots_for(n);
    c.large_begin = reinterpret_cast<uint64_t*>(p); p += align256(c.large_slots*8);
    c.large_end = reinterpret_cast<uint64_t*>(p); p += align256(c.large_slots*8);
    c.nbins = (uint64_t)(2.0 + sqrt((double)n)) + 1;
    c.bins = reinterpret_cast<uint32_t*>(p); p += align256(c.nbins*4);
    c.minmax = reinterpret_cast<unsigned long long*>(p);
    c.start = reinterpret_cast<double*>(p + 16);
    c.seg_counts = reinterpret_cast<unsigned int*>(p + 24);
    p += 256;
    c.temp = p;
    c.temp_bytes = bytes - (size_t)(p - static_cast<char*>(scratch));
    return c;
}

struct PulseScratch {
    double* time;
    int32_t* truth;
    uint32_t *lixel, *keep;
    uint8_t* slice;
    uint64_t* pos;
    void* temp;
    size_t temp_bytes;
};

size_t pulse_temp_bytes(uint64_t np) { return exclusive_sum_temp_bytes(np + 1); }

PulseScratch pulse_layout(uint64_t np, void* scratch, size_t bytes) {
    PulseScratch c;
    char* p = static_cast<char*>(scratch);
    c.time = reinterpret_cast<double*>(p); p += align256(np*8);
    c.truth = reinterpret_cast<int32_t*>(p); p += align256(np*4);
    c.lixel = reinterpret_cast<uint32_t*>(p); p += align256(np*4);
    c.keep = reinterpret_cast<uint32_t*>(p); p += align256((np + 1)*4);
    c.slice = reinterpret_cast<uint8_t*>(p); p += align256(np);
    c.pos = reinterpret_cast<uint64_t*>(p); p += align256((np + 1)*8);
    c.temp = p;
    c.temp_bytes = bytes - (size_t)(p - static_cast<char*>(scratch));
    return c;
}

}  // namespace

size_t signal_chain_photon_scratch_bytes(uint64_t n, uint32_t ns) {
    const uint64_t a4 = align256(n*4), a8 = align256(n*8), as = align256((uint64_t)(ns + 2)*8);
    const uint64_t nbins = (uint64_t)(2.0 + sqrt((double)n)) + 1;
    return 5*a4 + 4*a8 + 3*as + align256((uint64_t)(ns + 1)*4) +
           2*align256(large_slots_for(n)*8) + align256(nbins*4) + 256 +
           photon_temp_bytes(n, ns) + 256;
}

size_t signal_chain_pulse_scratch_bytes(uint64_t num_pulses) {
    const uint64_t np = num_pulses;
    return align256(np*8) + 2*align256(np*4) + align256((np + 1)*4) + align256(np) +
           align256((np + 1)*8) + pulse_temp_bytes(np) + 256;
}

// Steps 1-3a: pipelines, window, the conversion's counting pass and the scan
// of its counts.  *total_dev receives the electric pulses of the event,
// *start_dev the window start (both in the scratch).
cudaError_t launch_signal_chain_count(const SignalChainArgs& a, void* scratch, size_t bytes,
                                      int grid, cudaStream_t s, const uint64_t** total_dev,
                                      const double** start_dev) {
    const uint64_t n = a.num_photons;
    const uint32_t ns = a.num_sensors;
    if (n >= (1ull << 31) || ns >= (1u << 31)) return cudaErrorInvalidValue;
    const PhotonScratch c = photon_layout(n, ns, scratch, bytes);
    *total_dev = c.e_off + ns;
    *start_dev = c.start;
    cudaError_t e = cudaMemsetAsync(c.pipe_off, 0, (uint64_t)(ns + 1)*8, s);
    if (e != cudaSuccess) return e;
    // 1. by sensor, then every sensor's run by (time, input index)
    if (n > 0) {
        sc_sensor_keys_kernel<<<grid, 256, 0, s>>>(a.sensor, n, ns, c.skey_in, c.idx_in, a.err);
        // grouped by sensor (device_sort.cu: a counting sort, which also
        // gives each pipeline's offset; the order within a sensor is set by
        // the sort by (time, index) below)
        e = counting_sort(c.skey_in, n, ns + 1, c.idx_out, c.pipe_off, c.temp, s);
        if (e != cudaSuccess) return e;
        sc_time_keys_kernel<<<grid, 256, 0, s>>>(c.idx_out, a.time, c.pipe_off, ns, c.tkey_in);
        if (ns > 0) {
            e = cudaMemsetAsync(c.seg_counts, 0, 8, s);
            if (e != cudaSuccess) return e;
            e = cudaMemsetAsync(c.large_begin, 0, c.large_slots*8, s);
            if (e != cudaSuccess) return e;
            e = cudaMemsetAsync(c.large_end, 0, c.large_slots*8, s);
            if (e != cudaSuccess) return e;
            sc_segsort_warp_kernel<<<(ns + kSegWarps - 1)/kSegWarps, kSegWarps*32, 0, s>>>(
                c.tkey_in, c.idx_out, c.pipe_off, ns, c.tkey_out, c.idx_in, c.medium,
                c.seg_counts, c.large_begin, c.large_end, c.seg_counts + 1);
            if (n > kWarpSegment) {
                const uint64_t medium_max = n/(kWarpSegment + 1) + 1;
                const int blocks = (int)(medium_max < 296 ? medium_max : 296);
                sc_segsort_block_kernel<<<blocks, 512, kBlockSegment*12, s>>>(
                    c.tkey_in, c.idx_out, c.pipe_off, c.medium, c.seg_counts, c.tkey_out, c.idx_in);
            }
            if (n > kBlockSegment) {
                e = sort_long_runs(c.tkey_in, c.idx_out, c.tkey_out, c.idx_in, c.large_begin,
                                   c.large_end, (uint32_t)c.large_slots, s);
                if (e != cudaSuccess) return e;
            }
        }
        sc_gather_kernel<<<grid, 256, 0, s>>>(c.idx_in, a.time, a.wavelength, a.truth, c.pipe_off,
                                              ns, c.t, c.w, c.r);
    }
    // 2. the exposure window; minmax starts at the time keys of DBL_MAX and DBL_MIN
    static const unsigned long long init[2] = {0xffefffffffffffffull, 0x8010000000000000ull};
    e = cudaMemcpyAsync(c.minmax, init, sizeof(init), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    if (ns > 0)
        sc_minmax_kernel<<<(ns + 127)/128, 128, 0, s>>>(c.t, c.pipe_off, ns, c.minmax);
    e = cudaMemsetAsync(c.bins, 0, c.nbins*4, s);
    if (e != cudaSuccess) return e;
    const int use_smem = c.nbins <= (uint64_t)kSmemBins;
    if (n > 0)
        sc_histogram_kernel<<<grid, 256, use_smem ? c.nbins*4 : 0, s>>>(c.t, c.pipe_off, ns,
                                                                        c.minmax, c.bins,
                                                                        use_smem);
    sc_window_kernel<<<1, 1024, 0, s>>>(c.pipe_off, ns, c.minmax, c.bins, a.params.exposure_time,
                                        c.start);
    // 3a. the counting pass and the scan of the counts
    e = cudaMemsetAsync(c.counts, 0, (uint64_t)(ns + 1)*8, s);
    if (e != cudaSuccess) return e;
    if (ns > 0)
        sc_lixel_kernel<false><<<(ns + 127)/128, 128, 0, s>>>(
            a.params, a.seed, a.offset, c.pipe_off, c.t, c.w, c.r, a.efficiency, ns, c.start,
            c.counts, a.nsb_count, nullptr, nullptr, nullptr, nullptr, a.err);
    e = exclusive_sum_u64(c.counts, c.e_off, (uint64_t)ns + 1, c.temp, s);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// Steps 3b-4 up to the scan of the keep flags: the electric pulses written,
// extracted, their kept positions and the channel offsets.  *kept_dev
// receives the number of kept pulses (in the pulse scratch).
cudaError_t launch_signal_chain_extract(const SignalChainArgs& a, void* scratch, size_t bytes,
                                        void* pulse_scratch, size_t pulse_bytes,
                                        uint64_t num_pulses, int grid, cudaStream_t s,
                                        const uint64_t** kept_dev) {
    const uint32_t ns = a.num_sensors;
    const PhotonScratch c = photon_layout(a.num_photons, ns, scratch, bytes);
    const PulseScratch q = pulse_layout(num_pulses, pulse_scratch, pulse_bytes);
    *kept_dev = q.pos + num_pulses;
    if (num_pulses > 0) {
        const cudaError_t e = cudaMemsetAsync(q.lixel, 0xff, num_pulses*4, s);
        if (e != cudaSuccess) return e;
    }
    if (ns > 0)
        sc_lixel_kernel<true><<<(ns + 127)/128, 128, 0, s>>>(
            a.params, a.seed, a.offset, c.pipe_off, c.t, c.w, c.r, a.efficiency, ns, c.start,
            nullptr, nullptr, c.e_off, q.time, q.truth, q.lixel, a.err);
    sc_extract_kernel<<<grid, 256, 0, s>>>(a.params, a.seed, a.offset, c.e_off, q.time, q.lixel,
                                           num_pulses, ns, q.slice, q.keep);
    cudaError_t e = exclusive_sum_u32(q.keep, q.pos, num_pulses + 1, q.temp, s);
    if (e != cudaSuccess) return e;
    sc_channel_offsets_kernel<<<(ns + 1 + 127)/128, 128, 0, s>>>(c.e_off, q.pos, ns,
                                                                 a.channel_offset);
    return cudaGetLastError();
}

// Step 4 end: the kept pulses into the caller's photon stream.
cudaError_t launch_signal_chain_scatter(const SignalChainArgs& a, void* pulse_scratch,
                                        size_t pulse_bytes, uint64_t num_pulses, int grid,
                                        cudaStream_t s) {
    const PulseScratch q = pulse_layout(num_pulses, pulse_scratch, pulse_bytes);
    if (num_pulses > 0)
        sc_scatter_kernel<<<grid, 256, 0, s>>>(q.slice, q.truth, q.keep, q.pos, num_pulses,
                                               a.slice, a.slice_truth);
    return cudaGetLastError();
}

}  // namespace mlgpu
