// corsika.cu -- CORSIKA photon bunches to photons on the device: merlict's
// EventIoPhotonFactory (merlict_corsika/PhotonFactory.cpp:8-136).
//
// A bunch is 8 floats: x, y on the observation level (cm), direction
// cosines u, v, relative arrival time (ns), production height (cm), weight
// (photons in the bunch, 0..16), wavelength (nm).  It becomes floor(weight)
// photons plus one more if a uniform draw is <= the weight's fraction
// (PhotonFactory.cpp:14-24), all with the same support and direction: the
// direction of motion (u, v, -sqrt(1 - u^2 - v^2)) (:113-118), the support
// the ground point moved up the ray by c t + 1 km (:31-62), the wavelength
// |lambda| 1e-9 (:128-130).  The arithmetic is merlict's, in the same
// order, compiled with --fmad=false, so the photons are bit-identical to
// the reference's given the same draws.
//
// Three passes: counts per bunch, an exclusive scan, the expansion (a
// warp per 32 bunches, writing their photons as one contiguous run).
#include <cstdint>

#include "merlict_b200_philox.h"
#include "mlgpu_internal.h"

namespace mlgpu {
namespace {

constexpr int kScan = 1024;

__device__ __forceinline__ double bunch_uniform(const DevRng& r, uint64_t i) {
    if (r.mode == MLGPU_RNG_REPLAY) return __ldg(r.uniforms + i*(uint64_t)(r.stride ? r.stride : 1));
    return mlgpu_philox_uniform(r.seed, r.photon_offset + i, 0);
}

__global__ void __launch_bounds__(256)
corsika_count_kernel(const float* __restrict__ b, uint64_t n, DevRng rng,
                     uint32_t* __restrict__ count, unsigned int* __restrict__ err) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x) {
        const double w = (double)__ldg(b + 8*i + 6);
        uint32_t c = 0;
        if (!(w >= 0.0 && w <= 16.0)) {
            // EventIoPhotonFactory::assert_bunch_weight throws
            atomicCAS(err, 0u, (unsigned)MLGPU_ERR_INVALID_ARGUMENT);
        } else {
            c = (uint32_t)floor(w);
            if (bunch_uniform(rng, i) <= fmod(w, 1.0)) c += 1;
        }
        count[i] = c;
    }
}

// Exclusive scan of `n` counts in blocks of kScan; block sums to `sums`.
__global__ void __launch_bounds__(kScan)
scan_blocks_kernel(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, uint64_t n,
                   uint64_t* __restrict__ sums) {
    __shared__ uint64_t warp_sum[kScan/32];
    const uint64_t i = blockIdx.x*(uint64_t)kScan + threadIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t v = i < n ? in[i] : 0;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t s = warp_sum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;
    }
    __syncthreads();
    const uint64_t before = wid > 0 ? warp_sum[wid - 1] : 0;
    if (i < n) out[i] = before + x - v;
    if (threadIdx.x == kScan - 1) sums[blockIdx.x] = before + x;
}

// Exclusive scan of up to kScan * kScan block sums in one block (serial
// over chunks of kScan).
__global__ void __launch_bounds__(kScan)
scan_sums_kernel(uint64_t* __restrict__ sums, uint64_t blocks, uint64_t* __restrict__ total) {
    __shared__ uint64_t warp_sum[kScan/32];
    __shared__ uint64_t carry;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < blocks; base += kScan) {
        const uint64_t i = base + threadIdx.x;
        const uint64_t v = i < blocks ? sums[i] : 0;
        uint64_t x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            uint64_t s = warp_sum[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sum[lane] = s;
        }
        __syncthreads();
        const uint64_t before = (wid > 0 ? warp_sum[wid - 1] : 0) + carry;
        if (i < blocks) sums[i] = before + x - v;
        __syncthreads();
        if (threadIdx.x == kScan - 1) carry = before + x;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(256)
scan_add_kernel(uint64_t* __restrict__ out, uint64_t n, const uint64_t* __restrict__ sums) {
    for (uint64_t i = blockIdx.x*(uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x*blockDim.x)
        out[i] += sums[i/kScan];
}

// The expansion, a warp per 32 consecutive bunches: each lane computes its
// bunch's photon (merlict's arithmetic) into shared memory as four 16-byte
// words and marks the group's photons it owns in an owner list, then the
// warp writes the group's photons as one contiguous run -- lane p of a
// round writes photon p, reading its bunch from the owner list -- so that
// every store instruction covers consecutive addresses.
constexpr int kExpandWarps = 8;
constexpr int kGroupPhotons = 32*17;   // at most 17 photons per bunch

__global__ void __launch_bounds__(32*kExpandWarps)
corsika_expand_kernel(const float* __restrict__ b, uint64_t n, const uint32_t* __restrict__ count,
                      const uint64_t* __restrict__ offset, const int32_t* __restrict__ ids,
                      double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz,
                      double* __restrict__ dx, double* __restrict__ dy, double* __restrict__ dz,
                      double* __restrict__ wl, int32_t* __restrict__ out_id) {
    // per bunch: (support x, y), (support z, direction x), (direction y, z),
    // (wavelength, id bits)
    __shared__ double2 s_val[kExpandWarps][32][4];
    __shared__ uint8_t s_owner[kExpandWarps][kGroupPhotons];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t groups = (n + 31)/32;
    for (uint64_t grp = (uint64_t)blockIdx.x*kExpandWarps + warp; grp < groups;
         grp += (uint64_t)gridDim.x*kExpandWarps) {
        const uint64_t i = grp*32 + (uint64_t)lane;
        const uint32_t c = i < n ? count[i] : 0u;
        uint32_t incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
        if (c != 0) {
            const float* r = b + 8*i;
            // direction_of_motion, PhotonFactory.cpp:113-118
            const double u = (double)__ldg(r + 2), v = (double)__ldg(r + 3);
            const double z = sqrt(1.0 - u*u - v*v);
            const double cx = u, cy = v, cz = -z;
            // Ray(ground point, -direction): direction normalised (Ray.cpp:16-20)
            const double ux = cx*-1.0, uy = cy*-1.0, uz = cz*-1.0;
            const double un = sqrt(ux*ux + uy*uy + uz*uz);
            const double nx = ux/un, ny = uy/un, nz = uz/un;
            // ray_parameter_for_production_point, PhotonFactory.cpp:58-62
            const double t = (double)__ldg(r + 4)*1e-9;
            const double par = t*299792458.0 + 1e3;
            const double gx = (double)__ldg(r + 0)*1e-2, gy = (double)__ldg(r + 1)*1e-2, gz = 0.0;
            const int32_t id = ids ? __ldg(ids + i) : (int32_t)i;
            double2* sv = s_val[warp][lane];
            sv[0] = make_double2(gx + nx*par, gy + ny*par);
            sv[1] = make_double2(gz + nz*par, cx);
            sv[2] = make_double2(cy, cz);
            sv[3] = make_double2(fabs((double)__ldg(r + 7)*1e-9),
                                 __longlong_as_double((long long)(uint32_t)id));
            for (uint32_t k = incl - c; k < incl; k++) s_owner[warp][k] = (uint8_t)lane;
        }
        const uint64_t o0 = offset[grp*32];   // the group's first photon
        __syncwarp();
        for (uint32_t ph = (uint32_t)lane; ph < total; ph += 32) {
            const double2* sv = s_val[warp][s_owner[warp][ph]];
            const double2 v0 = sv[0], v1 = sv[1], v2 = sv[2], v3 = sv[3];
            const uint64_t o = o0 + ph;
            sx[o] = v0.x; sy[o] = v0.y; sz[o] = v1.x;
            dx[o] = v1.y; dy[o] = v2.x; dz[o] = v2.y;
            wl[o] = v3.x;
            if (out_id) out_id[o] = (int32_t)(uint32_t)__double_as_longlong(v3.y);
        }
        __syncwarp();   // the group's values are rewritten by the next one
    }
}

}  // namespace

size_t corsika_scratch_bytes(uint64_t n) {
    const uint64_t blocks = (n + kScan - 1)/kScan;
    return ((n*4 + 255) & ~uint64_t(255)) + ((n*8 + 255) & ~uint64_t(255)) + (blocks + 1)*8 + 256;
}

cudaError_t launch_corsika_count(const float* bunches, uint64_t n, const DevRng& rng, void* scratch,
                                 uint64_t* total_dev, unsigned int* err, int grid,
                                 cudaStream_t s) {
    uint32_t* count = static_cast<uint32_t*>(scratch);
    uint64_t* offset = reinterpret_cast<uint64_t*>(static_cast<char*>(scratch) +
                                                   ((n*4 + 255) & ~uint64_t(255)));
    uint64_t* sums = offset + ((n*8 + 255) & ~uint64_t(255))/8;
    const uint64_t blocks = (n + kScan - 1)/kScan;
    if (blocks > (uint64_t)kScan*kScan*64) return cudaErrorInvalidValue;
    corsika_count_kernel<<<grid, 256, 0, s>>>(bunches, n, rng, count, err);
    scan_blocks_kernel<<<(unsigned)blocks, kScan, 0, s>>>(count, offset, n, sums);
    scan_sums_kernel<<<1, kScan, 0, s>>>(sums, blocks, total_dev);
    scan_add_kernel<<<grid, 256, 0, s>>>(offset, n, sums);
    return cudaGetLastError();
}

cudaError_t launch_corsika_expand(const float* bunches, uint64_t n, const int32_t* ids,
                                  void* scratch, double* const* planes, int32_t* out_id, int grid,
                                  cudaStream_t s) {
    const uint32_t* count = static_cast<const uint32_t*>(scratch);
    const uint64_t* offset = reinterpret_cast<const uint64_t*>(
        static_cast<const char*>(scratch) + ((n*4 + 255) & ~uint64_t(255)));
    corsika_expand_kernel<<<grid, 32*kExpandWarps, 0, s>>>(bunches, n, count, offset, ids,
                                                          planes[0], planes[1], planes[2],
                                                          planes[3], planes[4], planes[5],
                                                          planes[6], out_id);
    return cudaGetLastError();
}

}  // namespace mlgpu
