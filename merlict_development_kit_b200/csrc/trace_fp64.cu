// trace_fp64.cu -- the plain FP64 tracer: one thread per photon, merlict's
// propagation state machine (merlict/PhotonAndFrame.cpp:13-124) with the
// frame-tree search of CausalIntersection (merlict/RayAndFrame.cpp:126-173)
// done as a stackless walk over the preorder node array.
//
// This translation unit is compiled with --fmad=false and without fast-math
// so that every add, multiply, divide and square root rounds exactly as in
// the reference's x86-64 build (no FMA contraction there either): given the
// same uniforms, photons end on the same surface with bit-identical
// positions, directions and times.  The only libm call on the path, exp()
// in the absorption test (PhotonAndFrame.cpp:32-38), may differ by one ulp
// from glibc; it is exactly 1 for merlict's default infinite absorption.
#include <cstdint>

#include "fp64_geometry.cuh"
#include "merlict_b200_philox.h"

namespace mlgpu {
namespace {

using namespace fp64;

template <typename T>
__device__ __forceinline__ double load_in(const void* p, uint64_t i) {
    return (double)__ldg(static_cast<const T*>(p) + i);
}

__device__ __forceinline__ void store_hist(mlgpu_history_entry* h, const Isec& is, int kind) {
    h->position[0] = is.pos.x; h->position[1] = is.pos.y; h->position[2] = is.pos.z;
    h->normal[0] = is.normal.x; h->normal[1] = is.normal.y; h->normal[2] = is.normal.z;
    h->distance = is.dist;
    h->leaf = is.leaf;
    h->interaction = (uint8_t)kind;
    h->from_outside_to_inside = (uint8_t)is.outside;
    h->pad[0] = 0; h->pad[1] = 0;
}

// The state of one photon between interactions (a merlict Photon: its ray,
// its history so far, its random stream).
struct PhotonState {
    v3 s, d;                 // ray support and direction
    Isec last;               // the latest intersection (history entry n_int - 1)
    v3 last_world, second_last_world;
    double lambda, tof;
    uint64_t i;              // photon index
    uint32_t n_int, k_draw;
    int32_t root;            // frame the next search is restricted to
    int interaction, err, tof_error;
};

// A new photon: merlict::Photon's constructor (Ray.cpp:16-20,
// RayForPropagation.cpp:52-64) and its wavelength check (Photon.cpp:20-28:
// merlict throws std::invalid_argument before propagating anything).
template <typename In>
__device__ __forceinline__ void start_photon(const TraceArgs& a, uint64_t i, PhotonState& p) {
    const DevScene& sc = a.scene;
    p.i = i;
    p.lambda = load_in<In>(a.photons.wavelength, i);
    if (p.lambda <= 0.0) raise_error(sc.error_word, MLGPU_ERR_INVALID_ARGUMENT);
    const v3 s0 = mk(load_in<In>(a.photons.sx, i), load_in<In>(a.photons.sy, i),
                     load_in<In>(a.photons.sz, i));
    p.s = s0;
    // Ray::set_support_and_direction normalises (Ray.cpp:16-20)
    p.d = normalized(mk(load_in<In>(a.photons.dx, i), load_in<In>(a.photons.dy, i),
                        load_in<In>(a.photons.dz, i)));
    p.last.leaf = MLGPU_LEAF_PHOTON_SOURCE; p.last.pos = p.s; p.last.normal = p.d;
    p.last.dist = 0.0;
    p.last.outside = dot(p.d, p.d) < 0.0;
    if (a.results.history)
        store_hist(a.results.history + i*(uint64_t)(a.max_interactions + 1), p.last,
                   MLGPU_PRODUCTION);
    p.last_world = position(IDENTITY, s0);
    p.second_last_world = p.last_world;
    p.n_int = 1;
    p.interaction = MLGPU_PRODUCTION;
    p.root = a.start_node;
    p.tof = 0.0;
    p.tof_error = 0;
    p.err = 0;
    p.k_draw = 0;
}

// One interaction of merlict's Propagator (PhotonAndFrame.cpp:13-124):
// the first causal intersection, then absorption, reflection or the
// Fresnel branches.  Returns true while the photon goes on.
__device__ __forceinline__ bool photon_step(const TraceArgs& a, PhotonState& p) {
    const DevScene& sc = a.scene;
    if (p.n_int > a.max_interactions) return false;
    const uint64_t i = p.i;
    const uint64_t stream = a.rng.photon_offset + i;
    auto draw = [&]() -> double {
        const uint32_t k = p.k_draw++;
        if (a.rng.mode == MLGPU_RNG_REPLAY) {
            if (k >= a.rng.stride) { if (!p.err) p.err = MLGPU_ERR_RUNTIME; return 0.5; }
            return __ldg(a.rng.uniforms + i*(uint64_t)a.rng.stride + k);
        }
        return mlgpu_philox_uniform(a.rng.seed, stream, k);
    };
    const double lambda = p.lambda;
    const v3 s = p.s, d = p.d;
    Isec is;
    if (p.root == 0 && sc.bvh_nodes > 0 && a.traversal == MLGPU_TRAVERSAL_BVH &&
        first_intersection_bvh(sc, s, d, &is)) {
    } else {
        is = first_intersection_tree(sc, p.root, s, d);
    }
    const bool hit = is.leaf >= 0;
    const LeafRec* L = hit ? sc.leaf + is.leaf : nullptr;
    double T[12];
    if (hit) {
#pragma unroll
        for (int k = 0; k < 12; k++) T[k] = __ldg(&L->T[k]);
    } else {
#pragma unroll
        for (int k = 0; k < 12; k++) T[k] = IDENTITY[k];
    }
    int32_t fn[6] = {0, 0, 0, 0, 0, 0};
    int32_t flags = 0, allowed = -1;
    if (hit) {
#pragma unroll
        for (int k = 0; k < 6; k++) fn[k] = __ldg(&L->fn[k]);
        flags = __ldg(&L->flags);
        allowed = __ldg(&L->allowed_node);
    }
    bool absorbed = false;
    if (hit) {
        const double depth = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_ABSORPTION
                                                          : MLGPU_SURF_INNER_ABSORPTION], lambda, &p.err);
        const double survival = exp(-is.dist/depth);
        absorbed = draw() > survival;
    }
    int kind;
    bool moved = false;
    v3 new_s = s, new_d = d;
    if (!hit || absorbed) {
        kind = MLGPU_ABSORPTION_IN_VOID;
    } else {
        const double refl = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFLECTION
                                                         : MLGPU_SURF_INNER_REFLECTION], lambda, &p.err);
        if (refl >= draw()) {
            kind = MLGPU_REFLECTION_ON_SURFACE;
            new_s = position(T, is.pos);
            new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
            moved = true;
        } else if (!(flags & MLGPU_FLAG_TRANSPARENT)) {
            kind = MLGPU_ABSORPTION_ON_SURFACE;
        } else {
            // Fresnel, merlict/Fresnel.cpp:7-38
            const v3 inc = orientation_inverse(T, d);
            const v3 nrm = is.outside ? is.normal : scale(is.normal, -1.0);
            const double n_from = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION
                                                               : MLGPU_SURF_INNER_REFRACTION], lambda, &p.err);
            const double n_to = func_eval(sc, fn[is.outside ? MLGPU_SURF_INNER_REFRACTION
                                                             : MLGPU_SURF_OUTER_REFRACTION], lambda, &p.err);
            const double cosI = dot(nrm, inc)*(-1.0);
            const double ratio = n_from/n_to;
            const double sinT2 = ratio*ratio*(1.0 - cosI*cosI);
            const double cosT = sqrt(1.0 - sinT2);
            double R;
            if (sinT2 > 1.0) {
                R = 1.0;
            } else {
                const double rOrth = (n_from*cosI - n_to*cosT) / (n_from*cosI + n_to*cosT);
                const double rPar = (n_to*cosI - n_from*cosT) / (n_to*cosI + n_from*cosT);
                R = (rOrth*rOrth + rPar*rPar) / 2.0;
            }
            if (R > draw()) {
                kind = MLGPU_FRESNEL_REFLECTION_ON_SURFACE;
                new_s = position(T, is.pos);
                new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                moved = true;
            } else {
                kind = is.outside ? MLGPU_REFRACTION_TO_INSIDE : MLGPU_REFRACTION_TO_OUTSIDE;
                const bool to_default = is.outside
                    ? (flags & MLGPU_FLAG_INNER_REFRACTION_DEFAULT) != 0
                    : (flags & MLGPU_FLAG_OUTER_REFRACTION_DEFAULT) != 0;
                p.root = (allowed >= 0 && !to_default) ? allowed : 0;
                const v3 refr = add(scale(inc, ratio), scale(nrm, ratio*cosI - cosT));
                new_s = position(T, is.pos);
                new_d = normalized(orientation(T, refr));
                moved = true;
            }
        }
    }
    if (a.results.history)
        store_hist(a.results.history + i*(uint64_t)(a.max_interactions + 1) + p.n_int, is, kind);
    {
        // time-of-flight term, merlict/Photon.cpp:37-56
        const int32_t f = hit
            ? fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION : MLGPU_SURF_INNER_REFRACTION]
            : sc.default_refraction;
        int terr = 0;
        const double n = func_eval(sc, f, lambda, &terr);
        if (terr && !p.tof_error) p.tof_error = terr;
        p.tof += n*is.dist/299792458.0;
    }
    p.second_last_world = p.last_world;
    p.last_world = moved ? new_s : position(T, is.pos);
    p.n_int++;
    p.interaction = kind;
    p.last = is;
    if (!moved) return false;
    p.s = new_s;
    p.d = new_d;
    return true;
}

// The photon's results: Sensor::assign_photon (Sensor.cpp:14-30) and the
// rest of its record.
template <typename Out>
__device__ __forceinline__ void finish_photon(const TraceArgs& a, PhotonState& p) {
    const DevScene& sc = a.scene;
    const uint64_t i = p.i;
    const uint32_t max_int = a.max_interactions;
    if (a.results.history) {
        mlgpu_history_entry* hist = a.results.history + i*(uint64_t)(max_int + 1);
        for (uint32_t k = p.n_int; k < max_int + 1; k++) {
            mlgpu_history_entry* h = &hist[k];
            h->position[0] = 0; h->position[1] = 0; h->position[2] = 0;
            h->normal[0] = 0; h->normal[1] = 0; h->normal[2] = 0;
            h->distance = 0; h->leaf = MLGPU_LEAF_PHOTON_SOURCE;
            h->interaction = 0; h->from_outside_to_inside = 0; h->pad[0] = 0; h->pad[1] = 0;
        }
    }
    const Isec& last = p.last;
    const int32_t sensor = last.leaf >= 0 ? __ldg(&sc.leaf[last.leaf].sensor) : -1;
    if (sensor >= 0 && p.tof_error && !p.err) p.err = p.tof_error;

    // final_intersection_incident_direction_wrt_frame, RayForPropagation.cpp:114-136
    v3 inc = mk(0.0, 0.0, 0.0);
    if (p.n_int > 1) {
        const v3 w = normalized(sub(p.last_world, p.second_last_world));
        if (last.leaf >= 0) {
            double T[12];
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = __ldg(&sc.leaf[last.leaf].T[k]);
            inc = orientation_inverse(T, w);
        } else {
            inc = orientation_inverse(IDENTITY, w);
        }
    }
    const DevResults& r = a.results;
    r.sensor[i] = sensor;
    if (r.x) static_cast<Out*>(r.x)[i] = (Out)last.pos.x;
    if (r.y) static_cast<Out*>(r.y)[i] = (Out)last.pos.y;
    if (r.time) r.time[i] = p.tof;
    if (r.theta_x) static_cast<Out*>(r.theta_x)[i] = (Out)(-1.0*inc.x);
    if (r.theta_y) static_cast<Out*>(r.theta_y)[i] = (Out)(-1.0*inc.y);
    if (r.final_leaf) r.final_leaf[i] = last.leaf;
    if (r.info)
        r.info[i] = (uint32_t)p.interaction | (p.n_int << 8) |
            ((p.k_draw > 255u ? 255u : p.k_draw) << 16) | ((uint32_t)p.err << 24);
    if (r.final_position) {
        r.final_position[3*i] = p.last_world.x;
        r.final_position[3*i + 1] = p.last_world.y;
        r.final_position[3*i + 2] = p.last_world.z;
    }
    if (r.final_direction) {
        r.final_direction[3*i] = p.d.x;
        r.final_direction[3*i + 1] = p.d.y;
        r.final_direction[3*i + 2] = p.d.z;
    }
    if (p.err) raise_error(sc.error_word, (unsigned int)p.err);
}

// One thread per photon, every interaction in a loop.
template <typename In, typename Out>
__global__ void __launch_bounds__(128)
trace_fp64_kernel(const TraceArgs a) {
    const uint64_t i = (uint64_t)blockIdx.x*blockDim.x + threadIdx.x;
    if (i >= a.num_photons) return;
    PhotonState p;
    start_photon<In>(a, i, p);
    while (photon_step(a, p)) {}
    finish_photon<Out>(a, p);
}

// One persistent launch over the whole batch, however its events are sized:
// every warp takes consecutive photons of the batch's tracing order from a
// device work queue (one atomic per warp and refill: a tile of as many
// photons as the warp has idle lanes) and advances its photons one
// interaction per round; a lane whose photon has ended takes the next one
// at the following round, so lanes stay busy while their neighbours'
// photons go on bouncing.  No thread ever waits for another: the queue is
// a counter, drained when it passes the batch size.
template <typename In, typename Out>
__global__ void __launch_bounds__(128)
queue_trace_kernel(const TraceArgs a, unsigned long long* queue) {
    const int lane = threadIdx.x & 31;
    const unsigned long long n = a.num_photons;
    PhotonState p;
    bool live = false;
    bool drained = false;   // warp-uniform: the queue gave out its last photon
    while (true) {
        const unsigned idle = __ballot_sync(0xffffffffu, !live);
        if (idle && !drained) {
            unsigned long long base = 0;
            if (lane == __ffs(idle) - 1) base = atomicAdd(queue, (unsigned long long)__popc(idle));
            base = __shfl_sync(0xffffffffu, base, __ffs(idle) - 1);
            if (base + __popc(idle) >= n) drained = true;
            if (!live) {
                const unsigned long long q = base + __popc(idle & ((1u << lane) - 1u));
                if (q < n) {
                    start_photon<In>(a, a.order ? (uint64_t)__ldg(a.order + q) : (uint64_t)q, p);
                    live = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, live)) break;
        if (live && !photon_step(a, p)) {
            finish_photon<Out>(a, p);
            live = false;
        }
    }
}

}  // namespace

cudaError_t launch_queue_trace(const TraceArgs& a, unsigned long long* queue, int grid,
                               cudaStream_t s) {
    if (a.num_photons == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F64)
        queue_trace_kernel<double, double><<<grid, 128, 0, s>>>(a, queue);
    else if (a.in_dtype == MLGPU_F32 && a.out_dtype == MLGPU_F64)
        queue_trace_kernel<float, double><<<grid, 128, 0, s>>>(a, queue);
    else if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F32)
        queue_trace_kernel<double, float><<<grid, 128, 0, s>>>(a, queue);
    else
        queue_trace_kernel<float, float><<<grid, 128, 0, s>>>(a, queue);
    return cudaGetLastError();
}

int queue_trace_blocks_per_sm() {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, queue_trace_kernel<double, double>,
                                                      128, 0) != cudaSuccess || blocks < 1)
        blocks = 1;
    return blocks;
}

cudaError_t launch_trace_fp64(const TraceArgs& a, int block, cudaStream_t s) {
    if (a.num_photons == 0) return cudaSuccess;
    block = 128;
    const uint64_t grid = (a.num_photons + block - 1) / block;
    if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F64)
        trace_fp64_kernel<double, double><<<(unsigned)grid, block, 0, s>>>(a);
    else if (a.in_dtype == MLGPU_F32 && a.out_dtype == MLGPU_F64)
        trace_fp64_kernel<float, double><<<(unsigned)grid, block, 0, s>>>(a);
    else if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F32)
        trace_fp64_kernel<double, float><<<(unsigned)grid, block, 0, s>>>(a);
    else
        trace_fp64_kernel<float, float><<<(unsigned)grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mlgpu
