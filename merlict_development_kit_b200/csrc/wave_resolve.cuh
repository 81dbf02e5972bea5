// wave_resolve.cuh -- the per-candidate and per-slot steps of the wavefront
// tracers, shared by the FP64 and FP32 forms:
//   intersect  one thread per (ray, candidate leaf): the distance to the
//              leaf's hit; the smallest distance of each ray is kept with a
//              64-bit atomic minimum on its bits (positive doubles order like
//              their bit patterns);
//   ties       one thread per candidate: among the candidates at exactly that
//              distance the lowest leaf index wins, which is the leaf merlict
//              visits first (RayAndFrame.cpp:160-173);
//   overflow   rays whose walk overflowed a queue get merlict's own walk of
//              the frame tree;
//   resolve    one thread per ray: the winner's full intersection, recomputed
//              by the same code, the interaction with the surface
//              (merlict/PhotonAndFrame.cpp:13-124), the history entry and the
//              time-of-flight term; survivors are compacted into the next
//              pool with a warp ballot and one atomic per warp, finished
//              photons write their results.
//
// kIsect selects the intersection arithmetic: FP64 (merlict's, bit-identical
// when the translation unit is compiled with --fmad=false), or the FP32
// intersections of fp32_geometry.cuh (with or without the FP64 Newton step).
// The interaction, positions and time of flight are FP64 in every form.
#ifndef MLGPU_WAVE_RESOLVE_CUH_
#define MLGPU_WAVE_RESOLVE_CUH_

#include <climits>
#include <cstdint>

#include "fp64_geometry.cuh"
#include "fp32_geometry.cuh"
#include "merlict_b200_philox.h"

namespace mlgpu {
namespace {

using namespace fp64;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kNoStep = -2;             // step state: the photon takes no step
constexpr int kStepNone = 0;            // it takes a step; nothing to queue (no candidates)
constexpr int kStepBvh = 1;             // it takes a step; the intake queues the BVH root
constexpr int kStepTree = 2;            // it takes a step; the intake walks its frame subtree
constexpr int32_t kNoLeaf = INT32_MAX;  // best_leaf of a ray without a hit
constexpr unsigned long long kNoKey = ~0ull;

constexpr int kIsectFp64 = 0;
constexpr int kIsectFp32 = 1;
constexpr int kIsectFp32Pure = 2;

template <typename T>
__device__ __forceinline__ double load_in(const void* p, uint64_t i) {
    return (double)__ldg(static_cast<const T*>(p) + i);
}

__device__ __forceinline__ void store_hist(mlgpu_history_entry* h, v3 pos, v3 nrm, double dist,
                                           int32_t leaf, int kind, bool outside) {
    h->position[0] = pos.x; h->position[1] = pos.y; h->position[2] = pos.z;
    h->normal[0] = nrm.x; h->normal[1] = nrm.y; h->normal[2] = nrm.z;
    h->distance = dist;
    h->leaf = leaf;
    h->interaction = (uint8_t)kind;
    h->from_outside_to_inside = (uint8_t)outside;
    h->pad[0] = 0; h->pad[1] = 0;
}

// Reserves n consecutive entries of a queue for every lane of the (full,
// converged) warp with one atomic; returns this lane's first index.
__device__ __forceinline__ uint32_t warp_reserve(unsigned int* counter, uint32_t n) {
    const int lane = threadIdx.x & 31;
    uint32_t x = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
    }
    const uint32_t sum = __shfl_sync(kFull, x, 31);
    uint32_t base = 0;
    if (lane == 31 && sum) base = atomicAdd(counter, sum);
    base = __shfl_sync(kFull, base, 31);
    return base + x - n;
}

// Sends a slot to merlict's own walk (once per iteration).
__device__ __forceinline__ void mark_overflow(const WaveBuffers& w, const RayPool& cur,
                                              uint32_t slot) {
    uint32_t* flag = cur.overflow_flag;
    if (atomicExch(flag + slot, 1u) == 0u)
        w.overflow[atomicAdd(&w.counters->overflow_len, 1u)] = slot;
}

// The first index of this warp in a grid-stride loop whose trip count is
// the same for every lane of a warp (so that warp_reserve sees full warps).
__device__ __forceinline__ uint32_t warp_first() {
    return blockIdx.x*blockDim.x + (threadIdx.x & ~31u);
}

// The FP64 ray of a slot from its 48-byte record.
__device__ __forceinline__ void load_ray(const RayPool& p, uint32_t slot, v3* s, v3* d) {
    const double2 a = p.sd[3*slot], b = p.sd[3*slot + 1], c = p.sd[3*slot + 2];
    *s = mk(a.x, a.y, b.x);
    *d = mk(b.y, c.x, c.y);
}

__device__ __forceinline__ void store_ray(const RayPool& p, uint32_t slot, v3 s, v3 d) {
    p.sd[3*slot] = make_double2(s.x, s.y);
    p.sd[3*slot + 1] = make_double2(s.z, d.x);
    p.sd[3*slot + 2] = make_double2(d.y, d.z);
}

// The box inflation of a ray's FP32 slab tests: its rounding to FP32.
__device__ __forceinline__ float box_inflation(const DevScene& sc, float ox, float oy, float oz) {
    return sc.bvh_eps + 4e-7f*(fabsf(ox) + fabsf(oy) + fabsf(oz));
}

// What the next intake queues for a ray about to take a step from s along d
// in the frame subtree `root`, and its FP32 walk record when that is the
// BVH: inside a lens (root != 0), or without a BVH, merlict's own walk of
// the subtree (kStepTree); else merlict tests the root frame's sphere first
// (RayAndFrame.cpp:137-149) and the BVH walk follows if the ray passes it.
__device__ __forceinline__ int prepare_walk(const TraceArgs& a, const RayPool& p, uint32_t slot,
                                            v3 s, v3 d, int32_t root) {
    const DevScene& sc = a.scene;
    if (root != 0 || sc.bvh_nodes == 0 || a.traversal == MLGPU_TRAVERSAL_FRAME_TREE)
        return kStepTree;
    const double2* np = reinterpret_cast<const double2*>(sc.node);
    const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
    if (!sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, dot(s, d))) return kStepNone;
    const float ox = (float)s.x, oy = (float)s.y, oz = (float)s.z;
    float fdx = (float)d.x, fdy = (float)d.y, fdz = (float)d.z;
    if (fabsf(fdx) < 1e-30f) fdx = copysignf(1e-30f, fdx);
    if (fabsf(fdy) < 1e-30f) fdy = copysignf(1e-30f, fdy);
    if (fabsf(fdz) < 1e-30f) fdz = copysignf(1e-30f, fdz);
    p.ray_o[slot] = make_float4(ox, oy, oz, box_inflation(sc, ox, oy, oz));
    p.ray_i[slot] = make_float4(1.0f/fdx, 1.0f/fdy, 1.0f/fdz, 0.0f);
    return kStepBvh;
}

template <int kIsect>
__global__ void __launch_bounds__(256)
wave_isect_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur) {
    const DevScene& sc = a.scene;
    const uint32_t n = w.counters->isect_len < w.isect_cap ? w.counters->isect_len : w.isect_cap;
    for (uint32_t e = blockIdx.x*blockDim.x + threadIdx.x; e < n; e += gridDim.x*blockDim.x) {
        const uint2 q = w.isect_q[e];
        const uint32_t slot = q.x;
        v3 s, d;
        load_ray(cur, slot, &s, &d);
        double dist = -1.0;
        if (kIsect == kIsectFp64) {
            double T[12], ti[3], pr[MLGPU_LEAF_PARAMS], r2;
            int32_t prim;
            load_leaf_slot(sc, q.y, T, ti, pr, &r2, &prim);
            // merlict's bounding-sphere test of the leaf (RayAndFrame.cpp:
            // 16-107; the sphere is centred on the frame's position,
            // Frame::position_in_world): the walk proposed the leaf with a
            // conservative single-precision version of it
            if (sphere_cull(make_double4(T[3], T[7], T[11], r2), s, d, dot(s, d))) {
                Isec h;
                intersect_leaf(sc, (int32_t)q.y, prim, pr, r2, position_inverse(T, ti, s),
                               orientation_inverse(T, d), &h);
                if (h.leaf >= 0) dist = h.dist;
            }
        } else {
            // by slot: the FP32 records in slot order, like the FP64 ones
            const fp32::Hit32 h = fp32::intersect32<false, true>(
                sc, (int32_t)q.y, fp32::dmk(s.x, s.y, s.z), fp32::dmk(d.x, d.y, d.z),
                kIsect == kIsectFp32Pure);
            if (h.leaf >= 0) dist = h.v;
        }
        w.isect_dist[e] = dist;
        if (dist >= 0.0) atomicMin(&cur.best_key[slot], (unsigned long long)__double_as_longlong(dist));
    }
}

__global__ void __launch_bounds__(256)
wave_tie_kernel(const WaveBuffers w, const RayPool cur) {
    const uint32_t n = w.counters->isect_len < w.isect_cap ? w.counters->isect_len : w.isect_cap;
    for (uint32_t e = blockIdx.x*blockDim.x + threadIdx.x; e < n; e += gridDim.x*blockDim.x) {
        const double dist = w.isect_dist[e];
        if (!(dist >= 0.0)) continue;
        const uint2 q = w.isect_q[e];
        if ((unsigned long long)__double_as_longlong(dist) == cur.best_key[q.x])
            atomicMin(&cur.best_leaf[q.x], __ldg(w.slot_leaf_of + q.y));
    }
}

// Rays whose walk overflowed a queue: merlict's own walk of the frame tree
// (FP64, in merlict's order) finds the closest hit.
__global__ void __launch_bounds__(128)
wave_overflow_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur) {
    const uint32_t n = w.counters->overflow_len;
    for (uint32_t e = blockIdx.x*blockDim.x + threadIdx.x; e < n; e += gridDim.x*blockDim.x) {
        const uint32_t slot = w.overflow[e];
        v3 s, d;
        load_ray(cur, slot, &s, &d);
        const Isec is = first_intersection_tree(a.scene, cur.root[slot], s, d);
        cur.best_leaf[slot] = is.leaf >= 0 ? is.leaf : kNoLeaf;
    }
}

// Three blocks per SM (80 registers, a few hundred bytes spilled): measured
// faster than two blocks at 126 registers.
template <typename Out, int kIsect>
__global__ void __launch_bounds__(256, 3)
wave_resolve_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur, const RayPool nxt) {
    const DevScene& sc = a.scene;
    // the property tables, staged in shared memory when they fit
    extern __shared__ double s_fn[];
    const double* fn_pts = sc.fn_points;
    const int32_t* fn_off = sc.fn_offset;
    if (w.fn_smem_bytes) {
        const int np = 3*sc.num_fn_points;
        int32_t* s_off = reinterpret_cast<int32_t*>(s_fn + np);
        for (int k = threadIdx.x; k < np; k += blockDim.x) s_fn[k] = __ldg(sc.fn_points + k);
        for (int k = threadIdx.x; k <= sc.num_functions; k += blockDim.x) s_off[k] = __ldg(sc.fn_offset + k);
        __syncthreads();
        fn_pts = s_fn;
        fn_off = s_off;
    }
    const uint32_t total = w.counters->total;
    const uint32_t slot = blockIdx.x*blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = slot < total;
    const uint32_t max_int = a.max_interactions;
    const uint32_t hist_len = max_int + 1;

    bool survive = false;
    int32_t finished_chunk = -1;   // fed propagation: the chunk of a photon that ends here
    // state of this slot after the step (written to the next pool if it survives)
    int32_t photon = 0, root = 0, n_next = 0, k_draw = 0, err = 0;
    v3 s = mk(0, 0, 0), d = mk(0, 0, 0);
    double lambda = 0.0, tof = 0.0;
    int32_t count = 0;
    if (valid) {
        load_ray(cur, slot, &s, &d);
        count = cur.step[slot];
    }

    if (valid) {
        photon = cur.photon[slot];
        lambda = cur.lambda[slot];
        tof = cur.tof[slot];
        root = cur.root[slot];
        const int32_t n_int = cur.n_int[slot];
        k_draw = cur.k_draw[slot];
        const int32_t err_word = cur.err[slot];
        err = err_word & 0xff;
        int tof_error = (err_word >> 8) & 0xff;
        const uint64_t stream = a.rng.photon_offset + (uint64_t)photon;
        mlgpu_history_entry* hist =
            a.results.history ? a.results.history + (uint64_t)photon*hist_len : nullptr;

        Isec is;
        int kind = MLGPU_PRODUCTION;
        bool moved = false;
        v3 new_s = s, new_d = d;
        double T[12];
        if (count == kNoStep) {
            is.leaf = MLGPU_LEAF_PHOTON_SOURCE;
            is.pos = s; is.normal = d; is.dist = 0.0; is.outside = dot(d, d) < 0.0;
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = IDENTITY[k];
        } else {
            // merlict's closest hit among the candidates: minimum distance,
            // ties to merlict's visiting order (RayAndFrame.cpp:160-173)
            {
                // the winner of the intersection and tie kernels (or of
                // merlict's own walk), recomputed by the same code
                const int32_t best = cur.best_leaf[slot];
                if (best == kNoLeaf) {
                    set_void(&is, s, d);
                } else if (kIsect == kIsectFp64) {
                    is = leaf_hit(sc, best, s, d);
                } else {
                    const fp32::Hit32 h = fp32::intersect32<true>(sc, best, fp32::dmk(s.x, s.y, s.z),
                                                            fp32::dmk(d.x, d.y, d.z),
                                                            kIsect == kIsectFp32Pure);
                    if (h.leaf < 0) {
                        set_void(&is, s, d);
                    } else {
                        is.leaf = h.leaf;
                        is.pos = mk(h.p.x, h.p.y, h.p.z);
                        is.normal = mk(h.n.x, h.n.y, h.n.z);
                        is.dist = h.v;
                        is.outside = h.outside;
                    }
                }
            }
            const bool hit = is.leaf >= 0;
            const LeafRec* L = hit ? sc.leaf + is.leaf : nullptr;
            if (hit) {
                const double2* q = reinterpret_cast<const double2*>(L->T);
#pragma unroll
                for (int k = 0; k < 6; k++) {
                    const double2 x = __ldg(q + k);
                    T[2*k] = x.x;
                    T[2*k + 1] = x.y;
                }
            } else {
#pragma unroll
                for (int k = 0; k < 12; k++) T[k] = IDENTITY[k];
            }
            int32_t fn[6] = {0, 0, 0, 0, 0, 0};
            int32_t flags = 0, allowed = -1;
            if (hit) {
                static_assert(offsetof(LeafRec, allowed_node) == 200 &&
                              offsetof(LeafRec, flags) == 204 && offsetof(LeafRec, fn) == 208,
                              "the resolve step reads these fields in 8- and 16-byte pieces");
                const int2 af = __ldg(reinterpret_cast<const int2*>(&L->allowed_node));
                const int4 f03 = __ldg(reinterpret_cast<const int4*>(L->fn));
                const int2 f45 = __ldg(reinterpret_cast<const int2*>(L->fn + 4));
                allowed = af.x;
                flags = af.y;
                fn[0] = f03.x; fn[1] = f03.y; fn[2] = f03.z; fn[3] = f03.w;
                fn[4] = f45.x; fn[5] = f45.y;
            }
            auto draw = [&]() -> double {
                const uint32_t k = (uint32_t)k_draw++;
                if (a.rng.mode == MLGPU_RNG_REPLAY) {
                    if (k >= a.rng.stride) { if (!err) err = MLGPU_ERR_RUNTIME; return 0.5; }
                    return __ldg(a.rng.uniforms + (uint64_t)photon*a.rng.stride + k);
                }
                return mlgpu_philox_uniform(a.rng.seed, stream, k);
            };
            bool absorbed = false;
            if (hit) {
                // absorbed_in_medium_before_reaching_surface, PhotonAndFrame.cpp:32-38
                const double depth = func_eval_tab(fn_pts, fn_off, fn[is.outside ? MLGPU_SURF_OUTER_ABSORPTION
                                                                  : MLGPU_SURF_INNER_ABSORPTION], lambda, &err);
                const double survival = exp(-is.dist/depth);
                absorbed = draw() > survival;
            }
            if (!hit || absorbed) {
                kind = MLGPU_ABSORPTION_IN_VOID;
            } else {
                const double refl = func_eval_tab(fn_pts, fn_off, fn[is.outside ? MLGPU_SURF_OUTER_REFLECTION
                                                                 : MLGPU_SURF_INNER_REFLECTION], lambda, &err);
                if (refl >= draw()) {
                    kind = MLGPU_REFLECTION_ON_SURFACE;
                    new_s = position(T, is.pos);
                    new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                    moved = true;
                } else if (!(flags & MLGPU_FLAG_TRANSPARENT)) {
                    kind = MLGPU_ABSORPTION_ON_SURFACE;
                } else {
                    const v3 inc = orientation_inverse(T, d);
                    const v3 nrm = is.outside ? is.normal : scale(is.normal, -1.0);
                    const double n_from = func_eval_tab(fn_pts, fn_off, fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION
                                                                       : MLGPU_SURF_INNER_REFRACTION], lambda, &err);
                    const double n_to = func_eval_tab(fn_pts, fn_off, fn[is.outside ? MLGPU_SURF_INNER_REFRACTION
                                                                     : MLGPU_SURF_OUTER_REFRACTION], lambda, &err);
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
                        root = (allowed >= 0 && !to_default) ? allowed : 0;
                        const v3 refr = add(scale(inc, ratio), scale(nrm, ratio*cosI - cosT));
                        new_s = position(T, is.pos);
                        new_d = normalized(orientation(T, refr));
                        moved = true;
                    }
                }
            }
            if (hist) store_hist(&hist[n_int], is.pos, is.normal, is.dist, is.leaf, kind, is.outside);
            {
                // time-of-flight term, merlict/Photon.cpp:37-56
                const int32_t f = hit
                    ? fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION : MLGPU_SURF_INNER_REFRACTION]
                    : sc.default_refraction;
                int terr = 0;
                const double n = func_eval_tab(fn_pts, fn_off, f, lambda, &terr);
                if (terr && !tof_error) tof_error = terr;
                tof += n*is.dist/299792458.0;
            }
        }
        const v3 step_start = s;
        n_next = n_int + (count == kNoStep ? 0 : 1);
        survive = moved && (uint32_t)n_next <= max_int;
        if (survive) {
            s = new_s;
            d = new_d;
            err = err | (tof_error << 8);
        } else {
            // the photon ends: its results (Sensor.cpp:14-30,
            // RayForPropagation.cpp:114-136)
            const v3 last_world = moved ? new_s : position(T, is.pos);
            const v3 second_last_world =
                count == kNoStep ? last_world : (n_int == 1 ? position(IDENTITY, step_start) : step_start);
            const v3 final_d = moved ? new_d : d;
            const int32_t sensor = is.leaf >= 0 ? __ldg(&sc.leaf[is.leaf].sensor) : -1;
            if (sensor >= 0 && tof_error && !err) err = tof_error;
            v3 inc = mk(0.0, 0.0, 0.0);
            if (n_next > 1) inc = orientation_inverse(T, normalized(sub(last_world, second_last_world)));
            const DevResults& r = a.results;
            const uint64_t p = (uint64_t)photon;
            r.sensor[p] = sensor;
            if (r.x) static_cast<Out*>(r.x)[p] = (Out)is.pos.x;
            if (r.y) static_cast<Out*>(r.y)[p] = (Out)is.pos.y;
            if (r.time) r.time[p] = tof;
            if (r.theta_x) static_cast<Out*>(r.theta_x)[p] = (Out)(-1.0*inc.x);
            if (r.theta_y) static_cast<Out*>(r.theta_y)[p] = (Out)(-1.0*inc.y);
            if (r.final_leaf) r.final_leaf[p] = is.leaf;
            if (r.info)
                r.info[p] = (uint32_t)kind | ((uint32_t)n_next << 8) |
                    ((k_draw > 255 ? 255u : (uint32_t)k_draw) << 16) | ((uint32_t)err << 24);
            if (r.final_position) {
                r.final_position[3*p] = last_world.x;
                r.final_position[3*p + 1] = last_world.y;
                r.final_position[3*p + 2] = last_world.z;
            }
            if (r.final_direction) {
                r.final_direction[3*p] = final_d.x;
                r.final_direction[3*p + 1] = final_d.y;
                r.final_direction[3*p + 2] = final_d.z;
            }
            if (hist)
                for (uint32_t k = (uint32_t)n_next; k < hist_len; k++)
                    store_hist(&hist[k], mk(0, 0, 0), mk(0, 0, 0), 0.0, MLGPU_LEAF_PHOTON_SOURCE, 0, false);
            if (err) raise_error(sc.error_word, (unsigned int)err);
            if (a.fed) {
                int32_t c = 0;
                while (c + 1 < a.feed_chunks && p >= a.feed_start[c + 1]) c++;
                finished_chunk = c;
            }
        }
    }
    // fed propagation: finished photons per chunk, one addition per chunk
    // and warp (a warp's photons mostly come from one chunk)
    if (a.fed) {
        const unsigned fin = __ballot_sync(kFull, finished_chunk >= 0);
        if (finished_chunk >= 0) {
            const unsigned same = __match_any_sync(fin, finished_chunk);
            if (lane == __ffs(same) - 1)
                atomicAdd(&w.counters->done[finished_chunk], (unsigned)__popc(same));
        }
    }
    // warp-ballot compaction of the surviving rays into the next pool
    const unsigned m = __ballot_sync(kFull, survive);
    if (m) {
        uint32_t base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(&w.counters->next, (unsigned)__popc(m));
        base = __shfl_sync(kFull, base, __ffs(m) - 1);
        if (survive) {
            const uint32_t o = base + __popc(m & ((1u << lane) - 1u));
            // the ray as the next iteration takes it: merlict's state, the
            // cleared closest hit, and what the intake has to queue
            nxt.photon[o] = photon;
            store_ray(nxt, o, s, d);
            nxt.lambda[o] = lambda;
            nxt.tof[o] = tof;
            nxt.root[o] = root;
            nxt.n_int[o] = n_next;
            nxt.k_draw[o] = k_draw;
            nxt.err[o] = err;
            nxt.best_key[o] = kNoKey;
            nxt.best_leaf[o] = kNoLeaf;
            nxt.overflow_flag[o] = 0u;
            nxt.step[o] = prepare_walk(a, nxt, o, s, d, root);
        }
    }
}

}  // namespace
}  // namespace mlgpu

#endif  // MLGPU_WAVE_RESOLVE_CUH_
