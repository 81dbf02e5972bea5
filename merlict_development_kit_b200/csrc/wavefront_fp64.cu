// wavefront_fp64.cu -- the wavefront FP64 tracer: merlict's propagation
// (merlict/PhotonAndFrame.cpp:13-124) split into per-step kernels over a
// fixed pool of ray slots, bit-identical to the plain tracer.
//
// One iteration over the pool:
//   walk     persistent kernel; every warp refills its idle lanes from a
//            per-warp chunk of slots (one atomic per 64 slots), takes new
//            photons into free slots, and walks the BVH of the scene,
//            recording the leaves that pass merlict's own bounding-sphere
//            test (RayAndFrame.cpp:16-107) as candidates;
//   resolve  one thread per slot: merlict's intersection of the candidates
//            (closest hit, ties in merlict's visiting order,
//            RayAndFrame.cpp:151-173) -- or, for a ray inside a lens,
//            merlict's walk of that lens's subtree -- the
//            interaction (absorption, reflection, Fresnel), the history
//            entry and the time-of-flight term; survivors are compacted
//            into the next pool with a warp ballot and one atomic per warp,
//            finished photons write their results.
// Separating the cheap, uniform tree walk from the heavy per-step work keeps
// a warp's lanes doing the same thing, which the one-thread-per-photon
// tracer cannot.  The arithmetic is the shared FP64 code, compiled with
// --fmad=false.
#include <cstdint>

#include "fp64_geometry.cuh"
#include "merlict_b200_philox.h"

namespace mlgpu {
namespace {

using namespace fp64;

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWaveCandidates = 32;     // candidate leaves recorded per ray step
constexpr int kWalkChunk = 64;          // slots a warp takes at a time
constexpr int kWalkBurst = 16;          // tree nodes a lane visits between refills
constexpr int kNoStep = -2;             // candidate count: photon takes no step

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

template <typename In>
__global__ void __launch_bounds__(256)
wave_walk_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur) {
    const DevScene& sc = a.scene;
    const uint32_t active = w.counters->active;
    const unsigned long long next_input = w.counters->next_input;
    const unsigned long long remaining = a.num_photons - next_input;
    const uint32_t room = w.pool - active;
    const uint32_t fresh = (uint32_t)(remaining < room ? remaining : room);
    const uint32_t total = active + fresh;
    const int lane = threadIdx.x & 31;
    const unsigned lower = (1u << lane) - 1u;
    const uint32_t max_int = a.max_interactions;
    const uint32_t hist_len = max_int + 1;

    uint32_t chunk_begin = 0, chunk_end = 0;   // warp-uniform
    bool exhausted = false;                    // warp-uniform
    int64_t item = -1;
    v3 s = mk(0, 0, 0), d = mk(0, 0, 0);
    double sd = 0.0;
    int nc = 0;
    bool overflow = false;
    bool tree_mode = false;                    // walking a frame's subtree
    int32_t i = 0, end = 0;                    // frame-tree walk cursor
    // BVH traversal state (single precision slab tests)
    float ox = 0.f, oy = 0.f, oz = 0.f, idx = 0.f, idy = 0.f, idz = 0.f, eps = 0.f;
    int32_t stack[kBvhStack];
    int sp = 0;
    while (true) {
        // hand idle lanes new slots from the warp's chunk
        unsigned idle = __ballot_sync(kFull, item < 0);
        while (idle && !exhausted) {
            if (chunk_begin >= chunk_end) {
                uint32_t b = 0;
                if (lane == 0) b = atomicAdd(&w.counters->walk_fetch, (unsigned)kWalkChunk);
                b = __shfl_sync(kFull, b, 0);
                if (b >= total) { exhausted = true; break; }
                chunk_begin = b;
                chunk_end = min(b + (uint32_t)kWalkChunk, total);
            }
            const uint32_t take = min((uint32_t)__popc(idle), chunk_end - chunk_begin);
            const int rank = __popc(idle & lower);
            if (item < 0 && rank < (int)take) {
                const uint32_t slot = chunk_begin + rank;
                item = slot;
                int32_t root;
                uint32_t n_int;
                if (slot >= active) {
                    // a new photon: merlict::Photon's constructor (Ray.cpp:16-20,
                    // RayForPropagation.cpp:52-64)
                    const uint64_t p = next_input + (slot - active);
                    s = mk(load_in<In>(a.photons.sx, p), load_in<In>(a.photons.sy, p),
                           load_in<In>(a.photons.sz, p));
                    d = normalized(mk(load_in<In>(a.photons.dx, p), load_in<In>(a.photons.dy, p),
                                      load_in<In>(a.photons.dz, p)));
                    root = a.start_node;
                    n_int = 1;
                    cur.photon[slot] = (int32_t)p;
                    cur.sx[slot] = s.x; cur.sy[slot] = s.y; cur.sz[slot] = s.z;
                    cur.dx[slot] = d.x; cur.dy[slot] = d.y; cur.dz[slot] = d.z;
                    cur.lambda[slot] = load_in<In>(a.photons.wavelength, p);
                    cur.tof[slot] = 0.0;
                    cur.root[slot] = root;
                    cur.n_int[slot] = 1;
                    cur.k_draw[slot] = 0;
                    cur.err[slot] = 0;
                    if (a.results.history)
                        store_hist(a.results.history + p*hist_len, s, d, 0.0,
                                   MLGPU_LEAF_PHOTON_SOURCE, MLGPU_PRODUCTION, dot(d, d) < 0.0);
                } else {
                    s = mk(cur.sx[slot], cur.sy[slot], cur.sz[slot]);
                    d = mk(cur.dx[slot], cur.dy[slot], cur.dz[slot]);
                    root = cur.root[slot];
                    n_int = (uint32_t)cur.n_int[slot];
                }
                if (n_int > max_int) {
                    w.cand_count[slot] = kNoStep;
                    item = -1;
                } else if (root != 0 || sc.bvh_nodes == 0 ||
                           a.traversal == MLGPU_TRAVERSAL_FRAME_TREE) {
                    // traversal restricted to a frame's subtree (inside a
                    // lens): merlict's own walk of that subtree
                    sd = dot(s, d);
                    nc = 0;
                    overflow = false;
                    tree_mode = true;
                    i = root;
                    end = __ldg(&sc.node_meta[root].x);
                } else {
                    sd = dot(s, d);
                    nc = 0;
                    overflow = false;
                    tree_mode = false;
                    sp = 0;
                    // merlict tests the root frame's own sphere first
                    const double2* np = reinterpret_cast<const double2*>(sc.node);
                    const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
                    if (sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, sd)) {
                        stack[sp++] = 0;
                        ox = (float)s.x; oy = (float)s.y; oz = (float)s.z;
                        float fdx = (float)d.x, fdy = (float)d.y, fdz = (float)d.z;
                        if (fabsf(fdx) < 1e-30f) fdx = copysignf(1e-30f, fdx);
                        if (fabsf(fdy) < 1e-30f) fdy = copysignf(1e-30f, fdy);
                        if (fabsf(fdz) < 1e-30f) fdz = copysignf(1e-30f, fdz);
                        idx = 1.0f/fdx; idy = 1.0f/fdy; idz = 1.0f/fdz;
                        eps = sc.bvh_eps + 4e-7f*(fabsf(ox) + fabsf(oy) + fabsf(oz));
                    }
                }
            }
            chunk_begin += take;
            idle = __ballot_sync(kFull, item < 0);
        }
        if (__ballot_sync(kFull, item >= 0) == 0) break;
        if (item >= 0) {
            // BVH traversal; each leaf it reaches gets merlict's own sphere
            // test (RayAndFrame.cpp:16-107) and, if it passes, becomes a
            // candidate.  The resolve kernel breaks ties in merlict's
            // visiting order, so the order here does not matter.
            int32_t* cand = w.cand + (size_t)item*kWaveCandidates;
            if (tree_mode) {
                // merlict's walk (RayAndFrame.cpp:137-149), candidates in its order
                for (int it = 0; it < kWalkBurst && i < end; it++) {
                    const double2* np = reinterpret_cast<const double2*>(sc.node + i);
                    const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
                    const int2 meta = __ldg(&sc.node_meta[i]);
                    if (!sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, sd)) {
                        i = meta.x;
                        continue;
                    }
                    if (meta.y >= 0) {
                        if (nc < kWaveCandidates) cand[nc] = meta.y;
                        nc++;
                    }
                    i++;
                }
                if (i >= end) {
                    w.cand_count[item] = nc;
                    item = -1;
                }
            } else {
            for (int it = 0; it < kWalkBurst && sp > 0; it++) {
                const int32_t ref = stack[--sp];
                if (ref < 0) {
                    const int32_t start = (ref & 0x7fffffff) >> 3;
                    const int32_t count = (ref & 7) + 1;
                    for (int32_t j = start; j < start + count; j++) {
                        const double2* q = reinterpret_cast<const double2*>(sc.bvh_sphere + j);
                        const double2 c01 = __ldg(q), c23 = __ldg(q + 1);
                        if (sphere_cull(make_double4(c01.x, c01.y, c23.x, c23.y), s, d, sd)) {
                            if (nc < kWaveCandidates) cand[nc] = __ldg(sc.bvh_leaf + j);
                            nc++;
                        }
                    }
                    continue;
                }
                const float4* nq = reinterpret_cast<const float4*>(sc.bvh + ref);
                const float4 lx = __ldg(nq), ly = __ldg(nq + 1), lz = __ldg(nq + 2);
                const float4 hx = __ldg(nq + 3), hy = __ldg(nq + 4), hz = __ldg(nq + 5);
                const int4 ch = __ldg(reinterpret_cast<const int4*>(nq + 6));
                const float lox[4] = {lx.x, lx.y, lx.z, lx.w}, loy[4] = {ly.x, ly.y, ly.z, ly.w};
                const float loz[4] = {lz.x, lz.y, lz.z, lz.w}, hix[4] = {hx.x, hx.y, hx.z, hx.w};
                const float hiy[4] = {hy.x, hy.y, hy.z, hy.w}, hiz[4] = {hz.x, hz.y, hz.z, hz.w};
                const int32_t child[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const float ax = (lox[k] - eps - ox)*idx, bx = (hix[k] + eps - ox)*idx;
                    const float ay = (loy[k] - eps - oy)*idy, by = (hiy[k] + eps - oy)*idy;
                    const float az = (loz[k] - eps - oz)*idz, bz = (hiz[k] + eps - oz)*idz;
                    const float tmin = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.0f));
                    const float tmax = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
                    if (tmin <= tmax && child[k] != kBvhEmpty) {
                        if (sp < kBvhStack) stack[sp++] = child[k];
                        else overflow = true;
                    }
                }
            }
            if (sp == 0) {
                w.cand_count[item] = overflow ? kWaveCandidates + 1 : nc;
                item = -1;
            }
            }
        }
    }
}

template <typename Out>
__global__ void __launch_bounds__(256)
wave_resolve_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur, const RayPool nxt) {
    const DevScene& sc = a.scene;
    const uint32_t total = w.counters->total;
    const uint32_t slot = blockIdx.x*blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const bool valid = slot < total;
    const uint32_t max_int = a.max_interactions;
    const uint32_t hist_len = max_int + 1;

    bool survive = false;
    // state of this slot after the step (written to the next pool if it survives)
    int32_t photon = 0, root = 0, n_next = 0, k_draw = 0, err = 0;
    v3 s = mk(0, 0, 0), d = mk(0, 0, 0);
    double lambda = 0.0, tof = 0.0;
    int32_t count = 0;
    if (valid) {
        s = mk(cur.sx[slot], cur.sy[slot], cur.sz[slot]);
        d = mk(cur.dx[slot], cur.dy[slot], cur.dz[slot]);
        count = w.cand_count[slot];
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
            if (count > kWaveCandidates) {
                is = first_intersection_tree(sc, root, s, d);
            } else {
                bool have = false;
                is.leaf = -1;
                const double sd = dot(s, d);
                const int32_t* cand = w.cand + (size_t)slot*kWaveCandidates;
                for (int k = 0; k < count; k++)
                    test_candidate(sc, cand[k], s, d, false, sd, &is, &have);
                if (!have) set_void(&is, s, d);
            }
            const bool hit = is.leaf >= 0;
            const LeafRec* L = hit ? sc.leaf + is.leaf : nullptr;
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
                const double depth = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_ABSORPTION
                                                                  : MLGPU_SURF_INNER_ABSORPTION], lambda, &err);
                const double survival = exp(-is.dist/depth);
                absorbed = draw() > survival;
            }
            if (!hit || absorbed) {
                kind = MLGPU_ABSORPTION_IN_VOID;
            } else {
                const double refl = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFLECTION
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
                    const double n_from = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION
                                                                       : MLGPU_SURF_INNER_REFRACTION], lambda, &err);
                    const double n_to = func_eval(sc, fn[is.outside ? MLGPU_SURF_INNER_REFRACTION
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
                const double n = func_eval(sc, f, lambda, &terr);
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
            if (err) atomicCAS(sc.error_word, 0u, (unsigned int)err);
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
            nxt.photon[o] = photon;
            nxt.sx[o] = s.x; nxt.sy[o] = s.y; nxt.sz[o] = s.z;
            nxt.dx[o] = d.x; nxt.dy[o] = d.y; nxt.dz[o] = d.z;
            nxt.lambda[o] = lambda;
            nxt.tof[o] = tof;
            nxt.root[o] = root;
            nxt.n_int[o] = n_next;
            nxt.k_draw[o] = k_draw;
            nxt.err[o] = err;
        }
    }
}

// counters between the kernels of an iteration
__global__ void wave_after_walk_kernel(WaveCounters* c, uint32_t pool, uint64_t num_photons) {
    const unsigned long long remaining = num_photons - c->next_input;
    const uint32_t room = pool - c->active;
    const uint32_t fresh = (uint32_t)(remaining < room ? remaining : room);
    c->total = c->active + fresh;
    c->next_input += fresh;
    c->next = 0;
}

__global__ void wave_after_resolve_kernel(WaveCounters* c) {
    c->active = c->next;
    c->walk_fetch = 0;
}

}  // namespace

cudaError_t launch_wave_fp64_iteration(const TraceArgs& a, const WaveBuffers& w,
                                       const RayPool& cur, const RayPool& nxt,
                                       int walk_blocks, cudaStream_t s) {
    const int resolve_blocks = (int)((w.pool + 255)/256);
    if (a.in_dtype == MLGPU_F64)
        wave_walk_kernel<double><<<walk_blocks, 256, 0, s>>>(a, w, cur);
    else
        wave_walk_kernel<float><<<walk_blocks, 256, 0, s>>>(a, w, cur);
    wave_after_walk_kernel<<<1, 1, 0, s>>>(w.counters, w.pool, a.num_photons);
    if (a.out_dtype == MLGPU_F64)
        wave_resolve_kernel<double><<<resolve_blocks, 256, 0, s>>>(a, w, cur, nxt);
    else
        wave_resolve_kernel<float><<<resolve_blocks, 256, 0, s>>>(a, w, cur, nxt);
    wave_after_resolve_kernel<<<1, 1, 0, s>>>(w.counters);
    return cudaGetLastError();
}

int wave_fp64_walk_blocks() {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave_walk_kernel<double>, 256, 0);
    if (per_sm < 1) per_sm = 1;
    return per_sm*sms;
}

}  // namespace mlgpu
