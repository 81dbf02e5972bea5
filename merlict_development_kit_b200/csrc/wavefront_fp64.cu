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

#include "wave_resolve.cuh"

namespace mlgpu {
namespace {

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
    int32_t spill = -1;                        // spill row of the current slot
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
                    spill = -1;
                    overflow = false;
                    tree_mode = true;
                    i = root;
                    end = __ldg(&sc.node_meta[root].x);
                } else {
                    sd = dot(s, d);
                    nc = 0;
                    spill = -1;
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
            // appends a candidate: the slot's own 32 entries, then a spill row
            auto push = [&](int32_t leaf) {
                if (nc < kWaveCandidates) {
                    cand[nc] = leaf;
                } else {
                    const int j = nc - kWaveCandidates;
                    if (j == 0) {
                        const uint32_t r = atomicAdd(&w.counters->spill_used, 1u);
                        if (r < kSpillRows) {
                            spill = (int32_t)r;
                            w.spill_slot[r] = (uint32_t)item;
                            w.spill_row[item] = spill;
                        }
                    }
                    if (spill >= 0 && j < kSpillCap) w.spill[(size_t)spill*kSpillCap + j] = leaf;
                }
                nc++;
            };
            // the count the queue sees: > 32 + kSpillCap sends the slot to
            // the overflow walk
            auto final_count = [&]() -> int32_t {
                if (overflow) return kWaveCandidates + kSpillCap + 1;
                if (nc > kWaveCandidates && (spill < 0 || nc > kWaveCandidates + kSpillCap))
                    return kWaveCandidates + kSpillCap + 1;
                return nc;
            };
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
                    if (meta.y >= 0) push(meta.y);
                    i++;
                }
                if (i >= end) {
                    w.cand_count[item] = final_count();
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
                        if (sphere_cull(make_double4(c01.x, c01.y, c23.x, c23.y), s, d, sd))
                            push(__ldg(sc.bvh_leaf + j));
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
                w.cand_count[item] = final_count();
                item = -1;
            }
            }
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
    c->queue_len = 0;
    c->overflow_len = 0;
}

__global__ void wave_after_resolve_kernel(WaveCounters* c) {
    c->active = c->next;
    c->walk_fetch = 0;
    c->spill_used = 0;
}

}  // namespace

cudaError_t launch_wave_iteration(const TraceArgs& a, const WaveBuffers& w, const RayPool& cur,
                                  const RayPool& nxt, int walk_blocks, int form, cudaStream_t s,
                                  cudaEvent_t* ev) {
    const int slot_blocks = (int)((w.pool + 255)/256);
    if (ev) cudaEventRecord(ev[0], s);
    if (a.in_dtype == MLGPU_F64)
        wave_walk_kernel<double><<<walk_blocks, 256, 0, s>>>(a, w, cur);
    else
        wave_walk_kernel<float><<<walk_blocks, 256, 0, s>>>(a, w, cur);
    if (ev) cudaEventRecord(ev[1], s);
    wave_after_walk_kernel<<<1, 1, 0, s>>>(w.counters, w.pool, a.num_photons);
    wave_enqueue_kernel<<<slot_blocks, 256, 0, s>>>(w);
    wave_overflow_kernel<<<kOverflowBlocks, 128, 0, s>>>(a, w, cur);
    if (ev) cudaEventRecord(ev[2], s);
    if (form == MLGPU_TRACER_FP64) {
        wave_isect_kernel<kIsectFp64><<<w.isect_blocks, 256, 0, s>>>(a, w, cur);
        if (ev) cudaEventRecord(ev[3], s);
        if (a.out_dtype == MLGPU_F64)
            wave_resolve_kernel<double, kIsectFp64><<<slot_blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
        else
            wave_resolve_kernel<float, kIsectFp64><<<slot_blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
    } else {
        const cudaError_t e = launch_wave32_isect_resolve(a, w, cur, nxt,
                                                          form == MLGPU_TRACER_FP32_PURE, s,
                                                          ev ? ev[3] : nullptr);
        if (e != cudaSuccess) return e;
    }
    wave_after_resolve_kernel<<<1, 1, 0, s>>>(w.counters);
    if (ev) cudaEventRecord(ev[4], s);
    return cudaGetLastError();
}

int wave_isect_blocks() {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, wave_isect_kernel<kIsectFp64>, 256, 0);
    if (per_sm < 1) per_sm = 1;
    return per_sm*sms;
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
