// wavefront_fp64.cu -- the wavefront FP64 tracer: merlict's propagation
// (merlict/PhotonAndFrame.cpp:13-124) split into per-step kernels over a
// fixed pool of ray slots, bit-identical to the plain tracer.
//
// One iteration over the pool, every stage a flat loop over uniform work
// items so that a warp's lanes do the same thing:
//   intake     one thread per slot: new photons enter free slots; a ray
//              inside a lens gets merlict's walk of that lens's subtree
//              (RayAndFrame.cpp:137-149), every other ray queues the root
//              of the BVH;
//   levels     one pass per BVH level, one thread per (ray, node) pair: the
//              eight child boxes; hit children go to the next level's queue;
//              the leaves of hit leaf ranges that pass a conservative FP32
//              version of merlict's bounding-sphere test become candidates
//              (merlict's exact test follows in the intersection step);
//   (or walk   one thread per ray: levels and sphere tests in one
//              depth-first walk with a stack, the same candidates;)
//   intersect, ties, overflow, resolve: wave_resolve.cuh.
// The arithmetic is the shared FP64 code, compiled with --fmad=false.
#include <cstdint>

#include "wave_resolve.cuh"

namespace mlgpu {
namespace {

constexpr int kTreeCands = 16;   // candidates of a frame-tree walk before it overflows
// staged nodes of a level: 20 KB of shared memory per block, which with the
// level kernel's own 24 KB stays under the 48 KB a block gets by default
constexpr int kMaxStagedNodes = 20480/(int)sizeof(QNode);

// The intake: new photons enter the free slots (merlict::Photon's
// constructor, Ray.cpp:16-20, RayForPropagation.cpp:52-64) and are prepared
// like the survivors the previous resolve step prepared; then every ray of
// the pool is queued -- the BVH root, or the candidates of merlict's own
// walk of its frame subtree (a ray inside a lens, RayAndFrame.cpp:137-149).
template <typename In>
__global__ void __launch_bounds__(256)
wave_intake_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur) {
    const DevScene& sc = a.scene;
    const uint32_t active = w.counters->active;
    const unsigned long long next_input = w.counters->next_input;
    // a fed propagation admits only the photons whose records have arrived
    const unsigned long long limit = a.fed ? w.counters->avail_snap : a.num_photons;
    const unsigned long long remaining = limit - next_input;
    const uint32_t room = w.pool - active;
    const uint32_t fresh = (uint32_t)(remaining < room ? remaining : room);
    const uint32_t total = active + fresh;
    const uint32_t slot = blockIdx.x*blockDim.x + threadIdx.x;
    const uint32_t max_int = a.max_interactions;
    const uint32_t hist_len = max_int + 1;
    bool bvh = false;          // queue the BVH root for this ray
    int nc = 0;                // candidates of a frame-tree walk
    int32_t cand[kTreeCands];
    if (slot < total) {
        int step;
        if (slot >= active) {
            const uint64_t q = next_input + (slot - active);
            uint64_t p;
            v3 s, d;
            double lambda;
            if (a.sorted) {
                // the photon's record in tracing order
                const double2* r = a.sorted + 4*q;
                const double2 r0 = __ldcg(r), r1 = __ldcg(r + 1), r2 = __ldcg(r + 2),
                              r3 = __ldcg(r + 3);
                s = mk(r0.x, r0.y, r1.x);
                d = normalized(mk(r1.y, r2.x, r2.y));
                lambda = r3.x;
                p = (uint64_t)__double_as_longlong(r3.y);
            } else {
                p = a.order ? (uint64_t)__ldg(a.order + q) : q;
                s = mk(load_in<In>(a.photons.sx, p), load_in<In>(a.photons.sy, p),
                       load_in<In>(a.photons.sz, p));
                d = normalized(mk(load_in<In>(a.photons.dx, p), load_in<In>(a.photons.dy, p),
                                  load_in<In>(a.photons.dz, p)));
                lambda = load_in<In>(a.photons.wavelength, p);
            }
            const int32_t root = a.start_node;
            cur.photon[slot] = (int32_t)p;
            store_ray(cur, slot, s, d);
            // Photon::assert_wavelength_is_positive (Photon.cpp:20-28):
            // merlict throws std::invalid_argument before propagating
            if (lambda <= 0.0) raise_error(sc.error_word, MLGPU_ERR_INVALID_ARGUMENT);
            cur.lambda[slot] = lambda;
            cur.tof[slot] = 0.0;
            cur.root[slot] = root;
            cur.n_int[slot] = 1;
            cur.k_draw[slot] = 0;
            cur.err[slot] = 0;
            cur.best_key[slot] = kNoKey;
            cur.best_leaf[slot] = kNoLeaf;
            cur.overflow_flag[slot] = 0u;
            if (a.results.history)
                store_hist(a.results.history + p*hist_len, s, d, 0.0,
                           MLGPU_LEAF_PHOTON_SOURCE, MLGPU_PRODUCTION, dot(d, d) < 0.0);
            step = 1u > max_int ? kNoStep : prepare_walk(a, cur, slot, s, d, root);
            cur.step[slot] = step;
        } else {
            step = cur.step[slot];   // prepared by the previous resolve step
        }
        bvh = step == kStepBvh;
        if (step == kStepTree) {
            // traversal restricted to a frame's subtree (inside a lens):
            // merlict's own walk of that subtree
            v3 s, d;
            load_ray(cur, slot, &s, &d);
            const double sd = dot(s, d);
            const int32_t root = cur.root[slot];
            bool over = false;
            int32_t i = root;
            const int32_t end = __ldg(&sc.node_meta[root].x);
            while (i < end) {
                const double2* np = reinterpret_cast<const double2*>(sc.node + i);
                const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
                const int2 meta = __ldg(&sc.node_meta[i]);
                if (!sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, sd)) {
                    i = meta.x;
                    continue;
                }
                if (meta.y >= 0) {
                    // candidates by slot; a leaf without geometry has none
                    // (and no intersection in merlict either)
                    const int32_t sl = __ldg(sc.leaf_slot + meta.y);
                    if (sl >= 0) {
                        if (nc < kTreeCands) cand[nc++] = sl;
                        else over = true;
                    }
                }
                i++;
            }
            if (over) {
                mark_overflow(w, cur, slot);
                nc = 0;
            }
        }
    }
    // queue the BVH root and the frame-tree candidates (all lanes take part)
    const uint32_t qb = warp_reserve(&w.counters->level_len[0], bvh ? 1u : 0u);
    if (bvh) {
        if (qb < w.level_cap) w.level_q[0][qb] = make_uint2(slot, 0u);
        else mark_overflow(w, cur, slot);
    }
    const uint32_t cb = warp_reserve(&w.counters->isect_len, (uint32_t)nc);
    for (int k = 0; k < nc; k++) {
        if (cb + k < w.isect_cap) w.isect_q[cb + k] = make_uint2(slot, (uint32_t)cand[k]);
        else mark_overflow(w, cur, slot);
    }
}

// The child references of a BVH node, four per int4 (kept in registers).
struct ChildRefs {
    int4 g0, g1;
};
static_assert(kBvhWidth == 8, "ChildRefs holds eight children");

__device__ __forceinline__ int32_t child_ref(const ChildRefs& c, int k) {
    const int4 q = k < 4 ? c.g0 : c.g1;
    switch (k & 3) {
    case 0: return q.x;
    case 1: return q.y;
    case 2: return q.z;
    default: return q.w;
    }
}

// The eight children of a quantised node (QNode, global memory through the
// read-only path or shared memory); their references into `child`.  A bound
// decodes as origin + q * 2^e; the slab distance (bound -+ o.w - o) * iv is
// evaluated as q * (2^e iv) + (origin -+ o.w - o) iv, one fused
// multiply-add per bound (the byte becomes a float by the exponent trick:
// 0x4b0000qq is 2^23 + q).  The rounding of that form stays inside the box
// inflation o.w, which covers several units in the last place of the
// scenery's extent and of the ray's origin.
template <bool kShared>
__device__ __forceinline__ uint32_t qnode_hits(const float4* nq, float4 o, float4 iv,
                                               ChildRefs* child) {
    auto ld = [nq](int k) { return kShared ? nq[k] : __ldg(nq + k); };
    const float4 w0 = ld(0), c0 = ld(1), c1 = ld(2), b0 = ld(3), b1 = ld(4), b2 = ld(5);
    child->g0 = make_int4(__float_as_int(c0.x), __float_as_int(c0.y), __float_as_int(c0.z),
                          __float_as_int(c0.w));
    child->g1 = make_int4(__float_as_int(c1.x), __float_as_int(c1.y), __float_as_int(c1.z),
                          __float_as_int(c1.w));
    const uint32_t ex = __float_as_uint(w0.w);
    const float sx = __uint_as_float((ex & 0xffu) << 23);
    const float sy = __uint_as_float(((ex >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((ex >> 16) & 0xffu) << 23);
    const float Sx = sx*iv.x, Sy = sy*iv.y, Sz = sz*iv.z;
    const float Lx = (w0.x - o.w - o.x)*iv.x, Hx = (w0.x + o.w - o.x)*iv.x;
    const float Ly = (w0.y - o.w - o.y)*iv.y, Hy = (w0.y + o.w - o.y)*iv.y;
    const float Lz = (w0.z - o.w - o.z)*iv.z, Hz = (w0.z + o.w - o.z)*iv.z;
    // bound words: lo x = (b0.x, b0.y), lo y = (b0.z, b0.w), lo z = (b1.x, b1.y),
    // hi x = (b1.z, b1.w), hi y = (b2.x, b2.y), hi z = (b2.z, b2.w)
    const uint32_t lox[2] = {__float_as_uint(b0.x), __float_as_uint(b0.y)};
    const uint32_t loy[2] = {__float_as_uint(b0.z), __float_as_uint(b0.w)};
    const uint32_t loz[2] = {__float_as_uint(b1.x), __float_as_uint(b1.y)};
    const uint32_t hix[2] = {__float_as_uint(b1.z), __float_as_uint(b1.w)};
    const uint32_t hiy[2] = {__float_as_uint(b2.x), __float_as_uint(b2.y)};
    const uint32_t hiz[2] = {__float_as_uint(b2.z), __float_as_uint(b2.w)};
    uint32_t hit = 0;
#pragma unroll
    for (int k = 0; k < kBvhWidth; k++) {
        const int g = k >> 2;
        const uint32_t sel = 0x7540u | (uint32_t)(k & 3);
        auto dq = [sel](uint32_t word) {
            return __uint_as_float(__byte_perm(word, 0x4b000000u, sel)) - 8388608.0f;
        };
        const float ax = __fmaf_rn(dq(lox[g]), Sx, Lx), bx = __fmaf_rn(dq(hix[g]), Sx, Hx);
        const float ay = __fmaf_rn(dq(loy[g]), Sy, Ly), by = __fmaf_rn(dq(hiy[g]), Sy, Hy);
        const float az = __fmaf_rn(dq(loz[g]), Sz, Lz), bz = __fmaf_rn(dq(hiz[g]), Sz, Hz);
        const float tmin = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.0f));
        const float tmax = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fmaxf(az, bz));
        if (tmin <= tmax && child_ref(*child, k) != kBvhEmpty) hit |= 1u << k;
    }
    return hit;
}

// merlict's bounding-sphere test of a leaf (RayAndFrame.cpp:16-107) in
// single precision on the walk's FP32 ray, with the radius widened by the
// rounding of the ray, the centre and the distance along the ray, so that
// every leaf the exact test passes also passes this one.  The FP64 tracer
// then repeats merlict's exact test on each candidate (wave_isect_kernel);
// the FP32 forms keep the candidates this test passes (their extra
// candidates are rejected by the intersection, whose hits lie inside the
// sphere).
__device__ __forceinline__ bool sphere_cull32(float4 c, float4 o, float3 dv) {
    const float wx = c.x - o.x, wy = c.y - o.y, wz = c.z - o.z;
    const float alpha = dv.x*wx + dv.y*wy + dv.z*wz;
    const float m = o.w + 4e-7f*(fabsf(c.x) + fabsf(c.y) + fabsf(c.z) + fabsf(alpha)) + 1e-6f*c.w;
    const float rr = (c.w + m)*(c.w + m);
    const float sx = wx - dv.x*alpha, sy = wy - dv.y*alpha, sz = wz - dv.z*alpha;
    if (sx*sx + sy*sy + sz*sz > rr) return false;
    if (alpha < -m) return wx*wx + wy*wy + wz*wz <= rr;
    return true;
}

// One BVH level: the child boxes of each queued (ray, node) pair, a lane
// per pair.  With `staged` > 0 the block first copies the level's `staged`
// nodes (a contiguous range, the tree being numbered breadth first) into
// shared memory and reads them from there.  (Eight lanes per pair, one child
// each, loads fewer sectors per request but repeats the ray's setup and the
// queue bookkeeping on every lane: measured 1.3x slower in total.)
//
// Hit leaf ranges: their leaves pass a conservative FP32 version of
// merlict's bounding-sphere test (sphere_cull32) or not; those that pass are
// the ray's candidates, queued as (ray slot, leaf slot).  A warp's hit
// ranges are spread over its lanes through shared memory -- one range per
// lane, as many rounds as the warp has ranges / 32 -- so that the up to
// eight tests of a range run beside the other lanes' instead of one lane at
// a time; a range's candidates stay adjacent in the queue, so that the
// intersection kernel reads neighbouring slot records with neighbouring
// threads.
constexpr int kLevelThreads = 256;
constexpr int kLevelWarps = kLevelThreads/32;

struct WalkRay {        // a lane's ray, published to its warp
    float4 o;           // origin, box inflation
    float4 dv;          // direction (from the reciprocal); w: the slot, as bits
};

__global__ void __launch_bounds__(kLevelThreads, 4)
wave_level_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur, int level,
                  int staged) {
    extern __shared__ float4 stage[];
    __shared__ WalkRay s_ray[kLevelWarps][32];
    __shared__ int2 s_range[kLevelWarps][32*kBvhWidth];   // (leaf-range reference, lane)
    const DevScene& sc = a.scene;
    // the ping-pong queues chosen by a select: an index into the parameter
    // array would make the compiler copy the whole parameter block to local
    // memory
    const uint2* in = (level & 1) ? w.level_q[1] : w.level_q[0];
    uint2* out = (level & 1) ? w.level_q[0] : w.level_q[1];
    const uint32_t len = w.counters->level_len[level];
    const uint32_t n = len < w.level_cap ? len : w.level_cap;
    const bool last = level + 1 >= kMaxBvhLevels;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int32_t base = sc.bvh_level_start[level];
    if (staged > 0) {
        const float4* src = reinterpret_cast<const float4*>(sc.bvh_q + base);
        const int words = staged*(int)(sizeof(QNode)/16);
        for (int t = threadIdx.x; t < words; t += blockDim.x) stage[t] = __ldg(src + t);
        __syncthreads();
    }
    for (uint32_t first = warp_first(); first < n; first += gridDim.x*blockDim.x) {
        const uint32_t e = first + (uint32_t)lane;
        uint32_t slot = 0;
        ChildRefs child;
        child.g0 = child.g1 = make_int4(kBvhEmpty, kBvhEmpty, kBvhEmpty, kBvhEmpty);
        uint32_t hit = 0;   // bit k: child k hit
        float4 o = make_float4(0.f, 0.f, 0.f, 0.f), iv = make_float4(1.f, 1.f, 1.f, 0.f);
        if (e < n) {
            const uint2 q = in[e];
            slot = q.x;
            o = cur.ray_o[slot];
            iv = cur.ray_i[slot];
            if ((uint32_t)((int32_t)q.y - base) < (uint32_t)staged)
                hit = qnode_hits<true>(stage + (sizeof(QNode)/16)*((int32_t)q.y - base), o, iv,
                                       &child);
            else
                hit = qnode_hits<false>(reinterpret_cast<const float4*>(sc.bvh_q + q.y), o, iv,
                                        &child);
        }
        uint32_t nn = 0, ranges = 0;   // bit k of ranges: child k is a hit leaf range
#pragma unroll
        for (int k = 0; k < kBvhWidth; k++)
            if (hit & (1u << k)) { if (child_ref(child, k) < 0) ranges |= 1u << k; else nn++; }
        uint32_t nb = warp_reserve(&w.counters->level_len[last ? level : level + 1], last ? 0u : nn);
#pragma unroll
        for (int k = 0; k < kBvhWidth; k++) {
            if (!(hit & (1u << k)) || child_ref(child, k) < 0) continue;
            if (!last && nb < w.level_cap) out[nb] = make_uint2(slot, (uint32_t)child_ref(child, k));
            else mark_overflow(w, cur, slot);
            nb++;
        }
        // the warp's hit leaf ranges, listed in shared memory
        const uint32_t nr = (uint32_t)__popc(ranges);
        uint32_t incl = nr;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(kFull, incl, d);
            if (lane >= d) incl += y;
        }
        const uint32_t total = __shfl_sync(kFull, incl, 31);
        if (total == 0) continue;   // warp-uniform
        s_ray[warp][lane].o = o;
        s_ray[warp][lane].dv = make_float4(1.0f/iv.x, 1.0f/iv.y, 1.0f/iv.z, __uint_as_float(slot));
        uint32_t at = incl - nr;
#pragma unroll
        for (int k = 0; k < kBvhWidth; k++)
            if ((ranges >> k) & 1u) s_range[warp][at++] = make_int2(child_ref(child, k), lane);
        __syncwarp();
        for (uint32_t r0 = 0; r0 < total; r0 += 32) {
            const uint32_t t = r0 + (uint32_t)lane;
            uint32_t pass = 0, src_slot = 0;   // bit j: leaf j of the range
            int32_t start = 0;
            if (t < total) {
                const int2 item = s_range[warp][t];
                const WalkRay rr = s_ray[warp][item.y];
                src_slot = __float_as_uint(rr.dv.w);
                start = (item.x & 0x7fffffff) >> 3;
                const int32_t count = (item.x & 7) + 1;
                const float3 dv = make_float3(rr.dv.x, rr.dv.y, rr.dv.z);
                for (int32_t j = 0; j < count; j++)
                    if (sphere_cull32(__ldg(sc.bvh_sphere_f + start + j), rr.o, dv))
                        pass |= 1u << j;
            }
            uint32_t cb = warp_reserve(&w.counters->isect_len, (uint32_t)__popc(pass));
            while (pass) {
                const int j = __ffs(pass) - 1;
                pass &= pass - 1u;
                // the candidate by its slot (leaf slots follow the BVH's ranges)
                if (cb < w.isect_cap) w.isect_q[cb] = make_uint2(src_slot, (uint32_t)(start + j));
                else mark_overflow(w, cur, src_slot);
                cb++;
            }
        }
        __syncwarp();   // the lists are rewritten by the next round of entries
    }
}

// The whole walk of a ray in one thread: a depth-first walk of the BVH with
// a stack, the same box tests as wave_level_kernel and the same sphere tests
// as wave_sphere_kernel, so the same candidate leaves; they are queued once
// per warp after the walk.  A ray whose stack or candidate list fills up
// goes to merlict's own walk (the overflow kernel).  One thread per ray of
// the root queue; the ray's FP64 state is read when its first leaf range
// is hit.
constexpr int kWalkStack = 3*kMaxBvhLevels + 4;
constexpr int kWalkCands = 32;

template <bool kF32>
__global__ void __launch_bounds__(256)
wave_walk_kernel(const TraceArgs a, const WaveBuffers w, const RayPool cur) {
    const DevScene& sc = a.scene;
    const uint32_t len = w.counters->level_len[0];
    const uint32_t n = len < w.level_cap ? len : w.level_cap;
    const int lane = threadIdx.x & 31;
    for (uint32_t first = warp_first(); first < n; first += gridDim.x*blockDim.x) {
        const uint32_t e = first + (uint32_t)lane;
        uint32_t slot = 0;
        int32_t cand[kWalkCands];
        uint32_t nc = 0;
        bool over = false;
        if (e < n) {
            const uint2 q = w.level_q[0][e];
            slot = q.x;
            const uint32_t root = q.y;
            const float4 o = cur.ray_o[slot], iv = cur.ray_i[slot];
            const float3 dv = make_float3(1.0f/iv.x, 1.0f/iv.y, 1.0f/iv.z);
            v3 s = mk(0, 0, 0), d = mk(0, 0, 0);
            double sd = 0.0;
            bool have_ray = false;
            int32_t stack[kWalkStack];
            int sp = 0;
            stack[sp++] = (int32_t)root;
            while (sp > 0 && !over) {
                ChildRefs child;
                const uint32_t hit = qnode_hits<false>(
                    reinterpret_cast<const float4*>(sc.bvh_q + stack[--sp]), o, iv, &child);
                for (int k = kBvhWidth - 1; k >= 0; k--) {
                    if (!(hit & (1u << k))) continue;
                    const int32_t ref = child_ref(child, k);
                    if (ref >= 0) {
                        if (sp < kWalkStack) stack[sp++] = ref;
                        else over = true;
                        continue;
                    }
                    const int32_t start = (ref & 0x7fffffff) >> 3;
                    const int32_t count = (ref & 7) + 1;
                    if (!kF32 && !have_ray) {
                        load_ray(cur, slot, &s, &d);
                        sd = dot(s, d);
                        have_ray = true;
                    }
                    for (int32_t j = start; j < start + count; j++) {
                        bool pass;
                        if (kF32) {
                            pass = sphere_cull32(__ldg(sc.bvh_sphere_f + j), o, dv);
                        } else {
                            const double2* c = reinterpret_cast<const double2*>(sc.bvh_sphere + j);
                            const double2 c01 = __ldg(c), c23 = __ldg(c + 1);
                            pass = sphere_cull(make_double4(c01.x, c01.y, c23.x, c23.y), s, d, sd);
                        }
                        if (pass) {
                            if (nc < (uint32_t)kWalkCands) cand[nc++] = j;   // the leaf's slot
                            else over = true;
                        }
                    }
                }
            }
        }
        if (over) {
            mark_overflow(w, cur, slot);
            nc = 0;
        }
        const uint32_t cb = warp_reserve(&w.counters->isect_len, nc);
        for (uint32_t k = 0; k < nc; k++) {
            if (cb + k < w.isect_cap) w.isect_q[cb + k] = make_uint2(slot, (uint32_t)cand[k]);
            else mark_overflow(w, cur, slot);
        }
    }
}

// counters between the kernels of an iteration
__global__ void wave_after_intake_kernel(WaveCounters* c, uint32_t pool, uint64_t num_photons,
                                         int fed) {
    const unsigned long long limit = fed ? c->avail_snap : num_photons;
    const unsigned long long remaining = limit - c->next_input;
    const uint32_t room = pool - c->active;
    const uint32_t fresh = (uint32_t)(remaining < room ? remaining : room);
    c->total = c->active + fresh;
    c->next_input += fresh;
    c->next = 0;
}

// The value of avail the next iteration admits photons up to: read once
// here, so that the intake and its counter kernel agree on it.  avail is
// raised by kernels of another stream after the records they publish are
// written, so a fence orders the read before the intake's record reads.
__device__ __forceinline__ void snapshot_avail(WaveCounters* c) {
    c->avail_snap = atomicAdd(&c->avail, 0ull);
    __threadfence();
}

__global__ void wave_after_resolve_kernel(WaveCounters* c, int fed) {
    if (threadIdx.x == 0) {
        if (fed) snapshot_avail(c);
        c->overflow_total += c->overflow_len;
        c->active = c->next;
        c->isect_len = 0;
        c->overflow_len = 0;
    }
    for (int k = threadIdx.x; k < kMaxBvhLevels; k += blockDim.x) c->level_len[k] = 0;
}

// Fed propagation: the records below `avail` are written (by the kernels
// before this one on its stream); raise the counter for the trace stream.
__global__ void feed_publish_kernel(WaveCounters* c, unsigned long long avail) {
    __threadfence();
    atomicMax(&c->avail, avail);
}

__global__ void feed_snapshot_kernel(WaveCounters* c) { snapshot_avail(c); }

// The counters into pinned host memory, stored by the SM rather than moved
// by a copy engine, so that the host's check after a period never queues
// behind bulk copies of results on another stream.
__global__ void wave_counters_to_host_kernel(const WaveCounters* c, WaveCounters* host) {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(c);
    uint32_t* dst = reinterpret_cast<uint32_t*>(host);
    for (int k = threadIdx.x; k < (int)(sizeof(WaveCounters)/4); k += blockDim.x) dst[k] = src[k];
}

}  // namespace

cudaError_t launch_feed_publish(WaveCounters* c, uint64_t avail, cudaStream_t s) {
    feed_publish_kernel<<<1, 1, 0, s>>>(c, (unsigned long long)avail);
    return cudaGetLastError();
}

cudaError_t launch_feed_snapshot(WaveCounters* c, cudaStream_t s) {
    feed_snapshot_kernel<<<1, 1, 0, s>>>(c);
    return cudaGetLastError();
}

cudaError_t launch_wave_counters_to_host(const WaveCounters* c, WaveCounters* host,
                                         cudaStream_t s) {
    wave_counters_to_host_kernel<<<1, 64, 0, s>>>(c, host);
    return cudaGetLastError();
}

cudaError_t launch_wave_iteration(const TraceArgs& a, const WaveBuffers& w, const RayPool& cur,
                                  const RayPool& nxt, int form, cudaStream_t s, cudaEvent_t* ev) {
    const int slot_blocks = (int)((w.pool + 255)/256);
    if (ev) cudaEventRecord(ev[0], s);
    if (a.in_dtype == MLGPU_F64)
        wave_intake_kernel<double><<<slot_blocks, 256, 0, s>>>(a, w, cur);
    else
        wave_intake_kernel<float><<<slot_blocks, 256, 0, s>>>(a, w, cur);
    wave_after_intake_kernel<<<1, 1, 0, s>>>(w.counters, w.pool, a.num_photons, a.fed);
    if (ev) cudaEventRecord(ev[1], s);
    if (w.walk == MLGPU_WALK_STACK) {
        if (form == MLGPU_TRACER_FP64) wave_walk_kernel<false><<<w.grid, 256, 0, s>>>(a, w, cur);
        else wave_walk_kernel<true><<<w.grid, 256, 0, s>>>(a, w, cur);
    } else {
        for (int k = 0; k < a.scene.bvh_levels; k++) {
            const int count = a.scene.bvh_level_start[k + 1] - a.scene.bvh_level_start[k];
            const int staged = k < w.staged_levels && count <= kMaxStagedNodes ? count : 0;
            wave_level_kernel<<<w.grid, 256, (size_t)staged*sizeof(QNode), s>>>(a, w, cur, k,
                                                                                   staged);
        }
    }
    if (ev) cudaEventRecord(ev[2], s);
    if (form == MLGPU_TRACER_FP64) {
        wave_isect_kernel<kIsectFp64><<<w.grid, 256, 0, s>>>(a, w, cur);
        wave_tie_kernel<<<w.grid, 256, 0, s>>>(w, cur);
        if (ev) cudaEventRecord(ev[3], s);
        wave_overflow_kernel<<<148, 128, 0, s>>>(a, w, cur);
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
    wave_after_resolve_kernel<<<1, 64, 0, s>>>(w.counters, a.fed);
    if (ev) cudaEventRecord(ev[4], s);
    return cudaGetLastError();
}

int wave_persistent_blocks() {
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return 8*sms;
}

}  // namespace mlgpu
