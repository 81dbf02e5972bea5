// capi.cu -- the extern "C" entry points of include/merlict_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <functional>
#include <string>
#include <mutex>
#include <vector>

#include "mlgpu_internal.h"

using namespace mlgpu;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(MLGPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define MLGPU_CUDA(call)                                   \
    do {                                                   \
        cudaError_t e_ = (call);                           \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

// A device buffer that grows on demand.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t n) {
        if (n <= bytes) return cudaSuccess;
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&ptr, n);
        if (e == cudaSuccess) bytes = n;
        return e;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
};

// CUDA-event timing of the kernel classes (mlgpu_scene_set_profiling).
// A chain is a run of events recorded on one stream with one kernel class
// between each neighbouring pair; chains stay pending until flushed.
struct Profiler {
    static constexpr int kMaxChain = 6;
    struct Chain {
        int n = 0;                          // events in the chain
        cudaEvent_t ev[kMaxChain];
        int cls[kMaxChain - 1];             // class between ev[k] and ev[k + 1]
        int launches[kMaxChain - 1];
    };
    bool on = false;
    std::vector<Chain> pending;
    std::vector<cudaEvent_t> spare;
    double ms[MLGPU_KERNEL_CLASSES] = {};
    uint64_t launches[MLGPU_KERNEL_CLASSES] = {};

    cudaEvent_t take() {
        if (!spare.empty()) { cudaEvent_t e = spare.back(); spare.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }
    // Takes n events; false (and none taken) if one cannot be created.
    bool take(int n, cudaEvent_t* out) {
        for (int k = 0; k < n; k++) {
            out[k] = take();
            if (!out[k]) {
                for (int j = 0; j < k; j++) spare.push_back(out[j]);
                return false;
            }
        }
        return true;
    }
    void add(const Chain& c) {
        pending.push_back(c);
        if (pending.size() > 4096) flush();   // bounds the pool of events
    }
    // Folds the pending chains into the totals (waits for their last events).
    cudaError_t flush() {
        cudaError_t err = cudaSuccess;
        for (const Chain& c : pending) {
            cudaError_t e = cudaEventSynchronize(c.ev[c.n - 1]);
            for (int k = 0; e == cudaSuccess && k + 1 < c.n; k++) {
                float t = 0.0f;
                e = cudaEventElapsedTime(&t, c.ev[k], c.ev[k + 1]);
                if (e == cudaSuccess) { ms[c.cls[k]] += t; launches[c.cls[k]] += c.launches[k]; }
            }
            if (e != cudaSuccess && err == cudaSuccess) err = e;
            for (int k = 0; k < c.n; k++) spare.push_back(c.ev[k]);
        }
        pending.clear();
        return err;
    }
    cudaError_t reset() {
        const cudaError_t e = flush();
        for (int k = 0; k < MLGPU_KERNEL_CLASSES; k++) { ms[k] = 0.0; launches[k] = 0; }
        return e;
    }
    void release() {
        flush();
        for (cudaEvent_t e : spare) cudaEventDestroy(e);
        spare.clear();
    }
};

}  // namespace

// Whole pieces of an mlgpu_propagate_host batch at most (plus one: the
// first and the last piece are halves).
constexpr int kHostChunks = 4;
constexpr int kHostPieces = kHostChunks + 1;

struct PendingUpload {
    std::vector<char> bytes;
    const void** out;
};

struct mlgpu_scene {
    int device = 0;
    DevScene dev;
    std::vector<void*> owned;        // device allocations of the scene
    std::vector<PendingUpload> pending;   // arrays staged while the scene is built
    void* arena = nullptr;           // the scene's read-only arrays, one allocation
    size_t arena_bytes = 0;
    unsigned int* error_word = nullptr;
    // staging for mlgpu_propagate_host and scratch for binning
    DeviceBuffer staging_in, staging_out, staging_hist, staging_rng, tune_out;
    DeviceBuffer staging_bins;           // counts and time histograms of a host call
    DeviceBuffer order;                  // tracing order of a batch and its sort scratch
    DeviceBuffer queue;                  // the work-queue tracer's counter
    int queue_blocks = 0;                // its resident blocks per SM
    DeviceBuffer corsika;                // bunch counts, offsets and the total
    DeviceBuffer stats;                  // sort buffers of the calibration statistics
    DeviceBuffer signal, signal_pulses, signal_tables;   // signal chain scratch, Func1 tables
    // ray pools of the wavefront tracers
    DeviceBuffer wave;
    WaveCounters* wave_host = nullptr;   // pinned copy of the counters
    WaveCounters* wave_host_dev = nullptr;   // its device address
    int wave_grid = 0;                   // default blocks of the persistent kernels
    // one check period of wavefront iterations as a CUDA graph, recorded on
    // a private stream and replayed on the caller's
    cudaGraphExec_t wave_graph = nullptr;
    cudaStream_t capture_stream = nullptr;
    uint64_t launches = 0;               // kernels launched for this scene
    mlgpu_wavefront_stats wave_stats = {0, 0, 0};
    // mlgpu_propagate_host's pipeline: trace, upload, download and ordering
    // streams; events: the caller's default stream, then per piece its
    // inputs, its sorted records and its results, then the cleared counters
    cudaStream_t host_stream[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t host_event[2 + 3*kMaxFeedChunks] = {};
    Profiler prof;
};

namespace {

// The scene's arrays are staged on the host while the scene is built and
// then copied into one device allocation (the scene arena), so that a single
// L2 access-policy window covers all of them.
template <typename T>
int upload(mlgpu_scene* s, const T* host, size_t count, const T** out) {
    if (count == 0) count = 1;
    PendingUpload u;
    u.bytes.assign(count*sizeof(T), 0);
    if (host) std::memcpy(u.bytes.data(), host, count*sizeof(T));
    u.out = reinterpret_cast<const void**>(out);
    s->pending.push_back(std::move(u));
    return MLGPU_OK;
}

// Allocates the arena, copies the staged arrays in (each on a 256-byte
// boundary) and sets the device pointers.
int finish_uploads(mlgpu_scene* s) {
    size_t total = 0;
    for (const PendingUpload& u : s->pending) total += (u.bytes.size() + 255) & ~size_t(255);
    void* arena = nullptr;
    MLGPU_CUDA(cudaMalloc(&arena, total));
    s->owned.push_back(arena);
    s->arena = arena;
    s->arena_bytes = total;
    std::vector<char> image(total, 0);
    size_t at = 0;
    for (const PendingUpload& u : s->pending) {
        std::memcpy(image.data() + at, u.bytes.data(), u.bytes.size());
        *u.out = static_cast<char*>(arena) + at;
        at += (u.bytes.size() + 255) & ~size_t(255);
    }
    s->pending.clear();
    MLGPU_CUDA(cudaMemcpy(arena, image.data(), total, cudaMemcpyHostToDevice));
    return MLGPU_OK;
}

// Host-side bounds checks of every index the kernels follow.
int validate(const mlgpu_flat_scene* f) {
    if (!f) return fail(MLGPU_ERR_INVALID_ARGUMENT, "flat scene is NULL");
    const int32_t nn = f->num_nodes, nl = f->num_leaves, nf = f->num_functions;
    if (nn < 1) return fail(MLGPU_ERR_INVALID_ARGUMENT, "scene has no nodes");
    if (nl < 0 || nf < 1) return fail(MLGPU_ERR_INVALID_ARGUMENT, "bad leaf or function count");
    if (!f->node_sphere || !f->node_skip || !f->node_leaf || !f->function_offset ||
        !f->function_points)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "missing scene array");
    if (nl > 0 && (!f->leaf_node || !f->leaf_frame2world || !f->leaf_primitive ||
                   !f->leaf_params || !f->leaf_surface || !f->leaf_sensor))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "missing leaf array");
    if (f->node_skip[0] != nn)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "node 0 must be the root of the whole tree");
    for (int32_t i = 0; i < nn; i++) {
        const int32_t k = f->node_skip[i];
        const int32_t leaf = f->node_leaf[i];
        if (k <= i || k > nn)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "node %d: skip %d out of range", i, k);
        if (leaf < -1 || leaf >= nl)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "node %d: leaf %d out of range", i, leaf);
        if ((leaf >= 0) != (k == i + 1))
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "node %d: leaf/subtree mismatch", i);
        if (leaf >= 0 && f->leaf_node[leaf] != i)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "node %d: leaf_node disagrees", i);
        // a frame's bounding sphere is centred on its position
        // (RayAndFrame.cpp:16-24, Frame::position_in_world = the frame-to-
        // world translation); the kernels take a leaf's centre from its
        // transform
        if (leaf >= 0 && f->leaf_frame2world) {
            const double* t = f->leaf_frame2world + 12*(size_t)leaf;
            const double* c = f->node_sphere + 4*(size_t)i;
            if (!(c[0] == t[3] && c[1] == t[7] && c[2] == t[11]))
                return fail(MLGPU_ERR_INVALID_ARGUMENT,
                            "leaf %d: bounding sphere not centred on the frame's position", leaf);
        }
        if (!(f->node_sphere[4*i + 3] >= 0.0))
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "node %d: negative bounding radius", i);
    }
    // merlict binds each sensor to one frame and no two sensors to the same
    // frame (Sensors::assert_no_two_sensors_have_same_frame,
    // Sensors.cpp:84-100); in the flat layout a sensor index on two leaves
    // is the same inconsistency
    if (f->num_sensors < 0) return fail(MLGPU_ERR_INVALID_ARGUMENT, "negative sensor count");
    std::vector<int32_t> leaf_of_sensor((size_t)f->num_sensors, -1);
    for (int32_t l = 0; l < nl; l++) {
        const int32_t sen = f->leaf_sensor[l];
        if (sen < 0 || sen >= f->num_sensors) continue;
        if (leaf_of_sensor[sen] >= 0)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "sensor %d is on leaves %d and %d", sen,
                        leaf_of_sensor[sen], l);
        leaf_of_sensor[sen] = l;
    }
    for (int32_t l = 0; l < nl; l++) {
        const int32_t prim = f->leaf_primitive[l];
        if (prim < 0 || prim >= MLGPU_PRIM_COUNT)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "leaf %d: unknown primitive %d", l, prim);
        const int32_t* su = f->leaf_surface + (size_t)l*MLGPU_SURF_COLUMNS;
        for (int c = 0; c < 6; c++)
            if (su[c] < 0 || su[c] >= nf)
                return fail(MLGPU_ERR_INVALID_ARGUMENT, "leaf %d: table id %d out of range", l, su[c]);
        if (su[MLGPU_SURF_ALLOWED_NODE] < -1 || su[MLGPU_SURF_ALLOWED_NODE] >= nn)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "leaf %d: allowed node out of range", l);
        if (f->leaf_sensor[l] < -1 || f->leaf_sensor[l] >= f->num_sensors)
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "leaf %d: sensor out of range", l);
    }
    if (f->function_offset[0] != 0)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "function offsets must start at 0");
    for (int32_t k = 0; k < nf; k++) {
        const int32_t b = f->function_offset[k], e = f->function_offset[k + 1];
        if (e - b < 1) return fail(MLGPU_ERR_INVALID_ARGUMENT, "function %d is empty", k);
        for (int32_t j = b + 1; j < e; j++)
            if (!(f->function_points[3*j] > f->function_points[3*(j - 1)]))
                return fail(MLGPU_ERR_INVALID_ARGUMENT,
                            "function %d: arguments not strictly increasing", k);
    }
    if (f->default_refraction < 0 || f->default_refraction >= nf)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "default refraction id out of range");
    return MLGPU_OK;
}

int build_device_scene(mlgpu_scene* s, const mlgpu_flat_scene* f) {
    const int32_t nn = f->num_nodes, nl = f->num_leaves, nf = f->num_functions;
    std::vector<double4> node(nn);
    std::vector<int2> meta(nn);
    for (int32_t i = 0; i < nn; i++) {
        const double* c = f->node_sphere + 4*(size_t)i;
        node[i] = make_double4(c[0], c[1], c[2], c[3]*c[3]);
        meta[i] = make_int2(f->node_skip[i], f->node_leaf[i]);
    }
    std::vector<LeafRec> leaf(nl > 0 ? nl : 1);
    std::vector<LeafRecF> leaf_f(nl > 0 ? nl : 1);
    std::vector<LeafAnchor> anchor(nl > 0 ? nl : 1);
    std::memset(anchor.data(), 0, anchor.size()*sizeof(LeafAnchor));
    std::memset(leaf.data(), 0, leaf.size()*sizeof(LeafRec));
    std::memset(leaf_f.data(), 0, leaf_f.size()*sizeof(LeafRecF));
    for (int32_t l = 0; l < nl; l++) {
        LeafRec& L = leaf[l];
        const double* t = f->leaf_frame2world + 12*(size_t)l;
        for (int k = 0; k < 12; k++) L.T[k] = t[k];
        // translation part of HomTra3::position_inverse, HomTra3.cpp:200-216
        L.tinv[0] = t[0]*t[3] + t[4]*t[7] + t[8]*t[11];
        L.tinv[1] = t[1]*t[3] + t[5]*t[7] + t[9]*t[11];
        L.tinv[2] = t[2]*t[3] + t[6]*t[7] + t[10]*t[11];
        for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) L.params[k] = f->leaf_params[MLGPU_LEAF_PARAMS*(size_t)l + k];
        const double r = f->node_sphere[4*(size_t)f->leaf_node[l] + 3];
        L.r2 = r*r;
        L.primitive = f->leaf_primitive[l];
        L.sensor = f->leaf_sensor[l];
        const int32_t* su = f->leaf_surface + (size_t)l*MLGPU_SURF_COLUMNS;
        L.allowed_node = su[MLGPU_SURF_ALLOWED_NODE];
        L.flags = su[MLGPU_SURF_FLAGS];
        for (int k = 0; k < 6; k++) L.fn[k] = su[k];

        LeafRecF& F = leaf_f[l];
        for (int rr = 0; rr < 3; rr++)
            for (int cc = 0; cc < 3; cc++) F.R[3*rr + cc] = (float)t[4*rr + cc];
        for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) F.params[k] = (float)L.params[k];
        F.r2 = (float)L.r2;
        F.primitive = L.primitive;
        F.sensor = L.sensor;
        F.allowed_node = L.allowed_node;
        F.flags = L.flags;
        for (int k = 0; k < 6; k++) F.fn[k] = L.fn[k];
        LeafAnchor& A = anchor[l];
        A.origin[0] = t[3]; A.origin[1] = t[7]; A.origin[2] = t[11];
        if (L.primitive == MLGPU_PRIM_SPHERE_CAP_HEX || L.primitive == MLGPU_PRIM_SPHERE_CAP_CYL ||
            L.primitive == MLGPU_PRIM_SPHERE_CAP_RECT) {
            // the cap's sphere: centre (0, 0, R) in the leaf frame
            const double R = L.params[0];
            A.R = R;
            A.center[0] = t[3] + R*t[2];
            A.center[1] = t[7] + R*t[6];
            A.center[2] = t[11] + R*t[10];
        }
    }
    const int32_t npts = f->function_offset[nf];
    s->dev.num_fn_points = npts;

    int st;
    if ((st = upload(s, node.data(), nn, &s->dev.node))) return st;
    if ((st = upload(s, meta.data(), nn, &s->dev.node_meta))) return st;
    if ((st = upload(s, leaf.data(), leaf.size(), &s->dev.leaf))) return st;
    if ((st = upload(s, f->function_points, 3*(size_t)npts, &s->dev.fn_points))) return st;
    if ((st = upload(s, f->function_offset, (size_t)nf + 1, &s->dev.fn_offset))) return st;
    if ((st = upload(s, leaf_f.data(), leaf_f.size(), &s->dev.leaf_f))) return st;
    if ((st = upload(s, anchor.data(), anchor.size(), &s->dev.leaf_anchor))) return st;
    {
        // BVH over the leaves; boxes widened for single-precision slab tests
        const double* root = f->node_sphere;
        const double extent = std::fabs(root[0]) + std::fabs(root[1]) + std::fabs(root[2]) +
            2.0*root[3];
        BvhHost bvh;
        build_bvh(f, 0.0, &bvh);
        if (!bvh.nodes.empty()) {
            if ((st = upload(s, bvh.nodes.data(), bvh.nodes.size(), &s->dev.bvh))) return st;
            std::vector<QNode> qn(bvh.nodes.size());
            for (size_t j = 0; j < qn.size(); j++) quantise_bvh_node(bvh.nodes[j], &qn[j]);
            if ((st = upload(s, qn.data(), qn.size(), &s->dev.bvh_q))) return st;
            if ((st = upload(s, bvh.leaf_ids.data(), bvh.leaf_ids.size(), &s->dev.bvh_leaf))) return st;
            // merlict's own bounding sphere of each leaf, in BVH order
            std::vector<double4> sph(bvh.leaf_ids.size());
            for (size_t j = 0; j < sph.size(); j++) sph[j] = node[f->leaf_node[bvh.leaf_ids[j]]];
            if ((st = upload(s, sph.data(), sph.size(), &s->dev.bvh_sphere))) return st;
            std::vector<float4> sph_f(sph.size());
            for (size_t j = 0; j < sph.size(); j++) {
                float r = (float)std::sqrt(sph[j].w);
                if ((double)r*(double)r < sph[j].w) r = std::nextafter(r, 3.0e38f);
                sph_f[j] = make_float4((float)sph[j].x, (float)sph[j].y, (float)sph[j].z, r);
            }
            if ((st = upload(s, sph_f.data(), sph_f.size(), &s->dev.bvh_sphere_f))) return st;
            s->dev.bvh_nodes = (int32_t)bvh.nodes.size();
            s->dev.bvh_levels = bvh.levels;
            for (int k = 0; k <= kMaxBvhLevels; k++)
                s->dev.bvh_level_start[k] = k <= bvh.levels ? bvh.level_start[k] : s->dev.bvh_nodes;
        }
        // the candidate records in slot order (the BVH's leaf order; every
        // leaf with geometry has a slot)
        {
            const size_t slots = bvh.leaf_ids.size();
            const size_t blocks = (slots + 7)/8;
            std::vector<double2> rec(blocks*96 > 0 ? blocks*96 : 1, make_double2(0.0, 0.0));
            std::vector<int32_t> leaf_slot(nl > 0 ? nl : 1, -1);
            for (size_t j = 0; j < slots; j++) {
                const double2* r = reinterpret_cast<const double2*>(&leaf[bvh.leaf_ids[j]]);
                for (int pr = 0; pr < 12; pr++) rec[(j >> 3)*96 + pr*8 + (j & 7)] = r[pr];
                leaf_slot[bvh.leaf_ids[j]] = (int32_t)j;
            }
            if ((st = upload(s, rec.data(), rec.size(), &s->dev.slot_rec))) return st;
            std::vector<uint4> rec_f(blocks*72 > 0 ? blocks*72 : 1, make_uint4(0u, 0u, 0u, 0u));
            for (size_t j = 0; j < slots; j++) {
                const uint4* f = reinterpret_cast<const uint4*>(&leaf_f[bvh.leaf_ids[j]]);
                const uint4* an = reinterpret_cast<const uint4*>(&anchor[bvh.leaf_ids[j]]);
                for (int u = 0; u < 5; u++) rec_f[(j >> 3)*72 + u*8 + (j & 7)] = f[u];
                for (int u = 0; u < 4; u++) rec_f[(j >> 3)*72 + (5 + u)*8 + (j & 7)] = an[u];
            }
            if ((st = upload(s, rec_f.data(), rec_f.size(), &s->dev.slot_rec_f))) return st;
            if ((st = upload(s, bvh.leaf_ids.data(), bvh.leaf_ids.size(), &s->dev.slot_leaf))) return st;
            if ((st = upload(s, leaf_slot.data(), leaf_slot.size(), &s->dev.leaf_slot))) return st;
            s->dev.num_slots = (int32_t)slots;
        }
        // a tree deeper than the walk's level queues: merlict's frame walk
        if (s->dev.bvh_levels >= kMaxBvhLevels) {
            s->dev.bvh_nodes = 0;
            s->dev.bvh_levels = 0;
        }
        s->dev.bvh_eps = (float)(1e-6 + 4e-7*extent);
    }
    const unsigned int* ew = nullptr;
    if ((st = upload<unsigned int>(s, nullptr, 1, &ew))) return st;
    if ((st = finish_uploads(s))) return st;
    s->error_word = const_cast<unsigned int*>(ew);
    s->dev.error_word = s->error_word;
    s->dev.num_nodes = nn;
    s->dev.num_leaves = nl;
    s->dev.num_functions = nf;
    s->dev.default_refraction = f->default_refraction;
    s->dev.num_sensors = f->num_sensors;
    for (int k = 0; k < 3; k++) {
        s->dev.hex_u[k] = f->hex_unit_u[k];
        s->dev.hex_v[k] = f->hex_unit_v[k];
        s->dev.hex_w[k] = f->hex_unit_w[k];
    }
    return MLGPU_OK;
}

int check_propagate_args(const mlgpu_scene* scene, const mlgpu_photons* ph,
                         const mlgpu_settings* st, const mlgpu_rng* rng,
                         const mlgpu_results* res) {
    if (!scene || !ph || !st || !rng || !res)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ph->dtype != MLGPU_F64 && ph->dtype != MLGPU_F32)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "photon dtype must be MLGPU_F64 or MLGPU_F32");
    if (res->dtype != MLGPU_F64 && res->dtype != MLGPU_F32)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "result dtype must be MLGPU_F64 or MLGPU_F32");
    if (!ph->support_x || !ph->support_y || !ph->support_z || !ph->direction_x ||
        !ph->direction_y || !ph->direction_z || !ph->wavelength)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "photon plane is NULL");
    if (!res->sensor) return fail(MLGPU_ERR_INVALID_ARGUMENT, "results.sensor is NULL");
    if (st->start_node < 0 || st->start_node >= scene->dev.num_nodes)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "start node %d out of range", st->start_node);
    if (st->max_num_interactions_per_photon > 254)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "max_num_interactions_per_photon must be <= 254");
    if (rng->mode != MLGPU_RNG_PHILOX && rng->mode != MLGPU_RNG_REPLAY)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown rng mode");
    if (rng->mode == MLGPU_RNG_REPLAY && !rng->uniforms)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "replay rng without uniforms");
    if (st->tracer != MLGPU_TRACER_FP64 && st->tracer != MLGPU_TRACER_FP32 &&
        st->tracer != MLGPU_TRACER_FP32_PURE && st->tracer != MLGPU_TRACER_FP64_PLAIN &&
        st->tracer != MLGPU_TRACER_FP64_QUEUE)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown tracer %d", st->tracer);
    if (st->traversal != MLGPU_TRAVERSAL_BVH && st->traversal != MLGPU_TRAVERSAL_FRAME_TREE)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown traversal %d", st->traversal);
    if (st->pool_size > (1u << 24) || (st->pool_size != 0 && st->pool_size < 1024))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "pool_size must be 0 or in [1024, 2^24]");
    if (st->check_period < 0 || st->check_period > 64)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "check_period must be in [0, 64]");
    if (st->grid_blocks < 0 || st->grid_blocks > 65535)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "grid_blocks must be in [0, 65535]");
    if (st->staged_levels < 0 || st->staged_levels > kMaxBvhLevels)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "staged_levels must be in [0, %d]", kMaxBvhLevels);
    if (st->use_graph != 0 && st->use_graph != 1)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "use_graph must be 0 or 1");
    if (st->photon_order < MLGPU_ORDER_DEFAULT || st->photon_order > MLGPU_ORDER_COHERENT)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown photon_order %d", st->photon_order);
    if (st->walk < MLGPU_WALK_DEFAULT || st->walk > MLGPU_WALK_STACK)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown walk %d", st->walk);
    if (st->queue_capacity != 0 && (st->queue_capacity < 32 || st->queue_capacity > (1u << 28)))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "queue_capacity must be 0 or in [32, 2^28]");
    return MLGPU_OK;
}

TraceArgs make_args(const mlgpu_scene* scene, const mlgpu_photons* ph, uint64_t n,
                    const mlgpu_settings* st, const mlgpu_rng* rng, const mlgpu_results* res) {
    TraceArgs a;
    std::memset(&a, 0, sizeof(a));
    a.scene = scene->dev;
    a.photons.sx = ph->support_x; a.photons.sy = ph->support_y; a.photons.sz = ph->support_z;
    a.photons.dx = ph->direction_x; a.photons.dy = ph->direction_y; a.photons.dz = ph->direction_z;
    a.photons.wavelength = ph->wavelength;
    a.in_dtype = ph->dtype;
    a.results.sensor = res->sensor;
    a.results.x = res->x; a.results.y = res->y; a.results.time = res->time;
    a.results.theta_x = res->theta_x; a.results.theta_y = res->theta_y;
    a.results.final_leaf = res->final_leaf; a.results.info = res->info;
    a.results.final_position = res->final_position;
    a.results.final_direction = res->final_direction;
    a.results.history = res->history;
    a.out_dtype = res->dtype;
    a.rng.mode = rng->mode; a.rng.stride = rng->stride; a.rng.seed = rng->seed;
    a.rng.photon_offset = rng->photon_offset; a.rng.uniforms = rng->uniforms;
    a.num_photons = n;
    a.max_interactions = st->max_num_interactions_per_photon;
    a.start_node = st->start_node;
    a.traversal = st->traversal;
    return a;
}

constexpr uint32_t kWavePool = 1u << 21;   // ray slots of the wavefront tracers

// Carves the two ray pools, the candidate lists and the counters out of
// one device buffer.
int wave_buffers(mlgpu_scene* scene, uint32_t pool, int grid, int staged, uint32_t queue_cap,
                 WaveBuffers* w, RayPool* p0, RayPool* p1) {
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t P = pool;
    const size_t level_cap = queue_cap ? queue_cap : 8*P;
    const size_t isect_cap = queue_cap ? queue_cap : 16*P;
    const size_t per_pool = up(P*48) + 3*up(P*8) + 8*up(P*4) + 2*up(P*16);
    const size_t rest = 2*up(level_cap*8) + up(isect_cap*8) + up(isect_cap*8) + up(P*4);
    MLGPU_CUDA(scene->wave.reserve(kWaveCounterBytes + 2*per_pool + rest));
    if (!scene->wave_host) MLGPU_CUDA(cudaMallocHost(&scene->wave_host, sizeof(WaveCounters)));
    if (!scene->wave_host_dev)
        MLGPU_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&scene->wave_host_dev),
                                            scene->wave_host, 0));
    if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
    char* b = static_cast<char*>(scene->wave.ptr);
    w->counters = reinterpret_cast<WaveCounters*>(b);
    b += kWaveCounterBytes;
    auto take = [&](size_t bytes) { char* p = b; b += up(bytes); return p; };
    RayPool* pools[2] = {p0, p1};
    for (RayPool* p : pools) {
        p->sd = reinterpret_cast<double2*>(take(P*48));
        p->lambda = reinterpret_cast<double*>(take(P*8));
        p->tof = reinterpret_cast<double*>(take(P*8));
        p->best_key = reinterpret_cast<unsigned long long*>(take(P*8));
        int32_t** i[7] = {&p->photon, &p->root, &p->n_int, &p->k_draw, &p->err, &p->step,
                          &p->best_leaf};
        for (int32_t** q : i) *q = reinterpret_cast<int32_t*>(take(P*4));
        p->overflow_flag = reinterpret_cast<uint32_t*>(take(P*4));
        p->ray_o = reinterpret_cast<float4*>(take(P*16));
        p->ray_i = reinterpret_cast<float4*>(take(P*16));
    }
    w->pool = pool;
    w->grid = grid > 0 ? grid : scene->wave_grid;
    w->staged_levels = staged;
    w->level_q[0] = reinterpret_cast<uint2*>(take(level_cap*8));
    w->level_q[1] = reinterpret_cast<uint2*>(take(level_cap*8));
    w->level_cap = (uint32_t)level_cap;
    w->isect_q = reinterpret_cast<uint2*>(take(isect_cap*8));
    w->slot_leaf_of = scene->dev.slot_leaf;
    w->isect_dist = reinterpret_cast<double*>(take(isect_cap*8));
    w->isect_cap = (uint32_t)isect_cap;
    w->overflow = reinterpret_cast<uint32_t*>(take(P*4));
    const size_t fn_bytes = (size_t)scene->dev.num_fn_points*3*sizeof(double) +
        ((size_t)scene->dev.num_functions + 1)*sizeof(int32_t);
    w->fn_smem_bytes = fn_bytes <= 16384 ? (int)fn_bytes : 0;
    return MLGPU_OK;
}

// Records `period` wavefront iterations (starting from ray pool 0) and the
// copy of the counters to the host as one CUDA graph, on the scene's private
// stream, and makes it the scene's executable graph (updated in place when
// the previous one has the same shape).
int record_wave_graph(mlgpu_scene* scene, const TraceArgs& a, const WaveBuffers& w,
                      const RayPool* pools, int form, int period) {
    if (!scene->capture_stream)
        MLGPU_CUDA(cudaStreamCreateWithFlags(&scene->capture_stream, cudaStreamNonBlocking));
    cudaStream_t cs = scene->capture_stream;
    MLGPU_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int g = 0; g < period && e == cudaSuccess; g++)
        e = launch_wave_iteration(a, w, pools[g & 1], pools[(g + 1) & 1], form, cs, nullptr);
    if (e == cudaSuccess) e = launch_wave_counters_to_host(w.counters, scene->wave_host_dev, cs);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cs, &graph);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return cuda_fail(e != cudaSuccess ? e : e2, "recording the wavefront graph");
    }
    bool updated = false;
    if (scene->wave_graph) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(scene->wave_graph, graph, &info) == cudaSuccess) updated = true;
        else {
            cudaGetLastError();
            cudaGraphExecDestroy(scene->wave_graph);
            scene->wave_graph = nullptr;
        }
    }
    if (!updated) e = cudaGraphInstantiate(&scene->wave_graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        scene->wave_graph = nullptr;
        return cuda_fail(e, "instantiating the wavefront graph");
    }
    return MLGPU_OK;
}

// Runs iterations of a wavefront tracer until every photon has finished,
// checking the counters on the host after every `check_period` iterations
// (one CUDA-graph launch per period with use_graph).  `form` selects the
// intersection arithmetic (FP64 or one of the FP32 forms).
// The order in which a batch's photons enter the tracers: coherent (a sort
// by support and direction, photon_order.cu) or the input order (a.order
// and a.sorted stay null).  With `records` the coherent order comes as the
// photons themselves, sorted into 64-byte records (a.sorted) that the
// wavefront intake reads in sequence, up to 2^28 photons (16 GiB of
// records); otherwise, and beyond that, as photon indices (a.order).
int tracing_order(mlgpu_scene* scene, TraceArgs* a, const mlgpu_settings* st,
                  cudaStream_t stream, bool records) {
    const bool coherent = a->num_photons < (1ull << 32) &&
        (st->photon_order == MLGPU_ORDER_COHERENT ||
         (st->photon_order == MLGPU_ORDER_DEFAULT && a->num_photons >= 65536));
    if (!coherent) return MLGPU_OK;
    const bool rec = records && a->num_photons <= (1ull << 28);
    const size_t obytes = (size_t)a->num_photons*(rec ? 4*sizeof(double2) : sizeof(uint32_t));
    MLGPU_CUDA(scene->order.reserve(obytes + 256 + photon_order_scratch_bytes(a->num_photons)));
    char* scratch = static_cast<char*>(scene->order.ptr) + ((obytes + 255) & ~size_t(255));
    if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
    uint32_t* order = rec ? nullptr : static_cast<uint32_t*>(scene->order.ptr);
    double2* sorted = rec ? static_cast<double2*>(scene->order.ptr) : nullptr;
    const cudaError_t e = launch_photon_order(a->photons, a->in_dtype, a->num_photons, order,
                                              sorted, 0, scratch, scene->wave_grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "photon order kernels");
    scene->launches += 7;
    a->order = order;
    a->sorted = sorted;
    return MLGPU_OK;
}

// A fed propagation (mlgpu_propagate_host's pipeline): the batch's photon
// planes arrive on the device piece by piece (in_ready[c] fires when piece
// c's planes are there); each piece is sorted into its records on the
// ordering stream and published to the tracer, and `download(c)` is called
// once every photon of piece c has finished.
struct FeedPlan {
    int pieces;
    uint64_t start[kMaxFeedChunks + 1];   // piece c: photons [start[c], start[c + 1])
    const void* planes[7];                // the whole batch's device planes
    cudaStream_t order;
    const cudaEvent_t* in_ready;
    const cudaEvent_t* ord_ready;
    cudaEvent_t ctr_ready;
    double2* records;
    void* scratch;                        // photon_order_scratch_bytes of the largest piece
    std::function<int(int)> download;
};

int run_wavefront(mlgpu_scene* scene, TraceArgs a, const mlgpu_settings* st,
                  cudaStream_t stream, const FeedPlan* feed = nullptr) {
    const int form = st->tracer;
    if (feed) {
        a.sorted = feed->records;
        a.order = nullptr;
        a.fed = 1;
        a.feed_chunks = feed->pieces;
        for (int c = 0; c <= feed->pieces; c++) a.feed_start[c] = feed->start[c];
    } else {
        const int ro = tracing_order(scene, &a, st, stream, true);
        if (ro) return ro;
    }
    const uint32_t want = st->pool_size ? st->pool_size : kWavePool;
    const uint32_t pool = (uint32_t)std::min<uint64_t>(a.num_photons, want);
    WaveBuffers w;
    RayPool pools[2];
    const int rc = wave_buffers(scene, pool, st->grid_blocks, st->staged_levels,
                                st->queue_capacity, &w, &pools[0], &pools[1]);
    if (rc) return rc;
    w.walk = st->walk == MLGPU_WALK_STACK ? MLGPU_WALK_STACK : MLGPU_WALK_LEVELS;
    // per-kernel events cannot be taken inside a graph: profiling runs launch by launch
    const bool graph = st->use_graph != 0 && !scene->prof.on;
    int period = st->check_period > 0 ? st->check_period : 4;
    if (graph && (period & 1)) period++;   // a graph starts and ends on ray pool 0
    if (graph) {
        const int r = record_wave_graph(scene, a, w, pools, form, period);
        if (r) return r;
    }
    MLGPU_CUDA(cudaMemsetAsync(w.counters, 0, sizeof(WaveCounters), stream));
    bool downloaded[kMaxFeedChunks] = {};
    if (feed) {
        // each piece: sorted into its records once its planes are on the
        // device, then published; the tracer starts with the first piece
        MLGPU_CUDA(cudaEventRecord(feed->ctr_ready, stream));
        MLGPU_CUDA(cudaStreamWaitEvent(feed->order, feed->ctr_ready, 0));
        const size_t ein = a.in_dtype == MLGPU_F64 ? 8 : 4;
        for (int c = 0; c < feed->pieces; c++) {
            const uint64_t a0 = feed->start[c], len = feed->start[c + 1] - a0;
            MLGPU_CUDA(cudaStreamWaitEvent(feed->order, feed->in_ready[c], 0));
            DevPhotons p;
            const void** dp[7] = {&p.sx, &p.sy, &p.sz, &p.dx, &p.dy, &p.dz, &p.wavelength};
            for (int k = 0; k < 7; k++)
                *dp[k] = static_cast<const char*>(feed->planes[k]) + a0*ein;
            cudaError_t e = launch_photon_order(p, a.in_dtype, len, nullptr, feed->records + 4*a0,
                                                a0, feed->scratch, scene->wave_grid, feed->order);
            if (e == cudaSuccess) e = launch_feed_publish(w.counters, a0 + len, feed->order);
            if (e == cudaSuccess) e = cudaEventRecord(feed->ord_ready[c], feed->order);
            if (e != cudaSuccess) return cuda_fail(e, "ordering a piece");
            scene->launches += 8;
        }
        MLGPU_CUDA(cudaStreamWaitEvent(stream, feed->ord_ready[0], 0));
        MLGPU_CUDA(launch_feed_snapshot(w.counters, stream));
        scene->launches++;
    }
    // every iteration advances each live photon by one step
    const uint64_t bound = (a.num_photons*(uint64_t)(a.max_interactions + 1))/pool +
        a.max_interactions + 16 + (uint64_t)period*(feed ? feed->pieces + 1 : 1);
    // launches per iteration: intake and its counters, the walk, intersections
    // and ties, the overflow walk, resolve and its counters
    const int walk_launches = w.walk == MLGPU_WALK_STACK ? 1 : scene->dev.bvh_levels;
    uint64_t iteration = 0;
    while (true) {
        if (graph) {
            MLGPU_CUDA(cudaGraphLaunch(scene->wave_graph, stream));
            iteration += (uint64_t)period;
            scene->launches += (uint64_t)period*((uint64_t)walk_launches + 7) + 1;
        } else {
            for (int g = 0; g < period; g++, iteration++) {
                const RayPool& cur = pools[iteration & 1];
                const RayPool& nxt = pools[(iteration + 1) & 1];
                Profiler::Chain ch;
                const bool timed = scene->prof.on && scene->prof.take(5, ch.ev);
                const cudaError_t e = launch_wave_iteration(a, w, cur, nxt, form, stream,
                                                            timed ? ch.ev : nullptr);
                if (e != cudaSuccess) return cuda_fail(e, "wavefront kernels");
                scene->launches += (uint64_t)walk_launches + 7;
                if (timed) {
                    ch.n = 5;
                    const int cls[4] = {MLGPU_KERNEL_INTAKE, MLGPU_KERNEL_WALK,
                                        MLGPU_KERNEL_INTERSECT, MLGPU_KERNEL_RESOLVE};
                    const int launches[4] = {2, walk_launches, 2, 3};
                    for (int k = 0; k < 4; k++) { ch.cls[k] = cls[k]; ch.launches[k] = launches[k]; }
                    scene->prof.add(ch);
                }
            }
            const cudaError_t e = launch_wave_counters_to_host(w.counters, scene->wave_host_dev,
                                                               stream);
            if (e != cudaSuccess) return cuda_fail(e, "wavefront counters");
            scene->launches++;
        }
        MLGPU_CUDA(cudaStreamSynchronize(stream));
        const WaveCounters& h = *scene->wave_host;
        if (feed) {
            // pieces whose photons have all finished go back to the host
            for (int c = 0; c < feed->pieces; c++) {
                if (downloaded[c] || h.done[c] < feed->start[c + 1] - feed->start[c]) continue;
                downloaded[c] = true;
                const int r = feed->download(c);
                if (r) return r;
            }
            // an empty pool with the next piece still on its way: the trace
            // stream waits for that piece (no kernel spins on it)
            if (h.active == 0 && h.next_input == h.avail_snap && h.next_input < a.num_photons) {
                int c = 0;
                while (c + 1 < feed->pieces && feed->start[c + 1] <= h.next_input) c++;
                MLGPU_CUDA(cudaStreamWaitEvent(stream, feed->ord_ready[c], 0));
                MLGPU_CUDA(launch_feed_snapshot(w.counters, stream));
                scene->launches++;
            }
        }
        if (h.active == 0 && h.next_input >= a.num_photons) break;
        if (iteration > bound)
            return fail(MLGPU_ERR_RUNTIME, "wavefront tracer did not drain its pool");
    }
    scene->wave_stats.calls++;
    scene->wave_stats.iterations += iteration;
    scene->wave_stats.overflow_rays += scene->wave_host->overflow_total;
    return MLGPU_OK;
}

int launch(mlgpu_scene* scene, const TraceArgs& a, const mlgpu_settings* st,
           cudaStream_t stream) {
    cudaError_t e;
    switch (st->tracer) {
    case MLGPU_TRACER_FP64:
    case MLGPU_TRACER_FP32:
    case MLGPU_TRACER_FP32_PURE: return run_wavefront(scene, a, st, stream);
    case MLGPU_TRACER_FP64_QUEUE: {
        TraceArgs q = a;
        const int ro = tracing_order(scene, &q, st, stream, false);
        if (ro) return ro;
        MLGPU_CUDA(scene->queue.reserve(256));
        int sms = 0, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (!scene->queue_blocks) scene->queue_blocks = queue_trace_blocks_per_sm();
        const int grid = st->grid_blocks > 0 ? st->grid_blocks : sms*scene->queue_blocks;
        Profiler::Chain ch;
        const bool timed = scene->prof.on && scene->prof.take(2, ch.ev);
        if (timed) cudaEventRecord(ch.ev[0], stream);
        e = launch_queue_trace(q, static_cast<unsigned long long*>(scene->queue.ptr), grid,
                               stream);
        scene->launches++;
        if (timed) {
            cudaEventRecord(ch.ev[1], stream);
            ch.n = 2; ch.cls[0] = MLGPU_KERNEL_PLAIN; ch.launches[0] = 1;
            scene->prof.add(ch);
        }
        break;
    }
    default: {
        Profiler::Chain ch;
        const bool timed = scene->prof.on && scene->prof.take(2, ch.ev);
        if (timed) cudaEventRecord(ch.ev[0], stream);
        e = launch_trace_fp64(a, st->block_size, stream);
        scene->launches++;
        if (timed) {
            cudaEventRecord(ch.ev[1], stream);
            ch.n = 2; ch.cls[0] = MLGPU_KERNEL_PLAIN; ch.launches[0] = 1;
            scene->prof.add(ch);
        }
        break;
    }
    }
    if (e != cudaSuccess) return cuda_fail(e, "trace kernel launch");
    return MLGPU_OK;
}

const char* device_error_text(unsigned int code) {
    switch (code) {
    case MLGPU_ERR_INVALID_ARGUMENT:
        return "Expected photon wavelength lambda > 0.0nm (Photon.cpp:20-28), but a "
               "photon's wavelength is <= 0";
    case MLGPU_ERR_OUT_OF_RANGE:
        return "a photon's wavelength is outside the argument range of a surface "
               "property table (Func1 limits [x_first, x_last))";
    case MLGPU_ERR_RUNTIME:
        return "a photon consumed more uniforms than its replay stream holds";
    default:
        return "device-side error";
    }
}

}  // namespace

namespace mlgpu {

int report_error(int code, const char* message) { return fail(code, "%s", message); }

const DevScene* device_scene(const mlgpu_scene* scene) { return &scene->dev; }

int scene_device(const mlgpu_scene* scene) { return scene->device; }

void profile_mark_begin(mlgpu_scene* scene, cudaStream_t s, ProfileMark* mark) {
    mark->timed = scene->prof.on && scene->prof.take(2, mark->ev);
    if (mark->timed) cudaEventRecord(mark->ev[0], s);
}

void profile_mark_end(mlgpu_scene* scene, cudaStream_t s, ProfileMark* mark, int cls,
                      int launches) {
    if (mark->timed) {
        cudaEventRecord(mark->ev[1], s);
        Profiler::Chain ch;
        ch.n = 2;
        ch.ev[0] = mark->ev[0];
        ch.ev[1] = mark->ev[1];
        ch.cls[0] = cls;
        ch.launches[0] = launches;
        scene->prof.add(ch);
    }
    scene->launches += (uint64_t)launches;
}

}  // namespace mlgpu

extern "C" {

int mlgpu_abi_version(void) { return MLGPU_ABI_VERSION; }

int mlgpu_host_alloc(uint64_t bytes, void** ptr) {
    if (!ptr) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    *ptr = nullptr;
    if (bytes == 0) return MLGPU_OK;
    const cudaError_t e = cudaMallocHost(ptr, bytes);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        return cuda_fail(e, "cudaMallocHost");
    }
    return MLGPU_OK;
}

int mlgpu_host_free(void* ptr) {
    if (!ptr) return MLGPU_OK;
    const cudaError_t e = cudaFreeHost(ptr);
    if (e != cudaSuccess) return cuda_fail(e, "cudaFreeHost");
    return MLGPU_OK;
}

int mlgpu_last_error(char* buffer, size_t buffer_size) {
    if (!buffer || buffer_size == 0) return (int)g_last_error.size();
    std::snprintf(buffer, buffer_size, "%s", g_last_error.c_str());
    return (int)g_last_error.size();
}

int mlgpu_scene_create(const mlgpu_flat_scene* flat, mlgpu_scene** scene) {
    if (!scene) return fail(MLGPU_ERR_INVALID_ARGUMENT, "scene out-pointer is NULL");
    *scene = nullptr;
    int st = validate(flat);
    if (st) return st;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return fail(MLGPU_ERR_NO_DEVICE, "no CUDA device is visible");
    mlgpu_scene* s = new mlgpu_scene;
    std::memset(&s->dev, 0, sizeof(s->dev));
    cudaGetDevice(&s->device);
    st = build_device_scene(s, flat);
    if (st) {
        mlgpu_scene_destroy(s);
        return st;
    }
    *scene = s;
    return MLGPU_OK;
}

int mlgpu_scene_destroy(mlgpu_scene* scene) {
    if (!scene) return MLGPU_OK;
    for (void* p : scene->owned) cudaFree(p);
    scene->staging_in.release();
    scene->staging_out.release();
    scene->staging_hist.release();
    scene->staging_rng.release();
    scene->staging_bins.release();
    scene->tune_out.release();
    scene->order.release();
    scene->queue.release();
    scene->corsika.release();
    scene->stats.release();
    scene->wave.release();
    if (scene->wave_host) cudaFreeHost(scene->wave_host);
    if (scene->wave_graph) cudaGraphExecDestroy(scene->wave_graph);
    if (scene->capture_stream) cudaStreamDestroy(scene->capture_stream);
    for (cudaStream_t hs : scene->host_stream)
        if (hs) cudaStreamDestroy(hs);
    for (cudaEvent_t he : scene->host_event)
        if (he) cudaEventDestroy(he);
    scene->prof.release();
    delete scene;
    return MLGPU_OK;
}

int mlgpu_propagate(mlgpu_scene* scene, const mlgpu_photons* photons, uint64_t num_photons,
                    const mlgpu_settings* settings, const mlgpu_rng* rng,
                    mlgpu_results* results, void* cuda_stream) {
    int st = check_propagate_args(scene, photons, settings, rng, results);
    if (st) return st;
    if (num_photons == 0) return MLGPU_OK;
    const TraceArgs a = make_args(scene, photons, num_photons, settings, rng, results);
    return launch(scene, a, settings, static_cast<cudaStream_t>(cuda_stream));
}

int mlgpu_scene_autotune(mlgpu_scene* scene, const mlgpu_photons* sample, uint64_t n,
                         const mlgpu_settings* base, const mlgpu_rng* rng,
                         mlgpu_settings* best, double* best_ms, void* cuda_stream) {
    if (!best) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    mlgpu_results res;
    std::memset(&res, 0, sizeof(res));
    res.dtype = MLGPU_F64;
    res.sensor = reinterpret_cast<int32_t*>(1);   // checked below against NULL only
    int st = check_propagate_args(scene, sample, base, rng, &res);
    if (st) return st;
    if (n == 0) return fail(MLGPU_ERR_INVALID_ARGUMENT, "empty sample");
    if (base->tracer == MLGPU_TRACER_FP64_PLAIN)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "only the wavefront tracers have knobs to tune");
    MLGPU_CUDA(scene->tune_out.reserve(4*n));
    res.sensor = static_cast<int32_t*>(scene->tune_out.ptr);
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    const bool prof = scene->prof.on;
    scene->prof.on = false;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    MLGPU_CUDA(cudaEventCreate(&ev[0]));
    MLGPU_CUDA(cudaEventCreate(&ev[1]));
    // times one setting: best of two runs after an untimed one
    auto time_of = [&](const mlgpu_settings& cand, double* ms) -> int {
        const TraceArgs a = make_args(scene, sample, n, &cand, rng, &res);
        double t_best = 1e300;
        for (int rep = 0; rep < 3; rep++) {
            if (cudaEventRecord(ev[0], stream) != cudaSuccess) return cuda_fail(cudaGetLastError(), "event");
            const int r = launch(scene, a, &cand, stream);
            if (r) return r;
            if (cudaEventRecord(ev[1], stream) != cudaSuccess) return cuda_fail(cudaGetLastError(), "event");
            const cudaError_t e = cudaEventSynchronize(ev[1]);
            if (e != cudaSuccess) return cuda_fail(e, "autotune run");
            float t = 0.0f;
            cudaEventElapsedTime(&t, ev[0], ev[1]);
            if (rep > 0) t_best = std::min(t_best, (double)t);
        }
        *ms = t_best;
        return MLGPU_OK;
    };
    int sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    mlgpu_settings cur = *base;
    cur.pool_size = 0; cur.check_period = 0; cur.use_graph = 1; cur.grid_blocks = 0;
    cur.staged_levels = 0;
    cur.photon_order = MLGPU_ORDER_DEFAULT;
    cur.walk = MLGPU_WALK_DEFAULT;
    double cur_ms = 0.0;
    st = time_of(cur, &cur_ms);
    // candidate values of each knob, tried one knob at a time
    const uint32_t pools[] = {1u << 19, 1u << 20, 1u << 21, 1u << 22};
    const int periods[] = {2, 4, 8, 16};
    const int grids[] = {4*sms, 8*sms, 16*sms};
    const int stages[] = {0, 3, 5};
    const int graphs[] = {0, 1};
    const int orders[] = {MLGPU_ORDER_INPUT, MLGPU_ORDER_COHERENT};
    const int walks[] = {MLGPU_WALK_LEVELS, MLGPU_WALK_STACK};
    for (int pass = 0; pass < 2 && st == MLGPU_OK; pass++) {
        const double start_ms = cur_ms;
        for (int knob = 0; knob < 7 && st == MLGPU_OK; knob++) {
            const int count = knob <= 1 ? 4 : knob <= 3 ? 3 : 2;
            for (int c = 0; c < count && st == MLGPU_OK; c++) {
                mlgpu_settings cand = cur;
                switch (knob) {
                case 0:
                    if (pools[c] > 2*n && c > 0) continue;   // larger than the sample
                    cand.pool_size = pools[c];
                    break;
                case 1: cand.check_period = periods[c]; break;
                case 2: cand.grid_blocks = grids[c]; break;
                case 3: cand.staged_levels = stages[c]; break;
                case 4: cand.use_graph = graphs[c]; break;
                case 5: cand.photon_order = orders[c]; break;
                default: cand.walk = walks[c]; break;
                }
                if (std::memcmp(&cand, &cur, sizeof(cand)) == 0) continue;
                double ms = 0.0;
                st = time_of(cand, &ms);
                if (st == MLGPU_OK && ms < cur_ms) { cur = cand; cur_ms = ms; }
            }
        }
        if (cur_ms > 0.98*start_ms) break;   // the pass gained little
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    scene->prof.on = prof;
    if (st) return st;
    *best = cur;
    if (best_ms) *best_ms = cur_ms;
    return MLGPU_OK;
}

int mlgpu_corsika_photons(mlgpu_scene* scene, const float* bunches, uint64_t n,
                          const int32_t* bunch_ids, const mlgpu_rng* rng,
                          mlgpu_photon_buffers* out, uint64_t* num_photons, void* cuda_stream) {
    if (!scene || !rng || !out || !num_photons)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    *num_photons = 0;
    if (n == 0) return MLGPU_OK;
    if (!bunches) return fail(MLGPU_ERR_INVALID_ARGUMENT, "bunches is NULL");
    if (rng->mode != MLGPU_RNG_PHILOX && rng->mode != MLGPU_RNG_REPLAY)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "unknown rng mode");
    if (rng->mode == MLGPU_RNG_REPLAY && !rng->uniforms)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "replay rng without uniforms");
    double* planes[7] = {out->support_x, out->support_y, out->support_z, out->direction_x,
                         out->direction_y, out->direction_z, out->wavelength};
    for (double* p : planes)
        if (!p) return fail(MLGPU_ERR_INVALID_ARGUMENT, "photon buffer is NULL");
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    MLGPU_CUDA(scene->corsika.reserve(corsika_scratch_bytes(n) + 256));
    if (!scene->wave_host) MLGPU_CUDA(cudaMallocHost(&scene->wave_host, sizeof(WaveCounters)));
    if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
    char* base = static_cast<char*>(scene->corsika.ptr);
    uint64_t* total_dev = reinterpret_cast<uint64_t*>(base);
    void* scratch = base + 256;
    DevRng r;
    r.mode = rng->mode; r.stride = rng->stride; r.seed = rng->seed;
    r.photon_offset = rng->photon_offset; r.uniforms = rng->uniforms;
    MLGPU_CUDA(cudaMemsetAsync(scene->error_word, 0, sizeof(unsigned int), stream));
    cudaError_t e = launch_corsika_count(bunches, n, r, scratch, total_dev, scene->error_word,
                                         scene->wave_grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "bunch count kernels");
    scene->launches += 4;
    // the total and the error word, back on the host (pinned staging)
    uint64_t* host = reinterpret_cast<uint64_t*>(scene->wave_host);
    MLGPU_CUDA(cudaMemcpyAsync(host, total_dev, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
    MLGPU_CUDA(cudaMemcpyAsync(host + 1, scene->error_word, sizeof(unsigned int),
                               cudaMemcpyDeviceToHost, stream));
    MLGPU_CUDA(cudaStreamSynchronize(stream));
    const uint64_t total = host[0];
    const unsigned int err = static_cast<unsigned int>(host[1] & 0xffffffffu);
    if (err) {
        MLGPU_CUDA(cudaMemset(scene->error_word, 0, sizeof(unsigned int)));
        return fail(MLGPU_ERR_INVALID_ARGUMENT,
                    "a bunch weight is outside [0, 16] (EventIoPhotonFactory::assert_bunch_weight)");
    }
    *num_photons = total;
    if (total > out->capacity)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "the bunches give %llu photons, the buffers hold %llu",
                    (unsigned long long)total, (unsigned long long)out->capacity);
    e = launch_corsika_expand(bunches, n, bunch_ids, scratch, planes, out->simulation_truth_id,
                              scene->wave_grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "bunch expansion kernel");
    scene->launches += 1;
    return MLGPU_OK;
}

int mlgpu_lixel_statistics(mlgpu_scene* scene, const int32_t* sensor, const float* cx,
                           const float* cy, const float* x, const float* y,
                           const float* time_delay, uint64_t n, double emitted,
                           float* statistics, void* cuda_stream) {
    if (!scene || !statistics) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (n > 0 && (!sensor || !cx || !cy || !x || !y || !time_delay))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL photon array");
    if (n >= (1ull << 31))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 photons per call");
    if (!(emitted > 0.0))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "photons_emitted_per_lixel must be > 0");
    const size_t bytes = lixel_stats_scratch_bytes(n);
    MLGPU_CUDA(scene->stats.reserve(bytes));
    if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
    const float* values[5] = {cx, cy, x, y, time_delay};
    const cudaError_t e = launch_lixel_stats(sensor, values, n, (uint32_t)scene->dev.num_sensors,
                                             emitted, statistics, scene->stats.ptr,
                                             scene->stats.bytes, scene->wave_grid,
                                             static_cast<cudaStream_t>(cuda_stream));
    if (e != cudaSuccess) return cuda_fail(e, "calibration statistics");
    scene->launches += 3;
    return MLGPU_OK;
}

int mlgpu_signal_chain(mlgpu_scene* scene, const mlgpu_signal_chain_config* cfg,
                       const int32_t* sensor, const double* arrival_time,
                       const double* wavelength, const int32_t* truth_id, uint64_t n,
                       const float* lixel_efficiency, uint32_t num_sensors, const mlgpu_rng* rng,
                       mlgpu_photon_stream* out, void* cuda_stream) {
    if (!scene || !cfg || !rng || !out) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    out->num_pulses = 0;
    out->nsb_exposure_start_time = 0.0;
    if (n > 0 && (!sensor || !arrival_time || !wavelength || !truth_id))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL photon array");
    if (n >= (1ull << 31))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "at most 2^31 - 1 photons per event");
    if (num_sensors > 0 && !lixel_efficiency)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "lixel_efficiency is NULL");
    if (!out->channel_offset || (out->capacity > 0 && (!out->arrival_time_slice ||
                                                        !out->simulation_truth_id)))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "photon stream buffer is NULL");
    if (rng->mode != MLGPU_RNG_PHILOX)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "the signal chain draws from the Philox streams");
    if (!(cfg->probability_for_second_puls < 1.0))
        return fail(MLGPU_ERR_INVALID_ARGUMENT,
                    "Expected config->probability_for_second_puls < 1.0, but actual it is: %g",
                    cfg->probability_for_second_puls);
    if (!cfg->quantum_efficiency || cfg->num_quantum_efficiency < 2 || !cfg->nsb_wavelength_cdf ||
        cfg->num_nsb_wavelength_cdf < 2)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "a Func1 table needs at least two points");
    if (cfg->num_lixel == 0 || !(cfg->time_slice_duration != 0.0))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "num_lixel and time_slice_duration must not be 0");
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    // the two Func1 tables, on the device
    const size_t nq = cfg->num_quantum_efficiency, nc = cfg->num_nsb_wavelength_cdf;
    MLGPU_CUDA(scene->signal_tables.reserve(3*(nq + nc)*sizeof(double)));
    double* tab = static_cast<double*>(scene->signal_tables.ptr);
    MLGPU_CUDA(cudaMemcpyAsync(tab, cfg->quantum_efficiency, 3*nq*sizeof(double),
                               cudaMemcpyHostToDevice, stream));
    MLGPU_CUDA(cudaMemcpyAsync(tab + 3*nq, cfg->nsb_wavelength_cdf, 3*nc*sizeof(double),
                               cudaMemcpyHostToDevice, stream));
    MLGPU_CUDA(scene->signal.reserve(signal_chain_photon_scratch_bytes(n, num_sensors)));
    if (!scene->wave_host) MLGPU_CUDA(cudaMallocHost(&scene->wave_host, sizeof(WaveCounters)));
    if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
    SignalChainArgs a;
    a.sensor = sensor; a.time = arrival_time; a.wavelength = wavelength; a.truth = truth_id;
    a.num_photons = n; a.efficiency = lixel_efficiency; a.num_sensors = num_sensors;
    a.seed = rng->seed; a.offset = rng->photon_offset;
    a.params.qe = tab; a.params.num_qe = (int32_t)nq;
    a.params.cdf = tab + 3*nq; a.params.num_cdf = (int32_t)nc;
    a.params.dark_rate = cfg->dark_rate;
    a.params.second_puls = cfg->probability_for_second_puls;
    a.params.total_integral = cfg->nsb_total_integral;
    a.params.nsb_rate = cfg->nsb_rate;
    a.params.num_lixel = (double)cfg->num_lixel;
    a.params.exposure_time = cfg->nsb_exposure_time;
    a.params.time_slice_duration = cfg->time_slice_duration;
    a.params.arrival_time_std = cfg->arrival_time_std;
    a.channel_offset = out->channel_offset;
    a.slice = out->arrival_time_slice;
    a.slice_truth = out->simulation_truth_id;
    a.nsb_count = out->nsb_count;
    a.err = scene->error_word;
    MLGPU_CUDA(cudaMemsetAsync(scene->error_word, 0, sizeof(unsigned int), stream));
    const uint64_t* total_dev = nullptr;
    const double* start_dev = nullptr;
    cudaError_t e = launch_signal_chain_count(a, scene->signal.ptr, scene->signal.bytes,
                                              scene->wave_grid, stream, &total_dev, &start_dev);
    if (e != cudaSuccess) return cuda_fail(e, "signal chain kernels");
    scene->launches += 10;
    // the electric pulses, the window start and the error word, on the host
    uint64_t* host = reinterpret_cast<uint64_t*>(scene->wave_host);
    auto read_back = [&](const uint64_t* count_dev) -> int {
        MLGPU_CUDA(cudaMemcpyAsync(host, count_dev, sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                   stream));
        MLGPU_CUDA(cudaMemcpyAsync(host + 1, start_dev, sizeof(double), cudaMemcpyDeviceToHost,
                                   stream));
        MLGPU_CUDA(cudaMemcpyAsync(host + 2, scene->error_word, sizeof(unsigned int),
                                   cudaMemcpyDeviceToHost, stream));
        MLGPU_CUDA(cudaStreamSynchronize(stream));
        const unsigned int err = static_cast<unsigned int>(host[2] & 0xffffffffu);
        if (!err) return MLGPU_OK;
        MLGPU_CUDA(cudaMemset(scene->error_word, 0, sizeof(unsigned int)));
        return fail((int)err, "signal chain: %s",
                    err == MLGPU_ERR_OUT_OF_RANGE
                        ? "a wavelength is outside the quantum efficiency table or a draw outside "
                          "the background's wavelength distribution (Func1 limits)"
                    : err == MLGPU_ERR_INVALID_ARGUMENT
                        ? "a photon's sensor index is not below num_sensors"
                        : "a lixel needs more draws than one Philox stream holds");
    };
    int st = read_back(total_dev);
    if (st) return st;
    const uint64_t electric = host[0];
    double start = 0.0;
    std::memcpy(&start, host + 1, sizeof(double));
    out->nsb_exposure_start_time = start;
    if (electric >= (1ull << 31))
        return fail(MLGPU_ERR_RUNTIME, "more than 2^31 - 1 electric pulses in one event");
    const size_t pulse_bytes = signal_chain_pulse_scratch_bytes(electric);
    MLGPU_CUDA(scene->signal_pulses.reserve(pulse_bytes));
    const uint64_t* kept_dev = nullptr;
    e = launch_signal_chain_extract(a, scene->signal.ptr, scene->signal.bytes,
                                    scene->signal_pulses.ptr, scene->signal_pulses.bytes, electric,
                                    scene->wave_grid, stream, &kept_dev);
    if (e != cudaSuccess) return cuda_fail(e, "signal chain extraction kernels");
    scene->launches += 6;
    // the kept pulses fit when the electric ones do; otherwise look first
    uint64_t kept = electric;
    const bool look_first = electric > out->capacity;
    if (look_first) {
        st = read_back(kept_dev);
        if (st) return st;
        kept = host[0];
        if (kept > out->capacity) {
            out->num_pulses = kept;
            return fail(MLGPU_ERR_INVALID_ARGUMENT,
                        "the event gives %llu pulses, the buffers hold %llu",
                        (unsigned long long)kept, (unsigned long long)out->capacity);
        }
    }
    e = launch_signal_chain_scatter(a, scene->signal_pulses.ptr, scene->signal_pulses.bytes,
                                    electric, scene->wave_grid, stream);
    if (e != cudaSuccess) return cuda_fail(e, "signal chain scatter kernel");
    scene->launches += 1;
    if (!look_first) {
        st = read_back(kept_dev);
        if (st) return st;
        kept = host[0];
    }
    out->num_pulses = kept;
    return MLGPU_OK;
}

int mlgpu_scene_sync_errors(mlgpu_scene* scene, void* cuda_stream) {
    if (!scene) return fail(MLGPU_ERR_INVALID_ARGUMENT, "scene is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    MLGPU_CUDA(cudaStreamSynchronize(s));
    unsigned int code = 0;
    MLGPU_CUDA(cudaMemcpy(&code, scene->error_word, sizeof(code), cudaMemcpyDeviceToHost));
    if (code) {
        MLGPU_CUDA(cudaMemset(scene->error_word, 0, sizeof(unsigned int)));
        return fail((int)code, "%s", device_error_text(code));
    }
    return MLGPU_OK;
}

}  // extern "C"

namespace {

// Per-sensor binning requested with a host-buffer propagation.
struct HostBinning {
    uint32_t* counts;        // host [num_sensors]
    uint32_t* time_hist;     // host [num_sensors][num_bins] or null
    uint32_t num_bins;
    double t_min, t_max;
};

int propagate_host(mlgpu_scene* scene, const mlgpu_photons* photons, uint64_t n,
                   const mlgpu_settings* settings, const mlgpu_rng* rng,
                   mlgpu_results* results, const HostBinning* bin) {
    int st = check_propagate_args(scene, photons, settings, rng, results);
    if (st) return st;
    if (bin) {
        if (!bin->counts) return fail(MLGPU_ERR_INVALID_ARGUMENT, "counts is NULL");
        if (bin->num_bins > 0 && (!bin->time_hist || !results->time || !(bin->t_max > bin->t_min)))
            return fail(MLGPU_ERR_INVALID_ARGUMENT,
                        "time histograms need results.time, an output and t_max > t_min");
        const uint64_t keys = (uint64_t)scene->dev.num_sensors*(bin->num_bins + 1ull);
        if (keys >= (1ull << 31))
            return fail(MLGPU_ERR_INVALID_ARGUMENT, "too many sensor x time bins");
    }
    if (n == 0) {
        if (bin) {
            std::memset(bin->counts, 0, sizeof(uint32_t)*(size_t)scene->dev.num_sensors);
            if (bin->num_bins)
                std::memset(bin->time_hist, 0,
                            sizeof(uint32_t)*(size_t)scene->dev.num_sensors*bin->num_bins);
        }
        return MLGPU_OK;
    }
    const size_t ein = photons->dtype == MLGPU_F64 ? 8 : 4;
    const size_t eout = results->dtype == MLGPU_F64 ? 8 : 4;
    const size_t hist_len = settings->max_num_interactions_per_photon + 1;
    const size_t hist_row = hist_len*sizeof(mlgpu_history_entry);
    const size_t stride = rng->mode == MLGPU_RNG_REPLAY ? rng->stride : 0;
    const void* planes[7] = {photons->support_x, photons->support_y, photons->support_z,
                             photons->direction_x, photons->direction_y, photons->direction_z,
                             photons->wavelength};
    // result planes: host pointer and bytes per photon
    struct Plane { void* host; size_t bytes; };
    const Plane back[] = {
        {results->sensor, 4}, {results->x, eout}, {results->y, eout}, {results->time, 8},
        {results->theta_x, eout}, {results->theta_y, eout}, {results->final_leaf, 4},
        {results->info, 4}, {results->final_position, 24}, {results->final_direction, 24},
        {results->history, hist_row},
    };
    constexpr int kPlanes = sizeof(back)/sizeof(back[0]);

    // device staging: the input planes one after another, the result planes
    // each on a 256-byte boundary
    MLGPU_CUDA(scene->staging_in.reserve(7*ein*n));
    size_t out_bytes = 0;
    size_t out_off[kPlanes];
    for (int k = 0; k < kPlanes - 1; k++) {
        out_off[k] = out_bytes;
        if (back[k].host) out_bytes += (back[k].bytes*n + 255) & ~size_t(255);
    }
    MLGPU_CUDA(scene->staging_out.reserve(out_bytes + 256));
    if (results->history) MLGPU_CUDA(scene->staging_hist.reserve(n*hist_row));
    if (stride) MLGPU_CUDA(scene->staging_rng.reserve(n*stride*sizeof(double)));
    char* din = static_cast<char*>(scene->staging_in.ptr);
    char* dout = static_cast<char*>(scene->staging_out.ptr);
    void* dev_plane[kPlanes];
    for (int k = 0; k < kPlanes - 1; k++) dev_plane[k] = back[k].host ? dout + out_off[k] : nullptr;
    dev_plane[kPlanes - 1] = results->history ? scene->staging_hist.ptr : nullptr;

    // Pieces of at least one ray pool each, when every host buffer is pinned
    // (copies from pageable memory would not overlap anything)
    auto pinned = [](const void* p) {
        if (!p) return true;
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeHost;
    };
    bool all_pinned = !stride || pinned(rng->uniforms);
    for (const void* p : planes) all_pinned = all_pinned && pinned(p);
    for (const Plane& b : back) all_pinned = all_pinned && pinned(b.host);
    const uint64_t pool = settings->tracer == MLGPU_TRACER_FP64_PLAIN || !settings->pool_size
        ? kWavePool : settings->pool_size;
    // A wavefront form in the coherent order is fed: one propagation over
    // the batch that admits each piece's photons as their sorted records
    // land, pieces of a quarter pool or more, each piece's results going
    // back as soon as its photons have all finished.  Otherwise each piece
    // is a propagation of its own, traced while the next one uploads.
    const bool wavefront = settings->tracer == MLGPU_TRACER_FP64 ||
        settings->tracer == MLGPU_TRACER_FP32 || settings->tracer == MLGPU_TRACER_FP32_PURE;
    const bool coherent = settings->photon_order == MLGPU_ORDER_COHERENT ||
        (settings->photon_order == MLGPU_ORDER_DEFAULT && n >= 65536);
    const bool fed = all_pinned && wavefront && coherent && n >= pool && n <= (1ull << 28);
    const int chunks = !all_pinned ? 1
        : fed ? (int)std::max<uint64_t>(1, std::min<uint64_t>(kMaxFeedChunks - 1, n/(pool/4)))
              : (int)std::max<uint64_t>(1, std::min<uint64_t>(kHostChunks, n/pool));
    // With two or more whole pieces the first and the last are halves: only
    // the first piece's inputs and the last piece's results wait uncovered.
    const int pieces = chunks > 1 ? chunks + 1 : 1;

    if (!scene->host_stream[0]) {
        for (cudaStream_t& hs : scene->host_stream)
            MLGPU_CUDA(cudaStreamCreateWithFlags(&hs, cudaStreamNonBlocking));
        for (cudaEvent_t& he : scene->host_event)
            MLGPU_CUDA(cudaEventCreateWithFlags(&he, cudaEventDisableTiming));
    }
    cudaStream_t trace = scene->host_stream[0], upload = scene->host_stream[1],
                 download = scene->host_stream[2], ordering = scene->host_stream[3];
    cudaEvent_t* in_ready = scene->host_event + 1;
    cudaEvent_t* ord_ready = scene->host_event + 1 + kMaxFeedChunks;
    cudaEvent_t* out_ready = scene->host_event + 1 + 2*kMaxFeedChunks;
    // after the caller's work on the legacy default stream, as a call on it would be
    MLGPU_CUDA(cudaEventRecord(scene->host_event[0], 0));
    MLGPU_CUDA(cudaStreamWaitEvent(upload, scene->host_event[0], 0));
    MLGPU_CUDA(cudaStreamWaitEvent(trace, scene->host_event[0], 0));
    // piece c starts at n * (2c - 1) / (2 chunks), clamped to [0, n]
    auto first = [&](int c) -> uint64_t {
        if (c <= 0) return 0;
        if (c >= pieces) return n;
        return pieces == 1 ? 0 : n*(2*(uint64_t)c - 1)/(2*(uint64_t)chunks);
    };
    // every piece's inputs are queued at once; each piece records its arrival
    for (int c = 0; c < pieces; c++) {
        const uint64_t a0 = first(c), len = first(c + 1) - a0;
        for (int k = 0; k < 7; k++)
            MLGPU_CUDA(cudaMemcpyAsync(din + (k*n + a0)*ein,
                                       static_cast<const char*>(planes[k]) + a0*ein, len*ein,
                                       cudaMemcpyHostToDevice, upload));
        if (stride)
            MLGPU_CUDA(cudaMemcpyAsync(static_cast<double*>(scene->staging_rng.ptr) + a0*stride,
                                       rng->uniforms + a0*stride, len*stride*sizeof(double),
                                       cudaMemcpyHostToDevice, upload));
        MLGPU_CUDA(cudaEventRecord(in_ready[c], upload));
    }
    // a failed piece leaves no copy in flight behind it
    auto drain = [&](int code) {
        cudaStreamSynchronize(upload);
        cudaStreamSynchronize(ordering);
        cudaStreamSynchronize(trace);
        cudaStreamSynchronize(download);
        return code;
    };
    // results of photons [a0, a0 + len) back to the host once the trace
    // stream's work so far is done
    auto results_back = [&](uint64_t a0, uint64_t len) -> int {
        if (cudaEventRecord(out_ready[0], trace) != cudaSuccess ||
            cudaStreamWaitEvent(download, out_ready[0], 0) != cudaSuccess)
            return cuda_fail(cudaGetLastError(), "pipeline event");
        for (int k = 0; k < kPlanes; k++) {
            if (!back[k].host) continue;
            const cudaError_t e = cudaMemcpyAsync(
                static_cast<char*>(back[k].host) + a0*back[k].bytes,
                static_cast<char*>(dev_plane[k]) + a0*back[k].bytes, len*back[k].bytes,
                cudaMemcpyDeviceToHost, download);
            if (e != cudaSuccess) return cuda_fail(e, "copying results to the host");
        }
        return MLGPU_OK;
    };
    if (fed) {
        uint64_t max_len = 0;
        for (int c = 0; c < pieces; c++) max_len = std::max(max_len, first(c + 1) - first(c));
        const size_t rbytes = (size_t)n*4*sizeof(double2);
        if (scene->order.reserve(rbytes + 256 + photon_order_scratch_bytes(max_len)) != cudaSuccess)
            return drain(cuda_fail(cudaGetLastError(), "photon records"));
        if (!scene->wave_grid) scene->wave_grid = wave_persistent_blocks();
        FeedPlan plan;
        plan.pieces = pieces;
        for (int c = 0; c <= pieces; c++) plan.start[c] = first(c);
        for (int k = 0; k < 7; k++) plan.planes[k] = din + k*n*ein;
        plan.order = ordering;
        plan.in_ready = in_ready;
        plan.ord_ready = ord_ready;
        plan.ctr_ready = scene->host_event[1 + 3*kMaxFeedChunks];
        plan.records = static_cast<double2*>(scene->order.ptr);
        plan.scratch = static_cast<char*>(scene->order.ptr) + ((rbytes + 255) & ~size_t(255));
        plan.download = [&](int c) { return results_back(first(c), first(c + 1) - first(c)); };
        mlgpu_photons dph = *photons;
        const void** dp[7] = {&dph.support_x, &dph.support_y, &dph.support_z, &dph.direction_x,
                              &dph.direction_y, &dph.direction_z, &dph.wavelength};
        for (int k = 0; k < 7; k++) *dp[k] = din + k*n*ein;
        dph.simulation_truth_id = nullptr;
        mlgpu_rng drng = *rng;
        if (stride) drng.uniforms = static_cast<const double*>(scene->staging_rng.ptr);
        mlgpu_results dres;
        std::memset(&dres, 0, sizeof(dres));
        dres.dtype = results->dtype;
        dres.sensor = static_cast<int32_t*>(dev_plane[0]);
        dres.x = dev_plane[1];
        dres.y = dev_plane[2];
        dres.time = static_cast<double*>(dev_plane[3]);
        dres.theta_x = dev_plane[4];
        dres.theta_y = dev_plane[5];
        dres.final_leaf = static_cast<int32_t*>(dev_plane[6]);
        dres.info = static_cast<uint32_t*>(dev_plane[7]);
        dres.final_position = static_cast<double*>(dev_plane[8]);
        dres.final_direction = static_cast<double*>(dev_plane[9]);
        dres.history = static_cast<mlgpu_history_entry*>(dev_plane[10]);
        const TraceArgs a = make_args(scene, &dph, n, settings, &drng, &dres);
        st = run_wavefront(scene, a, settings, trace, &plan);
        if (st) return drain(st);
    }
    for (int c = 0; !fed && c < pieces; c++) {
        const uint64_t a0 = first(c), len = first(c + 1) - a0;
        if (cudaStreamWaitEvent(trace, in_ready[c], 0) != cudaSuccess)
            return drain(cuda_fail(cudaGetLastError(), "pipeline event"));
        // photon i of the piece is photon a0 + i of the batch
        mlgpu_photons dph = *photons;
        const void** dp[7] = {&dph.support_x, &dph.support_y, &dph.support_z, &dph.direction_x,
                              &dph.direction_y, &dph.direction_z, &dph.wavelength};
        for (int k = 0; k < 7; k++) *dp[k] = din + (k*n + a0)*ein;
        dph.simulation_truth_id = nullptr;
        mlgpu_rng drng = *rng;
        drng.photon_offset = rng->photon_offset + a0;
        if (stride) drng.uniforms = static_cast<const double*>(scene->staging_rng.ptr) + a0*stride;
        mlgpu_results dres;
        std::memset(&dres, 0, sizeof(dres));
        dres.dtype = results->dtype;
        void* piece[kPlanes];
        for (int k = 0; k < kPlanes; k++)
            piece[k] = dev_plane[k] ? static_cast<char*>(dev_plane[k]) + a0*back[k].bytes : nullptr;
        dres.sensor = static_cast<int32_t*>(piece[0]);
        dres.x = piece[1];
        dres.y = piece[2];
        dres.time = static_cast<double*>(piece[3]);
        dres.theta_x = piece[4];
        dres.theta_y = piece[5];
        dres.final_leaf = static_cast<int32_t*>(piece[6]);
        dres.info = static_cast<uint32_t*>(piece[7]);
        dres.final_position = static_cast<double*>(piece[8]);
        dres.final_direction = static_cast<double*>(piece[9]);
        dres.history = static_cast<mlgpu_history_entry*>(piece[10]);
        const TraceArgs a = make_args(scene, &dph, len, settings, &drng, &dres);
        st = launch(scene, a, settings, trace);
        if (st) return drain(st);
        // the piece's results go back while the next piece is traced
        if (cudaEventRecord(out_ready[c], trace) != cudaSuccess ||
            cudaStreamWaitEvent(download, out_ready[c], 0) != cudaSuccess)
            return drain(cuda_fail(cudaGetLastError(), "pipeline event"));
        for (int k = 0; k < kPlanes; k++) {
            if (!back[k].host) continue;
            const cudaError_t e = cudaMemcpyAsync(static_cast<char*>(back[k].host) + a0*back[k].bytes,
                                                  piece[k], len*back[k].bytes,
                                                  cudaMemcpyDeviceToHost, download);
            if (e != cudaSuccess) return drain(cuda_fail(e, "copying results to the host"));
        }
    }
    if (bin) {
        // the whole batch's sensors (and times) are on the device once the
        // last piece is traced: bin them there, copy the bins back
        const size_t ns = (size_t)scene->dev.num_sensors;
        const size_t keys = ns*(bin->num_bins + 1ull);
        if (scene->staging_bins.reserve(keys*sizeof(uint32_t)) != cudaSuccess)
            return drain(cuda_fail(cudaGetLastError(), "binning buffers"));
        uint32_t* dcounts = static_cast<uint32_t*>(scene->staging_bins.ptr);
        uint32_t* dhist = bin->num_bins ? dcounts + ns : nullptr;
        cudaError_t e = launch_bin_arrivals(
            scene->dev, static_cast<const int32_t*>(dev_plane[0]),
            static_cast<const double*>(dev_plane[3]), n, dcounts, dhist, bin->num_bins,
            bin->t_min, bin->t_max, trace);
        if (e != cudaSuccess) return drain(cuda_fail(e, "binning kernels"));
        scene->launches += 2;
        e = cudaMemcpyAsync(bin->counts, dcounts, ns*sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            trace);
        if (e == cudaSuccess && dhist)
            e = cudaMemcpyAsync(bin->time_hist, dhist, ns*bin->num_bins*sizeof(uint32_t),
                                cudaMemcpyDeviceToHost, trace);
        if (e != cudaSuccess) return drain(cuda_fail(e, "copying bins to the host"));
    }
    const cudaError_t e = cudaStreamSynchronize(download);
    if (e != cudaSuccess) return drain(cuda_fail(e, "copying results to the host"));
    return mlgpu_scene_sync_errors(scene, trace);
}

}  // namespace

extern "C" {

int mlgpu_propagate_host(mlgpu_scene* scene, const mlgpu_photons* photons, uint64_t n,
                         const mlgpu_settings* settings, const mlgpu_rng* rng,
                         mlgpu_results* results) {
    return propagate_host(scene, photons, n, settings, rng, results, nullptr);
}

int mlgpu_propagate_and_bin_host(mlgpu_scene* scene, const mlgpu_photons* photons, uint64_t n,
                                 const mlgpu_settings* settings, const mlgpu_rng* rng,
                                 mlgpu_results* results, uint32_t* counts, uint32_t* time_hist,
                                 uint32_t num_time_bins, double t_min, double t_max) {
    const HostBinning bin = {counts, time_hist, num_time_bins, t_min, t_max};
    return propagate_host(scene, photons, n, settings, rng, results, &bin);
}

int mlgpu_bin_arrivals(mlgpu_scene* scene, const int32_t* sensor, const double* time,
                       uint64_t n, uint32_t* counts, uint32_t* time_hist,
                       uint32_t num_time_bins, double t_min, double t_max,
                       void* cuda_stream) {
    if (!scene || !sensor || !counts)
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (num_time_bins > 0 && (!time || !time_hist || !(t_max > t_min)))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "time histogram needs times, output and t_max > t_min");
    const uint64_t keys = (uint64_t)scene->dev.num_sensors * (num_time_bins + 1ull);
    if (keys >= (1ull << 31))
        return fail(MLGPU_ERR_INVALID_ARGUMENT, "too many sensor x time bins");
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    Profiler::Chain ch;
    const bool timed = scene->prof.on && scene->prof.take(2, ch.ev);
    if (timed) cudaEventRecord(ch.ev[0], stream);
    const cudaError_t e = launch_bin_arrivals(
        scene->dev, sensor, time, n, counts, num_time_bins ? time_hist : nullptr,
        num_time_bins, t_min, t_max, stream);
    if (timed) {
        cudaEventRecord(ch.ev[1], stream);
        ch.n = 2; ch.cls[0] = MLGPU_KERNEL_BIN; ch.launches[0] = 2;
        scene->prof.add(ch);
    }
    if (e != cudaSuccess) return cuda_fail(e, "binning kernels");
    scene->launches += 2;
    return MLGPU_OK;
}

int mlgpu_scene_wavefront_stats(mlgpu_scene* scene, mlgpu_wavefront_stats* stats, int reset) {
    if (!scene) return fail(MLGPU_ERR_INVALID_ARGUMENT, "scene is NULL");
    if (stats) *stats = scene->wave_stats;
    if (reset) scene->wave_stats = mlgpu_wavefront_stats{0, 0, 0};
    return MLGPU_OK;
}

int mlgpu_scene_kernel_launches(const mlgpu_scene* scene, uint64_t* launches) {
    if (!scene || !launches) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    *launches = scene->launches;
    return MLGPU_OK;
}

int mlgpu_scene_set_profiling(mlgpu_scene* scene, int enable) {
    if (!scene) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    const cudaError_t e = scene->prof.reset();
    scene->prof.on = enable != 0;
    if (e != cudaSuccess) return cuda_fail(e, "profiling events");
    return MLGPU_OK;
}

int mlgpu_scene_kernel_times(mlgpu_scene* scene, double* ms, uint64_t* launches) {
    if (!scene) return fail(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    const cudaError_t e = scene->prof.flush();
    if (e != cudaSuccess) return cuda_fail(e, "profiling events");
    for (int k = 0; k < MLGPU_KERNEL_CLASSES; k++) {
        if (ms) ms[k] = scene->prof.ms[k];
        if (launches) launches[k] = scene->prof.launches[k];
    }
    return MLGPU_OK;
}

}  // extern "C"
