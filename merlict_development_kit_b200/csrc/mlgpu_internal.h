// mlgpu_internal.h -- device-side scene layout and launch interfaces shared
// by the kernels and the C ABI implementation.
#ifndef MLGPU_INTERNAL_H_
#define MLGPU_INTERNAL_H_

#include <cstddef>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "merlict_b200.h"

namespace mlgpu {

// One leaf surface in 256 bytes (two 128-byte lines).  The first line holds
// what every candidate test needs -- the 3x4 frame-to-world transform, the
// translation part of its inverse, the primitive and sensor -- the second
// the squared bounding radius beside the primitive parameters (so that a
// one-parameter primitive, the lixels and pixels, adds one 16-byte load),
// then the surface's flags and property-table ids.
struct __align__(256) LeafRec {
    double T[12];          // rows of the 3x4 homogeneous transform
    double tinv[3];        // T00*T03 + T10*T13 + T20*T23, ... (HomTra3.cpp:200-216)
    int32_t primitive;
    int32_t sensor;
    double r2;             // bounding sphere radius squared
    double params[MLGPU_LEAF_PARAMS];
    int32_t allowed_node;
    int32_t flags;
    int32_t fn[6];         // outer/inner reflection, refraction, absorption
    int32_t pad[6];
};
static_assert(sizeof(LeafRec) == 256, "LeafRec must be 256 bytes");
static_assert(offsetof(LeafRec, primitive) == 120 && offsetof(LeafRec, r2) == 128 &&
              offsetof(LeafRec, params) == 136, "LeafRec's first line ends with the primitive");

// FP32 image of a leaf for the batched tracer: transform relative to the
// leaf's own origin, parameters in float, 128 bytes.
struct __align__(128) LeafRecF {
    float R[9];            // rotation rows
    float params[MLGPU_LEAF_PARAMS];
    float r2;
    int32_t primitive;
    int32_t sensor;
    int32_t allowed_node;
    int32_t flags;
    int32_t fn[6];
    int32_t pad[2];
};
static_assert(sizeof(LeafRecF) == 128, "LeafRecF must be 128 bytes");

// FP64 anchor of a leaf for the FP32 forms (64 bytes): the leaf's origin
// (the FP32 geometry is relative to it) and, for spherical caps, the world
// centre and radius of the cap's sphere (origin + R * the frame's z axis),
// on which the FP64 Newton step of a cap root is taken.
// Laid out for 16-byte loads: (origin x, y), (origin z, R), (centre x, y),
// (centre z, pad).
struct __align__(64) LeafAnchor {
    double origin[3];
    double R;              // cap curvature radius (0: not a spherical cap)
    double center[3];
    double pad;
};
static_assert(sizeof(LeafAnchor) == 64, "LeafAnchor must be 64 bytes");
static_assert(offsetof(LeafAnchor, R) == 24 && offsetof(LeafAnchor, center) == 32,
              "LeafAnchor fields must sit where the 16-byte loads expect them");

// BVH node of kBvhWidth children: child boxes as [axis][child] (float,
// rounded outwards) and child references: a node index, a leaf range
// (kBvhLeafFlag | start << 3 | count - 1, into DevScene::bvh_leaf) or
// kBvhEmpty.  The kernels read it as 16-byte words, four children at a
// time: word a*G + g holds the low bounds on axis a of children 4g..4g+3,
// word (3 + a)*G + g the high bounds, word 6*G + g their references
// (G = kBvhWidth/4).
constexpr int kBvhWidth = 8;
constexpr int kBvhGroups = kBvhWidth/4;
struct __align__(128) BvhNode {
    float lo[3][kBvhWidth];
    float hi[3][kBvhWidth];
    int32_t child[kBvhWidth];
    int32_t pad[kBvhWidth == 4 ? 4 : 8];
};
static_assert(sizeof(BvhNode) == 32*kBvhWidth, "BvhNode must be 32 bytes per child");
static_assert(offsetof(BvhNode, child) == 6*kBvhGroups*16,
              "BvhNode references must follow the boxes");
// The same node quantised to 96 bytes (the level kernels' copy): per axis
// a float origin (the children's smallest low bound) and a power-of-two
// step 2^e, and per child and axis 8-bit low and high bounds in steps,
// rounded outwards, so that origin + q * 2^e bounds the float box of the
// BvhNode.  Read as six 16-byte words: (origin, the three biased exponents
// in bytes 0-2 of w), the references of children 0-3 and 4-7, then the
// bounds, each axis and side as two words of four children's bytes:
// lo x, lo y | lo z, hi x | hi y, hi z.
struct __align__(16) QNode {
    float origin[3];
    uint32_t exps;
    int32_t child[kBvhWidth];
    uint32_t qlo[3][2];
    uint32_t qhi[3][2];
};
static_assert(sizeof(QNode) == 96 && kBvhWidth == 8, "QNode: six 16-byte words, eight children");
void quantise_bvh_node(const BvhNode& n, QNode* q);

constexpr int32_t kBvhLeafFlag = (int32_t)0x80000000u;
constexpr int32_t kBvhEmpty = 0x7fffffff;
constexpr int kBvhStack = 64;
constexpr int kMaxBvhLevels = 48;

struct DevScene {
    const double4* node;        // x, y, z, radius^2
    const int2* node_meta;      // skip, leaf
    const LeafRec* leaf;
    const double* fn_points;    // (x, y, slope) triplets
    const int32_t* fn_offset;
    // FP32 copies for the batched tracer
    const LeafRecF* leaf_f;
    const LeafAnchor* leaf_anchor;  // [num_leaves] FP64 origin and cap sphere of each leaf
    int32_t num_nodes;
    int32_t num_leaves;
    int32_t num_functions;
    int32_t num_fn_points;      // fn_offset[num_functions]
    int32_t default_refraction;
    int32_t num_sensors;
    double hex_u[3], hex_v[3], hex_w[3];
    unsigned int* error_word;   // first device-side error code
    // BVH over the leaves with geometry (empty: walk the frame tree)
    const BvhNode* bvh;
    const QNode* bvh_q;         // the same nodes quantised (the level kernels read these)
    const int32_t* bvh_leaf;
    // The candidate records: the first 192 bytes of the leaf record of
    // every leaf with geometry, in slot order (the BVH's leaf order), eight
    // slots to a block of 96 double2 holding pair p of slot 8b + i at
    // 96 b + 8 p + i -- the up to eight leaves of a leaf range, tested by
    // neighbouring lanes, share one 128-byte line per pair.
    const double2* slot_rec;
    // The FP32 forms' candidate records in the same slot order: the first
    // 80 bytes of LeafRecF and the 64 of LeafAnchor (origin, R, cap centre)
    // as nine 16-byte units, eight slots to a block of 72, unit u of slot
    // 8 b + i at 72 b + 8 u + i.
    const uint4* slot_rec_f;
    const int32_t* slot_leaf;   // [slots] leaf of each slot
    const int32_t* leaf_slot;   // [num_leaves] slot of each leaf, -1: no geometry
    int32_t num_slots;
    const double4* bvh_sphere;  // per BVH leaf slot: world centre and radius^2 of that leaf
    const float4* bvh_sphere_f; // the same in FP32: centre (rounded) and radius (rounded up)
    int32_t bvh_nodes;
    int32_t bvh_levels;         // node levels of the BVH (nodes of level k are visited by pass k)
    float bvh_eps;              // box inflation per ray: bvh_eps + 4e-7 |origin|_1
    int32_t bvh_level_start[kMaxBvhLevels + 1];   // nodes of level k: [start[k], start[k+1])
};

constexpr int kMaxFeedChunks = 16;   // chunks of a fed propagation

struct DevPhotons {
    const void* sx; const void* sy; const void* sz;
    const void* dx; const void* dy; const void* dz;
    const void* wavelength;
};

struct DevResults {
    int32_t* sensor;
    void* x; void* y;
    double* time;
    void* theta_x; void* theta_y;
    int32_t* final_leaf;
    uint32_t* info;
    double* final_position;
    double* final_direction;
    mlgpu_history_entry* history;
};

struct DevRng {
    int32_t mode;
    uint32_t stride;
    uint64_t seed;
    uint64_t photon_offset;
    const double* uniforms;
};

struct TraceArgs {
    DevScene scene;
    DevPhotons photons;
    int32_t in_dtype;
    DevResults results;
    int32_t out_dtype;
    DevRng rng;
    uint64_t num_photons;
    uint32_t max_interactions;
    int32_t start_node;
    int32_t traversal;          // MLGPU_TRAVERSAL_*
    const uint32_t* order;      // tracing order of the photons, or null (input order)
    // or the photons themselves in tracing order, 64 bytes each (then
    // `order` is null): (sx, sy), (sz, dx), (dy, dz), (wavelength, index bits)
    const double2* sorted;
    // Fed propagation (the host call's pipeline): the records arrive chunk
    // by chunk; the intake admits photons up to WaveCounters::avail_snap
    // instead of num_photons, and finished photons are counted per chunk
    // (chunk c holds the photon indices [feed_start[c], feed_start[c + 1])).
    int32_t fed;
    int32_t feed_chunks;
    uint64_t feed_start[kMaxFeedChunks + 1];
};

struct BvhHost {
    std::vector<BvhNode> nodes;         // breadth first: each level is an index range
    std::vector<int32_t> leaf_ids;
    std::vector<int32_t> level_start;    // levels + 1 entries
    int levels = 0;              // depth of the tree (root alone: 1)
};
void build_bvh(const mlgpu_flat_scene* f, double inflate, BvhHost* out);

// wavefront tracers: a pool of ray slots, two of them (current, next)
struct WaveCounters {
    unsigned long long next_input;   // photons taken into the pool so far
    unsigned int active;             // rays carried over into the current pool
    unsigned int total;              // active + new photons of this iteration
    unsigned int next;               // survivors written to the next pool
    unsigned int isect_len;          // (slot, leaf) candidates to intersect
    unsigned int overflow_len;       // slots sent to merlict's own walk
    unsigned int level_len[kMaxBvhLevels];   // (slot, node) pairs of each BVH level
    unsigned long long overflow_total;       // overflow_len summed over the iterations
    // fed propagation: photons whose records have arrived (raised by the
    // chunks' publish kernels on another stream), its value as the current
    // iteration uses it, and the finished photons of each chunk
    unsigned long long avail;
    unsigned long long avail_snap;
    unsigned int done[kMaxFeedChunks];
};
constexpr size_t kWaveCounterBytes = 512;
static_assert(sizeof(WaveCounters) <= kWaveCounterBytes,
              "the counters sit in the first 512 bytes of the pool");

// One pool of ray slots; two pools alternate between iterations.  The
// resolve step of an iteration writes each surviving ray into the next
// pool ready to walk -- its FP64 record, its FP32 walk record, its cleared
// closest hit and what the intake has to queue for it -- so that the next
// intake only queues survivors and fills the free slots with new photons.
struct RayPool {
    int32_t* photon;
    double2* sd;             // [pool][3] support and direction, one 48-byte record per slot
    double* lambda;
    double* tof;
    int32_t* root;
    int32_t* n_int;
    int32_t* k_draw;
    int32_t* err;            // error | time-of-flight error << 8
    int32_t* step;           // kNoStep, or what to queue: kStepNone, kStepBvh, kStepTree
    float4* ray_o;           // single-precision origin, box inflation (kStepBvh rays)
    float4* ray_i;           // reciprocal direction (kStepBvh rays)
    unsigned long long* best_key;   // smallest hit distance (bits of a positive double)
    int32_t* best_leaf;      // leaf of the closest hit, lowest index on ties
    uint32_t* overflow_flag; // the slot is queued for merlict's own walk
};

struct WaveBuffers {
    WaveCounters* counters;
    uint32_t pool;
    int grid;                // blocks of the persistent (grid-stride) kernels
    int staged_levels;       // BVH levels whose nodes each block stages in shared memory
    int walk;                // MLGPU_WALK_LEVELS or MLGPU_WALK_STACK
    int fn_smem_bytes;       // property tables staged in shared memory (0: read from global)
    uint2* level_q[2];       // (slot, node) pairs, ping-pong between BVH levels
    uint32_t level_cap;
    uint2* isect_q;          // (ray slot, leaf slot) candidates
    const int32_t* slot_leaf_of;   // the scene's slot -> leaf map (DevScene::slot_leaf)
    double* isect_dist;      // distance to each candidate's hit, -1: none
    uint32_t isect_cap;
    uint32_t* overflow;      // [pool] slots for merlict's own walk
};

// One iteration of a wavefront tracer: walk, queue and intersect the
// candidates, resolve.  `form` is MLGPU_TRACER_FP64, _FP32 or _FP32_PURE;
// the FP32 forms' kernels live in wavefront_fp32.cu.
// With `ev` non-null, events ev[0..4] are recorded before the intake, after
// it, after the BVH walk, after the intersections and after the resolve step.
cudaError_t launch_wave_iteration(const TraceArgs& a, const WaveBuffers& w, const RayPool& cur,
                                  const RayPool& nxt, int form, cudaStream_t s, cudaEvent_t* ev);
// The counters to `host`: the device address of pinned host memory.
cudaError_t launch_wave_counters_to_host(const WaveCounters* c, WaveCounters* host,
                                         cudaStream_t s);
// the FP32 forms' intersection and resolve kernels; `mid` (may be null) is
// recorded between them
cudaError_t launch_wave32_isect_resolve(const TraceArgs& a, const WaveBuffers& w,
                                        const RayPool& cur, const RayPool& nxt, bool pure,
                                        cudaStream_t s, cudaEvent_t mid);

cudaError_t launch_trace_fp64(const TraceArgs& a, int block, cudaStream_t s);
// The persistent work-queue tracer (trace_fp64.cu): `grid` blocks of 128
// threads drain the batch through the counter `queue` (zeroed here).
cudaError_t launch_queue_trace(const TraceArgs& a, unsigned long long* queue, int grid,
                               cudaStream_t s);
int queue_trace_blocks_per_sm();
// CORSIKA bunches to photons (corsika.cu): counts and offsets into
// `scratch` (corsika_scratch_bytes), the total to *total_dev; then the
// expansion into the seven FP64 planes.
size_t corsika_scratch_bytes(uint64_t n);
cudaError_t launch_corsika_count(const float* bunches, uint64_t n, const DevRng& rng, void* scratch,
                                 uint64_t* total_dev, unsigned int* err, int grid, cudaStream_t s);
cudaError_t launch_corsika_expand(const float* bunches, uint64_t n, const int32_t* ids,
                                  void* scratch, double* const* planes, int32_t* out_id, int grid,
                                  cudaStream_t s);
// Per-sensor calibration statistics (lixel_stats.cu): `values` = cx, cy,
// x, y, time delay; `out` [num_sensors][12].
size_t lixel_stats_scratch_bytes(uint64_t n);
cudaError_t launch_lixel_stats(const int32_t* sensor, const float* const* values, uint64_t n,
                               uint32_t num_sensors, double emitted, float* out, void* scratch,
                               size_t scratch_bytes, int grid, cudaStream_t s);
// The signal chain after binning for one event (signal_chain.cu).
struct SignalChainParams {
    const double* qe;                // Func1 points (x, y, slope) on the device
    int32_t num_qe;
    const double* cdf;               // the background's inverse wavelength CDF
    int32_t num_cdf;
    double dark_rate, second_puls, total_integral, nsb_rate, num_lixel, exposure_time;
    double time_slice_duration, arrival_time_std;
};
struct SignalChainArgs {
    const int32_t* sensor;
    const double* time;
    const double* wavelength;
    const int32_t* truth;
    uint64_t num_photons;
    const float* efficiency;
    uint32_t num_sensors;
    uint64_t seed, offset;
    SignalChainParams params;
    uint64_t* channel_offset;        // [num_sensors + 1]
    uint8_t* slice;
    int32_t* slice_truth;
    int32_t* nsb_count;              // may be null
    unsigned int* err;
};
// Three launches with two host reads between them: count (the electric
// pulses of the event -> *total_dev), extract (-> *kept_dev, the channel
// offsets), scatter (the kept pulses into the caller's buffers).
size_t signal_chain_photon_scratch_bytes(uint64_t n, uint32_t num_sensors);
size_t signal_chain_pulse_scratch_bytes(uint64_t num_pulses);
cudaError_t launch_signal_chain_count(const SignalChainArgs& a, void* scratch, size_t bytes,
                                      int grid, cudaStream_t s, const uint64_t** total_dev,
                                      const double** start_dev);
cudaError_t launch_signal_chain_extract(const SignalChainArgs& a, void* scratch, size_t bytes,
                                        void* pulse_scratch, size_t pulse_bytes,
                                        uint64_t num_pulses, int grid, cudaStream_t s,
                                        const uint64_t** kept_dev);
cudaError_t launch_signal_chain_scatter(const SignalChainArgs& a, void* pulse_scratch,
                                        size_t pulse_bytes, uint64_t num_pulses, int grid,
                                        cudaStream_t s);
// A coherent tracing order of a photon batch (photon_order.cu): `order`
// receives n photon indices or, when `sorted` is not null, `sorted` receives
// the photons themselves in that order (TraceArgs::sorted's 64-byte
// records; `order` is then unused); `scratch` holds
// photon_order_scratch_bytes(n).
size_t photon_order_scratch_bytes(uint64_t n);
cudaError_t launch_photon_order(const DevPhotons& p, int in_dtype, uint64_t n, uint32_t* order,
                                double2* sorted, uint64_t index_base, void* scratch, int grid,
                                cudaStream_t s);
// Fed propagation: raises WaveCounters::avail to `avail` once the work
// before it on `s` is done; copies avail into avail_snap.
cudaError_t launch_feed_publish(WaveCounters* c, uint64_t avail, cudaStream_t s);
cudaError_t launch_feed_snapshot(WaveCounters* c, cudaStream_t s);
int wave_persistent_blocks();
// device_sort.cu: a stable LSD radix sort of (key, value) pairs on the low
// key_bits bits of the keys (ping-pong through key_tmp/val_tmp; `temp`
// holds radix_sort_temp_bytes(n)), exclusive sums into 64-bit offsets
// (`temp`: exclusive_sum_temp_bytes(n); in and out may be the same array
// for the 64-bit form), and a sort of each listed run [begin[t], end[t])
// of a segmented array by (64-bit key, value) into key_out/val_out (key_in
// and val_in are overwritten; empty runs are skipped).
size_t radix_sort_temp_bytes(uint64_t n);
cudaError_t radix_sort_pairs(const uint32_t* key_in, const uint32_t* val_in, uint32_t* key_out,
                             uint32_t* val_out, uint32_t* key_tmp, uint32_t* val_tmp, uint64_t n,
                             int key_bits, void* temp, cudaStream_t s);
size_t exclusive_sum_temp_bytes(uint64_t n);
cudaError_t exclusive_sum_u64(const uint64_t* in, uint64_t* out, uint64_t n, void* temp,
                              cudaStream_t s);
cudaError_t exclusive_sum_u32(const uint32_t* in, uint64_t* out, uint64_t n, void* temp,
                              cudaStream_t s);
cudaError_t sort_long_runs(uint64_t* key_in, uint32_t* val_in, uint64_t* key_out,
                           uint32_t* val_out, const uint64_t* begin, const uint64_t* end,
                           uint32_t runs, cudaStream_t s);
// A counting sort by keys in [0, keys): index_out receives the input
// indices grouped by key (ascending keys; the order within a key is not
// defined), offset[k] where key k starts (keys + 1 entries, the last the
// total).  `temp`: counting_sort_temp_bytes(n, keys).  n < 2^32.
size_t counting_sort_temp_bytes(uint64_t n, uint32_t keys);
cudaError_t counting_sort(const uint32_t* key, uint64_t n, uint32_t keys, uint32_t* index_out,
                          uint64_t* offset, void* temp, cudaStream_t s);

// Zeroes counts (and time_hist) and bins n arrivals into them: two kernel
// launches, no scratch memory (bin.cu).
cudaError_t launch_bin_arrivals(const DevScene& sc, const int32_t* sensor,
                                const double* time, uint64_t n, uint32_t* counts,
                                uint32_t* time_hist, uint32_t num_bins,
                                double t_min, double t_max, cudaStream_t s);

// Records a message for mlgpu_last_error and returns `code` (capi.cu).
int report_error(int code, const char* message);
// The device scene of a handle (capi.cu).
const DevScene* device_scene(const mlgpu_scene* scene);
// The CUDA device the scene was created on (capi.cu).
int scene_device(const mlgpu_scene* scene);
// Launch accounting for entry points outside capi.cu: profile_mark_begin
// records the first event of a timed chain on `s` when the scene's profiling
// is on (with events the profiler already holds or creates, never device
// memory); profile_mark_end closes it with `launches` kernels of class `cls`
// and adds the launches to the scene's count (mlgpu_scene_kernel_launches).
struct ProfileMark {
    cudaEvent_t ev[2];
    bool timed;
};
void profile_mark_begin(mlgpu_scene* scene, cudaStream_t s, ProfileMark* mark);
void profile_mark_end(mlgpu_scene* scene, cudaStream_t s, ProfileMark* mark, int cls,
                      int launches);

}  // namespace mlgpu

#endif  // MLGPU_INTERNAL_H_
