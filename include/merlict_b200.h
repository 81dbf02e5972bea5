/*
 * merlict_b200.h -- C ABI of the B200 photon-propagation engine.
 *
 * The engine replaces merlict's per-photon propagation loop and the
 * arrival binning that follows it:
 *
 *   merlict::propagate_photons_in_frame_with_config(
 *       std::vector<Photon>*, const Frame*, const PropagationConfig*,
 *       random::Generator*)                    merlict/Photons.h:12-16
 *   merlict::propagate_photons_in_frame_with_config_multi_thread(...)
 *                                 merlict_multi_thread/merlict_multi_thread.h:12-16
 *   merlict::sensor::Sensors::assign_photons(const std::vector<Photon>*)
 *                                              merlict/sensor/Sensors.h:35
 *
 * The caller first flattens its frame tree (merlict/Frame.h) into an
 * mlgpu_flat_scene: nodes in depth-first preorder with escape indices,
 * leaf surfaces with their 3x4 frame-to-world transforms and primitive
 * parameters, and the piecewise-linear property tables (merlict/function/
 * Func1.h).  The scene is uploaded once; photons are then traced in batches.
 *
 * No C++ types cross this boundary: plain pointers and sizes only.  Every
 * entry point returns an int status (MLGPU_OK == 0).  On failure a message
 * is kept per thread and can be read with mlgpu_last_error().
 */
#ifndef MERLICT_B200_H_
#define MERLICT_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MLGPU_ABI_VERSION 8

/* ---- status codes ------------------------------------------------------ */
enum {
    MLGPU_OK = 0,
    MLGPU_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference */
    MLGPU_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range, e.g. a wavelength
                                       outside a Func1 table, Limits.cpp:37-46 */
    MLGPU_ERR_RUNTIME = 3,          /* std::runtime_error */
    MLGPU_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    MLGPU_ERR_NO_DEVICE = 5
};

/* ---- interactions, same numbering as merlict/RayForPropagation.h:14-28 -- */
enum {
    MLGPU_PRODUCTION = 0,
    MLGPU_ABSORPTION_IN_VOID = 1,
    MLGPU_ABSORPTION_IN_MEDIUM = 2,
    MLGPU_ABSORPTION_ON_SURFACE = 3,
    MLGPU_FRESNEL_REFLECTION_ON_SURFACE = 4,
    MLGPU_REFLECTION_ON_SURFACE = 5,
    MLGPU_REFRACTION_TO_OUTSIDE = 6,
    MLGPU_REFRACTION_TO_INSIDE = 7
};

/* ---- leaf primitives (merlict/scenery/primitive/primitive.h:5-19) -------
 * Parameters per leaf (leaf_params, 8 doubles, unused slots are 0):      */
enum {
    MLGPU_PRIM_NONE = 0,             /* frame or surface without geometry   */
    MLGPU_PRIM_SPHERE_CAP_HEX = 1,   /* R, hex inner radius                 */
    MLGPU_PRIM_SPHERE_CAP_CYL = 2,   /* R, bound radius^2                   */
    MLGPU_PRIM_SPHERE_CAP_RECT = 3,  /* R, half x width, half y width       */
    MLGPU_PRIM_ELLIPTIC_CAP_HEX = 4, /* A, B, C, 1/A^2, 1/B^2, 1/C^2, hex inner */
    MLGPU_PRIM_DISC = 5,             /* radius^2                            */
    MLGPU_PRIM_HEX_PLANE = 6,        /* hex inner radius                    */
    MLGPU_PRIM_PLANE = 7,            /* half x width, half y width          */
    MLGPU_PRIM_ANNULUS = 8,          /* outer radius^2, inner radius^2      */
    MLGPU_PRIM_PLANE_DUAL_SPHERE = 9,/* circ1 x, circ1 y, circ2 x, circ2 y, circle radius */
    MLGPU_PRIM_TRIANGLE = 10,        /* Ax, Ay, Bx, By, Cx, Cy              */
    MLGPU_PRIM_CYLINDER = 11,        /* radius, length                      */
    MLGPU_PRIM_SPHERE = 12,          /* radius                              */
    MLGPU_PRIM_COUNT = 13
};

#define MLGPU_LEAF_PARAMS 8

/* leaf_surface columns: six property-table ids, the node a refraction into
 * the medium restricts traversal to (or -1), and flag bits.                */
enum {
    MLGPU_SURF_OUTER_REFLECTION = 0,
    MLGPU_SURF_INNER_REFLECTION = 1,
    MLGPU_SURF_OUTER_REFRACTION = 2,
    MLGPU_SURF_INNER_REFRACTION = 3,
    MLGPU_SURF_OUTER_ABSORPTION = 4,
    MLGPU_SURF_INNER_ABSORPTION = 5,
    MLGPU_SURF_ALLOWED_NODE = 6,
    MLGPU_SURF_FLAGS = 7,
    MLGPU_SURF_COLUMNS = 8
};

enum {
    MLGPU_FLAG_TRANSPARENT = 1,            /* SurfaceEntity.cpp:67-74        */
    MLGPU_FLAG_INNER_REFRACTION_DEFAULT = 2, /* inner_refraction is the default table */
    MLGPU_FLAG_OUTER_REFRACTION_DEFAULT = 4  /* outer_refraction is the default table */
};

/* Special leaf ids in results and histories. */
#define MLGPU_LEAF_VOID (-1)           /* no surface hit: VOID_SURFACE_ENTITY   */
#define MLGPU_LEAF_PHOTON_SOURCE (-2)  /* only the production entry exists     */

/* Flattened frame tree.  All pointers are host pointers. */
typedef struct mlgpu_flat_scene {
    /* Nodes: the frames of the tree in depth-first preorder, children in
     * their stored order (merlict/RayAndFrame.cpp:137-149).  Node 0 is the
     * tree root.  The subtree of node i is the index range
     * [i, node_skip[i]).                                                  */
    int32_t num_nodes;
    const double* node_sphere;   /* [num_nodes][4]: world x, y, z, bounding radius */
    const int32_t* node_skip;    /* [num_nodes]                                    */
    const int32_t* node_leaf;    /* [num_nodes]: leaf index, -1 if the frame has children */

    /* Leaves: frames without children. */
    int32_t num_leaves;
    const int32_t* leaf_node;        /* [num_leaves]                         */
    const double* leaf_frame2world;  /* [num_leaves][12]: rows of the 3x4 T  */
    const int32_t* leaf_primitive;   /* [num_leaves]                         */
    const double* leaf_params;       /* [num_leaves][MLGPU_LEAF_PARAMS]      */
    const int32_t* leaf_surface;     /* [num_leaves][MLGPU_SURF_COLUMNS]     */
    const int32_t* leaf_sensor;      /* [num_leaves]: sensor index or -1     */

    /* Property tables Func1: points (x, y, slope) sorted by x. */
    int32_t num_functions;
    const int32_t* function_offset;  /* [num_functions + 1] into the points  */
    const double* function_points;   /* [total points][3]                    */
    int32_t default_refraction;      /* id of the default refraction table   */

    /* Unit vectors of the hexagonal bound (HexagonalPrismZ.h:11-17), as the
     * host computed them, so that host and device agree bit for bit.      */
    double hex_unit_u[3];
    double hex_unit_v[3];
    double hex_unit_w[3];

    int32_t num_sensors;             /* sensor indices are 0 .. num_sensors-1 */
} mlgpu_flat_scene;

/* Photon batch: seven planes of one element type plus optional ids.
 * Pointers are device pointers for mlgpu_propagate and host pointers for
 * mlgpu_propagate_host.                                                   */
enum { MLGPU_F64 = 0, MLGPU_F32 = 1 };

typedef struct mlgpu_photons {
    int32_t dtype;                    /* MLGPU_F64 or MLGPU_F32            */
    const void* support_x;
    const void* support_y;
    const void* support_z;
    const void* direction_x;
    const void* direction_y;
    const void* direction_z;
    const void* wavelength;           /* metres                            */
    const int32_t* simulation_truth_id; /* may be NULL                     */
} mlgpu_photons;

/* One entry of a photon's history (Intersection + Interaction,
 * merlict/RayForPropagation.h:32-64). */
typedef struct mlgpu_history_entry {
    double position[3];   /* in the object frame of the surface            */
    double normal[3];     /* surface normal in the object frame            */
    double distance;      /* from the ray support to the intersection      */
    int32_t leaf;         /* leaf index, MLGPU_LEAF_VOID or _PHOTON_SOURCE */
    uint8_t interaction;
    uint8_t from_outside_to_inside;
    uint8_t pad[2];
} mlgpu_history_entry;

/* Per-photon results.  Any pointer may be NULL to skip that output, except
 * `sensor`.  x, y (and time) are written as `dtype` (x, y) and double (time).
 * info = interaction | num_interactions << 8 | uniforms used << 16
 *        | error << 24.                                                   */
typedef struct mlgpu_results {
    int32_t dtype;            /* element type of x, y, theta_x, theta_y     */
    int32_t* sensor;          /* sensor index of the final surface or -1    */
    void* x;                  /* final intersection, object frame (Sensor.cpp:14-30) */
    void* y;
    double* time;             /* time of flight, Photon.cpp:44-56           */
    void* theta_x;            /* -incident direction in the sensor frame    */
    void* theta_y;
    int32_t* final_leaf;
    uint32_t* info;
    double* final_position;   /* [n][3] world position of the final intersection */
    double* final_direction;  /* [n][3] direction of the photon at the end  */
    mlgpu_history_entry* history; /* [n][max_num_interactions_per_photon + 1] */
} mlgpu_results;

/* Random numbers.  PHILOX: Philox4x32-10 keyed by `seed`, photon i draws
 * from the counter stream (photon_offset + i); the k-th uniform of a photon
 * is (bits >> 11) * 2^-53 of the k-th block.  REPLAY: photon i consumes
 * uniforms[i * stride + k], k < stride (an exhausted stream is an error). */
enum { MLGPU_RNG_PHILOX = 0, MLGPU_RNG_REPLAY = 1 };

typedef struct mlgpu_rng {
    int32_t mode;
    uint32_t stride;
    uint64_t seed;
    uint64_t photon_offset;
    const double* uniforms;   /* device pointer (host for _host calls)    */
} mlgpu_rng;

/* Tracer forms.  Both FP64 forms reproduce merlict bit for bit; the
 * wavefront forms run per-step kernels over a pool of ray slots and wait
 * on the stream a few times per call to learn when the pool has drained. */
enum {
    MLGPU_TRACER_FP64 = 0,        /* wavefront, FP64                                  */
    MLGPU_TRACER_FP32 = 1,        /* wavefront, FP32 bulk math, FP64 where needed     */
    MLGPU_TRACER_FP32_PURE = 2,   /* FP32 everywhere (precision study only)           */
    MLGPU_TRACER_FP64_PLAIN = 3,  /* one thread per photon, FP64                      */
    MLGPU_TRACER_FP64_QUEUE = 4   /* FP64 in one persistent launch: warps take tiles
                                     of photons from a device work queue and advance
                                     them one interaction per round, refilling the
                                     lanes whose photons have ended                  */
};

/* How candidate surfaces are found for a ray in the whole tree.
 * BVH: an 8-wide bounding-volume hierarchy built at scene creation proposes
 * candidates; each still passes merlict's own bounding-sphere test of the
 * leaf and merlict's intersection, ties broken in merlict's visiting order.
 * FRAME_TREE: merlict's own walk over the frame tree's bounding spheres
 * (RayAndFrame.cpp:137-149).  Traversal restricted to a lens (an allowed
 * frame) always walks the frame tree.                                     */
enum { MLGPU_TRAVERSAL_BVH = 0, MLGPU_TRAVERSAL_FRAME_TREE = 1 };

/* PropagationConfig (merlict/PropagationConfig.h:10-13) plus engine knobs.
 * The knobs after `traversal` tune the wavefront tracers and never change
 * results; 0 selects the default.  mlgpu_scene_autotune picks them.       */
typedef struct mlgpu_settings {
    uint32_t max_num_interactions_per_photon;
    int32_t start_node;     /* node of the `world` frame passed by the caller */
    int32_t tracer;         /* MLGPU_TRACER_*                                 */
    int32_t block_size;     /* 0 = default                                    */
    int32_t traversal;      /* MLGPU_TRAVERSAL_*                              */
    uint32_t pool_size;     /* ray slots of the wavefront pool (2^21)         */
    int32_t check_period;   /* iterations between host checks of the pool (4) */
    int32_t use_graph;      /* 1: each check period is one CUDA-graph launch  */
    int32_t grid_blocks;    /* blocks of the grid-stride kernels (8 per SM)   */
    int32_t staged_levels;  /* top BVH levels read from shared memory (0)     */
    int32_t photon_order;   /* MLGPU_ORDER_*: the order photons enter the pool */
    int32_t walk;           /* MLGPU_WALK_*: how rays walk the BVH             */
    uint32_t queue_capacity; /* entries of each wavefront work queue: the
                               (ray, BVH node) queues, the (ray, leaf range)
                               queue and the (ray, candidate) queue; 0 = 8, 16
                               and 16 entries per ray slot.  A ray whose
                               entries do not fit takes merlict's own frame
                               walk instead (same results); a small capacity
                               only makes that fallback common.  0 or at
                               least 32.                                     */
} mlgpu_settings;

/* walk: LEVELS runs one kernel per BVH level over queued (ray, node) pairs
 * and one over the hit leaf ranges; STACK walks each ray's whole BVH in one
 * thread with a stack.  Both test the same boxes and bounding spheres and
 * find the same candidate leaves, so the results are the same.  DEFAULT is
 * LEVELS.                                                                  */
enum { MLGPU_WALK_DEFAULT = 0, MLGPU_WALK_LEVELS = 1, MLGPU_WALK_STACK = 2 };

/* photon_order: COHERENT sorts the batch by a 4-D cell key of support and
 * direction before tracing, so that neighbouring ray slots follow nearly
 * the same path (results are the same in any order).  DEFAULT is COHERENT
 * for batches of at least 65,536 photons and INPUT below.                  */
enum { MLGPU_ORDER_DEFAULT = 0, MLGPU_ORDER_INPUT = 1, MLGPU_ORDER_COHERENT = 2 };

typedef struct mlgpu_scene mlgpu_scene;

/* ---- library -------------------------------------------------------- */
int mlgpu_abi_version(void);
int mlgpu_last_error(char* buffer, size_t buffer_size);

/* ---- scene ---------------------------------------------------------- *
 * Replaces the per-call frame-tree walk of CausalIntersection
 * (merlict/RayAndFrame.cpp:126-173) by a device copy of the tree.
 * Validates the flat scene (index ranges, sorted tables) and uploads it to
 * the current CUDA device.                                              */
int mlgpu_scene_create(const mlgpu_flat_scene* flat, mlgpu_scene** scene);
int mlgpu_scene_destroy(mlgpu_scene* scene);

/* Kernel launches this scene has made so far (all entry points), for
 * callers that account for GPU work.                                      */
int mlgpu_scene_kernel_launches(const mlgpu_scene* scene, uint64_t* launches);

/* Kernel classes timed by the profiling hook below.  No counterpart in the
 * reference: it exists so that callers can put a roofline on each stage of
 * the device pipeline.                                                    */
enum {
    MLGPU_KERNEL_WALK = 0,       /* BVH levels and leaf-sphere tests          */
    MLGPU_KERNEL_INTAKE = 1,     /* photon intake, lens walks, pool counters  */
    MLGPU_KERNEL_INTERSECT = 2,  /* one thread per candidate, closest hit     */
    MLGPU_KERNEL_RESOLVE = 3,    /* interaction, compaction, results          */
    MLGPU_KERNEL_PLAIN = 4,      /* one-thread-per-photon tracer              */
    MLGPU_KERNEL_BIN = 5,        /* arrival binning                           */
    MLGPU_KERNEL_CLASSES = 6
};

/* Turns CUDA-event timing of every kernel class on (enable != 0) or off
 * and clears the totals.  While on, each launch is bracketed by events on
 * the caller's stream, which costs a few microseconds per launch.        */
int mlgpu_scene_set_profiling(mlgpu_scene* scene, int enable);

/* Device milliseconds and launches per kernel class since profiling was
 * last turned on; waits for the outstanding timed launches.  `ms` and
 * `launches` hold MLGPU_KERNEL_CLASSES entries each (either may be NULL). */
int mlgpu_scene_kernel_times(mlgpu_scene* scene, double* ms, uint64_t* launches);

/* Counters of the wavefront tracers since the scene was created (or since
 * the last call with reset != 0): propagations, iterations (each advances
 * every live ray by one interaction) and rays that did not fit a work
 * queue and were resolved by merlict's own walk of the frame tree
 * (RayAndFrame.cpp:126-173), counted once per ray and iteration.  No
 * counterpart in the reference.  Reads host-side totals only.            */
typedef struct mlgpu_wavefront_stats {
    uint64_t calls;
    uint64_t iterations;
    uint64_t overflow_rays;
} mlgpu_wavefront_stats;

int mlgpu_scene_wavefront_stats(mlgpu_scene* scene, mlgpu_wavefront_stats* stats, int reset);

/* The current GPU's FP64 arithmetic rate in FLOP/s, measured by a short
 * kernel of independent FP64 operation chains on every SM (about a tenth
 * of a second; synchronises `cuda_stream`).  fma != 0: fused multiply-adds
 * (2 FLOP each); fma == 0: separate adds and multiplies (1 FLOP each), the
 * only forms the bit-exact FP64 tracers use.  No counterpart in the
 * reference: it is the measured denominator of the tracers' compute
 * roofline, whose numerators are the reference's own operation counts.   */
int mlgpu_probe_fp64_rate(int fma, double* flops_per_second, void* cuda_stream);

/* ---- propagation ------------------------------------------------------ *
 * Replaces propagate_photons_in_frame_with_config (merlict/Photons.cpp:9-22)
 * and its thread-pool twin (merlict_multi_thread.cpp:28-55).
 * Device pointers, asynchronous on `cuda_stream` (a cudaStream_t, NULL =
 * default stream).  Errors found on the device (a wavelength outside a
 * property table, an exhausted replay stream) are reported by
 * mlgpu_scene_sync_errors().                                             */
int mlgpu_propagate(
    mlgpu_scene* scene,
    const mlgpu_photons* photons,
    uint64_t num_photons,
    const mlgpu_settings* settings,
    const mlgpu_rng* rng,
    mlgpu_results* results,
    void* cuda_stream);

/* Waits for `cuda_stream` and returns the first device-side error raised
 * since the previous call (then clears it).                             */
int mlgpu_scene_sync_errors(mlgpu_scene* scene, void* cuda_stream);

/* Same as mlgpu_propagate but with host pointers: copies the photons in,
 * traces, copies the results out and synchronises.  This is the call the
 * reference-side C++ shim makes.  When every buffer is page-locked
 * (cudaHostAlloc, cudaHostRegister, torch pin_memory) the batch moves in
 * pieces whose copies overlap the tracing.  With a wavefront form in the
 * coherent photon order one propagation is fed piece by piece (up to
 * sixteen pieces of at least a quarter ray pool, the first and the last
 * half as large): each piece is sorted on the device as soon as it has
 * landed and its photons are admitted from then on, and each piece's
 * results are copied back as soon as all its photons have finished.
 * Otherwise each piece (up to four of at least one ray pool) is a
 * propagation of its own, traced while the next one uploads.  Either way
 * the results are those of one call.
 * Ordered after earlier work on the legacy default stream.               */
int mlgpu_propagate_host(
    mlgpu_scene* scene,
    const mlgpu_photons* photons,
    uint64_t num_photons,
    const mlgpu_settings* settings,
    const mlgpu_rng* rng,
    mlgpu_results* results);

/* Page-locked host memory for the buffers of the host-buffer calls
 * (cudaMallocHost / cudaFreeHost), for callers that do not link the CUDA
 * runtime themselves, such as the reference-side C++ shim: with every
 * buffer of mlgpu_propagate_host in such memory the batch moves in pieces
 * whose copies overlap the tracing.  *ptr is NULL after a failure and for
 * 0 bytes; freeing NULL does nothing.                                    */
int mlgpu_host_alloc(uint64_t bytes, void** ptr);
int mlgpu_host_free(void* ptr);

/* Propagation and arrival binning in one host-buffer call: the pair a
 * merlict application runs per event, propagate_photons_in_frame_with_config
 * then Sensors::assign_photons (merlict/Photons.cpp:9-22,
 * merlict/sensor/Sensors.cpp:79-81), for callers that want per-sensor
 * statistics beside the per-photon results.  As mlgpu_propagate_host; then,
 * on the device, mlgpu_bin_arrivals' counts and time histograms of the whole
 * batch, copied to counts[num_sensors] and time_hist[num_sensors]
 * [num_time_bins] (host; time_hist and results->time are needed only when
 * num_time_bins > 0).                                                      */
int mlgpu_propagate_and_bin_host(
    mlgpu_scene* scene,
    const mlgpu_photons* photons,
    uint64_t num_photons,
    const mlgpu_settings* settings,
    const mlgpu_rng* rng,
    mlgpu_results* results,
    uint32_t* counts,
    uint32_t* time_hist,
    uint32_t num_time_bins,
    double t_min,
    double t_max);

/* ---- CORSIKA photon bunches --------------------------------------------- *
 * Replaces merlict::EventIoPhotonFactory (merlict_corsika/PhotonFactory.cpp:
 * 8-136) for a whole event at once, on the device.  `bunches` holds
 * num_bunches rows of 8 floats (x, y [cm], u, v, time [ns], production
 * height [cm], weight, wavelength [nm]); bunch i gives floor(weight) photons
 * plus one if its uniform draw is <= the weight's fraction, each with the
 * support, direction and wavelength merlict's factory gives it, and
 * simulation_truth_id = bunch_ids[i] (or i if bunch_ids is NULL).  The
 * draws: PHILOX stream (photon_offset + i), first uniform; REPLAY
 * uniforms[i].  Photons are written in bunch order.  The call waits for
 * `cuda_stream`; *num_photons receives the number of photons; if it exceeds
 * out->capacity nothing is written and MLGPU_ERR_INVALID_ARGUMENT is
 * returned (call again with larger buffers).  A weight outside [0, 16] is
 * MLGPU_ERR_INVALID_ARGUMENT (merlict throws std::invalid_argument).     */
typedef struct mlgpu_photon_buffers {
    double* support_x;
    double* support_y;
    double* support_z;
    double* direction_x;
    double* direction_y;
    double* direction_z;
    double* wavelength;
    int32_t* simulation_truth_id;     /* may be NULL                       */
    uint64_t capacity;                /* photons each buffer holds          */
} mlgpu_photon_buffers;

int mlgpu_corsika_photons(
    mlgpu_scene* scene,
    const float* bunches,
    uint64_t num_bunches,
    const int32_t* bunch_ids,
    const mlgpu_rng* rng,
    mlgpu_photon_buffers* out,
    uint64_t* num_photons,
    void* cuda_stream);

/* ---- calibration statistics ----------------------------------------------- *
 * Replaces plenoscope::calibration::LixelStatisticsFiller (merlict_portal_
 * plenoscope/calibration/LixelStatisticsFiller.cpp:20-62): for every sensor
 * s, of the photons with sensor[i] == s in their order i, the count and the
 * online mean and standard deviation (OnlineStatistics.cpp:15-50, variance
 * m2/n) of cx, cy (incident direction), x, y (support on the aperture) and
 * time_delay.  statistics[s][12] receives LixelStatistic's fields as merlict
 * computes them: efficiency = count/photons_emitted_per_lixel,
 * efficiency_std = sqrt(count)/photons_emitted_per_lixel, then cx, cy, x,
 * y, time_delay as (mean, std) pairs (NaN where merlict's are NaN).
 * Device pointers; asynchronous on `cuda_stream`.                        */
int mlgpu_lixel_statistics(
    mlgpu_scene* scene,
    const int32_t* sensor,
    const float* cx,
    const float* cy,
    const float* x,
    const float* y,
    const float* time_delay,
    uint64_t num_photons,
    double photons_emitted_per_lixel,
    float* statistics,
    void* cuda_stream);

/* ---- the signal chain after binning --------------------------------------- *
 * Replaces, for one event, the steps plenoscope_propagation.cpp:201-247
 * chains after Sensors::assign_photons: signal_processing::
 * get_photon_pipelines (PipelinePhoton.cpp:25-65), plenoscope::
 * night_sky_background::inject_nsb_into_photon_pipeline (Injector.cpp:
 * 8-98), PhotoElectricConverter::Converter::get_pulse_pipeline_for_photon_
 * pipeline (PhotoElectricConverter.cpp:31-90) and extract_pulses
 * (pulse_extraction.cpp:9-52).
 *
 * Photon i (device arrays) reached sensor[i] (< 0: none) at arrival_time[i]
 * with wavelength[i] and simulation_truth_id truth_id[i]; sensor s is lixel
 * s with calibrated efficiency lixel_efficiency[s] (float, as
 * calibration::read_efficiencies gives it).  Func1 tables are merlict's
 * Func1 points (x, y, slope) sorted by x, n of them, host memory: the
 * quantum efficiency and the background light's inverse wavelength CDF
 * (night_sky_background::Light::wavelength_probability, with its
 * total integral); nsb_rate is Light::rate and num_lixel the light-field
 * sensor's lixel count (Light.cpp:8-24).
 *
 * The draws: PHILOX only; stage s (1 background, 2 conversion, 3
 * extraction) of lixel i draws uniforms k = 0, 1, ... of stream
 * ((0xF0 | s) << 56) | (photon_offset + i) in the order merlict's code asks
 * for them; a normal deviate is mean + std sqrt(-2 ln(1 - u1)) cos(2 pi u2).
 *
 * Output: channel c's pulses are arrival_time_slice / simulation_truth_id
 * [channel_offset[c], channel_offset[c + 1]) (device, channel_offset has
 * num_sensors + 1 entries) in merlict's order; nsb_count (device, may be
 * NULL) the background photons of each lixel; num_pulses and
 * nsb_exposure_start_time (host) are set.  The call waits for
 * `cuda_stream` once; if num_pulses exceeds `capacity` only the offsets are
 * written and MLGPU_ERR_INVALID_ARGUMENT is returned (call again with
 * larger buffers).  A wavelength outside the quantum efficiency's table is
 * MLGPU_ERR_OUT_OF_RANGE (merlict throws std::out_of_range);
 * probability_for_second_puls >= 1 is MLGPU_ERR_INVALID_ARGUMENT.        */
typedef struct mlgpu_signal_chain_config {
    const double* quantum_efficiency;       /* Func1 points, host             */
    uint32_t num_quantum_efficiency;
    uint32_t num_nsb_wavelength_cdf;
    const double* nsb_wavelength_cdf;       /* Func1 points, host             */
    double nsb_total_integral;
    double nsb_rate;                        /* 1/s into the whole sensor      */
    double dark_rate;                       /* 1/s per lixel                  */
    double probability_for_second_puls;     /* crosstalk, < 1                 */
    double nsb_exposure_time;               /* s                              */
    double time_slice_duration;             /* s                              */
    double arrival_time_std;                /* single_photon_arrival_time_resolution, s */
    uint32_t num_lixel;
    uint32_t reserved;
} mlgpu_signal_chain_config;

typedef struct mlgpu_photon_stream {
    uint64_t* channel_offset;               /* [num_sensors + 1], device      */
    uint8_t* arrival_time_slice;            /* [capacity], device             */
    int32_t* simulation_truth_id;           /* [capacity], device             */
    int32_t* nsb_count;                     /* [num_sensors], device, or NULL */
    uint64_t capacity;
    uint64_t num_pulses;                    /* out                            */
    double nsb_exposure_start_time;         /* out, s                         */
} mlgpu_photon_stream;

int mlgpu_signal_chain(
    mlgpu_scene* scene,
    const mlgpu_signal_chain_config* config,
    const int32_t* sensor,
    const double* arrival_time,
    const double* wavelength,
    const int32_t* truth_id,
    uint64_t num_photons,
    const float* lixel_efficiency,
    uint32_t num_sensors,
    const mlgpu_rng* rng,
    mlgpu_photon_stream* out,
    void* cuda_stream);

/* ---- tuning ------------------------------------------------------------ *
 * No counterpart in the reference (merlict has no device parameters).
 * Picks the wavefront knobs of `base` (pool_size, check_period, use_graph,
 * grid_blocks, staged_levels, photon_order) for this scene by timing
 * mlgpu_propagate on a
 * sample of photons (device pointers, as for mlgpu_propagate): coordinate
 * descent from the defaults, each candidate timed with CUDA events on
 * `cuda_stream` (best of two runs after one untimed run).  Writes the
 * fastest settings to `best` (the other fields copied from `base`) and its
 * time in milliseconds to `best_ms` (may be NULL).  Results of the sample
 * runs are discarded; the tracer form is `base->tracer` (a wavefront
 * form).  The knobs never change what a propagation computes.            */
int mlgpu_scene_autotune(
    mlgpu_scene* scene,
    const mlgpu_photons* sample,
    uint64_t num_photons,
    const mlgpu_settings* base,
    const mlgpu_rng* rng,
    mlgpu_settings* best,
    double* best_ms,
    void* cuda_stream);

/* ---- arrival binning ------------------------------------------------- *
 * Replaces Sensors::assign_photons (merlict/sensor/Sensors.cpp:79-81) for
 * callers that want per-sensor statistics rather than arrival lists:
 * counts[s] = photons whose final surface is sensor s; time_hist[s][b] =
 * those arrivals with time in bin b of [t_min, t_max) (num_time_bins, may
 * be 0).  Device pointers.  `counts` and `time_hist` are overwritten.
 * Sensor ids outside [0, num_sensors) (no arrival: -1) are not counted.
 * Two kernel launches (zero the outputs, one pass of atomic additions);
 * allocates no device memory.                                            */
int mlgpu_bin_arrivals(
    mlgpu_scene* scene,
    const int32_t* sensor,
    const double* time,
    uint64_t num_photons,
    uint32_t* counts,
    uint32_t* time_hist,
    uint32_t num_time_bins,
    double t_min,
    double t_max,
    void* cuda_stream);

/* ---- allocation-free arrival binning ------------------------------------ *
 * No counterpart in the reference (merlict bins arrivals on the host).
 *
 * The same counts and time histograms as mlgpu_bin_arrivals, for callers
 * that must not allocate device memory once they are running: a host
 * application whose GPU memory is handed out by its own pool or caching
 * allocator (a cudaMalloc behind its back can exceed its fixed budget or
 * fragment the pool), or an event loop with real-time deadlines, where
 * cudaMalloc and cudaFree may synchronise the device and stall the other
 * streams.  The binning kernels accumulate in the caller's output buffers
 * and use no scratch, so neither entry point allocates; this one also
 * checks that the scene's device is the current device (else
 * MLGPU_ERR_INVALID_ARGUMENT) before it launches anything.  The inputs and
 * outputs are the caller's device buffers, as for mlgpu_bin_arrivals.  Its
 * two kernel launches count in mlgpu_scene_kernel_launches and, while
 * profiling is on, in the MLGPU_KERNEL_BIN times.  Calls share no state,
 * so calls on different streams may overlap.                             */
int mlgpu_bin_arrivals_noalloc(
    mlgpu_scene* scene,
    const int32_t* sensor,
    const double* time,
    uint64_t num_photons,
    uint32_t* counts,
    uint32_t* time_hist,
    uint32_t num_time_bins,
    double t_min,
    double t_max,
    void* cuda_stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif  /* MERLICT_B200_H_ */
