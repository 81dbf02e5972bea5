// bin_noalloc.cu -- mlgpu_bin_arrivals_noalloc: per-sensor arrival counts
// and time histograms for callers that must not allocate device memory
// while running (see include/merlict_b200.h).  The binning kernels
// (bin.cu) accumulate in the caller's output buffers and need no scratch,
// so this entry point allocates nothing; it adds the check that the scene's
// device is the current one, so that the launches cannot land on another
// GPU's context.
#include <cstdio>

#include "mlgpu_internal.h"

extern "C" int mlgpu_bin_arrivals_noalloc(
    mlgpu_scene* scene, const int32_t* sensor, const double* time, uint64_t n,
    uint32_t* counts, uint32_t* time_hist, uint32_t num_time_bins, double t_min,
    double t_max, void* cuda_stream) {
    if (!scene || !sensor || !counts)
        return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    if (num_time_bins > 0 && (!time || !time_hist || !(t_max > t_min)))
        return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT,
                                   "time histogram needs times, output and t_max > t_min");
    const mlgpu::DevScene* dev = mlgpu::device_scene(scene);
    const uint64_t keys = (uint64_t)dev->num_sensors * (num_time_bins + 1ull);
    if (keys >= (1ull << 31))
        return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT, "too many sensor x time bins");
    // the launches go to the current device: it must be the scene's
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return mlgpu::report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    if (device != mlgpu::scene_device(scene)) {
        char msg[160];
        std::snprintf(msg, sizeof(msg),
                      "the current device (%d) is not the scene's device (%d)", device,
                      mlgpu::scene_device(scene));
        return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT, msg);
    }
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    mlgpu::ProfileMark mark;
    mlgpu::profile_mark_begin(scene, stream, &mark);
    e = mlgpu::launch_bin_arrivals(*dev, sensor, time, n, counts,
                                   num_time_bins ? time_hist : nullptr, num_time_bins, t_min,
                                   t_max, stream);
    mlgpu::profile_mark_end(scene, stream, &mark, MLGPU_KERNEL_BIN, 2);
    if (e != cudaSuccess) return mlgpu::report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}
