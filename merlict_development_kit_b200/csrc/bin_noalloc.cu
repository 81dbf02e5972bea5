// bin_noalloc.cu -- mlgpu_bin_arrivals_noalloc: per-sensor arrival counts
// and time histograms for callers that must not allocate device memory
// while running (see include/merlict_b200.h).  The partial histograms that
// mlgpu_bin_arrivals keeps in a buffer grown with cudaMalloc live here in a
// fixed array compiled into the library instead.
#include <cstdio>
#include <mutex>

#include "mlgpu_internal.h"

namespace {

// The scratch: MLGPU_NOALLOC_BIN_SCRATCH_WORDS words on every device that
// loads this library, for the life of the process.  In host code its name
// is only a stand-in for the symbol, never a device address: the address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_bin_scratch[MLGPU_NOALLOC_BIN_SCRATCH_WORDS];

constexpr int kMaxDevices = 128;
std::mutex g_setup_mutex;
uint32_t* g_scratch_address[kMaxDevices] = {};

// Once per device, with that device current: the array's device address.
int scratch_of_current_device(uint32_t** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        return mlgpu::report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices)
        return mlgpu::report_error(MLGPU_ERR_RUNTIME, "device ordinal beyond the set-up table");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_address[device]) {
        void* address = nullptr;
        e = cudaGetSymbolAddress(&address, g_bin_scratch);
        if (e != cudaSuccess) {
            char msg[256];
            std::snprintf(msg, sizeof(msg),
                          "cudaGetSymbolAddress of the binning scratch failed: %s",
                          cudaGetErrorString(e));
            return mlgpu::report_error(MLGPU_ERR_CUDA, msg);
        }
        g_scratch_address[device] = static_cast<uint32_t*>(address);
    }
    *out = g_scratch_address[device];
    return MLGPU_OK;
}

}  // namespace

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
    if (keys > MLGPU_NOALLOC_BIN_SCRATCH_WORDS) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "sensors x (time bins + 1) = %llu exceeds the fixed scratch of "
                      "%u keys of mlgpu_bin_arrivals_noalloc",
                      (unsigned long long)keys, (unsigned)MLGPU_NOALLOC_BIN_SCRATCH_WORDS);
        return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT, msg);
    }
    // the array used is the current device's: it must be the scene's
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
    uint32_t* scratch = nullptr;
    const int st = scratch_of_current_device(&scratch);
    if (st != MLGPU_OK) return st;
    const cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    mlgpu::ProfileMark mark;
    mlgpu::profile_mark_begin(scene, stream, &mark);
    // The tile kernel stores every word of the partial histograms before
    // the reduction reads it, so the scratch needs no clearing.
    e = mlgpu::launch_bin_arrivals(
        *dev, sensor, time, n, counts, num_time_bins ? time_hist : nullptr, num_time_bins,
        t_min, t_max, scratch, MLGPU_NOALLOC_BIN_SCRATCH_WORDS, stream);
    mlgpu::profile_mark_end(scene, stream, &mark, MLGPU_KERNEL_BIN, 2);
    if (e != cudaSuccess) return mlgpu::report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    return MLGPU_OK;
}
