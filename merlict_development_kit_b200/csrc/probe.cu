// probe.cu -- mlgpu_probe_fp64_rate: the FP64 arithmetic rate of the
// current GPU, measured, as the denominator of the tracer's compute
// roofline (the reference's operation counts are FP64 adds, multiplies,
// divides and square roots).
//
// Every thread runs kChains independent dependency chains of FP64
// operations (enough to cover the pipe's latency) for `iterations` rounds;
// the grid fills every SM several times over.  With fma = 1 each operation
// is a fused multiply-add (2 FLOP); with fma = 0 it is an add or a
// multiply (1 FLOP each), the only forms the bit-exact tracer may use (it
// is compiled without contraction).  The result is kept live by a store
// that depends on every chain.
#include <cstdint>

#include "mlgpu_internal.h"

namespace {

constexpr int kChains = 8;
constexpr int kUnroll = 16;

template <bool kFma>
__global__ void __launch_bounds__(256)
fp64_rate_kernel(double seed, int iterations, double* sink) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++) x[c] = seed + (double)(threadIdx.x + c);
    const double m = 1.0000001, a = 1e-9;
    for (int it = 0; it < iterations; it++) {
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
#pragma unroll
            for (int c = 0; c < kChains; c++) {
                if (kFma) {
                    x[c] = fma(x[c], m, a);
                } else if (u & 1) {
                    x[c] = __dadd_rn(x[c], a);
                } else {
                    x[c] = __dmul_rn(x[c], m);
                }
            }
        }
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; c++) s += x[c];
    if (s == 12345.678) sink[0] = s;   // never true; keeps the chains
}

}  // namespace

extern "C" int mlgpu_probe_fp64_rate(int fma, double* flops_per_second, void* cuda_stream) {
    if (!flops_per_second) return mlgpu::report_error(MLGPU_ERR_INVALID_ARGUMENT, "NULL argument");
    const cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = 8*sms, threads = 256, iterations = 4096;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t e = cudaEventCreate(&ev[0]);
    if (e == cudaSuccess) e = cudaEventCreate(&ev[1]);
    float ms = 0.0f;
    for (int rep = 0; rep < 3 && e == cudaSuccess; rep++) {   // the first run warms up
        e = cudaEventRecord(ev[0], s);
        if (fma) fp64_rate_kernel<true><<<blocks, threads, 0, s>>>(1.0, iterations, nullptr);
        else fp64_rate_kernel<false><<<blocks, threads, 0, s>>>(1.0, iterations, nullptr);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(ev[1], s);
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ev[0], ev[1]);
    }
    if (ev[0]) cudaEventDestroy(ev[0]);
    if (ev[1]) cudaEventDestroy(ev[1]);
    if (e != cudaSuccess) return mlgpu::report_error(MLGPU_ERR_CUDA, cudaGetErrorString(e));
    const double ops = (double)blocks*threads*iterations*kUnroll*kChains;
    *flops_per_second = ops*(fma ? 2.0 : 1.0)/(ms*1e-3);
    return MLGPU_OK;
}
