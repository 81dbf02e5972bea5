// trace_fp32.cu -- placeholder until the batched FP32 tracer lands.
#include "mlgpu_internal.h"

namespace mlgpu {

cudaError_t launch_trace_fp32(const TraceArgs& a, int block, bool pure, cudaStream_t s) {
    (void)a; (void)block; (void)pure; (void)s;
    return cudaErrorNotSupported;
}

}  // namespace mlgpu
