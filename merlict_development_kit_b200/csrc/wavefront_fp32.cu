// wavefront_fp32.cu -- the batched FP32 tracer: the wavefront iteration of
// wavefront_fp64.cu (the same BVH walk, which proposes the leaves passing
// merlict's bounding-sphere test as candidates) with the candidates
// intersected in single precision (fp32_geometry.cuh).  Positions, the
// interaction and the time of flight stay FP64, so the only difference to
// merlict is the rounding of each intersection -- about 1e-7 of the leaf's
// size -- which moves a photon to another sensor only when it lands within
// that distance of a pixel's edge.
//
// This translation unit is compiled with the default --fmad=true: the FP32
// form makes no bit-identity claim, and the contractions shorten the
// intersection arithmetic.
#include <cstdint>

#include "wave_resolve.cuh"

namespace mlgpu {

cudaError_t launch_wave32_isect_resolve(const TraceArgs& a, const WaveBuffers& w,
                                        const RayPool& cur, const RayPool& nxt, bool pure,
                                        cudaStream_t s, cudaEvent_t mid) {
    const int blocks = (int)((w.pool + 255)/256);
    if (pure) wave_isect_kernel<kIsectFp32Pure><<<w.grid, 256, 0, s>>>(a, w, cur);
    else wave_isect_kernel<kIsectFp32><<<w.grid, 256, 0, s>>>(a, w, cur);
    wave_tie_kernel<<<w.grid, 256, 0, s>>>(w, cur);
    if (mid) cudaEventRecord(mid, s);
    wave_overflow_kernel<<<148, 128, 0, s>>>(a, w, cur);
    if (pure) {
        if (a.out_dtype == MLGPU_F64)
            wave_resolve_kernel<double, kIsectFp32Pure><<<blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
        else
            wave_resolve_kernel<float, kIsectFp32Pure><<<blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
    } else {
        if (a.out_dtype == MLGPU_F64)
            wave_resolve_kernel<double, kIsectFp32><<<blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
        else
            wave_resolve_kernel<float, kIsectFp32><<<blocks, 256, w.fn_smem_bytes, s>>>(a, w, cur, nxt);
    }
    return cudaGetLastError();
}

}  // namespace mlgpu
