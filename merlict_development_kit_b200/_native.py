"""Loads libmerlict_b200.so (the CUDA engine) and declares its C ABI.

There is no CPU fallback: if the library is missing or was built for another
GPU, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libmerlict_b200.so")

_lib = None


class EngineError(RuntimeError):
    """An engine status other than MLGPU_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def _exception_for(status: int, message: str) -> Exception:
    # the std:: exceptions merlict throws for the same conditions
    if status == abi.ERR_INVALID_ARGUMENT:
        return ValueError(message)
    if status == abi.ERR_OUT_OF_RANGE:
        return IndexError(message)
    return EngineError(status, message)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with "
                "`python -m merlict_development_kit_b200.build` (needs nvcc)")
        L = C.CDLL(LIB_PATH)
        L.mlgpu_abi_version.restype = C.c_int
        L.mlgpu_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.mlgpu_last_error.restype = C.c_int
        L.mlgpu_scene_create.argtypes = [C.POINTER(abi.mlgpu_flat_scene), C.POINTER(C.c_void_p)]
        L.mlgpu_scene_destroy.argtypes = [C.c_void_p]
        L.mlgpu_propagate.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64,
            C.POINTER(abi.mlgpu_settings), C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_results), C.c_void_p]
        L.mlgpu_propagate_host.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64,
            C.POINTER(abi.mlgpu_settings), C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_results)]
        L.mlgpu_propagate_and_bin_host.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64,
            C.POINTER(abi.mlgpu_settings), C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_results), C.c_void_p, C.c_void_p, C.c_uint32, C.c_double,
            C.c_double]
        L.mlgpu_scene_sync_errors.argtypes = [C.c_void_p, C.c_void_p]
        L.mlgpu_probe_fp64_rate.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_void_p]
        L.mlgpu_bin_arrivals.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
            C.c_uint32, C.c_double, C.c_double, C.c_void_p]
        L.mlgpu_scene_kernel_launches.argtypes = [C.c_void_p, C.POINTER(C.c_uint64)]
        L.mlgpu_scene_wavefront_stats.argtypes = [C.c_void_p,
                                                  C.POINTER(abi.mlgpu_wavefront_stats), C.c_int]
        L.mlgpu_scene_set_profiling.argtypes = [C.c_void_p, C.c_int]
        L.mlgpu_scene_kernel_times.argtypes = [C.c_void_p, C.POINTER(C.c_double),
                                               C.POINTER(C.c_uint64)]
        L.mlgpu_bin_arrivals_noalloc.argtypes = [
            C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
            C.c_uint32, C.c_double, C.c_double, C.c_void_p]
        L.mlgpu_corsika_photons.argtypes = [
            C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_photon_buffers), C.POINTER(C.c_uint64), C.c_void_p]
        L.mlgpu_lixel_statistics.argtypes = [C.c_void_p] + [C.c_void_p] * 6 + [
            C.c_uint64, C.c_double, C.c_void_p, C.c_void_p]
        L.mlgpu_signal_chain.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_signal_chain_config)] + [C.c_void_p] * 4 + [
            C.c_uint64, C.c_void_p, C.c_uint32, C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_photon_stream), C.c_void_p]
        L.mlgpu_scene_autotune.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64,
            C.POINTER(abi.mlgpu_settings), C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_settings), C.POINTER(C.c_double), C.c_void_p]
        _declare_surrogate(L)
        for name in ("mlgpu_scene_create", "mlgpu_scene_destroy", "mlgpu_propagate",
                     "mlgpu_scene_autotune", "mlgpu_corsika_photons", "mlgpu_lixel_statistics",
                     "mlgpu_signal_chain",
                     "mlgpu_propagate_host", "mlgpu_propagate_and_bin_host",
                     "mlgpu_scene_sync_errors", "mlgpu_bin_arrivals",
                     "mlgpu_bin_arrivals_noalloc", "mlgpu_scene_kernel_launches",
                     "mlgpu_scene_wavefront_stats", "mlgpu_probe_fp64_rate"):
            getattr(L, name).restype = C.c_int
        if L.mlgpu_abi_version() != abi.ABI_VERSION:
            raise ImportError("libmerlict_b200.so ABI version mismatch")
        _lib = L
    return _lib


class mlgpu_sg_sensor_grid(C.Structure):
    _fields_ = [
        ("num_sensors", C.c_uint32),
        ("center", C.c_void_p), ("rotation", C.c_void_p), ("inner", C.c_void_p),
        ("sensor_id", C.c_void_p),
        ("x0", C.c_double), ("y0", C.c_double), ("cell", C.c_double),
        ("nx", C.c_uint32), ("ny", C.c_uint32),
        ("cell_start", C.c_void_p), ("cell_items", C.c_void_p),
        ("hex_u", C.c_double * 2), ("hex_v", C.c_double * 2), ("hex_w", C.c_double * 2),
    ]


def _declare_surrogate(L) -> None:
    """ctypes signatures of include/merlict_b200_surrogate.h."""
    vp, u32, u64, f32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float
    L.mlgpu_sg_image_offset.argtypes = [u32, u32, u32]
    L.mlgpu_sg_image_offset.restype = C.c_size_t
    L.mlgpu_sg_param_count.restype = u64
    L.mlgpu_sg_image_bytes.restype = u64
    L.mlgpu_sg_workspace_bytes.argtypes = [u32, C.c_int]
    L.mlgpu_sg_workspace_bytes.restype = u64
    L.mlgpu_sg_gemm_f32.argtypes = [vp, u32, vp, u32, u32, u32, u32, vp, vp, vp]
    L.mlgpu_sg_pack_weights.argtypes = [vp, vp, vp]
    L.mlgpu_sg_forward.argtypes = [vp, vp, vp, u32, vp, vp, vp]
    L.mlgpu_sg_forward_layered.argtypes = [vp, vp, vp, u32, vp, vp, vp]
    L.mlgpu_sg_train_step.argtypes = [vp, vp, vp, vp, vp, vp, vp, u32, u32, f32, vp, vp, vp, vp]
    L.mlgpu_sg_sample.argtypes = [vp, vp, u32, vp, vp, f32, f32, u64, u64,
                                  C.POINTER(mlgpu_sg_sensor_grid), vp, vp, vp, vp, vp, vp, vp]
    L.mlgpu_sg_sync_errors.argtypes = [vp]
    for name in ("mlgpu_sg_gemm_f32", "mlgpu_sg_pack_weights", "mlgpu_sg_forward",
                 "mlgpu_sg_forward_layered",
                 "mlgpu_sg_train_step", "mlgpu_sg_sample", "mlgpu_sg_sync_errors"):
        getattr(L, name).restype = C.c_int


def last_error() -> str:
    buf = C.create_string_buffer(2048)
    lib().mlgpu_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != abi.OK:
        raise _exception_for(status, last_error())


# every symbol include/merlict_b200.h declares
EXPORTED = (
    "mlgpu_abi_version", "mlgpu_last_error", "mlgpu_scene_create", "mlgpu_scene_destroy",
    "mlgpu_propagate", "mlgpu_scene_sync_errors", "mlgpu_propagate_host",
    "mlgpu_propagate_and_bin_host", "mlgpu_host_alloc", "mlgpu_host_free",
    "mlgpu_bin_arrivals", "mlgpu_bin_arrivals_noalloc", "mlgpu_scene_kernel_launches",
    "mlgpu_scene_wavefront_stats", "mlgpu_probe_fp64_rate",
    "mlgpu_scene_set_profiling", "mlgpu_scene_kernel_times", "mlgpu_scene_autotune",
    "mlgpu_corsika_photons", "mlgpu_lixel_statistics", "mlgpu_signal_chain",
    # include/merlict_b200_surrogate.h
    "mlgpu_sg_image_offset", "mlgpu_sg_gemm_f32", "mlgpu_sg_param_count", "mlgpu_sg_image_bytes",
    "mlgpu_sg_pack_weights", "mlgpu_sg_workspace_bytes", "mlgpu_sg_forward",
    "mlgpu_sg_forward_layered",
    "mlgpu_sg_train_step", "mlgpu_sg_sample", "mlgpu_sg_sync_errors",
)
