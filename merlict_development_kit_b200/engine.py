"""Device scene and propagation calls over the engine's C ABI.

PyTorch provides device memory and streams; the work is done by the CUDA
kernels in libmerlict_b200.so.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import abi
from ._native import check, lib
from .photons import PLANES

TRACERS = {"fp64": abi.TRACER_FP64, "fp32": abi.TRACER_FP32, "fp32_pure": abi.TRACER_FP32_PURE,
           "fp64_plain": abi.TRACER_FP64_PLAIN, "fp64_queue": abi.TRACER_FP64_QUEUE}
TRAVERSALS = {"bvh": abi.TRAVERSAL_BVH, "frame_tree": abi.TRAVERSAL_FRAME_TREE}


@dataclass
class PropagationConfig:
    """merlict::PropagationConfig (merlict/PropagationConfig.h:10-13)."""
    max_num_interactions_per_photon: int = 5


class Philox:
    """Counter-based generator: photon i of a call draws from stream
    (photon_offset + i) of key `seed`.  Stands in for merlict's
    random::Generator on the device."""

    def __init__(self, seed: int = 0, photon_offset: int = 0):
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.photon_offset = int(photon_offset)

    def _struct(self, n: int):
        r = abi.mlgpu_rng()
        r.mode = abi.RNG_PHILOX
        r.seed = self.seed
        r.photon_offset = self.photon_offset
        return r, None

    def advance(self, n: int) -> None:
        self.photon_offset += int(n)


class Replay:
    """Replays recorded uniforms: photon i consumes uniforms[i, k], k = 0, 1,
    ... (an exhausted row is an error)."""

    def __init__(self, uniforms):
        self.uniforms = uniforms

    def _struct(self, n: int):
        u = self.uniforms
        if not isinstance(u, torch.Tensor):
            u = torch.as_tensor(np.ascontiguousarray(u, dtype=np.float64))
        u = u.to(device="cuda", dtype=torch.float64).contiguous()
        if u.dim() != 2 or u.shape[0] < n:
            raise ValueError("replay uniforms must have shape [num_photons, stride]")
        r = abi.mlgpu_rng()
        r.mode = abi.RNG_REPLAY
        r.stride = int(u.shape[1])
        r.uniforms = u.data_ptr()
        return r, u

    def advance(self, n: int) -> None:
        pass


def _stream_handle(stream) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def photons_to_device(batch: dict, dtype=torch.float64) -> dict:
    """Copies a photon batch (numpy or torch) to the current CUDA device."""
    out = {}
    for k in PLANES:
        v = batch[k]
        t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
        out[k] = t.to(device="cuda", dtype=dtype, non_blocking=True).contiguous()
    if batch.get("id") is not None:
        v = batch["id"]
        t = v if isinstance(v, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(v))
        out["id"] = t.to(device="cuda", dtype=torch.int32).contiguous()
    return out


def _settings(config: PropagationConfig, start_node: int, tracer: str, traversal: str,
              tuning: dict | None) -> abi.mlgpu_settings:
    st = abi.mlgpu_settings(int(config.max_num_interactions_per_photon), int(start_node),
                            TRACERS[tracer], 0, TRAVERSALS[traversal])
    for k, v in (tuning or {}).items():
        if k not in abi.mlgpu_settings.TUNING:
            raise ValueError(f"unknown tuning knob {k!r}")
        setattr(st, k, int(v))
    return st


def _photon_struct(photons: dict, n: int) -> abi.mlgpu_photons:
    in_dtype = photons["wavelength"].dtype
    ph = abi.mlgpu_photons()
    ph.dtype = abi.F64 if in_dtype == torch.float64 else abi.F32
    for k in PLANES:
        t = photons[k]
        if t.dtype != in_dtype or not t.is_cuda or not t.is_contiguous() or t.shape[0] != n:
            raise ValueError(f"photon plane {k} must be a contiguous CUDA tensor of {in_dtype}")
        setattr(ph, k, t.data_ptr())
    return ph


class Scene:
    """A flattened frame tree resident on the current CUDA device."""

    def __init__(self, flat: abi.FlatScene):
        if not torch.cuda.is_available():
            raise RuntimeError("merlict_development_kit_b200 needs a CUDA device")
        torch.cuda.init()
        flat.validate()
        self.flat = flat
        self._struct = flat.as_struct()
        h = C.c_void_p()
        check(lib().mlgpu_scene_create(C.byref(self._struct), C.byref(h)))
        self._h = h
        self.num_sensors = flat.num_sensors

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().mlgpu_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def propagate(self, photons: dict, config: PropagationConfig | None = None,
                  rng=None, tracer: str = "fp64", start_node: int = 0,
                  outputs=("sensor", "x", "y", "time"), history: bool = False,
                  out_dtype=torch.float64, stream=None, sync: bool = True,
                  results: dict | None = None, traversal: str = "bvh",
                  tuning: dict | None = None) -> dict:
        """Traces a batch of device-resident photons.

        `photons` is a dict of CUDA tensors (see photons.PLANES).  Returns a
        dict of CUDA tensors with the requested outputs.  With sync=True the
        call waits and raises on device-side errors (a wavelength outside a
        property table raises IndexError, like merlict's std::out_of_range).
        `tuning` sets the wavefront knobs of mlgpu_settings (pool_size,
        check_period, use_graph, grid_blocks, staged_levels), e.g. the dict
        `autotune` returns; they never change the results.
        """
        config = config or PropagationConfig()
        rng = rng if rng is not None else Philox(0)
        n = int(photons["wavelength"].shape[0])
        ph = _photon_struct(photons, n)
        dev = photons["wavelength"].device
        res = abi.mlgpu_results()
        res.dtype = abi.F64 if out_dtype == torch.float64 else abi.F32
        out = {} if results is None else results
        spec = {
            "sensor": ((n,), torch.int32), "x": ((n,), out_dtype), "y": ((n,), out_dtype),
            "time": ((n,), torch.float64), "theta_x": ((n,), out_dtype),
            "theta_y": ((n,), out_dtype), "final_leaf": ((n,), torch.int32),
            "info": ((n,), torch.int32), "final_position": ((n, 3), torch.float64),
            "final_direction": ((n, 3), torch.float64),
        }
        wanted = set(outputs) | {"sensor"}
        for k, (shape, dt) in spec.items():
            if k in wanted:
                if k not in out or out[k].shape[0] < n:
                    out[k] = torch.empty(shape, dtype=dt, device=dev)
                setattr(res, k, out[k].data_ptr())
        if history:
            m = config.max_num_interactions_per_photon + 1
            out["history"] = torch.empty((n, m, abi.HISTORY_DTYPE.itemsize), dtype=torch.uint8, device=dev)
            res.history = out["history"].data_ptr()
        st = _settings(config, start_node, tracer, traversal, tuning)
        r, keep = rng._struct(n)
        sh = _stream_handle(stream)
        check(lib().mlgpu_propagate(self._h, C.byref(ph), n, C.byref(st), C.byref(r),
                                    C.byref(res), C.c_void_p(sh)))
        rng.advance(n)
        if sync:
            check(lib().mlgpu_scene_sync_errors(self._h, C.c_void_p(sh)))
        del keep
        return out

    def autotune(self, photons: dict, config: PropagationConfig | None = None,
                 rng=None, tracer: str = "fp64", stream=None) -> tuple[dict, float]:
        """Picks the wavefront knobs for this scene by timing propagations
        of the sample `photons` (mlgpu_scene_autotune); returns the tuning
        dict for `propagate` and the sample's best time in ms."""
        config = config or PropagationConfig()
        rng = rng if rng is not None else Philox(0)
        n = int(photons["wavelength"].shape[0])
        ph = _photon_struct(photons, n)
        base = _settings(config, 0, tracer, "bvh", None)
        best = abi.mlgpu_settings()
        ms = C.c_double(0.0)
        r, keep = rng._struct(n)
        check(lib().mlgpu_scene_autotune(self._h, C.byref(ph), n, C.byref(base), C.byref(r),
                                         C.byref(best), C.byref(ms),
                                         C.c_void_p(_stream_handle(stream))))
        del keep
        return best.tuning(), float(ms.value)

    def corsika_photons(self, bunches: torch.Tensor, rng=None, bunch_ids: torch.Tensor | None = None,
                        capacity: int | None = None, stream=None) -> dict:
        """Photons of CORSIKA bunches ([n][8] float32 CUDA tensor: x, y [cm],
        u, v, time [ns], production height [cm], weight, wavelength [nm]),
        made on the device the way merlict's EventIoPhotonFactory makes them
        (mlgpu_corsika_photons); planes as for `propagate`, plus "id".
        A weight outside [0, 16] raises ValueError, like merlict."""
        if bunches.dtype != torch.float32 or not bunches.is_cuda or bunches.dim() != 2 \
                or bunches.shape[1] != 8:
            raise ValueError("bunches must be a [n][8] float32 CUDA tensor")
        b = bunches.contiguous()
        n = int(b.shape[0])
        rng = rng if rng is not None else Philox(0)
        r, keep = rng._struct(n)
        cap = 17 * n if capacity is None else int(capacity)
        out = {k: torch.empty(cap, dtype=torch.float64, device=b.device) for k in PLANES}
        out["id"] = torch.empty(cap, dtype=torch.int32, device=b.device)
        buf = abi.mlgpu_photon_buffers()
        for k in PLANES:
            setattr(buf, k, out[k].data_ptr())
        buf.simulation_truth_id = out["id"].data_ptr()
        buf.capacity = cap
        total = C.c_uint64(0)
        ids = bunch_ids.contiguous() if bunch_ids is not None else None
        check(lib().mlgpu_corsika_photons(self._h, C.c_void_p(b.data_ptr()), n,
                                          C.c_void_p(ids.data_ptr() if ids is not None else None),
                                          C.byref(r), C.byref(buf), C.byref(total),
                                          C.c_void_p(_stream_handle(stream))))
        rng.advance(n)
        del keep
        t = int(total.value)
        return {k: v[:t] for k, v in out.items()}

    def kernel_launches(self) -> int:
        """Kernels this scene has launched so far."""
        v = C.c_uint64(0)
        check(lib().mlgpu_scene_kernel_launches(self._h, C.byref(v)))
        return int(v.value)

    def wavefront_stats(self, reset: bool = False) -> dict:
        """Wavefront propagations, iterations and rays resolved by merlict's
        own frame walk after a work queue overflowed, since the scene was
        created or the last reset."""
        s = abi.mlgpu_wavefront_stats()
        check(lib().mlgpu_scene_wavefront_stats(self._h, C.byref(s), int(bool(reset))))
        return {"calls": int(s.calls), "iterations": int(s.iterations),
                "overflow_rays": int(s.overflow_rays)}

    KERNEL_CLASSES = ("walk", "intake", "intersect", "resolve", "plain", "bin")

    def set_profiling(self, enable: bool) -> None:
        """Turns CUDA-event timing of the kernel classes on or off (and
        clears the totals)."""
        check(lib().mlgpu_scene_set_profiling(self._h, int(bool(enable))))

    def kernel_times(self) -> dict:
        """{class: (device ms, launches)} since profiling was turned on."""
        n = len(self.KERNEL_CLASSES)
        ms = (C.c_double * n)()
        launches = (C.c_uint64 * n)()
        check(lib().mlgpu_scene_kernel_times(self._h, ms, launches))
        return {k: (float(ms[i]), int(launches[i])) for i, k in enumerate(self.KERNEL_CLASSES)}

    def sync_errors(self, stream=None) -> None:
        check(lib().mlgpu_scene_sync_errors(self._h, C.c_void_p(_stream_handle(stream))))

    def bin_arrivals(self, sensor: torch.Tensor, time: torch.Tensor | None = None,
                     num_time_bins: int = 0, t_min: float = 0.0, t_max: float = 1.0,
                     stream=None):
        """Per-sensor counts (and time histograms) of device results."""
        n = int(sensor.shape[0])
        counts = torch.empty(self.num_sensors, dtype=torch.int32, device=sensor.device)
        hist = None
        tp = None
        if num_time_bins:
            hist = torch.empty((self.num_sensors, num_time_bins), dtype=torch.int32,
                               device=sensor.device)
            tp = time.data_ptr()
        check(lib().mlgpu_bin_arrivals(
            self._h, C.c_void_p(sensor.data_ptr()), C.c_void_p(tp), n,
            C.c_void_p(counts.data_ptr()), C.c_void_p(hist.data_ptr() if hist is not None else None),
            int(num_time_bins), float(t_min), float(t_max), C.c_void_p(_stream_handle(stream))))
        return counts, hist


def history_to_numpy(h: torch.Tensor) -> np.ndarray:
    """Device history bytes -> structured numpy array of mlgpu_history_entry."""
    a = h.cpu().numpy()
    return a.view(abi.HISTORY_DTYPE).reshape(a.shape[0], a.shape[1])
