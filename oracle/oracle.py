"""TEST INFRASTRUCTURE -- Python access to the checkers under oracle/.

* `Oracle` wraps _build/libmerlict_oracle.so, the C restatement of merlict's
  propagation (merlict_oracle.c), run on a FlatScene.
* `RefScene` wraps _ref/libmerlict_ref_harness.so: a scene built with the
  reference library's own classes and factories, flattened by the product's
  shim, and propagated by the reference's own Propagator.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from merlict_development_kit_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
ORACLE_SO = os.path.join(HERE, "_build", "libmerlict_oracle.so")
HARNESS_SO = os.path.join(HERE, "_ref", "libmerlict_ref_harness.so")
SHIM_HARNESS_SO = os.path.join(HERE, "_ref", "libmerlict_shim_harness.so")
SANITIZE_EXE = os.path.join(HERE, "_ref", "sanitize_shim")
ENGINE_SO = os.path.join(REPO, "merlict_development_kit_b200", "_build", "libmerlict_b200.so")
# the reference source tree: $MERLICT_REFERENCE_DIR, else `reference` beside
# the repository; without it the reference-built checkers are not rebuilt
REFERENCE_DIR = os.environ.get("MERLICT_REFERENCE_DIR",
                               os.path.join(os.path.dirname(REPO), "reference"))


class OracleCounters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "nodes", "leaves", "caps", "cap_bounds", "planes", "others",
        "reflections", "fresnels", "segments", "funcs", "steps")] + [
        ("leaves_per_step", C.c_uint64 * 65)]

    def as_dict(self) -> dict:
        d = {k: int(getattr(self, k)) for k, _ in self._fields_ if k != "leaves_per_step"}
        d["leaves_per_step"] = [int(v) for v in self.leaves_per_step]
        return d


def build(reference: bool = True) -> None:
    """Builds the oracle, and -- when the reference sources are present --
    the reference harness, the sanitizer check of the drop-in's host code
    and (once the engine library is built) the drop-in's test harness."""
    targets = ["oracle"]
    if reference and os.path.isdir(REFERENCE_DIR):
        targets += ["ref", "sanitize"]
        if os.path.exists(ENGINE_SO):
            targets.append("shim")
    subprocess.run(["make", "-s", "-C", HERE, f"-j{os.cpu_count() or 4}",
                    f"REF={REFERENCE_DIR}"] + targets, check=True)


def harness_available() -> bool:
    return os.path.exists(HARNESS_SO)


def shim_harness_available() -> bool:
    return os.path.exists(SHIM_HARNESS_SO)


def _photon_struct(ph: dict) -> tuple[abi.mlgpu_photons, list]:
    keep = []
    s = abi.mlgpu_photons()
    s.dtype = abi.F64
    for name in ("support_x", "support_y", "support_z", "direction_x",
                 "direction_y", "direction_z", "wavelength"):
        a = np.ascontiguousarray(ph[name], dtype=np.float64)
        keep.append(a)
        setattr(s, name, a.ctypes.data)
    if ph.get("id") is not None:
        a = np.ascontiguousarray(ph["id"], dtype=np.int32)
        keep.append(a)
        s.simulation_truth_id = a.ctypes.data
    return s, keep


def alloc_results(n: int, max_interactions: int, history: bool):
    out = {
        "sensor": np.zeros(n, np.int32),
        "x": np.zeros(n), "y": np.zeros(n), "time": np.zeros(n),
        "theta_x": np.zeros(n), "theta_y": np.zeros(n),
        "final_leaf": np.zeros(n, np.int32), "info": np.zeros(n, np.uint32),
        "final_position": np.zeros((n, 3)), "final_direction": np.zeros((n, 3)),
    }
    if history:
        out["history"] = np.zeros((n, max_interactions + 1), abi.HISTORY_DTYPE)
    r = abi.mlgpu_results()
    r.dtype = abi.F64
    for k, a in out.items():
        setattr(r, k, a.ctypes.data)
    return r, out


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build(reference=False)
        self.lib = C.CDLL(path)
        self.lib.oracle_propagate.restype = C.c_int
        self.lib.oracle_propagate.argtypes = [
            C.POINTER(abi.mlgpu_flat_scene), C.POINTER(abi.mlgpu_photons), C.c_uint64,
            C.POINTER(abi.mlgpu_settings), C.POINTER(abi.mlgpu_rng),
            C.POINTER(abi.mlgpu_results), C.POINTER(OracleCounters)]
        self.lib.oracle_bin_arrivals.restype = None
        assert self.lib.oracle_sizeof_history_entry() == 64

    def propagate(self, scene: abi.FlatScene, photons: dict, max_interactions: int = 5,
                  seed: int = 0, uniforms: np.ndarray | None = None,
                  start_node: int = 0, history: bool = False,
                  photon_offset: int = 0):
        """Returns (status, results dict, counters dict)."""
        n = len(photons["wavelength"])
        ps, keep = _photon_struct(photons)
        st = abi.mlgpu_settings(max_interactions, start_node, abi.TRACER_FP64, 0)
        rng = abi.mlgpu_rng()
        if uniforms is not None:
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            keep.append(u)
            rng.mode = abi.RNG_REPLAY
            rng.stride = u.shape[1]
            rng.uniforms = u.ctypes.data
        else:
            rng.mode = abi.RNG_PHILOX
            rng.seed = seed
            rng.photon_offset = photon_offset
        rs, out = alloc_results(n, max_interactions, history)
        cnt = OracleCounters()
        fs = scene.as_struct()
        status = self.lib.oracle_propagate(C.byref(fs), C.byref(ps), n, C.byref(st),
                                           C.byref(rng), C.byref(rs), C.byref(cnt))
        return status, out, cnt.as_dict()

    def bin_arrivals(self, sensor, time, num_sensors, num_bins=0, t_min=0.0, t_max=1.0):
        sensor = np.ascontiguousarray(sensor, np.int32)
        time = np.ascontiguousarray(time, np.float64)
        counts = np.zeros(num_sensors, np.uint32)
        hist = np.zeros((num_sensors, max(num_bins, 1)), np.uint32)
        self.lib.oracle_bin_arrivals(
            sensor.ctypes.data_as(C.c_void_p), time.ctypes.data_as(C.c_void_p),
            C.c_uint64(len(sensor)), C.c_int32(num_sensors),
            counts.ctypes.data_as(C.c_void_p),
            hist.ctypes.data_as(C.c_void_p) if num_bins else None,
            C.c_uint32(num_bins), C.c_double(t_min), C.c_double(t_max))
        return counts, (hist if num_bins else None)


_harness = {}


def harness(path: str = HARNESS_SO):
    """The reference harness library (or, with SHIM_HARNESS_SO, the same
    harness with the C++ drop-in linked in), its functions declared."""
    if path not in _harness:
        if not os.path.exists(path):
            raise RuntimeError(f"{os.path.basename(path)} not built (oracle/Makefile)")
        lib = C.CDLL(path)
        lib.ref_scene_build.restype = C.c_void_p
        lib.ref_scene_build.argtypes = [C.c_char_p, C.POINTER(C.c_double), C.c_int]
        lib.ref_scene_free.argtypes = [C.c_void_p]
        lib.ref_scene_flat.argtypes = [C.c_void_p, C.POINTER(abi.mlgpu_flat_scene)]
        lib.ref_scene_num_sensors.argtypes = [C.c_void_p]
        lib.ref_last_error.restype = C.c_char_p
        lib.ref_scene_from_json.restype = C.c_void_p
        lib.ref_scene_from_json.argtypes = [C.c_char_p, C.c_int]
        lib.ref_scene_sensor_ids.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        for name in ("ref_json_photons", "ref_table_photons"):
            getattr(lib, name).restype = C.c_int64
            getattr(lib, name).argtypes = [C.c_char_p, C.c_void_p, C.c_uint64]
        lib.ref_json_propagation_config.argtypes = [C.c_char_p, C.POINTER(C.c_uint64)]
        lib.ref_mt19937_uniforms.argtypes = [C.c_uint64, C.c_uint64, C.c_void_p]
        lib.ref_propagate.restype = C.c_int
        lib.ref_propagate.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64, C.c_uint32,
            C.c_int, C.c_uint64, C.c_void_p, C.c_uint32, C.c_int,
            C.POINTER(abi.mlgpu_results), C.POINTER(C.c_double)]
        lib.ref_last_supports.restype = C.c_uint64
        lib.ref_last_supports.argtypes = [C.c_void_p, C.c_void_p]
        lib.ref_rebuild_photons.restype = C.c_int
        lib.ref_rebuild_photons.argtypes = [
            C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64, C.c_uint32, C.c_void_p,
            C.c_void_p, C.c_void_p, C.POINTER(abi.mlgpu_results)]
        if hasattr(lib, "shim_propagate"):
            lib.shim_propagate.restype = C.c_int
            lib.shim_propagate.argtypes = [
                C.c_void_p, C.POINTER(abi.mlgpu_photons), C.c_uint64, C.c_uint32, C.c_int,
                C.c_uint64, C.POINTER(C.c_uint64), C.POINTER(abi.mlgpu_results)]
        _harness[path] = lib
    return _harness[path]


# propagation modes of ref_propagate
REPLAY_PHILOX = 0
REPLAY_UNIFORMS = 1
REFERENCE_SINGLE_THREAD = 2
REFERENCE_MULTI_THREAD = 3


class RefScene:
    """A scene built and propagated by the reference library."""

    def __init__(self, kind: str, params=(), lib_path: str = HARNESS_SO):
        self.lib = harness(lib_path)
        p = (C.c_double * max(len(params), 1))(*params)
        self.h = self.lib.ref_scene_build(kind.encode(), p, len(params))
        if not self.h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        self.kind = kind
        self.params = tuple(params)

    @classmethod
    def from_json(cls, path: str, plenoscope: bool = False) -> "RefScene":
        """A scenery read by the reference's own JSON reader (merlict's, or
        with `plenoscope` its plenoscope extension)."""
        self = cls.__new__(cls)
        self.lib = harness()
        self.h = self.lib.ref_scene_from_json(os.fspath(path).encode(), int(plenoscope))
        if not self.h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        self.kind = "json"
        self.params = (os.fspath(path), bool(plenoscope))
        return self

    def sensor_ids(self) -> np.ndarray:
        n = self.lib.ref_scene_sensor_ids(self.h, None, 0)
        ids = np.zeros(max(n, 1), dtype=np.uint64)
        self.lib.ref_scene_sensor_ids(self.h, ids.ctypes.data, n)
        return ids[:n]

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_scene_free(self.h)
            self.h = None

    def flat(self) -> abi.FlatScene:
        s = abi.mlgpu_flat_scene()
        if self.lib.ref_scene_flat(self.h, C.byref(s)) != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return abi.FlatScene.from_struct(s)

    def propagate(self, photons: dict, max_interactions: int = 5,
                  mode: int = REPLAY_PHILOX, seed: int = 0,
                  uniforms: np.ndarray | None = None, threads: int = 1,
                  history: bool = False, results: bool = True):
        """Returns (status, results dict or None, seconds)."""
        n = len(photons["wavelength"])
        ps, keep = _photon_struct(photons)
        up, stride = None, 0
        if uniforms is not None:
            u = np.ascontiguousarray(uniforms, dtype=np.float64)
            keep.append(u)
            up, stride = u.ctypes.data, u.shape[1]
        out = None
        rs_ptr = None
        if results:
            rs, out = alloc_results(n, max_interactions, history)
            rs_ptr = C.byref(rs)
        sec = C.c_double(0.0)
        status = self.lib.ref_propagate(self.h, C.byref(ps), n, max_interactions, mode,
                                        seed, up, stride, threads, rs_ptr, C.byref(sec))
        if status != 0 and out is None:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return status, out, sec.value

    def last_supports(self) -> np.ndarray:
        """[n][3]: the ray support of each photon after the last propagation."""
        n = int(self.lib.ref_last_supports(self.h, None))
        out = np.zeros((max(n, 1), 3))
        self.lib.ref_last_supports(self.h, out.ctypes.data)
        return out[:n]

    def rebuild(self, photons: dict, max_interactions: int, results: dict):
        """merlict_b200::rebuild_histories on fresh photons from the exported
        `results` (history, info, final_direction), then merlict's
        Sensors::assign_photons; returns (status, results dict)."""
        n = len(photons["wavelength"])
        ps, keep = _photon_struct(photons)
        hist = np.ascontiguousarray(results["history"])
        info = np.ascontiguousarray(results["info"], dtype=np.uint32)
        fd = np.ascontiguousarray(results["final_direction"], dtype=np.float64)
        rs, out = alloc_results(n, max_interactions, True)
        status = self.lib.ref_rebuild_photons(self.h, C.byref(ps), n, max_interactions,
                                              hist.ctypes.data, info.ctypes.data,
                                              fd.ctypes.data, C.byref(rs))
        return status, out

    def shim_propagate(self, photons: dict, max_interactions: int, mode: int, mt_seed: int):
        """The C++ drop-in on this scene (needs SHIM_HARNESS_SO): mode 0
        propagate_photons_in_frame_with_config + merlict's assign_photons, 1
        the _multi_thread twin, 2 propagate_and_assign_photons.  Returns
        (status, results dict, the Philox seed the drop-in drew)."""
        n = len(photons["wavelength"])
        ps, keep = _photon_struct(photons)
        rs, out = alloc_results(n, max_interactions, True)
        seed = C.c_uint64(0)
        status = self.lib.shim_propagate(self.h, C.byref(ps), n, max_interactions, mode,
                                         mt_seed, C.byref(seed), C.byref(rs))
        return status, out, int(seed.value)

    def last_error(self) -> str:
        return self.lib.ref_last_error().decode()


def corsika_photons_reference(bunches: np.ndarray, uniforms: np.ndarray) -> dict:
    """merlict's own EventIoPhotonFactory (through the harness) on bunches
    [n][8] float32, bunch i drawing uniforms[i]."""
    L = C.CDLL(HARNESS_SO)
    b = np.ascontiguousarray(bunches, dtype=np.float32)
    u = np.ascontiguousarray(uniforms, dtype=np.float64)
    n = b.shape[0]
    cap = 17 * n
    planes = {k: np.zeros(cap) for k in ("support_x", "support_y", "support_z", "direction_x",
                                          "direction_y", "direction_z", "wavelength")}
    ids = np.zeros(cap, np.int32)
    total = C.c_uint64(0)
    L.ref_corsika_photons.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p] + [C.c_void_p] * 8 + [
        C.c_uint64, C.POINTER(C.c_uint64)]
    L.ref_last_error.restype = C.c_char_p
    st = L.ref_corsika_photons(b.ctypes.data, n, u.ctypes.data, *[planes[k].ctypes.data for k in planes],
                               ids.ctypes.data, cap, C.byref(total))
    if st != 0:
        raise ValueError(L.ref_last_error().decode())
    t = int(total.value)
    out = {k: v[:t] for k, v in planes.items()}
    out["id"] = ids[:t]
    return out


def corsika_photons_numpy(bunches: np.ndarray, uniforms: np.ndarray) -> dict:
    """A NumPy restatement of EventIoPhotonFactory (merlict_corsika/
    PhotonFactory.cpp:8-136) in merlict's operation order; the direction is
    returned as the Photon holds it (normalised, Ray.cpp:16-20)."""
    b = np.asarray(bunches, dtype=np.float32).astype(np.float64)
    w = b[:, 6]
    if np.any((w < 0.0) | (w > 16.0)):
        raise ValueError("bunch weight outside [0, 16]")
    count = np.floor(w).astype(np.int64) + (np.asarray(uniforms) <= np.fmod(w, 1.0))
    u, v = b[:, 2], b[:, 3]
    z = np.sqrt(1.0 - u * u - v * v)
    cx, cy, cz = u, v, -z
    ux, uy, uz = cx * -1.0, cy * -1.0, cz * -1.0
    un = np.sqrt(ux * ux + uy * uy + uz * uz)
    par = (b[:, 4] * 1e-9) * 299792458.0 + 1e3
    sx, sy, sz = b[:, 0] * 1e-2 + (ux / un) * par, b[:, 1] * 1e-2 + (uy / un) * par, 0.0 + (uz / un) * par
    dn = np.sqrt(cx * cx + cy * cy + cz * cz)
    rep = lambda a: np.repeat(a, count)
    return {"support_x": rep(sx), "support_y": rep(sy), "support_z": rep(sz),
            "direction_x": rep(cx / dn), "direction_y": rep(cy / dn), "direction_z": rep(cz / dn),
            "wavelength": rep(np.abs(b[:, 7] * 1e-9)),
            "id": rep(np.arange(b.shape[0], dtype=np.int32))}


def lixel_statistics_reference(sensor, cx, cy, x, y, t, num_lixel: int, num_blocks: int,
                               photons_per_block: int) -> np.ndarray:
    """merlict's own LixelStatisticsFiller (through the harness) on one block
    of per-photon results; returns [num_lixel][12] float32."""
    L = C.CDLL(HARNESS_SO)
    arrs = [np.ascontiguousarray(sensor, dtype=np.int32)] + [
        np.ascontiguousarray(a, dtype=np.float32) for a in (cx, cy, x, y, t)]
    out = np.zeros((num_lixel, 12), np.float32)
    L.ref_lixel_statistics.argtypes = [C.c_void_p] * 6 + [C.c_uint64] * 4 + [C.c_void_p]
    st = L.ref_lixel_statistics(*[a.ctypes.data for a in arrs], arrs[0].size, num_lixel,
                                num_blocks, photons_per_block, out.ctypes.data)
    if st != 0:
        raise RuntimeError("reference statistics failed")
    return out


def _ref_rows(fn, path: str) -> np.ndarray:
    L = harness()
    n = getattr(L, fn)(os.fspath(path).encode(), None, 0)
    if n < 0:
        raise RuntimeError(L.ref_last_error().decode())
    rows = np.zeros((max(n, 1), 8))
    getattr(L, fn)(os.fspath(path).encode(), rows.ctypes.data, n)
    return rows[:n]


def json_photons_reference(path: str) -> np.ndarray:
    """merlict's json::load_photons, as rows [id, support, direction, wavelength]."""
    return _ref_rows("ref_json_photons", path)


def table_photons_reference(path: str) -> np.ndarray:
    """merlict's raw_matrix2photons(tsvio::gen_table_from_file), as rows."""
    return _ref_rows("ref_table_photons", path)


def json_propagation_config_reference(path: str) -> int:
    """merlict's json::load_PropagationConfig: max_num_interactions_per_photon."""
    L = harness()
    v = C.c_uint64(0)
    if L.ref_json_propagation_config(os.fspath(path).encode(), C.byref(v)) != 0:
        raise RuntimeError(L.ref_last_error().decode())
    return int(v.value)


def mt19937_uniforms_reference(seed: int, n: int) -> np.ndarray:
    """merlict's Mt19937(seed).uniform(), n times."""
    out = np.zeros(max(int(n), 1))
    harness().ref_mt19937_uniforms(int(seed), int(n), out.ctypes.data)
    return out[:int(n)]


def signal_chain_reference(mode: int, seed: int, offset: int, sensor, time, wavelength, truth,
                           num_sensors: int, lixel_efficiency, qe_xy, dark_rate: float,
                           probability_for_second_puls: float, flux_xy, lfs, exposure_time: float,
                           time_slice_duration: float, arrival_time_std: float, nsb_count=None):
    """merlict's own signal chain for one event (see ref_signal_chain):
    mode 0 replays the engine's per-lixel Philox draws (nsb_count gives the
    background photons per lixel), mode 1 runs merlict's Mt19937(seed).
    Returns a dict of numpy arrays plus the start time and the seconds the
    chain took."""
    L = harness()
    if not hasattr(L, "_signal_declared"):
        L.ref_signal_chain.restype = C.c_void_p
        L.ref_signal_chain.argtypes = [C.c_int, C.c_uint64, C.c_uint64] + [C.c_void_p] * 4 + [
            C.c_uint64, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint32, C.c_double, C.c_double,
            C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_signal_result.restype = C.c_uint64
        L.ref_signal_result.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.ref_signal_start_time.restype = C.c_double
        L.ref_signal_start_time.argtypes = [C.c_void_p]
        L.ref_signal_seconds.restype = C.c_double
        L.ref_signal_seconds.argtypes = [C.c_void_p]
        L.ref_signal_free.argtypes = [C.c_void_p]
        L._signal_declared = True
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        keep.append(a)
        return a.ctypes.data

    n = len(sensor)
    qe = np.ascontiguousarray(qe_xy, dtype=np.float64).reshape(-1, 2)
    flux = np.ascontiguousarray(flux_xy, dtype=np.float64).reshape(-1, 2)
    nc = None if nsb_count is None else arr(nsb_count, np.uint32)
    h = L.ref_signal_chain(int(mode), int(seed), int(offset), arr(sensor, np.int32),
                           arr(time, np.float64), arr(wavelength, np.float64), arr(truth, np.int32),
                           n, int(num_sensors), arr(lixel_efficiency, np.float32), arr(qe, np.float64),
                           qe.shape[0], float(dark_rate), float(probability_for_second_puls),
                           arr(flux, np.float64), flux.shape[0], arr(lfs, np.float64),
                           arr([exposure_time, time_slice_duration, arrival_time_std], np.float64), nc)
    if not h:
        raise RuntimeError(L.ref_last_error().decode())
    try:
        types = [np.uint64] * 3 + [np.float64, np.float64, np.int32, np.float64, np.int32, np.uint8,
                                   np.int32]
        names = ["pipeline_offset", "pulse_offset", "channel_offset", "pipeline_time",
                 "pipeline_wavelength", "pipeline_truth", "pulse_time", "pulse_truth",
                 "channel_slice", "channel_truth"]
        out = {}
        for which, (name, dt) in enumerate(zip(names, types)):
            m = L.ref_signal_result(h, which, None)
            a = np.zeros(max(int(m), 1), dtype=dt)
            L.ref_signal_result(h, which, a.ctypes.data)
            out[name] = a[:int(m)]
        out["nsb_exposure_start_time"] = L.ref_signal_start_time(h)
        out["seconds"] = L.ref_signal_seconds(h)
        return out
    finally:
        L.ref_signal_free(h)


def photon_stream_write_reference(path: str, truth_path: str, offsets, slices, truth,
                                  time_slice_duration: float) -> None:
    """merlict's PhotonStream::write and write_simulation_truth."""
    L = harness()
    L.ref_photon_stream_write.argtypes = [C.c_char_p, C.c_char_p] + [C.c_void_p] * 3 + [
        C.c_uint32, C.c_float]
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    sl = np.ascontiguousarray(slices, dtype=np.uint8)
    tr = np.ascontiguousarray(truth, dtype=np.int32)
    if L.ref_photon_stream_write(os.fspath(path).encode(), os.fspath(truth_path).encode(),
                                 o.ctypes.data, sl.ctypes.data, tr.ctypes.data, len(o) - 1,
                                 float(time_slice_duration)) != 0:
        raise RuntimeError(L.ref_last_error().decode())


def corsika_file_reference(path: str, kind: str) -> dict:
    """A CORSIKA file through merlict's own reader: kind 'eventio'
    (eventio::Run) or 'event_tape' (event_tape::Run)."""
    L = harness()
    L.ref_corsika_file_read.restype = C.c_void_p
    L.ref_corsika_file_read.argtypes = [C.c_char_p, C.c_int]
    L.ref_corsika_file_result.restype = C.c_uint64
    L.ref_corsika_file_result.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.ref_corsika_file_free.argtypes = [C.c_void_p]
    h = L.ref_corsika_file_read(os.fspath(path).encode(), 0 if kind == "eventio" else 1)
    if not h:
        raise RuntimeError(L.ref_last_error().decode())
    try:
        names = ["run_header", "telescope_positions", "event_headers", "telescope_offsets",
                 "offset_start", "bunches", "bunch_start", "input_card"]
        types = [np.float32] * 4 + [np.uint64, np.float32, np.uint64, np.uint8]
        out = {}
        for which, (name, dt) in enumerate(zip(names, types)):
            m = int(L.ref_corsika_file_result(h, which, None))
            a = np.zeros(max(m, 1), dtype=dt)
            L.ref_corsika_file_result(h, which, a.ctypes.data)
            out[name] = a[:m]
        out["input_card"] = out["input_card"].tobytes().decode("latin-1")
        return out
    finally:
        L.ref_corsika_file_free(h)
