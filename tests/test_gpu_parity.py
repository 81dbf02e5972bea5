"""GPU parity: the CUDA FP64 tracer against the reference's own outputs
(golden fixtures) and against the CPU oracle, through the C ABI."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_names, load_golden
from merlict_development_kit_b200 import photons as P
from parity import history_mismatches, mismatches

pytestmark = pytest.mark.gpu

ALL_OUTPUTS = ("sensor", "x", "y", "time", "theta_x", "theta_y", "final_leaf", "info",
               "final_position", "final_direction")


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from merlict_development_kit_b200 import engine
    return engine


def run_gpu(eng, flat, photons, max_int, seed=0, uniforms=None, history=False,
            tracer="fp64", outputs=ALL_OUTPUTS):
    scene = eng.Scene(flat)
    dev = eng.photons_to_device(photons)
    rng = eng.Replay(uniforms) if uniforms is not None else eng.Philox(seed)
    out = scene.propagate(dev, eng.PropagationConfig(max_int), rng, tracer=tracer,
                          outputs=outputs, history=history)
    got = {k: v.cpu().numpy() for k, v in out.items() if k != "history"}
    if "info" in got:
        got["info"] = got["info"].view(np.uint32)
    if history:
        got["history"] = eng.history_to_numpy(out["history"])
    scene.close()
    return got


FP64_TRACERS = ("fp64", "fp64_plain", "fp64_queue")


@pytest.mark.parametrize("tracer", FP64_TRACERS)
@pytest.mark.parametrize("name", golden_names())
def test_fp64_tracer_matches_reference_bit_for_bit(eng, name, tracer):
    flat, photons, ref, meta = load_golden(name)
    got = run_gpu(eng, flat, photons, meta["max_interactions"], seed=meta["seed"],
                  uniforms=meta["uniforms"], history=True, tracer=tracer)
    assert mismatches(ref, got) == {}
    assert history_mismatches(ref["history"], got["history"]) == {}


@pytest.mark.parametrize("tracer", FP64_TRACERS)
@pytest.mark.parametrize("name,n", [("reflector_camera", 200_000),
                                    ("light_field_small", 100_000),
                                    ("primitive_zoo", 200_000)])
def test_fp64_tracer_matches_oracle_on_larger_batches(eng, oracle, name, n, tracer):
    from merlict_development_kit_b200 import photons as P
    flat, _, _, meta = load_golden(name)
    if name == "primitive_zoo":
        ph = P.isotropic_shell_source(n, 123, 4.0, 2.5)
    elif name == "light_field_small":
        ph = P.downward_disc_source(n, 123, 5.55, 21.4, 0.5)
    else:
        ph = P.downward_disc_source(n, 123, 2.0, 10.0, 1.5)
    status, ref, _ = oracle.propagate(flat, ph, meta["max_interactions"], seed=77)
    assert status == 0
    got = run_gpu(eng, flat, ph, meta["max_interactions"], seed=77, tracer=tracer)
    assert mismatches(ref, got) == {}


@pytest.mark.parametrize("max_int", [0, 1, 2, 3])
def test_interaction_limit_and_zero_limit(eng, oracle, max_int):
    """PhotonAndFrame.cpp:18-21: the limit counts the production entry."""
    flat, photons, ref, meta = load_golden("light_field_small")
    status, ref, _ = oracle.propagate(flat, photons, max_int, seed=3, history=True)
    for tracer in FP64_TRACERS:
        got = run_gpu(eng, flat, photons, max_int, seed=3, history=True, tracer=tracer)
        assert mismatches(ref, got) == {}, tracer
        assert history_mismatches(ref["history"], got["history"]) == {}, tracer


def test_propagate_host_entry_point(eng):
    """mlgpu_propagate_host: host buffers in and out, as the C++ shim calls it."""
    from merlict_development_kit_b200 import _native, abi
    from oracle.oracle import _photon_struct, alloc_results
    flat, photons, ref, meta = load_golden("reflector_camera")
    scene = eng.Scene(flat)
    ps, keep = _photon_struct(photons)
    n = len(photons["wavelength"])
    rs, out = alloc_results(n, meta["max_interactions"], history=True)
    st = abi.mlgpu_settings(meta["max_interactions"], 0, abi.TRACER_FP64, 0, abi.TRAVERSAL_BVH)
    rng = abi.mlgpu_rng()
    rng.mode = abi.RNG_PHILOX
    rng.seed = meta["seed"]
    _native.check(_native.lib().mlgpu_propagate_host(scene.handle, C.byref(ps), n, C.byref(st),
                                                     C.byref(rng), C.byref(rs)))
    assert mismatches(ref, out) == {}
    assert history_mismatches(ref["history"], out["history"]) == {}


def test_propagate_and_bin_host_entry_point(eng, oracle):
    """mlgpu_propagate_and_bin_host: the per-photon results of
    mlgpu_propagate_host plus per-sensor counts and time histograms of the
    whole batch, equal to the oracle's binning of those results."""
    from merlict_development_kit_b200 import _native, abi
    from oracle.oracle import _photon_struct, alloc_results
    flat, _, _, meta = load_golden("light_field_small")
    photons = P.downward_disc_source(300_000, 4, 5.55, 21.4, 0.5)
    scene = eng.Scene(flat)
    ps, keep = _photon_struct(photons)
    n = len(photons["wavelength"])
    st = abi.mlgpu_settings(meta["max_interactions"], 0, abi.TRACER_FP64, 0, abi.TRAVERSAL_BVH)
    st.pool_size = 65536   # several pieces when the buffers are pinned; pageable here
    rng = abi.mlgpu_rng()
    rng.mode = abi.RNG_PHILOX
    rng.seed = 12
    L = _native.lib()
    rs0, want = alloc_results(n, meta["max_interactions"], history=False)
    _native.check(L.mlgpu_propagate_host(scene.handle, C.byref(ps), n, C.byref(st), C.byref(rng),
                                         C.byref(rs0)))
    t = want["time"][want["sensor"] >= 0]
    t0, t1, nb = float(t.min()) - 1e-12, float(t.max()) + 1e-12, 24
    rs1, got = alloc_results(n, meta["max_interactions"], history=False)
    counts = np.full(flat.num_sensors, 7, np.uint32)
    hist = np.full((flat.num_sensors, nb), 7, np.uint32)
    _native.check(L.mlgpu_propagate_and_bin_host(
        scene.handle, C.byref(ps), n, C.byref(st), C.byref(rng), C.byref(rs1),
        counts.ctypes.data, hist.ctypes.data, nb, t0, t1))
    assert mismatches(want, got) == {}
    ref_counts, ref_hist = oracle.bin_arrivals(want["sensor"], want["time"], flat.num_sensors,
                                               nb, t0, t1)
    assert np.array_equal(counts, ref_counts)
    assert np.array_equal(hist, ref_hist)
    # counts only
    counts[:] = 7
    _native.check(L.mlgpu_propagate_and_bin_host(
        scene.handle, C.byref(ps), n, C.byref(st), C.byref(rng), C.byref(rs1),
        counts.ctypes.data, None, 0, 0.0, 0.0))
    assert np.array_equal(counts, ref_counts)
    scene.close()


def host_call_pinned(scene, photons, max_int, tracer, pool, seed=0, uniforms=None,
                     order=None):
    """mlgpu_propagate_host on page-locked buffers (so that it pipelines the
    batch in pieces of at least `pool` photons, or a quarter pool when it
    feeds one propagation)."""
    import torch
    from merlict_development_kit_b200 import _native, abi
    n = len(photons["wavelength"])
    keep = []

    def pinned(shape, dtype):
        dt = np.dtype(dtype)
        t = torch.empty(int(np.prod(shape)) * dt.itemsize, dtype=torch.uint8).pin_memory()
        keep.append(t)
        return t.numpy().view(dt).reshape(shape)

    ps = abi.mlgpu_photons()
    ps.dtype = abi.F64
    for name in ("support_x", "support_y", "support_z", "direction_x", "direction_y",
                 "direction_z", "wavelength"):
        a = pinned((n,), np.float64)
        a[:] = photons[name]
        setattr(ps, name, a.ctypes.data)
    out = {"sensor": pinned((n,), np.int32), "x": pinned((n,), np.float64),
           "y": pinned((n,), np.float64), "time": pinned((n,), np.float64),
           "theta_x": pinned((n,), np.float64), "theta_y": pinned((n,), np.float64),
           "final_leaf": pinned((n,), np.int32), "info": pinned((n,), np.uint32),
           "final_position": pinned((n, 3), np.float64),
           "final_direction": pinned((n, 3), np.float64),
           "history": pinned((n, max_int + 1), abi.HISTORY_DTYPE)}
    rs = abi.mlgpu_results()
    rs.dtype = abi.F64
    for k, a in out.items():
        setattr(rs, k, a.ctypes.data)
    tracers = {"fp64": abi.TRACER_FP64, "fp32": abi.TRACER_FP32, "fp64_plain": abi.TRACER_FP64_PLAIN}
    st = abi.mlgpu_settings(max_int, 0, tracers[tracer], 0, abi.TRAVERSAL_BVH)
    st.pool_size = pool
    if order is not None:
        st.photon_order = order
    rng = abi.mlgpu_rng()
    if uniforms is None:
        rng.mode = abi.RNG_PHILOX
        rng.seed = seed
    else:
        u = pinned(uniforms.shape, np.float64)
        u[:] = uniforms
        rng.mode = abi.RNG_REPLAY
        rng.stride = uniforms.shape[1]
        rng.uniforms = u.ctypes.data
    _native.check(_native.lib().mlgpu_propagate_host(scene.handle, C.byref(ps), n, C.byref(st),
                                                     C.byref(rng), C.byref(rs)))
    return {k: v.copy() for k, v in out.items()}


@pytest.mark.parametrize("tracer", ["fp64", "fp32"])
@pytest.mark.parametrize("rng_mode", ["philox", "replay"])
@pytest.mark.parametrize("fed", [False, True])
def test_propagate_host_in_pieces(eng, tracer, rng_mode, fed):
    """Pinned host buffers and a 1024-slot pool.  In the input order
    mlgpu_propagate_host traces the 4000 photons in four pieces (666, 1334,
    1333 and 667 photons: three whole pieces, the first and the last cut in
    half), one propagation each, whose copies overlap the tracing.  In the
    coherent order it feeds one propagation: sixteen pieces (133 photons
    first and last, 266 or 267 between) sorted on their own stream as they
    land, admitted as they are published, their results copied back as
    their photons finish -- one wavefront call instead of four.
    Photon i keeps its own random stream, so every result and history entry
    equals one call on device buffers (and, for the FP64 tracer with Philox
    draws, merlict's own)."""
    from merlict_development_kit_b200 import abi
    flat, photons, ref, meta = load_golden("light_field_small")
    uniforms = None
    if rng_mode == "replay":
        uniforms = np.random.default_rng(5).random((len(photons["wavelength"]), 64))
    scene = eng.Scene(flat)
    calls0 = scene.wavefront_stats()["calls"]
    got = host_call_pinned(scene, photons, meta["max_interactions"], tracer, 1024,
                           seed=meta["seed"], uniforms=uniforms,
                           order=abi.ORDER_COHERENT if fed else abi.ORDER_INPUT)
    assert scene.wavefront_stats()["calls"] - calls0 == (1 if fed else 4)
    scene.close()
    want = run_gpu(eng, flat, photons, meta["max_interactions"], seed=meta["seed"],
                   uniforms=uniforms, history=True, tracer=tracer)
    assert mismatches(want, got) == {}
    assert history_mismatches(want["history"], got["history"]) == {}
    if tracer == "fp64" and rng_mode == "philox":
        assert mismatches(ref, got) == {}
        assert history_mismatches(ref["history"], got["history"]) == {}


def test_wavelength_outside_property_table_raises(eng):
    flat, photons, ref, meta = load_golden("mirror_absorber")
    ph = {k: v.copy() for k, v in photons.items()}
    ph["wavelength"][:] = 1500e-9
    with pytest.raises(IndexError):
        run_gpu(eng, flat, ph, 5, seed=1)
    # the scene stays usable afterwards
    got = run_gpu(eng, flat, photons, 5, seed=meta["seed"])
    assert mismatches(ref, got) == {}


def test_exhausted_replay_stream_raises(eng):
    flat, photons, ref, meta = load_golden("reflector_camera_replay")
    with pytest.raises(Exception):
        run_gpu(eng, flat, photons, 5, uniforms=meta["uniforms"][:, :1])


def test_known_answer_statistics(eng):
    """PhotonTest.cpp:84-302 on 1e5 photons each."""
    from merlict_development_kit_b200 import photons as P
    n = 100_000
    flat, *_ = load_golden("mirror_absorber")
    ph = P.make_batch(np.tile([-2.0, 0, 0], (n, 1)), np.tile([1.0, 0, 0], (n, 1)),
                      np.arange(1, n + 1) / n * 100e-9 + 250e-9)
    got = run_gpu(eng, flat, ph, 5, seed=5, outputs=("sensor",))
    assert abs((got["sensor"] >= 0).mean() - 0.42) < 0.02
    flat, *_ = load_golden("water_box")
    ph = P.make_batch(np.zeros((n, 3)), np.tile([0, 0, 1.0], (n, 1)), np.full(n, 433e-9))
    got = run_gpu(eng, flat, ph, 5, seed=6, outputs=("sensor", "time"))
    hit = got["sensor"] >= 0
    assert abs(hit.mean() - 0.95) < 0.02
    assert abs(got["time"][hit].mean() - (2.0 + 1.33) / 299792458.0) < 1e-10
    flat, *_ = load_golden("absorbing_box")
    got = run_gpu(eng, flat, ph, 5, seed=7, outputs=("sensor",))
    assert abs((got["sensor"] >= 0).mean() - 0.367) < 0.02


def test_bin_arrivals_matches_oracle(eng, oracle):
    import torch
    from merlict_development_kit_b200 import photons as P
    flat, _, _, meta = load_golden("light_field_small")
    ph = P.downward_disc_source(300_000, 9, 5.55, 21.4, 0.5)
    scene = eng.Scene(flat)
    out = scene.propagate(eng.photons_to_device(ph), eng.PropagationConfig(10), eng.Philox(3),
                          outputs=("sensor", "time"))
    t = out["time"][out["sensor"] >= 0]
    t0, t1 = float(t.min()) - 1e-12, float(t.max()) + 1e-12
    counts, hist = scene.bin_arrivals(out["sensor"], out["time"], 16, t0, t1)
    ref_counts, ref_hist = oracle.bin_arrivals(out["sensor"].cpu().numpy(), out["time"].cpu().numpy(),
                                               flat.num_sensors, 16, t0, t1)
    assert np.array_equal(counts.cpu().numpy().astype(np.uint32), ref_counts)
    assert np.array_equal(hist.cpu().numpy().astype(np.uint32), ref_hist)
    counts2, _ = scene.bin_arrivals(out["sensor"])
    assert np.array_equal(counts2.cpu().numpy().astype(np.uint32), ref_counts)
    torch.cuda.synchronize()


def test_production_mode_histograms_match_the_reference(eng):
    """Production RNG on the config-0 camera: merlict's own multi-threaded
    path (Mt19937 seeds per photon) against the GPU's Philox stream --
    per-pixel counts by chi-squared, arrival times by a two-sample KS test."""
    from scipy import stats
    from oracle import oracle as O
    if not O.harness_available():
        pytest.skip("reference harness not built")
    params = (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2)
    scene_ref = O.RefScene("reflector_camera", params)
    flat = scene_ref.flat()
    ph = P.downward_disc_source(400_000, 12, 2.0, 10.0, 1.5)
    _, ref, _ = scene_ref.propagate(ph, 5, O.REFERENCE_MULTI_THREAD, seed=3)
    scene = eng.Scene(flat)
    out = scene.propagate(eng.photons_to_device(ph), eng.PropagationConfig(5), eng.Philox(77),
                          outputs=("sensor", "time"))
    got = {k: v.cpu().numpy() for k, v in out.items()}
    scene.close()
    a = np.bincount(ref["sensor"][ref["sensor"] >= 0], minlength=flat.num_sensors)
    b = np.bincount(got["sensor"][got["sensor"] >= 0], minlength=flat.num_sensors)
    m = (a + b) > 0
    chi2 = (((a - b) ** 2)[m] / (a + b)[m]).sum()
    dof = int(m.sum())
    assert chi2 < dof + 5 * np.sqrt(2 * dof), (chi2, dof)
    ks = stats.ks_2samp(ref["time"][ref["sensor"] >= 0], got["time"][got["sensor"] >= 0])
    assert ks.pvalue > 1e-3, ks


@pytest.mark.parametrize("name,n", [("reflector_camera", 200_000), ("light_field_small", 100_000),
                                    ("primitive_zoo", 200_000)])
def test_stack_walk_finds_the_same_hits(eng, oracle, name, n):
    """walk=STACK (one thread walks a ray's whole BVH) against the oracle,
    and against walk=LEVELS for the FP32 forms: the same candidates, so
    the same results."""
    flat, _, _, meta = load_golden(name)
    if name == "primitive_zoo":
        ph = P.isotropic_shell_source(n, 321, 4.0, 2.5)
    elif name == "light_field_small":
        ph = P.downward_disc_source(n, 321, 5.55, 21.4, 0.5)
    else:
        ph = P.downward_disc_source(n, 321, 2.0, 10.0, 1.5)
    status, ref, _ = oracle.propagate(flat, ph, meta["max_interactions"], seed=78)
    assert status == 0
    scene = eng.Scene(flat)
    dev = eng.photons_to_device(ph)
    outs = ("sensor", "x", "y", "time", "final_leaf")
    for tracer in ("fp64", "fp32"):
        got = {}
        for walk in (1, 2):
            o = scene.propagate(dev, eng.PropagationConfig(meta["max_interactions"]),
                                eng.Philox(78), tracer=tracer, outputs=outs,
                                tuning={"walk": walk})
            got[walk] = {k: v.cpu().numpy() for k, v in o.items()}
        for k in outs:
            assert np.array_equal(got[1][k], got[2][k]), (tracer, k)
        if tracer == "fp64":
            assert mismatches(ref, got[2]) == {}
    scene.close()


@pytest.mark.parametrize("n", [1_000_000, 40_000_000])
def test_bin_arrivals_counters_wide_and_narrow(eng, n):
    """The binning keeps 16-bit per-warp counters when no warp can count
    past 65,535 photons in one slice and 32-bit ones otherwise; 4e7 arrivals
    on a scene of few sensors take the 32-bit path, 1e6 the 16-bit one.
    Both against numpy's bincount, with time histograms, one sensor taking
    a tenth of all arrivals (more than 65,535 per warp and slice)."""
    import torch
    flat, _, _, _ = load_golden("light_field_small")
    scene = eng.Scene(flat)
    g = torch.Generator(device="cuda").manual_seed(5)
    ns = flat.num_sensors
    sensor = torch.randint(-1, ns, (n,), device="cuda", dtype=torch.int32, generator=g)
    sensor[::10] = 3
    time = torch.rand(n, device="cuda", dtype=torch.float64, generator=g) * 1e-8
    counts, hist = scene.bin_arrivals(sensor, time, 5, 0.0, 1e-8)
    s = sensor.cpu().numpy()
    t = time.cpu().numpy()
    ok = s >= 0
    ref_counts = np.bincount(s[ok], minlength=ns)
    f = (t[ok] - 0.0) / (1e-8 - 0.0) * 5.0
    inside = (f >= 0.0) & (f < 5.0)
    ref_hist = np.zeros((ns, 5), np.int64)
    np.add.at(ref_hist, (s[ok][inside], f[inside].astype(np.int64)), 1)
    assert np.array_equal(counts.cpu().numpy(), ref_counts)
    assert np.array_equal(hist.cpu().numpy(), ref_hist)
    counts2, _ = scene.bin_arrivals(sensor)
    assert np.array_equal(counts2.cpu().numpy(), ref_counts)
    scene.close()
