"""GPU parity on the benchmarked configurations themselves, at 1e6 photons
each, against merlict's own Propagator (the reference library compiled from
its sources) replaying the same Philox streams photon by photon -- the
pattern of merlict_multi_thread.cpp:12-26 with the engine's generator:

* config 0: the 30-facet reflector with the 1,440-pixel camera;
* config 1: the light-field telescope the bench traces (252 facets, 1,039
  lenses, 63,379 lixels, 78,378 leaves);
* config 3: the 5,388-facet R = 213 m reflector with 8,443 pixels.

The GPU traces the scene built by this package's own builder (the product
path); the reference traces the scene built by merlict's own factories.
FP64: every per-photon output bit for bit (sensor, final leaf, interaction
and count, x, y, theta, time, final position and direction).  FP32 on the
same photons: at least 99.99 % on the same sensor.

Also here: the wavefront's overflow fallback.  A ray whose entries do not
fit one of the work queues takes merlict's own frame-tree walk
(RayAndFrame.cpp:118-173); `queue_capacity` shrinks the queues so that
the fallback carries a large share of the rays, and the results must stay
bit for bit the same."""
import os

import numpy as np
import pytest

import bench
from conftest import load_golden
from merlict_development_kit_b200 import factories as F, photons as P
from oracle import oracle as O
from parity import mismatches

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")]

N = 1_000_000
THREADS = max(1, os.cpu_count() or 1)

CONFIGS = {
    "config0_camera": dict(
        kind="reflector_camera", params=(4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2),
        build=lambda: F.reflector_camera(), source=(2.0, 10.0, 1.5), max_int=5),
    "config1_light_field_telescope": dict(
        kind="light_field_sensor",
        params=(bench.SCENE["focal_length"], bench.SCENE["aperture_radius"],
                bench.SCENE["fov_deg"], bench.SCENE["pixel_fov_deg"],
                bench.SCENE["paxels_on_diagonal"], bench.SCENE["housing_overhead"],
                bench.SCENE["reflectivity"]),
        build=lambda: F.light_field_telescope(**bench.SCENE),
        source=(bench.SOURCE["disc_radius"], bench.SOURCE["height"],
                bench.SOURCE["max_zenith_deg"]),
        max_int=bench.MAX_INTERACTIONS),
    "config3_large_reflector": dict(
        kind="large_reflector", params=(106.5, 35.5, 0.0, 0.45, 0.01, 6.5, 0.06667, 0.9),
        build=lambda: F.large_reflector_camera(), source=(40.0, 110.0, 3.5), max_int=5),
}

OUTPUTS = ("sensor", "x", "y", "time", "theta_x", "theta_y", "final_leaf", "info",
           "final_position", "final_direction")


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from merlict_development_kit_b200 import engine
    return engine


def gpu_trace(eng, flat, ph, max_int, seed, tracer="fp64", tuning=None, scene=None):
    import torch
    own = scene is None
    scene = scene or eng.Scene(flat)
    dtype = torch.float32 if tracer == "fp32" else torch.float64
    outs = OUTPUTS if tracer == "fp64" else ("sensor", "x", "y", "time")
    out = scene.propagate(eng.photons_to_device(ph, dtype=dtype), eng.PropagationConfig(max_int),
                          eng.Philox(seed), tracer=tracer, outputs=outs, out_dtype=dtype,
                          tuning=tuning)
    got = {k: v.cpu().numpy() for k, v in out.items()}
    if "info" in got:
        got["info"] = got["info"].view(np.uint32)
    if own:
        scene.close()
    return got


def rounded_to_f32(ph):
    return {k: v.astype(np.float32).astype(np.float64) for k, v in ph.items()}


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_benchmarked_configuration_matches_reference(eng, name):
    c = CONFIGS[name]
    flat = c["build"]().flatten()
    ref_scene = O.RefScene(c["kind"], c["params"])
    ph = rounded_to_f32(P.downward_disc_source(N, 4711, *c["source"]))
    status, ref, _ = ref_scene.propagate(ph, c["max_int"], O.REPLAY_PHILOX, seed=2024,
                                         threads=THREADS)
    assert status == 0, ref_scene.last_error()
    got = gpu_trace(eng, flat, ph, c["max_int"], 2024)
    on_sensor = (ref["sensor"] >= 0).mean()
    assert on_sensor > 0.2, on_sensor
    assert mismatches(ref, got) == {}
    # FP32 form on the same (FP32-exact) photons and streams
    got32 = gpu_trace(eng, flat, ph, c["max_int"], 2024, tracer="fp32")
    agreement = (got32["sensor"] == ref["sensor"]).mean()
    assert agreement >= 0.9999, agreement


def test_overflow_fallback_is_exact_on_light_field_small(eng, oracle):
    """Queues of 1,024 entries for a pool of 100,000 rays: most rays of
    every iteration overflow and are resolved by merlict's frame walk."""
    flat, _, _, meta = load_golden("light_field_small")
    ph = P.downward_disc_source(100_000, 99, 5.55, 21.4, 0.5)
    status, want, _ = oracle.propagate(flat, ph, meta["max_interactions"], seed=5)
    assert status == 0
    scene = eng.Scene(flat)
    scene.wavefront_stats(reset=True)
    got = gpu_trace(eng, flat, ph, meta["max_interactions"], 5,
                    tuning={"queue_capacity": 1024}, scene=scene)
    stats = scene.wavefront_stats(reset=True)
    assert stats["overflow_rays"] > 50_000, stats
    assert mismatches(want, got) == {}
    # the same photons with the default queues: no overflow, same results
    again = gpu_trace(eng, flat, ph, meta["max_interactions"], 5, scene=scene)
    assert scene.wavefront_stats()["overflow_rays"] == 0
    assert mismatches(want, again) == {}
    scene.close()


@pytest.mark.parametrize("capacity", [65_536, 1 << 20])
def test_overflow_fallback_is_exact_on_light_field_telescope(eng, capacity):
    """The benchmarked telescope with queues that hold a part of what the
    pool of 2e5 rays needs, against the reference Propagator."""
    c = CONFIGS["config1_light_field_telescope"]
    flat = c["build"]().flatten()
    ref_scene = O.RefScene(c["kind"], c["params"])
    ph = P.downward_disc_source(200_000, 17, *c["source"])
    status, want, _ = ref_scene.propagate(ph, c["max_int"], O.REPLAY_PHILOX, seed=31,
                                          threads=THREADS)
    assert status == 0
    scene = eng.Scene(flat)
    scene.wavefront_stats(reset=True)
    got = gpu_trace(eng, flat, ph, c["max_int"], 31, scene=scene,
                    tuning={"queue_capacity": capacity, "pool_size": 200_000})
    stats = scene.wavefront_stats()
    assert stats["overflow_rays"] > 0, stats
    assert mismatches(want, got) == {}
    # the FP32 form through the same fallback
    got32 = gpu_trace(eng, flat, ph, c["max_int"], 31, tracer="fp32", scene=scene,
                      tuning={"queue_capacity": capacity, "pool_size": 200_000})
    assert (got32["sensor"] == want["sensor"]).mean() >= 0.9999
    scene.close()


def test_queue_capacity_is_validated(eng):
    flat, photons, _, meta = load_golden("reflector_camera")
    with pytest.raises(ValueError):
        gpu_trace(eng, flat, photons, meta["max_interactions"], 1, tuning={"queue_capacity": 8})


def test_production_mode_on_the_light_field_telescope(eng):
    """Production random streams on the benchmarked telescope: merlict's own
    multi-threaded path (an Mt19937 per photon, seeded from one generator,
    merlict_multi_thread.cpp:12-55) against the GPU's Philox streams on
    the same 2e6 photons.  Per-lixel counts: chi-squared within five sigma
    of its degrees of freedom, and a Jensen-Shannon divergence no larger
    than the noise floor between two GPU runs with independent seeds (plus
    a tenth of it); arrival times: a two-sample KS test."""
    from scipy import stats
    from merlict_development_kit_b200.precision import js_divergence
    c = CONFIGS["config1_light_field_telescope"]
    flat = c["build"]().flatten()
    ref_scene = O.RefScene(c["kind"], c["params"])
    ph = P.downward_disc_source(2_000_000, 23, *c["source"])
    status, ref, _ = ref_scene.propagate(ph, c["max_int"], O.REFERENCE_MULTI_THREAD, seed=5,
                                         threads=THREADS)
    assert status == 0, ref_scene.last_error()
    a = gpu_trace(eng, flat, ph, c["max_int"], 101)
    b = gpu_trace(eng, flat, ph, c["max_int"], 202)
    ns = flat.num_sensors

    def hist(r):
        s = r["sensor"]
        return np.bincount(s[s >= 0], minlength=ns).astype(np.float64)
    h_ref, h_a, h_b = hist(ref), hist(a), hist(b)
    assert h_ref.sum() > 0.2 * len(ph["wavelength"])
    m = (h_ref + h_a) > 0
    chi2 = (((h_ref - h_a) ** 2)[m] / (h_ref + h_a)[m]).sum()
    dof = int(m.sum())
    assert chi2 < dof + 5 * np.sqrt(2 * dof), (chi2, dof)
    floor = js_divergence(h_a, h_b)
    assert js_divergence(h_ref, h_a) <= 1.1 * floor, (js_divergence(h_ref, h_a), floor)
    t_ref = ref["time"][ref["sensor"] >= 0]
    t_gpu = a["time"][a["sensor"] >= 0]
    rng = np.random.default_rng(0)
    ks = stats.ks_2samp(rng.choice(t_ref, 200_000, replace=False),
                        rng.choice(t_gpu, 200_000, replace=False))
    assert ks.pvalue > 1e-3, ks
