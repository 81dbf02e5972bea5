"""The C++ drop-in (shim/merlict_b200_shim.h) on the GPU, called the way a
merlict application calls the reference's functions: scenes built by
merlict's own factories, photons as merlict Photon objects, merlict's
Mt19937 as the generator, and merlict's own unchanged
Sensors::assign_photons afterwards (merlict/sensor/Sensors.cpp:20-81).

The drop-in draws one seed from the generator (Generator::create_seed) for
the engine's Philox streams; merlict's Propagator replaying those streams
photon by photon must give the same photons: arrivals, histories rebuilt
through RayForPropagation::push_back_intersection_and_interaction
(RayForPropagation.h:49-51), the ray each photon ends with, and the
PhotonArrival rows of the fast path (Sensor.cpp:14-30)."""
import os

import numpy as np
import pytest

import bench
from merlict_development_kit_b200 import photons as P
from oracle import oracle as O
from parity import history_mismatches, mismatches

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.shim_harness_available(),
                                 reason="drop-in test harness not built (oracle/Makefile shim)")]

THREADS = max(1, os.cpu_count() or 1)
SCENES = {
    "light_field_telescope": ("light_field_sensor",
                              (10.7, 5.35, 6.5, 0.186, 9, 1.1, 0.9),
                              (bench.SOURCE["disc_radius"], bench.SOURCE["height"],
                               bench.SOURCE["max_zenith_deg"]), bench.MAX_INTERACTIONS),
    "reflector_camera": ("reflector_camera", (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2),
                         (2.0, 10.0, 1.5), 5),
}
ARRIVAL = ("sensor", "x", "y", "time", "theta_x", "theta_y")


@pytest.fixture(scope="module")
def scenes():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    # kept for the whole module: the drop-in caches its device copy by the
    # address of the world frame
    return {k: O.RefScene(kind, params, lib_path=O.SHIM_HARNESS_SO)
            for k, (kind, params, _, _) in SCENES.items()}


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("name", sorted(SCENES))
def test_drop_in_then_merlicts_assign_photons(scenes, name, mode):
    _, _, source, max_int = SCENES[name]
    sc = scenes[name]
    ph = P.downward_disc_source(200_000, 8 + mode, *source)
    status, got, seed = sc.shim_propagate(ph, max_int, mode, mt_seed=123 + mode)
    assert status == 0, sc.last_error()
    support_got = sc.last_supports()
    status, want, _ = sc.propagate(ph, max_int, O.REPLAY_PHILOX, seed=seed, threads=THREADS,
                                   history=True)
    assert status == 0, sc.last_error()
    support_want = sc.last_supports()
    assert (want["sensor"] >= 0).mean() > 0.2
    assert mismatches(want, got, info_mask=0xFFFF) == {}
    assert history_mismatches(want["history"], got["history"]) == {}
    assert np.array_equal(support_got, support_want)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_drop_in_fast_path_writes_merlicts_arrivals(scenes, name):
    """propagate_and_assign_photons: PhotonArrival rows written straight
    into the sensors, in Sensors::assign_photons' photon order."""
    _, _, source, max_int = SCENES[name]
    sc = scenes[name]
    ph = P.downward_disc_source(200_000, 21, *source)
    status, got, seed = sc.shim_propagate(ph, max_int, 2, mt_seed=7)
    assert status == 0, sc.last_error()
    status, want, _ = sc.propagate(ph, max_int, O.REPLAY_PHILOX, seed=seed, threads=THREADS)
    assert status == 0
    # only arrivals exist on this path: the photons themselves stay fresh
    assert np.array_equal(got["sensor"], want["sensor"])
    hit = want["sensor"] >= 0
    assert hit.mean() > 0.2
    for k in ARRIVAL[1:]:
        assert np.array_equal(got[k][hit], want[k][hit]), k


def test_drop_in_fast_path_above_one_ray_pool(scenes):
    """propagate_and_assign_photons stages its inputs and results in
    page-locked memory, so a batch of more than one ray pool (2^21 photons)
    is fed to one propagation piece by piece: the arrivals are still
    merlict's, photon for photon."""
    _, _, source, max_int = SCENES["light_field_telescope"]
    sc = scenes["light_field_telescope"]
    ph = P.downward_disc_source(2_200_000, 33, *source)
    status, got, seed = sc.shim_propagate(ph, max_int, 2, mt_seed=11)
    assert status == 0, sc.last_error()
    status, want, _ = sc.propagate(ph, max_int, O.REPLAY_PHILOX, seed=seed, threads=THREADS)
    assert status == 0
    assert np.array_equal(got["sensor"], want["sensor"])
    hit = want["sensor"] >= 0
    assert hit.mean() > 0.2
    for k in ARRIVAL[1:]:
        assert np.array_equal(got[k][hit], want[k][hit]), k


def test_drop_in_raises_merlicts_exception_type(scenes):
    """A wavelength outside a property table: merlict's Func1 throws
    std::out_of_range (function/Limits.cpp:37-46); the drop-in raises the
    same type from the engine's status."""
    _, _, source, max_int = SCENES["light_field_telescope"]
    sc = scenes["light_field_telescope"]
    ph = P.downward_disc_source(1000, 3, *source)
    ph["wavelength"][:] = 1500e-9
    status, _, _ = sc.shim_propagate(ph, max_int, 0, mt_seed=1)
    assert status == O.abi.ERR_OUT_OF_RANGE, sc.last_error()
    assert "range" in sc.last_error()
    # merlict's own single-thread path throws in the calling thread
    ref_status, _, _ = sc.propagate(ph, max_int, O.REFERENCE_SINGLE_THREAD, seed=1)
    assert ref_status == O.abi.ERR_OUT_OF_RANGE
    # the scene stays usable
    ph = P.downward_disc_source(1000, 3, *source)
    status, _, _ = sc.shim_propagate(ph, max_int, 0, mt_seed=1)
    assert status == 0
