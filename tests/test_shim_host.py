"""The C++ drop-in's host code without a GPU: its history rebuild
(merlict_b200::rebuild_histories) fed with merlict's own export must give
back merlict's photons, and the flattener plus the rebuild run clean under
AddressSanitizer and UndefinedBehaviorSanitizer."""
import os
import subprocess

import numpy as np
import pytest

import bench
from merlict_development_kit_b200 import photons as P
from oracle import oracle as O
from parity import history_mismatches, mismatches

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")


@needs_ref
def test_history_rebuild_round_trip_on_the_light_field_telescope():
    """merlict's Propagator on the full benchmarked telescope, its histories
    exported as the engine exports them, rebuilt into fresh merlict photons,
    binned by merlict's Sensors::assign_photons: every result, every history
    entry and the ray each photon ends with come back bit for bit."""
    sc = O.RefScene("light_field_sensor", (10.7, 5.35, 6.5, 0.186, 9, 1.1, 0.9))
    ph = P.downward_disc_source(20_000, 5, bench.SOURCE["disc_radius"], bench.SOURCE["height"],
                                bench.SOURCE["max_zenith_deg"])
    status, want, _ = sc.propagate(ph, bench.MAX_INTERACTIONS, O.REPLAY_PHILOX, seed=9,
                                   threads=8, history=True)
    assert status == 0
    support_want = sc.last_supports()
    status, got = sc.rebuild(ph, bench.MAX_INTERACTIONS, want)
    assert status == 0, sc.last_error()
    assert (want["sensor"] >= 0).mean() > 0.3
    assert mismatches(want, got, info_mask=0xFFFF) == {}
    assert history_mismatches(want["history"], got["history"]) == {}
    assert np.array_equal(sc.last_supports(), support_want)


@needs_ref
def test_history_rebuild_rejects_an_unknown_leaf():
    sc = O.RefScene("reflector_camera", (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2))
    ph = P.downward_disc_source(100, 5, 2.0, 10.0, 1.5)
    status, want, _ = sc.propagate(ph, 5, O.REPLAY_PHILOX, seed=9, history=True)
    assert status == 0
    bad = dict(want)
    bad["history"] = want["history"].copy()
    bad["history"]["leaf"][:, 1] = 10 ** 6
    status, _ = sc.rebuild(ph, 5, bad)
    assert status == O.abi.ERR_RUNTIME
    assert "unknown leaf" in sc.last_error()


@pytest.mark.skipif(not os.path.exists(O.SANITIZE_EXE), reason="sanitizer build not made")
def test_drop_in_host_code_under_address_and_undefined_behaviour_sanitizers():
    r = subprocess.run([O.SANITIZE_EXE], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "all scenes round-tripped" in r.stdout
    assert "ERROR: AddressSanitizer" not in r.stderr
    assert "runtime error" not in r.stderr


@pytest.mark.skipif(not O.shim_harness_available(), reason="drop-in harness not built")
def test_drop_in_harness_links_the_engine_and_exports_the_drop_in():
    """No GPU call: the library with merlict's signatures loads beside the
    engine and exposes its entry point."""
    lib = O.harness(O.SHIM_HARNESS_SO)
    assert hasattr(lib, "shim_propagate")
    maps = open(f"/proc/{os.getpid()}/maps").read()
    assert "libmerlict_b200.so" in maps
