"""CORSIKA photon bunches -> photons (merlict's EventIoPhotonFactory,
merlict_corsika/PhotonFactory.cpp:8-136): the NumPy restatement against
the reference factory itself on the CPU, and the device kernels
(mlgpu_corsika_photons) against the reference on the GPU."""
import numpy as np
import pytest

from oracle import oracle as O

PLANES = ("support_x", "support_y", "support_z", "direction_x", "direction_y", "direction_z",
          "wavelength")


def random_bunches(n, seed):
    rng = np.random.default_rng(seed)
    b = np.zeros((n, 8), np.float32)
    b[:, 0] = rng.uniform(-15000, 15000, n)          # cm
    b[:, 1] = rng.uniform(-15000, 15000, n)
    th = np.deg2rad(rng.uniform(0, 4, n))
    ph = rng.uniform(0, 2 * np.pi, n)
    b[:, 2] = np.sin(th) * np.cos(ph)
    b[:, 3] = np.sin(th) * np.sin(ph)
    b[:, 4] = rng.normal(0, 5, n)                     # ns
    b[:, 5] = rng.uniform(5e5, 2e6, n)                # cm
    w = rng.uniform(0, 16, n)
    w[::7] = np.floor(w[::7])                         # whole weights: no extra photon
    w[::11] = 0.0
    b[:, 6] = w
    b[:, 7] = rng.uniform(-700, -250, n)              # CORSIKA may store it negative
    return b, rng.random(n)


def normalised(d):
    n = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    return d[0] / n, d[1] / n, d[2] / n


@pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")
def test_numpy_restatement_matches_the_reference_factory():
    b, u = random_bunches(5000, 1)
    ref = O.corsika_photons_reference(b, u)
    got = O.corsika_photons_numpy(b, u)
    assert ref["id"].size > 20000
    for k in PLANES + ("id",):
        assert np.array_equal(ref[k], got[k]), k


@pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")
def test_reference_factory_rejects_weights_outside_range():
    b, u = random_bunches(10, 2)
    b[3, 6] = 17.0
    with pytest.raises(ValueError):
        O.corsika_photons_reference(b, u)
    with pytest.raises(ValueError):
        O.corsika_photons_numpy(b, u)


@pytest.mark.gpu
def test_device_bunches_match_the_reference_factory():
    import torch
    from merlict_development_kit_b200 import engine
    from conftest import load_golden
    b, u = random_bunches(20000, 3)
    ref = (O.corsika_photons_reference(b, u) if O.harness_available()
           else O.corsika_photons_numpy(b, u))
    scene = engine.Scene(load_golden("sphere")[0])
    got = scene.corsika_photons(torch.as_tensor(b, device="cuda"),
                                engine.Replay(torch.as_tensor(u[:, None], device="cuda")))
    got = {k: v.cpu().numpy() for k, v in got.items()}
    for k in ("support_x", "support_y", "support_z", "wavelength", "id"):
        assert np.array_equal(got[k], ref[k]), k
    d = normalised((got["direction_x"], got["direction_y"], got["direction_z"]))
    for k, v in zip(("direction_x", "direction_y", "direction_z"), d):
        assert np.array_equal(v, ref[k]), k
    # Philox draws: the expected number of photons is the sum of the weights
    big, _ = random_bunches(200000, 4)
    n = scene.corsika_photons(torch.as_tensor(big, device="cuda"), engine.Philox(5))["id"].numel()
    w = big[:, 6].astype(np.float64)
    frac = np.fmod(w, 1.0)
    assert abs(n - w.sum()) < 6 * np.sqrt((frac * (1 - frac)).sum()) + 1
    with pytest.raises(ValueError):
        bad = big[:10].copy()
        bad[2, 6] = -1.0
        scene.corsika_photons(torch.as_tensor(bad, device="cuda"), engine.Philox(5))
    scene.close()


@pytest.mark.gpu
def test_event_tape_bunches_through_the_device_factory(tmp_path):
    """An event tape written and read back by corsika_io, its events'
    bunches expanded on the device: the reference factory's photons."""
    import torch
    from merlict_development_kit_b200 import corsika_io as CI, engine
    from conftest import load_golden
    p = str(tmp_path / "run.tar")
    w = CI.EventTapeWriter(p, buffer_size=1000)
    w.write_runh(CI.header_block("RUNH", {1: 9}))
    sizes = [3000, 1, 2500]
    for e, n in enumerate(sizes, start=1):
        w.write_evth(CI.header_block("EVTH", {1: e, 43: 9}))
        w.write_bunches(random_bunches(n, 10 + e)[0])
    w.close()
    scene = engine.Scene(load_golden("sphere")[0])
    for e, ev in enumerate(CI.EventTapeRun(p), start=1):
        b = ev.photons
        assert len(b) == sizes[e - 1]
        u = np.random.default_rng(e).random(len(b))
        ref = (O.corsika_photons_reference(b, u) if O.harness_available()
               else O.corsika_photons_numpy(b, u))
        got = scene.corsika_photons(torch.as_tensor(b, device="cuda"),
                                    engine.Replay(torch.as_tensor(u[:, None], device="cuda")))
        for k in ("support_x", "support_y", "support_z", "wavelength", "id"):
            assert np.array_equal(got[k].cpu().numpy(), ref[k]), k
    scene.close()
