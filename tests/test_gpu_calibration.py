"""Plenoscope calibration on the GPU: the per-lixel statistics kernel bit
for bit against merlict's own LixelStatisticsFiller, and a calibration run
of the 1-degree light-field sensor."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_lixel_statistics_match_the_reference_filler():
    import torch
    from merlict_development_kit_b200 import calibration as CAL, engine
    if not O.harness_available():
        pytest.skip("reference harness not built")
    flat = load_golden("light_field_small")[0]
    scene = engine.Scene(flat)
    n = 300_000
    rng = np.random.default_rng(7)
    sensor = rng.integers(-1, flat.num_sensors, size=n).astype(np.int32)
    sensor[rng.random(n) < 0.3] = -1
    sensor[sensor == 5] = 6            # a lixel without photons (NaN statistics)
    sensor[sensor == 7] = -1
    sensor[np.flatnonzero(sensor == 8)[1:]] = -1   # a lixel with one photon
    vals = [rng.normal(size=n).astype(np.float32) * s for s in (0.02, 0.02, 20.0, 20.0, 3e-9)]
    ref = O.lixel_statistics_reference(sensor, *vals, flat.num_sensors, 4, n // 4)
    dev = [torch.as_tensor(v, device="cuda") for v in [sensor] + vals]
    got = CAL.lixel_statistics(scene, *dev, (4 * (n // 4)) / flat.num_sensors)
    got = np.stack([got[f] for f in CAL.FIELDS], axis=1)
    assert np.array_equal(got, ref, equal_nan=True)
    assert np.isnan(got[5, 2]) and np.isnan(got[8, 3]) and not np.isnan(got[8, 2])
    scene.close()


def test_calibration_of_the_small_light_field_sensor():
    from merlict_development_kit_b200 import calibration as CAL, engine
    flat = load_golden("light_field_small")[0]
    scene = engine.Scene(flat)
    # the fixture's imaging system: f = 10.7 m, aperture radius 5.35 m, 1 degree field
    st = CAL.calibrate(scene, 5.35, np.deg2rad(0.5), num_photons=2_000_000, seed=3)
    eff = st["efficiency"]
    assert np.all(np.isfinite(eff)) and eff.mean() > 0.05
    seen = eff > 0.2 * eff.mean()
    # each lixel sees the sky through a small cone and the aperture through a
    # small patch: its spread in both is far below the calibration range's
    assert np.nanmedian(st["cx_std"][seen]) < 0.3 * np.deg2rad(0.6)
    assert np.nanmedian(st["x_std"][seen]) < 0.3 * 5.35 * 1.05
    assert np.all(np.abs(st["time_delay_mean"][seen]) < 1e-7)
    scene.close()
