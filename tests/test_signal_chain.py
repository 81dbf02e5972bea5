"""The signal chain after binning: the oracle's restatement (the checker of
the CUDA kernels) against merlict's own background injection, conversion
and extraction driven by the same per-lixel draws; the light, the photon
stream files and merlict's own known answers."""
import os

import numpy as np
import pytest

from merlict_development_kit_b200 import factories as F
from merlict_development_kit_b200 import signal_chain as SC
from merlict_development_kit_b200.scenery import Func1, deg2rad
from oracle import oracle as O
from oracle import signal_oracle as SO

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")

LFS = [10.7, 5.35, 2.0, 0.2, 5, 1.1]          # 1,387 lixels
FLUX = [[250e-9, 1e17], [400e-9, 3e17], [700e-9, 2e17]]
QE = [[200e-9, 0.0], [450e-9, 0.6], [1200e-9, 0.0]]


def geometry(lfs=LFS):
    n = Func1([[200e-9, 1.5], [1200e-9, 1.5]])
    cfg = F.LightFieldSensorConfig(lfs[0], lfs[1], deg2rad(lfs[2]), deg2rad(lfs[3]), int(lfs[4]),
                                   lfs[5], n, n)
    return F.LightFieldSensorGeometry(cfg)


def event(seed, n, num_lixel, spread=3e-9, one_lixel=None):
    rng = np.random.default_rng(seed)
    sensor = rng.integers(-1, num_lixel, n).astype(np.int32)
    if one_lixel is not None:
        sensor[:] = one_lixel
    t = rng.normal(30e-9, spread, n)
    w = rng.uniform(300e-9, 600e-9, n)
    tr = rng.integers(0, 5000, n).astype(np.int32)
    eff = rng.uniform(0.0, 1.0, num_lixel).astype(np.float32)
    return sensor, t, w, tr, eff


def chain_kwargs(light, num_lixel, dark=5e6, p2=0.1, T=50e-9, dt=0.5e-9, sigma=0.4e-9, seed=99,
                 offset=7, qe=QE):
    return dict(qe=Func1(qe), dark_rate=dark, probability_for_second_puls=p2,
                nsb_cdf=light.wavelength_probability.cumulative_distribution_function,
                nsb_total_integral=light.wavelength_probability.total_integral_of_distribution,
                nsb_rate=light.rate, num_lixel=num_lixel, nsb_exposure_time=T,
                time_slice_duration=dt, arrival_time_std=sigma, seed=seed, offset=offset)


def flat(o):
    ch = o["channels"]
    off = np.cumsum([0] + [len(c) for c in ch]).astype(np.uint64)
    sl = np.array([p[0] for c in ch for p in c], dtype=np.uint8)
    tr = np.array([p[1] for c in ch for p in c], dtype=np.int32)
    pt = np.array([x[0] for p in o["photon_pipelines"] for x in p])
    pw = np.array([x[1] for p in o["photon_pipelines"] for x in p])
    pu = np.array([x[0] for p in o["electric_pipelines"] for x in p])
    return off, sl, tr, pt, pw, pu


def run_both(sensor, t, w, tr, eff, g, flux=FLUX, **kw):
    light = SC.NightSkyBackgroundLight(g, Func1(flux))
    k = chain_kwargs(light, g.num_lixels, **kw)
    o = SO.signal_chain(sensor, t, w, tr, g.num_lixels, eff, **k)
    r = O.signal_chain_reference(0, k["seed"], k["offset"], sensor, t, w, tr, g.num_lixels, eff,
                                 kw.get("qe", QE), k["dark_rate"], k["probability_for_second_puls"],
                                 flux, [g.cfg.expected_imaging_system_focal_length,
                                        g.cfg.expected_imaging_system_max_aperture_radius,
                                        LFS[2], LFS[3], LFS[4], LFS[5]],
                                 k["nsb_exposure_time"], k["time_slice_duration"],
                                 k["arrival_time_std"], nsb_count=o["nsb_count"])
    return o, r


def assert_same(o, r):
    off, sl, tr, pt, pw, pu = flat(o)
    assert o["nsb_exposure_start_time"] == r["nsb_exposure_start_time"]
    assert np.array_equal(pt, r["pipeline_time"])
    assert np.array_equal(pw, r["pipeline_wavelength"])
    assert np.array_equal(pu, r["pulse_time"])
    assert np.array_equal(off, r["channel_offset"])
    assert np.array_equal(sl, r["channel_slice"])
    assert np.array_equal(tr, r["channel_truth"])


@needs_ref
@pytest.mark.parametrize("case", ["default", "no_background", "no_dark", "crosstalk", "empty",
                                  "one_lixel", "wide_spread", "no_sensor_hit"])
def test_oracle_matches_merlicts_chain_on_the_same_draws(case):
    g = geometry()
    nl = g.num_lixels
    kw = {}
    n, one, spread, flux = 5000, None, 3e-9, FLUX
    if case == "no_background":
        flux = [[250e-9, 0.0], [700e-9, 1e-30]]
    elif case == "no_dark":
        kw["dark"] = 0.0
    elif case == "crosstalk":
        kw["p2"] = 0.6
    elif case == "empty":
        n = 0
    elif case == "one_lixel":
        n, one = 400, 17
    elif case == "wide_spread":
        spread = 400e-9
    sensor, t, w, tr, eff = event(3, n, nl, spread, one)
    if case == "no_sensor_hit":
        sensor[:] = -1
    o, r = run_both(sensor, t, w, tr, eff, g, flux=flux, **kw)
    assert_same(o, r)
    if case not in ("empty", "no_sensor_hit"):
        assert len(r["channel_slice"]) > 0


@needs_ref
def test_quantum_efficiency_out_of_range_fails_in_both():
    g = geometry()
    sensor, t, w, tr, eff = event(4, 200, g.num_lixels)
    w[5] = 150e-9
    with pytest.raises(IndexError):
        run_both(sensor, t, w, tr, eff, g)
    with pytest.raises(RuntimeError):
        O.signal_chain_reference(1, 1, 0, sensor, t, w, tr, g.num_lixels, eff, QE, 0.0, 0.0, FLUX,
                                 LFS, 50e-9, 0.5e-9, 0.4e-9)


@needs_ref
def test_crosstalk_probability_one_is_refused():
    g = geometry()
    sensor, t, w, tr, eff = event(4, 10, g.num_lixels)
    with pytest.raises(RuntimeError):
        O.signal_chain_reference(1, 1, 0, sensor, t, w, tr, g.num_lixels, eff, QE, 0.0, 1.0, FLUX,
                                 LFS, 50e-9, 0.5e-9, 0.4e-9)
    with pytest.raises(ValueError):
        SC.PhotoElectricConverterConfig(Func1(QE), 0.0, 1.0).check()


@needs_ref
def test_production_mode_agrees_in_distribution():
    """merlict's own Mt19937 threaded through all lixels against the
    per-lixel Philox streams: the same pulse counts and slice distribution
    within their statistical errors."""
    g = geometry()
    sensor, t, w, tr, eff = event(8, 40000, g.num_lixels)
    light = SC.NightSkyBackgroundLight(g, Func1(FLUX))
    k = chain_kwargs(light, g.num_lixels, dark=2e7)
    counts_o, counts_r = [], []
    hist_o, hist_r = np.zeros(100), np.zeros(100)
    for s in range(3):
        k["seed"] = 100 + s
        o = SO.signal_chain(sensor, t, w, tr, g.num_lixels, eff, **k)
        _, sl, *_ = flat(o)
        r = O.signal_chain_reference(1, 100 + s, 0, sensor, t, w, tr, g.num_lixels, eff, QE, 2e7,
                                     0.1, FLUX, LFS, 50e-9, 0.5e-9, 0.4e-9)
        counts_o.append(len(sl))
        counts_r.append(len(r["channel_slice"]))
        hist_o += np.bincount(sl, minlength=100)
        hist_r += np.bincount(r["channel_slice"], minlength=100)
    a, b = sum(counts_o), sum(counts_r)
    assert abs(a - b) < 5 * np.sqrt(a + b)
    m = (hist_o + hist_r) > 20
    chi2 = np.sum((hist_o[m] / a - hist_r[m] / b) ** 2 / ((hist_o[m] + hist_r[m]) / (a * b)))
    assert chi2 / m.sum() < 2.0


# ---- the light and the window ------------------------------------------------------

def test_light_rate_follows_merlicts_formula():
    g = geometry()
    light = SC.NightSkyBackgroundLight(g, Func1(FLUX))
    fov = 1.20 * deg2rad(LFS[2]) / 2.0
    area = np.pi * (1.05 * LFS[1]) ** 2
    integral = (0.5 * (1e17 + 3e17) * 150e-9 + 0.5 * (3e17 + 2e17) * 300e-9)
    assert light.rate == pytest.approx(integral * area * 2 * np.pi * (1 - np.cos(fov)), rel=2e-3)
    w = [light.wavelength_probability.draw(u) for u in np.linspace(0, 0.999, 50)]
    assert min(w) >= 250e-9 and max(w) < 700e-9 and np.all(np.diff(w) >= 0)


def test_window_is_centred_on_the_mode():
    rng = np.random.default_rng(1)
    times = np.concatenate([rng.normal(20e-9, 1e-9, 5000), rng.uniform(0, 100e-9, 500)])
    pipes = [sorted([(float(x), 400e-9, 0) for x in times[i::7]]) for i in range(7)]
    S = SO.nsb_exposure_start_time(pipes, 200e-9)
    assert abs((S + 100e-9) - 20e-9) < 2e-9
    assert SO.nsb_exposure_start_time([[], []], 200e-9) == -100e-9


# ---- converter known answers (PhotoElectricConverterTest.cpp) -----------------------

def test_converter_known_answers():
    photons = [(i * 1e-9, 433e-9, i) for i in range(1337)]
    d = SO.Draws(0, SO.STAGE_PEC, 0, 0)
    assert SO.photo_electric([], SC.ZERO_EFFICIENCY, 0.0, 0.0, 1.0, d) == []
    assert SO.photo_electric(photons, SC.ZERO_EFFICIENCY, 0.0, 0.0, 1337e-9, d) == []
    one = Func1([[200e-9, 1.0], [1200e-9, 1.0]])
    out = SO.photo_electric(photons, one, 0.0, 0.0, 1337e-9, SO.Draws(0, SO.STAGE_PEC, 0, 1))
    assert [p[0] for p in out] == [p[0] for p in photons]
    dark = SO.photo_electric([], SC.ZERO_EFFICIENCY, 100e6, 0.0, 1e-6,
                             SO.Draws(0, SO.STAGE_PEC, 0, 2))
    assert abs(len(dark) - 100) < 35
    assert all(p[1] == SO.PHOTO_ELECTRIC_CONVERTER_ACCIDENTAL for p in dark)


def test_extraction_keeps_slices_0_to_99():
    pulses = [(t * 1e-9, 1) for t in (-5.0, 0.0, 0.2, 49.6, 99.4, 99.6, 150.0)]
    out = SO.extract(pulses, 1e-9, 0.0, SO.Draws(0, SO.STAGE_EXTRACT, 0, 0))
    assert [s for s, _ in out] == [0, 0, 50, 99]


# ---- photon stream files (PhotonStream.cpp) ----------------------------------------

def stream_example():
    ch = [[(3, 7), (4, -100)], [], [(99, -201)], [], [(0, 1), (0, 2), (12, -202)]]
    return SC.PhotonStream.from_channels(ch, 0.5e-9)


@needs_ref
def test_photon_stream_files_match_merlicts(tmp_path):
    s = stream_example()
    mine, mine_t = str(tmp_path / "a.phs"), str(tmp_path / "a.truth")
    ref, ref_t = str(tmp_path / "b.phs"), str(tmp_path / "b.truth")
    SC.write(s, mine)
    SC.write_simulation_truth(s, mine_t)
    O.photon_stream_write_reference(ref, ref_t, s.channel_offset, s.arrival_time_slice,
                                    s.simulation_truth_id, s.time_slice_duration)
    assert open(mine, "rb").read() == open(ref, "rb").read()
    assert open(mine_t, "rb").read() == open(ref_t, "rb").read()
    back = SC.read_with_simulation_truth(ref, ref_t)
    assert np.array_equal(back.channel_offset, s.channel_offset)
    assert np.array_equal(back.arrival_time_slice, s.arrival_time_slice)
    assert np.array_equal(back.simulation_truth_id, s.simulation_truth_id)


def test_photon_stream_round_trip_and_rules(tmp_path):
    s = stream_example()
    p = str(tmp_path / "s.phs")
    SC.write(s, p)
    assert SC.num_symbols_to_represent(s) == 6 + 4
    back = SC.read(p)
    assert back.num_channels == 5
    assert np.array_equal(back.channel_offset, s.channel_offset)
    assert back.time_slice_duration == np.float32(0.5e-9)
    bad = SC.PhotonStream.from_channels([[(255, 0)]], 1e-9)
    with pytest.raises(RuntimeError):
        SC.write(bad, str(tmp_path / "bad.phs"))
    empty = SC.PhotonStream.from_channels([], 1e-9)
    SC.write(empty, p)
    assert SC.read(p).num_channels == 0
    with pytest.raises(RuntimeError):
        SC.read(str(tmp_path / "missing.phs"))
    assert os.path.getsize(p) == 16


def test_lixel_statistics_file_round_trip(tmp_path):
    from merlict_development_kit_b200 import calibration as CAL
    rng = np.random.default_rng(2)
    st = {f: rng.normal(size=7).astype(np.float32) for f in CAL.FIELDS}
    p = str(tmp_path / "lixel_statistics.bin")
    CAL.write(st, p)
    assert os.path.getsize(p) == 7 * 48
    with open(p, "ab") as f:
        f.write(b"\0" * 20)                       # a partial record is not read
    back = CAL.read(p)
    for f in CAL.FIELDS:
        assert np.array_equal(back[f], st[f])
    assert np.array_equal(CAL.read_efficiencies(p), st["efficiency"])
