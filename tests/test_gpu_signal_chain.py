"""GPU parity of the signal chain (csrc/signal_chain.cu through
mlgpu_signal_chain): against the oracle's restatement on the same per-lixel
Philox draws, and against merlict's own background injection, conversion
and extraction replaying those draws.  Integer outputs (background photons
per lixel, pulse offsets, slices, truth ids) and the window start are
compared exactly."""
import numpy as np
import pytest

from merlict_development_kit_b200 import signal_chain as SC
from merlict_development_kit_b200.scenery import Func1
from oracle import oracle as O
from oracle import signal_oracle as SO
from test_signal_chain import FLUX, LFS, QE, chain_kwargs, event, flat, geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from merlict_development_kit_b200 import engine
    return engine


@pytest.fixture(scope="module")
def scene(eng):
    from conftest import load_golden
    flat_scene, *_ = load_golden("sphere")
    s = eng.Scene(flat_scene)
    yield s
    s.close()


def config(g, flux=FLUX, dark=5e6, p2=0.1, qe=QE, T=50e-9, dt=0.5e-9, sigma=0.4e-9):
    light = SC.NightSkyBackgroundLight(g, Func1(flux))
    return SC.SignalChainConfig(SC.PhotoElectricConverterConfig(Func1(qe), dark, p2), light, T, dt,
                                sigma), light


def gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, seed, offset, capacity=None):
    import torch
    dev = torch.device("cuda")
    ps = SC.run(scene, cfg, torch.as_tensor(sensor, device=dev), torch.as_tensor(t, device=dev),
                torch.as_tensor(w, device=dev), torch.as_tensor(tr, device=dev),
                torch.as_tensor(eff, device=dev), eng.Philox(seed, offset), capacity=capacity)
    return (ps.channel_offset.cpu().numpy().astype(np.uint64), ps.arrival_time_slice.cpu().numpy(),
            ps.simulation_truth_id.cpu().numpy(), ps.nsb_exposure_start_time,
            ps.nsb_count.cpu().numpy())


@pytest.mark.parametrize("case", ["default", "no_dark", "crosstalk", "empty", "one_lixel",
                                  "wide_spread", "bright_lixel"])
def test_gpu_matches_oracle_and_merlict(eng, scene, case):
    g = geometry()
    nl = g.num_lixels
    kw = {}
    n, one, spread = 5000, None, 3e-9
    if case == "no_dark":
        kw["dark"] = 0.0
    elif case == "crosstalk":
        kw["p2"] = 0.6
    elif case == "empty":
        n = 0
    elif case == "one_lixel":
        n, one = 400, 17
    elif case == "bright_lixel":
        # a run longer than one block's shared-memory sort (4,096 photons):
        # the stable radix sort of long runs
        n, one = 12_000, 17
    elif case == "wide_spread":
        spread = 400e-9
    sensor, t, w, tr, eff = event(3, n, nl, spread, one)
    cfg, light = config(g, **kw)
    off, sl, trg, start, nsb = gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 99, 7)
    o = SO.signal_chain(sensor, t, w, tr, nl, eff, **chain_kwargs(light, nl, **kw))
    o_off, o_sl, o_tr, *_ = flat(o)
    assert start == o["nsb_exposure_start_time"]
    assert np.array_equal(nsb, np.array(o["nsb_count"], dtype=np.int32))
    assert np.array_equal(off, o_off)
    assert np.array_equal(sl, o_sl)
    assert np.array_equal(trg, o_tr)
    if O.harness_available():
        r = O.signal_chain_reference(0, 99, 7, sensor, t, w, tr, nl, eff, QE, kw.get("dark", 5e6),
                                     kw.get("p2", 0.1), FLUX, LFS, 50e-9, 0.5e-9, 0.4e-9,
                                     nsb_count=nsb)
        assert r["nsb_exposure_start_time"] == start
        assert np.array_equal(off, r["channel_offset"])
        assert np.array_equal(sl, r["channel_slice"])
        assert np.array_equal(trg, r["channel_truth"])


def test_capacity_too_small_is_retried(eng, scene):
    g = geometry()
    sensor, t, w, tr, eff = event(5, 3000, g.num_lixels)
    cfg, _ = config(g)
    a = gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 1, 0)
    b = gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 1, 0, capacity=1)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))


def test_wavelength_outside_the_efficiency_table_raises(eng, scene):
    g = geometry()
    sensor, t, w, tr, eff = event(6, 300, g.num_lixels)
    sensor[:] = 3
    w[7] = 150e-9
    cfg, _ = config(g)
    with pytest.raises(IndexError):
        gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 1, 0)
    # the scene stays usable
    w[7] = 400e-9
    gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 1, 0)


def test_sensor_index_beyond_the_lixels_raises(eng, scene):
    g = geometry()
    sensor, t, w, tr, eff = event(6, 300, g.num_lixels)
    sensor[0] = g.num_lixels
    cfg, _ = config(g)
    with pytest.raises(ValueError):
        gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 1, 0)


def test_full_light_field_sensor_event(eng, scene):
    """A config-1-sized event (63,379 lixels, 2e6 photons): the window start
    and 150 sampled lixels against the oracle, and the stream's invariants."""
    import random
    g = geometry([10.7, 5.35, 6.5, 0.186, 9, 1.1])
    nl = g.num_lixels
    assert nl == 63379
    sensor, t, w, tr, eff = event(11, 2_000_000, nl)
    cfg, light = config(g)
    off, sl, trg, start, nsb = gpu_chain(eng, scene, cfg, sensor, t, w, tr, eff, 5, 0)
    kw = chain_kwargs(light, nl, seed=5, offset=0)
    pipes = SO.photon_pipelines(sensor, t, w, tr, nl)
    S = SO.nsb_exposure_start_time(pipes, 50e-9)
    assert start == S
    assert np.all(np.diff(off.astype(np.int64)) >= 0) and int(off[-1]) == len(sl)
    assert sl.max() < 100
    for lix in random.Random(0).sample(range(nl), 150):
        p, k = SO.inject_nsb_lixel(pipes[lix], S, 50e-9, eff[lix], light.rate, nl, kw["nsb_cdf"],
                                   kw["nsb_total_integral"], SO.Draws(5, SO.STAGE_NSB, 0, lix))
        assert k == nsb[lix]
        e = SO.photo_electric(p, kw["qe"], 5e6, 0.1, 50e-9, SO.Draws(5, SO.STAGE_PEC, 0, lix))
        x = SO.extract(e, 0.5e-9, 0.4e-9, SO.Draws(5, SO.STAGE_EXTRACT, 0, lix))
        a, b = int(off[lix]), int(off[lix + 1])
        assert [s for s, _ in x] == list(sl[a:b])
        assert [i for _, i in x] == list(trg[a:b])
