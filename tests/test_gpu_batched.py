"""The batched form: many air-shower-like events of very uneven sizes traced
as one photon stream through the wavefront tracer's pool (CUDA-graph
launches, autotuned knobs), against one call per event.  Each photon draws
from its own Philox stream (key seed, counter = its index in the whole
stream), so batching changes nothing in the results: FP64 results must be
bit-identical to the per-event calls of merlict's single-event API."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

OUTPUTS = ("sensor", "x", "y", "time", "final_leaf", "info")


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available()
    from merlict_development_kit_b200 import engine
    return engine


@pytest.fixture(scope="module")
def events():
    from merlict_development_kit_b200 import photons as P
    sizes = P.cherenkov_event_sizes(40, 3, min_photons=50, max_photons=20_000)
    # events aimed at the small (1 degree) light-field sensor of the test scene
    batch, offsets = P.cherenkov_events(sizes, 4, device="cuda", clip_radius=6.0,
                                        max_axis_zenith_deg=0.2, cone_deg=0.25,
                                        cone_spread_deg=0.05)
    return batch, offsets


def host(out):
    return {k: v.cpu().numpy() for k, v in out.items() if k in OUTPUTS}


def assert_same(a, b):
    for k in OUTPUTS:
        assert np.array_equal(a[k], b[k], equal_nan=True), k


def test_one_batched_call_equals_per_event_calls(eng, events):
    batch, off = events
    flat = load_golden("light_field_small")[0]
    scene = eng.Scene(flat)
    cfg = eng.PropagationConfig(10)
    whole = host(scene.propagate(batch, cfg, eng.Philox(9), outputs=OUTPUTS,
                                 tuning=dict(use_graph=1, check_period=4)))
    assert (whole["sensor"] >= 0).mean() > 0.05   # the events do light the sensor
    for e in range(len(off) - 1):
        a, b = int(off[e]), int(off[e + 1])
        part = {k: v[a:b].contiguous() for k, v in batch.items()}
        got = host(scene.propagate(part, cfg, eng.Philox(9, photon_offset=a), outputs=OUTPUTS,
                                   tuning=dict(use_graph=0)))
        assert_same(got, {k: v[a:b] for k, v in whole.items()})
    scene.close()


@pytest.mark.parametrize("tuning", [
    dict(pool_size=1024, check_period=1, use_graph=0, photon_order=1),
    dict(pool_size=1024, check_period=3, use_graph=1, photon_order=2),   # odd period: the graph takes 4
    dict(pool_size=4096, grid_blocks=148, staged_levels=5, use_graph=1),
    dict(pool_size=1 << 20, check_period=16, grid_blocks=2368, staged_levels=3, use_graph=1,
         photon_order=1),
])
@pytest.mark.parametrize("tracer", ["fp64", "fp32"])
def test_tuning_knobs_do_not_change_results(eng, events, tuning, tracer):
    import torch
    batch, _ = events
    if tracer == "fp32":
        batch = {k: v.float() for k, v in batch.items()}
    out_dtype = torch.float32 if tracer == "fp32" else torch.float64
    flat = load_golden("light_field_small")[0]
    scene = eng.Scene(flat)
    cfg = eng.PropagationConfig(10)
    ref = host(scene.propagate(batch, cfg, eng.Philox(21), tracer=tracer, outputs=OUTPUTS,
                               out_dtype=out_dtype))
    got = host(scene.propagate(batch, cfg, eng.Philox(21), tracer=tracer, outputs=OUTPUTS,
                               out_dtype=out_dtype, tuning=tuning))
    assert_same(got, ref)
    scene.close()


def test_autotune_picks_knobs_from_its_candidates(eng, events):
    batch, _ = events
    flat = load_golden("light_field_small")[0]
    scene = eng.Scene(flat)
    cfg = eng.PropagationConfig(10)
    sample = {k: v[:200_000].contiguous() for k, v in batch.items()}
    tuning, ms = scene.autotune(sample, cfg, eng.Philox(1))
    assert ms > 0.0
    assert tuning["pool_size"] in (0, 1 << 19, 1 << 20, 1 << 21, 1 << 22)
    assert tuning["check_period"] in (0, 2, 4, 8, 16)
    assert tuning["use_graph"] in (0, 1)
    assert tuning["staged_levels"] in (0, 3, 5)
    assert tuning["photon_order"] in (0, 1, 2)
    ref = host(scene.propagate(batch, cfg, eng.Philox(5), outputs=OUTPUTS))
    got = host(scene.propagate(batch, cfg, eng.Philox(5), outputs=OUTPUTS, tuning=tuning))
    assert_same(got, ref)
    scene.close()


def test_invalid_tuning_is_rejected(eng, events):
    batch, _ = events
    flat = load_golden("light_field_small")[0]
    scene = eng.Scene(flat)
    for bad in (dict(pool_size=100), dict(check_period=65), dict(use_graph=2),
                dict(grid_blocks=-1), dict(staged_levels=49), dict(photon_order=3)):
        with pytest.raises(ValueError):
            scene.propagate(batch, eng.PropagationConfig(10), eng.Philox(1), tuning=bad)
    scene.close()


@pytest.mark.parametrize("grid_blocks", [0, 3, 1000])
def test_persistent_work_queue_equals_per_event_calls(eng, events, grid_blocks):
    """The whole batch of uneven events in one persistent launch whose warps
    pull photon tiles from a device work queue (tracer fp64_queue), with the
    default grid, a grid far smaller than the GPU (3 blocks drain the whole
    queue) and a larger one: bit-identical to per-event wavefront calls."""
    batch, off = events
    flat = load_golden("light_field_small")[0]
    scene = eng.Scene(flat)
    cfg = eng.PropagationConfig(10)
    launches0 = scene.kernel_launches()
    queued = host(scene.propagate(batch, cfg, eng.Philox(9), outputs=OUTPUTS, tracer="fp64_queue",
                                  tuning=dict(grid_blocks=grid_blocks)))
    # one launch for the queue (plus the tracing order's kernels)
    assert scene.kernel_launches() - launches0 <= 8
    for e in range(len(off) - 1):
        a, b = int(off[e]), int(off[e + 1])
        part = {k: v[a:b].contiguous() for k, v in batch.items()}
        got = host(scene.propagate(part, cfg, eng.Philox(9, photon_offset=a), outputs=OUTPUTS))
        assert_same(got, {k: v[a:b] for k, v in queued.items()})
    scene.close()
