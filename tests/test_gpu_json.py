"""GPU parity for sceneries and photon sources read from JSON: the CUDA
tracer on the package's reading of a file against merlict's Propagator on
merlict's own reading of the same file, bit for bit (the Philox stream
replayed on both sides)."""
import os

import numpy as np
import pytest

from merlict_development_kit_b200 import json_scenery as J
from merlict_development_kit_b200 import scenery as S
from oracle import oracle as O
from parity import mismatches
from test_gpu_parity import run_gpu
from test_json_scenery import path, sensors_of, stl_scenery

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")]


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from merlict_development_kit_b200 import engine
    return engine


def check(eng, scenery_path, plenoscope, photons, max_int=8, seed=41):
    sc = J.load_scenery(scenery_path, plenoscope=plenoscope)
    flat = S.flatten(sc.root, sensors_of(sc, plenoscope))
    ref_scene = O.RefScene.from_json(scenery_path, plenoscope)
    status, ref, _ = ref_scene.propagate(photons, max_int, mode=O.REPLAY_PHILOX, seed=seed)
    assert status == 0
    got = run_gpu(eng, flat, photons, max_int, seed=seed)
    assert mismatches(ref, got) == {}
    return ref


@pytest.mark.parametrize("tracer_photons", ["point_source.json", "parallel_disc.json"])
def test_primitives_from_json(eng, tracer_photons):
    ph = J.load_photons(path(tracer_photons))
    if tracer_photons == "parallel_disc.json":
        ph = J.transform_photons(J.loads('{"pos": [0, 0, 12], "rot": [0, 0, 0]}'), ph)
    ref = check(eng, path("primitives.json"), False, ph)
    assert (ref["sensor"] >= 0).sum() > 100


def test_hexagonal_reflector_from_json(eng):
    ph = J.to_photons(J.loads('{"parallel_disc": {"disc_radius": 2.3, "num_photons": 50000}, '
                              '"pos": [0, 0, 8], "rot": [3.14159265358979, 0, 0]}'))
    ref = check(eng, path("reflector_hex.json"), False, ph, max_int=5)
    assert (ref["sensor"] == 0).sum() > 1000


def test_plenoscope_from_json(eng):
    ph = J.to_photons(J.loads('{"parallel_disc": {"disc_radius": 5.3, "num_photons": 100000}, '
                              '"pos": [0, 0, 20], "rot": [3.1355, 0.004, 0]}'))
    ref = check(eng, path("plenoscope.json"), True, ph, max_int=10)
    assert (ref["sensor"] >= 0).sum() > 1000


def test_stl_scenery_from_json(eng, tmp_path):
    p = stl_scenery(tmp_path)
    ph = J.to_photons(J.loads('{"point_source": {"opening_angle": 0.4, "num_photons": 20000}, '
                              '"pos": [0, 0, 5], "rot": [3.14159265358979, 0, 0]}'))
    check(eng, p, False, ph)
