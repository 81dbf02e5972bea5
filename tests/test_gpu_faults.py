"""Malformed inputs on the GPU, answered the way merlict answers them (the
CPU side of the same cases is tests/test_faults.py): a wavelength <= 0
fails the call with MLGPU_ERR_INVALID_ARGUMENT (merlict's Photon
constructor throws std::invalid_argument, Photon.cpp:20-28), ahead of any
out-of-range wavelength in the same batch; NaN and infinite inputs are
propagated with merlict's NaN arithmetic, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from merlict_development_kit_b200 import abi, photons as P
from oracle import oracle as O
from parity import mismatches
from test_faults import ODD_ROWS, with_bad_rows

pytestmark = pytest.mark.gpu

OUTPUTS = ("sensor", "x", "y", "time", "theta_x", "theta_y", "final_leaf", "info",
           "final_position", "final_direction")


@pytest.fixture(scope="module")
def eng():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from merlict_development_kit_b200 import engine
    return engine


@pytest.mark.parametrize("tracer", ["fp64", "fp64_plain", "fp32"])
def test_nonpositive_wavelength_is_an_invalid_argument(eng, tracer):
    import torch
    from conftest import load_golden
    flat, photons, ref, meta = load_golden("reflector_camera")
    scene = eng.Scene(flat)
    dtype = torch.float32 if tracer == "fp32" else torch.float64
    cfg = eng.PropagationConfig(meta["max_interactions"])
    # one photon at 0 nm among photons outside the property tables: the
    # invalid argument is the error the call reports
    bad = with_bad_rows(photons, {7: {"wavelength": 0.0}})
    bad["wavelength"][100:200] = 1500e-9
    with pytest.raises(ValueError, match="wavelength"):
        scene.propagate(eng.photons_to_device(bad, dtype=dtype), cfg, eng.Philox(1),
                        tracer=tracer, out_dtype=dtype)
    bad = with_bad_rows(photons, {len(photons["wavelength"]) - 1: {"wavelength": -5e-7}})
    with pytest.raises(ValueError):
        scene.propagate(eng.photons_to_device(bad, dtype=dtype), cfg, eng.Philox(1),
                        tracer=tracer, out_dtype=dtype)
    # the scene is usable afterwards and gives merlict's results
    out = scene.propagate(eng.photons_to_device(photons), cfg, eng.Philox(meta["seed"]),
                          outputs=("sensor", "x", "y", "time"))
    got = {k: v.cpu().numpy() for k, v in out.items()}
    assert mismatches(ref, got) == {}
    scene.close()


def test_nonpositive_wavelength_through_the_host_call(eng):
    from conftest import load_golden
    from merlict_development_kit_b200 import _native
    from oracle.oracle import _photon_struct, alloc_results
    flat, photons, _, meta = load_golden("reflector_camera")
    bad = with_bad_rows(photons, {0: {"wavelength": 0.0}})
    scene = eng.Scene(flat)
    ps, keep = _photon_struct(bad)
    n = len(bad["wavelength"])
    rs, _ = alloc_results(n, meta["max_interactions"], history=False)
    st = abi.mlgpu_settings(meta["max_interactions"], 0, abi.TRACER_FP64, 0, abi.TRAVERSAL_BVH)
    rng = abi.mlgpu_rng()
    rng.mode = abi.RNG_PHILOX
    status = _native.lib().mlgpu_propagate_host(scene.handle, C.byref(ps), n, C.byref(st),
                                                C.byref(rng), C.byref(rs))
    assert status == abi.ERR_INVALID_ARGUMENT
    scene.close()


@pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")
@pytest.mark.parametrize("tracer", ["fp64", "fp64_plain"])
@pytest.mark.parametrize("kind,params,source,max_int", [
    ("primitive_zoo", (), None, 10),
    ("light_field_sensor", (10.7, 5.35, 1.0, 0.186, 9, 1.1, 0.9), (5.55, 21.4, 0.5), 10),
])
def test_nan_and_infinite_inputs_match_the_reference(eng, kind, params, source, max_int, tracer):
    sc = O.RefScene(kind, params)
    base = (P.isotropic_shell_source(5000, 8, 4.0, 2.5) if source is None
            else P.downward_disc_source(5000, 8, *source))
    ph = with_bad_rows(base, ODD_ROWS)
    status, ref, _ = sc.propagate(ph, max_int, O.REPLAY_PHILOX, seed=3)
    assert status == 0
    scene = eng.Scene(sc.flat())
    out = scene.propagate(eng.photons_to_device(ph), eng.PropagationConfig(max_int),
                          eng.Philox(3), tracer=tracer, outputs=OUTPUTS)
    got = {k: v.cpu().numpy() for k, v in out.items()}
    got["info"] = got["info"].view(np.uint32)
    scene.close()
    assert mismatches(ref, got) == {}
