"""Malformed inputs, on the CPU: the engine's checker and the C ABI answer
them the way merlict does.

* A wavelength <= 0: merlict's Photon constructor throws
  std::invalid_argument (merlict/Photon.cpp:20-28) before anything is
  propagated; the engine fails the call with MLGPU_ERR_INVALID_ARGUMENT.
* A NaN or zero direction, a NaN wavelength, an infinite support: merlict
  throws nothing (Ray::set_support_and_direction normalises to NaN,
  Func1's limits let NaN through, Limits.cpp:37-46); the photon is
  propagated with NaN arithmetic and the engine must give the same bits.
* Two sensors on one frame: merlict's Sensors throws DuplicateFrame, a
  std::invalid_argument (Sensors.cpp:84-100); in the flat layout that is a
  sensor index on two leaves, rejected before any device work."""
import ctypes as C

import numpy as np
import pytest

from merlict_development_kit_b200 import abi, factories as F, photons as P
from merlict_development_kit_b200 import scenery as S
from oracle import oracle as O
from parity import mismatches

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")


def with_bad_rows(ph, rows):
    """A copy of the batch with some photons replaced: rows = {index: {plane: value}}."""
    out = {k: np.array(v, copy=True) for k, v in ph.items()}
    for i, planes in rows.items():
        for k, v in planes.items():
            out[k][i] = v
    return out


NAN = float("nan")
ODD_ROWS = {
    3: {"direction_x": NAN},
    10: {"direction_x": 0.0, "direction_y": 0.0, "direction_z": 0.0},
    17: {"wavelength": NAN},
    25: {"support_z": float("inf")},
    31: {"direction_z": float("-inf")},
    40: {"support_x": NAN},
}


@needs_ref
@pytest.mark.parametrize("wavelength", [0.0, -450e-9])
def test_nonpositive_wavelength_fails_before_propagation(oracle, wavelength):
    sc = O.RefScene("reflector_camera", (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2))
    ph = with_bad_rows(P.downward_disc_source(1000, 2, 2.0, 10.0, 1.5),
                       {500: {"wavelength": wavelength}})
    status, _, _ = sc.propagate(ph, 5, O.REPLAY_PHILOX, seed=1)
    assert status == abi.ERR_INVALID_ARGUMENT
    st, _, _ = oracle.propagate(sc.flat(), ph, 5, seed=1)
    assert st == abi.ERR_INVALID_ARGUMENT


@needs_ref
@pytest.mark.parametrize("kind,params,source,max_int", [
    ("primitive_zoo", (), None, 10),
    ("light_field_sensor", (10.7, 5.35, 1.0, 0.186, 9, 1.1, 0.9), (5.55, 21.4, 0.5), 10),
])
def test_nan_and_infinite_inputs_propagate_like_the_reference(oracle, kind, params, source,
                                                              max_int):
    sc = O.RefScene(kind, params)
    base = (P.isotropic_shell_source(2000, 8, 4.0, 2.5) if source is None
            else P.downward_disc_source(2000, 8, *source))
    ph = with_bad_rows(base, ODD_ROWS)
    status, ref, _ = sc.propagate(ph, max_int, O.REPLAY_PHILOX, seed=3)
    assert status == 0
    st, got, _ = oracle.propagate(sc.flat(), ph, max_int, seed=3)
    assert st == 0
    assert mismatches(ref, got) == {}
    assert all(ref["sensor"][i] == -1 for i in (3, 10, 40))


def test_flat_scene_with_a_sensor_on_two_leaves_is_rejected():
    flat = F.reflector_camera().flatten()
    sensor = np.array(flat.leaf_sensor, copy=True)
    pixels = np.flatnonzero(sensor >= 0)
    sensor[pixels[1]] = sensor[pixels[0]]
    bad = abi.FlatScene(**{**flat.__dict__, "leaf_sensor": sensor})
    with pytest.raises(ValueError, match="two leaves"):
        bad.validate()
    from merlict_development_kit_b200 import _native
    L = _native.lib()
    fs = bad.as_struct()
    h = C.c_void_p()
    assert L.mlgpu_scene_create(C.byref(fs), C.byref(h)) == abi.ERR_INVALID_ARGUMENT
    assert "two leaves" in _native.last_error() or "is on leaves" in _native.last_error()
    assert not h.value


def test_builder_rejects_two_sensors_on_one_frame():
    sc = S.Scenery()
    disc = sc.root.add(S.Disc("d", (0.0, 0.0, 0.0), S.ROT3_UNITY))
    disc.set_radius(1.0)
    sc.add_sensor(0, disc)
    sc.add_sensor(1, disc)
    with pytest.raises(ValueError):
        sc.init()
