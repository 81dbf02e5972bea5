"""The package's own scene builder reproduces scenes built by merlict's own
classes and factories, array by array and bit for bit."""
import numpy as np
import pytest

from merlict_development_kit_b200 import abi, factories as F
from merlict_development_kit_b200 import scenery as S
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")


def flat_diff(a, b):
    bad = []
    for k in abi.FlatScene.ARRAYS:
        x, y = getattr(a, k), getattr(b, k)
        if x.shape != y.shape:
            bad.append((k, "shape", x.shape, y.shape))
            continue
        eq = (x == y) | (np.isnan(x) & np.isnan(y)) if x.dtype.kind == "f" else (x == y)
        if not eq.all():
            bad.append((k, int((~eq).sum())))
    for k in ("default_refraction", "num_sensors"):
        if getattr(a, k) != getattr(b, k):
            bad.append(k)
    return bad


@needs_ref
def test_reflector_camera_matches_reference_factory():
    mine = F.reflector_camera().flatten()
    ref = O.RefScene("reflector_camera", (4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2)).flat()
    assert flat_diff(mine, ref) == []


def test_reflector_camera_pixels_tile_without_overlap():
    """Every point of the focal plane lies in at most one pixel hexagon: the
    closest hit never has to choose between two coplanar pixels at the same
    distance."""
    flat = F.reflector_camera().flatten()
    T = np.asarray(flat.leaf_frame2world).reshape(-1, 3, 4)
    P = np.asarray(flat.leaf_params).reshape(-1, abi.LEAF_PARAMS)
    U = np.array([flat.hex_unit_u, flat.hex_unit_v, flat.hex_unit_w])
    pixels = [l for l in range(flat.num_leaves) if flat.leaf_sensor[l] >= 0]
    assert len(pixels) == 1440
    rng = np.random.default_rng(1)
    pts = np.c_[rng.uniform(-0.15, 0.15, (100_000, 2)), np.full(100_000, 4.9)]
    covered = np.zeros(len(pts), int)
    for l in pixels:
        local = (pts - T[l][:, 3]) @ T[l][:, :3]
        covered += (np.abs(local @ U.T) < P[l][0]).all(1)
    assert covered.max() == 1
    assert covered.mean() > 0.2


@needs_ref
def test_light_field_telescope_matches_reference_factory():
    """The full config-1 scene: 93,459 nodes, 78,378 leaves, 63,379 lixels."""
    mine = F.light_field_telescope().flatten()
    ref = O.RefScene("light_field_sensor", (10.7, 5.35, 6.5, 0.186, 9, 1.1, 0.9)).flat()
    assert mine.num_nodes == 93459 and mine.num_leaves == 78378 and mine.num_sensors == 63379
    assert flat_diff(mine, ref) == []


def test_builder_matches_golden_scenes():
    """Without the reference: the committed fixtures hold merlict-built scenes."""
    from conftest import load_golden
    for name, build in [("reflector_camera", lambda: F.reflector_camera()),
                        ("light_field_small", lambda: F.light_field_telescope(fov_deg=1.0))]:
        ref, *_ = load_golden(name)
        assert flat_diff(build().flatten(), ref) == [], name


def test_octant_clustering_groups_more_than_16_children():
    sc = S.Scenery()
    for i in range(40):
        p = sc.root.add(S.Disc(f"d{i}", (np.cos(i) * 3, np.sin(i) * 3, 0.1 * i), S.ROT3_UNITY))
        p.set_radius(0.1)
    sc.init()
    assert len(sc.root.children) <= 8
    assert all(c.name.startswith("oct_") or not c.children for c in sc.root.children)
    flat = sc.flatten()
    flat.validate()
    assert flat.num_leaves == 40


def test_func1_evaluate_and_range():
    f = S.Func1([[300e-9, 1.0], [200e-9, 2.0], [400e-9, 3.0]])
    assert f.limits == (200e-9, 400e-9)
    with pytest.raises(IndexError):
        f.evaluate(400e-9)
    with pytest.raises(ValueError):
        S.Func1([[1.0, 1.0], [1.0, 2.0]])
