"""The JSON reader: sceneries, propagation settings and photon sources read
from merlict's JSON files match what merlict's own reader makes of the
same files -- the flattened scenes array by array, the photons bit for bit
-- and the reader keeps merlict's keys, defaults and errors."""
import json
import os
import struct

import numpy as np
import pytest

from merlict_development_kit_b200 import json_scenery as J
from merlict_development_kit_b200 import photons as P
from merlict_development_kit_b200 import scenery as S
from merlict_development_kit_b200.prng import Mt19937
from oracle import oracle as O
from test_builder import flat_diff

needs_ref = pytest.mark.skipif(not O.harness_available(), reason="reference harness not built")
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "json")
SCENERIES = [("primitives", False), ("reflector_hex", False), ("plenoscope", True),
             ("plenoscope_demonstration", True)]


def path(name):
    return os.path.join(HERE, name)


def sensors_of(sc, plenoscope):
    return sc.plenoscopes[0].light_field_channels if plenoscope else sc.sensors


def write_binary_stl(p, facets, header=b"binary stl written by the tests"):
    """facets: (normal, a, b, c) triples of 3-vectors."""
    with open(p, "wb") as f:
        f.write(header.ljust(80, b" "))
        f.write(struct.pack("<I", len(facets)))
        for n, a, b, c in facets:
            f.write(struct.pack("<12f", *n, *a, *b, *c))
            f.write(struct.pack("<H", 0))


def pyramid_facets():
    top = (0.0, 0.0, 1.0)
    base = [(-1.0, -1.0, 0.0), (1.0, -1.0, 0.0), (1.0, 1.0, 0.0), (-1.0, 1.0, 0.0)]
    out = []
    for i in range(4):
        a, b = base[i], base[(i + 1) % 4]
        u = np.subtract(b, a)
        v = np.subtract(top, a)
        n = np.cross(u, v)
        n = n / np.linalg.norm(n)
        out.append((tuple(n), a, b, top))
    # a facet whose normal is exactly +z: no rotation
    out.append(((0.0, 0.0, 1.0), (2.0, 2.0, 0.5), (3.0, 2.0, 0.5), (2.0, 3.0, 0.5)))
    return out


def stl_scenery(tmp_path):
    write_binary_stl(str(tmp_path / "pyramid.stl"), pyramid_facets())
    scenery = {
        "functions": [{"name": "mirror", "argument_versus_value": [[200e-9, 0.7], [1200e-9, 0.7]]}],
        "colors": [],
        "children": [
            {"type": "StereoLitography", "name": "pyramid", "pos": [0.1, 0.0, 2.0],
             "rot": [0.0, 0.2, 0.0], "scale": 0.5, "path": "pyramid.stl",
             "surface": {"outer_reflection": "mirror"}, "children": []},
            {"type": "Disc", "name": "floor", "pos": [0, 0, -1], "rot": [0, 0, 0], "radius": 5.0,
             "surface": {}, "children": [], "sensor_id": 1},
        ],
    }
    p = tmp_path / "stl_scenery.json"
    p.write_text(json.dumps(scenery))
    return str(p)


# ---- the reader against merlict's ---------------------------------------------------

@needs_ref
@pytest.mark.parametrize("name,plenoscope", SCENERIES)
def test_scenery_matches_the_reference_reader(name, plenoscope):
    p = path(name + ".json")
    sc = J.load_scenery(p, plenoscope=plenoscope)
    sensors = sensors_of(sc, plenoscope)
    ref = O.RefScene.from_json(p, plenoscope)
    assert flat_diff(S.flatten(sc.root, sensors), ref.flat()) == []
    assert [s.id for s in sensors] == [int(i) for i in ref.sensor_ids()]


@needs_ref
def test_stl_scenery_matches_the_reference_reader(tmp_path):
    p = stl_scenery(tmp_path)
    sc = J.load_scenery(p)
    mine = sc.flatten()
    assert flat_diff(mine, O.RefScene.from_json(p).flat()) == []
    pyramid = sc.root.children[0]
    assert [c.name for c in pyramid.children] == [f"triangle_{i}" for i in range(5)]
    assert all(c.outer_reflection is pyramid.outer_reflection for c in pyramid.children)


@needs_ref
@pytest.mark.parametrize("name", ["point_source.json", "parallel_disc.json"])
def test_photon_sources_match_the_reference_bit_for_bit(name):
    mine = P.photons2raw_matrix(J.load_photons(path(name)))
    ref = O.json_photons_reference(path(name))
    assert mine.shape == ref.shape
    assert np.array_equal(mine, ref)


@needs_ref
def test_photon_table_matches_the_reference():
    mine = P.photons2raw_matrix(P.load_photon_table(path("photons.tsv")))
    ref = O.table_photons_reference(path("photons.tsv"))
    assert np.array_equal(mine, ref)


@needs_ref
def test_propagation_config_matches_the_reference():
    assert (J.load_PropagationConfig(path("propagation_config.json")).max_num_interactions_per_photon
            == O.json_propagation_config_reference(path("propagation_config.json")) == 1337)


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 12345, 2**63 + 17])
def test_mt19937_matches_the_reference(seed):
    assert np.array_equal(Mt19937(seed).uniforms(5000), O.mt19937_uniforms_reference(seed, 5000))


@needs_ref
@pytest.mark.parametrize("mutate", [
    lambda j: j["children"][0].pop("name"),                                  # MissingKey
    lambda j: j["children"][0]["children"][0].pop("surface"),                 # MissingKey
    lambda j: j["children"][0]["children"][0].pop("children"),                # MissingKey
    lambda j: j["children"][0].__setitem__("pos", [1, 2]),                    # BadTriple
    lambda j: j["children"][0].__setitem__("pos", "up"),                      # BadTriple
    lambda j: j["colors"].append({"name": "grey", "rgb": [0, 0, 0]}),          # colour reused
    lambda j: j["functions"].append(j["functions"][0]),                       # function reused
    lambda j: j["children"][0]["children"][0]["surface"].__setitem__("outer_reflection", "nope"),
    lambda j: j["children"][0]["children"][1].__setitem__("sensor_id", 7),    # sensor id reused
    lambda j: j["children"][0]["children"][6].pop("length"),                  # MissingKey
    lambda j: j["children"][0]["children"][7].pop("start_pos"),               # neither form
    lambda j: j["children"][0]["children"][7].__setitem__("end_pos", [-0.6, 0.5, 2.0]),
    lambda j: j["children"][0]["children"][5].__setitem__("radius", 0.0),     # Sphere radius
    lambda j: j["children"][0]["children"][4].__setitem__("Bx", -0.2),        # degenerate edge
    lambda j: j["children"][0].__setitem__("name", "two words"),              # frame name
    lambda j: j["functions"][0].__setitem__("argument_versus_value", [[1.0, 2.0, 3.0]]),
])
def test_errors_where_the_reference_reader_errs(tmp_path, mutate):
    with open(path("primitives.json")) as f:
        j = json.load(f)
    mutate(j)
    p = tmp_path / "bad.json"
    p.write_text(json.dumps(j))
    with pytest.raises(RuntimeError):
        O.RefScene.from_json(str(p))
    with pytest.raises((KeyError, IndexError, ValueError, TypeError)):
        J.load_scenery(str(p))


@needs_ref
def test_two_light_field_sensors_collide_in_the_colour_map(tmp_path):
    """The light-field sensor factory registers its colours by fixed names,
    so a second light-field sensor in one scenery fails, in merlict too."""
    with open(path("plenoscope.json")) as f:
        j = json.load(f)
    second = dict(j["children"][1], name="second", pos=[30.0, 0.0, 10.7])
    j["children"].append(second)
    p = tmp_path / "two.json"
    p.write_text(json.dumps(j))
    with pytest.raises(RuntimeError):
        O.RefScene.from_json(str(p), True)
    with pytest.raises(S.KeyAlreadyInUse):
        J.load_scenery(str(p), plenoscope=True)


# ---- the reader on its own (merlict_json/tests/JsonTest.cpp) ------------------------------

def test_mt19937_known_answer():
    """The C++ standard's check of std::mt19937_64: the 10000th output of a
    default-seeded engine (seed 5489)."""
    assert int(Mt19937(5489).words(10000)[-1]) == 9981545732273789042


def test_getters_follow_nlohmann_conversions():
    o = J.loads('{"f8": -0.898, "hans": {"A": 1, "B": 2}, "peter": [1, 2, 3], "flag": true}')
    assert o.f8("f8") == -0.898
    assert o.i8("f8") == 0                    # get<int64_t> truncates
    with pytest.raises(TypeError):
        o.st("f8")
    assert o.obj("hans").i8("A") == 1 and o.obj("hans").i8("B") == 2
    with pytest.raises(J.MissingKey):
        o.obj("peter").i8("A")
    assert o.obj("peter").size() == 3
    assert [o.obj("peter").i8(i) for i in range(3)] == [1, 2, 3]
    with pytest.raises(J.ListTooShort):
        o.obj("peter").i8(3)
    assert o.vec3("peter") == (1.0, 2.0, 3.0)
    assert o.b1("flag") is True
    with pytest.raises(TypeError):
        o.b1("f8")
    with pytest.raises(J.MissingKey):
        o.f8("missing")


@pytest.mark.parametrize("bad", ['{"peter": [1, 2]}', '{"peter": "woot"}', '{"peter": [1, "a", 3]}'])
def test_bad_triples(bad):
    with pytest.raises(J.BadTriple):
        J.loads(bad).vec3("peter")


def test_triples_are_read_as_float32():
    """json.cpp:29-43 reads triples with get<float>()."""
    v = J.loads('{"pos": [0.1, 4.889, -2.3]}').vec3("pos")
    assert v == tuple(float(np.float32(x)) for x in (0.1, 4.889, -2.3))
    assert v[0] != 0.1


def test_json_has_no_nan_literals():
    with pytest.raises(ValueError):
        J.loads('{"x": NaN}')


def test_colors_and_functions():
    sc = J.JsonScenery()
    J.add_colors(sc.colors, J.loads('[{"name": "red", "rgb": [255, 0, 0]}, '
                                    '{"name": "blue", "rgb": [0, 0, 255]}]'))
    assert sc.colors.get("red") == (255.0, 0.0, 0.0) and sc.colors.has("blue")
    J.add_colors(sc.colors, J.loads("{}"))        # an empty object adds nothing
    J.add_functions(sc.functions, J.loads(
        '[{"name": "foo", "argument_versus_value": [[0, 5], [1, 4], [2, 3], [3, 2], [4, 1], [5, 0]]}]'))
    foo = sc.functions.get("foo")
    assert foo.limits == (0.0, 5.0)
    assert foo.evaluate(0.0) == pytest.approx(5.0, abs=1e-9)
    assert foo.evaluate(0.5) == pytest.approx(4.5, abs=1e-9)
    assert foo.evaluate(4.999) == pytest.approx(0.0, abs=2e-3)
    with pytest.raises(S.NoSuchKey):
        sc.functions.get("bar")
    with pytest.raises(S.KeyAlreadyInUse):
        sc.colors.add("red", (1, 1, 1))


def test_sensor_ids_and_unknown_types():
    sc = J.load_scenery(path("primitives.json"))
    assert [s.id for s in sc.sensors] == [7, 3, 11, 12, 99]
    assert sc.sensor_map.get(7).frame.name == "disc"
    assert sc.sensor_map.get(99).frame.name == "ceiling"
    with pytest.raises(S.NoSuchKey):
        sc.sensor_map.get(0)
    names = set()
    stack = [sc.root]
    while stack:
        f = stack.pop()
        names.add(f.name)
        stack.extend(f.children)
    assert "not_a_merlict_type" not in names and "skipped" not in names


def test_missing_rotation_is_no_rotation():
    """merlict leaves the Rot3 of a frame without "rot" or "rot_axis"
    default-constructed, i.e. uninitialised (json.cpp:180-192); this reader
    gives it no rotation."""
    sc = J.JsonScenery()
    J.append_to_frame_in_scenery(sc.root, sc, J.loads(
        '{"functions": [], "colors": [], "children": [{"type": "Frame", "name": "f", '
        '"pos": [1, 2, 3], "children": []}]}'))
    f = sc.root.children[0]
    assert f.rot.xyz == (0.0, 0.0, 0.0)


def test_plenoscope_reader_ignores_sensor_ids():
    sc = J.load_scenery(path("plenoscope_demonstration.json"), plenoscope=True)
    assert sc.sensors == []
    pis = sc.plenoscopes[0]
    assert pis.frame.name == "demonstration"
    assert [s.id for s in pis.light_field_channels] == list(range(len(pis.light_field_channels)))


def test_point_source_known_answers():
    """JsonTest.cpp PointSource and PointSource_rotated."""
    b = J.to_photons(J.loads('{"point_source": {"opening_angle": 0.01, "num_photons": 137}, '
                             '"pos": [0, 2, 0], "rot": [0, 0, 0]}'))
    assert len(b["wavelength"]) == 137
    assert np.all(b["support_x"] == 0.0) and np.all(b["support_y"] == 2.0)
    assert np.all(b["support_z"] == 0.0)
    assert np.allclose(b["direction_z"], 1.0, atol=0.1)
    b = J.to_photons(J.loads('{"point_source": {"opening_angle": 0.01, "num_photons": 13}, '
                             '"pos": [0, 2, 0], "rot": [0, 1.5705, 0]}'))
    assert len(b["wavelength"]) == 13
    assert np.allclose(b["direction_x"], -1.0, atol=0.1)
    b = J.to_photons(J.loads('{"parallel_disc": {"disc_radius": 2.5, "num_photons": 13}, '
                             '"pos": [0, 0, 0], "rot": [0, 1.5705, 0]}'))
    assert np.allclose(b["direction_x"], -1.0, atol=0.1)
    assert np.all(np.hypot(b["support_y"], b["support_z"]) <= 2.5 + 1e-12)
    with pytest.raises(J.UnkownTypeOfLightSource):
        J.to_photons(J.loads('{"laser": {}, "pos": [0, 0, 0], "rot": [0, 0, 0]}'))


def test_parallel_disc_consumes_the_stream_like_merlict():
    """Rejection sampling uses one pair of draws per attempt; the stream
    continues right after the last accepted pair."""
    g = Mt19937(3)
    P.parallel_towards_z_from_xy_disc(1.0, 500, g)
    u = Mt19937(3).uniforms(4000).reshape(-1, 2)
    x, y = u[:, 0] * 2.0 - 1.0, u[:, 1] * 2.0 - 1.0
    used = 2 * (np.flatnonzero(~(x * x + y * y > 1.0))[499] + 1)
    assert g.uniform() == Mt19937(3).uniforms(used + 1)[-1]


def test_photon_table_rules(tmp_path):
    t = P.gen_table_from_string("# header\n\n 1 2\t3 \n#\n4 0x1p-2 -inf\n")
    assert t == [[1.0, 2.0, 3.0], [4.0, 0.25, -np.inf]]
    with pytest.raises(ValueError):
        P.gen_table_from_string("1 2 x\n")
    with pytest.raises(ValueError):
        P.raw_matrix2photons([[0, 1, 2, 3, 0, 0, 1]])
    with pytest.raises(ValueError):
        P.raw_matrix2photons([[0, 1, 2, 3, 0, 0, 1, -5e-7]])
    with pytest.raises(RuntimeError):
        P.gen_table_from_file(str(tmp_path / "missing.tsv"))


def test_ascii_stl_is_refused(tmp_path):
    p = tmp_path / "a.stl"
    p.write_bytes(b"solid cube\n" + b" " * 100)
    with pytest.raises(ValueError):
        J.read_binary_stl(str(p))


def test_hex_aperture_reflector():
    """Geometry.cpp:32-67: the facet centres of a hexagonal aperture lie in
    the hexagon (strictly) and outside the inner disc."""
    from merlict_development_kit_b200 import factories as F
    cfg = F.ReflectorConfig(4.889, 0.5, 2.1, 0.2, 0.3, 0.01, True)
    g = F.ReflectorGeometry(cfg)
    xy = np.array([p[:2] for p in g.facet_positions])
    spacing = g.facet_spacing
    R = np.sqrt(3) / 2 * (2.1 - spacing / 2)
    for phi in (0.0, 2 * np.pi / 3, -2 * np.pi / 3):
        proj = xy @ np.array([np.cos(phi), np.sin(phi)])
        assert np.all(np.abs(proj) < R + 1e-12)
    assert np.all(np.hypot(xy[:, 0], xy[:, 1]) > 0.2 + spacing / 2)
    assert g.num_facets != F.ReflectorGeometry(F.ReflectorConfig(4.889, 0.5, 2.1, 0.2, 0.3, 0.01,
                                                                 False)).num_facets
