"""Sceneries, propagation settings and photon sources from JSON.

The reader of merlict's JSON files (merlict_json/json.cpp) and of its
plenoscope extension (merlict_portal_plenoscope/json_to_plenoscope.h),
with the same names, keys, defaults and errors, building this package's
scene model (scenery.py, factories.py) instead of merlict's.  A loaded
scenery flattens into the drop-in layout of include/merlict_b200.h like
any other:

    sc = json_scenery.load_scenery("scenery.json")          # merlict's reader
    scene = engine.Scene(sc.flatten())                      # sensors by sensor_id

    sc = json_scenery.load_scenery("plenoscope.json", plenoscope=True)
    scene = engine.Scene(scenery.flatten(sc.root, sc.plenoscopes[0].light_field_channels))

Two details of merlict's reader decide the numbers and are kept:
triples ("pos", "rot", "rot_axis", "start_pos", "rgb", ...) are read as
32-bit floats and widened to double (json.cpp:29-43), every other number
as a double; and unknown "type"s are skipped together with their
children (json.cpp:209-228).  The plenoscope reader adds the types
"LightFieldSensor" and "LightFieldSensor_for_demonstration" and, unlike
merlict's, does not register "sensor_id"s (json_to_plenoscope.h:85-120).

merlict's rendering settings (visual::Config, json.cpp:469-508) are not
read: nothing on the propagation path uses them.
"""
from __future__ import annotations

import json as _json
import os
import struct
from dataclasses import dataclass, field

import numpy as np

from . import factories, photons as _photons
from .engine import PropagationConfig
from .prng import Mt19937
from .scenery import (ROT3_UNITY, Annulus, BiConvexLensHexBound, Cylinder, Disc, Frame, Func1,
                      HexPlane, Plane, ResourceMap, Rot3, Scenery, Sensor, Sphere,
                      SphereCapWithHexagonalBound, SphereCapWithRectangularBound, SurfaceEntity,
                      Triangle, deg2rad, t_from_rot_pos)


# ---- errors (merlict_json/json.h) ----------------------------------------------

class MissingKey(KeyError):
    """json::MissingKey: an object lacks a required key."""


class ListTooShort(IndexError):
    """json::ListTooShort: a list is shorter than the index asked for."""


class BadTriple(ValueError):
    """json::BadTriple: not a list of three numbers."""


class UnkownTypeOfLightSource(ValueError):
    """json::UnkownTypeOfLightSource: neither 'point_source' nor 'parallel_disc'."""


# ---- the value wrapper, json.cpp:48-131 -------------------------------------------

def _type_name(v) -> str:
    if v is None:
        return "null"
    if isinstance(v, bool):
        return "boolean"
    if isinstance(v, (int, float)):
        return "number"
    if isinstance(v, str):
        return "string"
    if isinstance(v, list):
        return "array"
    return "object"


def _number(v, what: str) -> float:
    """nlohmann's get<double>(): numbers only."""
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise TypeError(f"type must be number, but is {_type_name(v)} ({what})")
    return float(v)


def _f32(v) -> float:
    """get<float>() widened back to double: numbers and booleans."""
    if isinstance(v, bool):
        return float(v)
    if not isinstance(v, (int, float)):
        raise TypeError(_type_name(v))
    with np.errstate(over="ignore"):
        return float(np.float32(v))


def _to_triple(v):
    """json.cpp:29-43."""
    try:
        if not isinstance(v, list) or len(v) < 3:
            raise IndexError
        return (_f32(v[0]), _f32(v[1]), _f32(v[2]))
    except (IndexError, TypeError):
        raise BadTriple("Expected triple to be an array of three floats: [x, y, z]', but "
                        f"actually it is{_json.dumps(v)}'.") from None


class Object:
    """merlict::json::Object: a JSON value with merlict's typed getters.
    Getters by key need an object holding the key (MissingKey); getters by
    index need a list long enough (ListTooShort)."""

    def __init__(self, j):
        self.j = j.j if isinstance(j, Object) else j

    # -- access
    def key(self, k: str) -> bool:
        return isinstance(self.j, dict) and k in self.j

    def _at_key(self, k: str):
        if not self.key(k):
            raise MissingKey(f"Expected key: '{k}' in {_json.dumps(self.j)}")
        return self.j[k]

    def _at_idx(self, i: int):
        if self.size() <= i:
            raise ListTooShort(f"Expected at least size {i + 1} for object {_json.dumps(self.j)}")
        if not isinstance(self.j, list):
            raise TypeError(f"cannot use at() with {_type_name(self.j)}")
        return self.j[i]

    def _get(self, k):
        return self._at_idx(k) if isinstance(k, int) else self._at_key(k)

    def size(self) -> int:
        if self.j is None:
            return 0
        if isinstance(self.j, (list, dict)):
            return len(self.j)
        return 1

    # -- typed getters
    def f8(self, k) -> float:
        return _number(self._get(k), str(k))

    def i8(self, k) -> int:
        v = self._get(k)
        return int(_number(v, str(k))) if isinstance(v, float) else int(_integer(v, k))

    def u8(self, k) -> int:
        v = self._get(k)
        if isinstance(v, float):
            return int(v)
        return int(_integer(v, k)) & ((1 << 64) - 1)

    def st(self, k) -> str:
        v = self._get(k)
        if not isinstance(v, str):
            raise TypeError(f"type must be string, but is {_type_name(v)} ({k})")
        return v

    def b1(self, k) -> bool:
        v = self._get(k)
        if not isinstance(v, bool):
            raise TypeError(f"type must be boolean, but is {_type_name(v)} ({k})")
        return v

    def obj(self, k) -> "Object":
        return Object(self._get(k))

    def vec3(self, k):
        return _to_triple(self._get(k))

    def rot3(self, k) -> Rot3:
        a = _to_triple(self._get(k))
        return Rot3(a[0], a[1], a[2])

    def color(self, k):
        return _to_triple(self._get(k))

    def str(self) -> str:
        return _json.dumps(self.j)


def _integer(v, k):
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise TypeError(f"type must be number, but is {_type_name(v)} ({k})")
    return v


def _reject_constant(name):
    raise ValueError(f"parse error: invalid literal '{name}'")


def loads(text: str) -> Object:
    """Parses JSON text (NaN and Infinity are not JSON, as in nlohmann's parser)."""
    return Object(_json.loads(text, parse_constant=_reject_constant))


def load(path: str) -> Object:
    """json::load, json.cpp:133-147."""
    try:
        with open(path, "r") as f:
            text = f.read()
    except OSError:
        raise RuntimeError(f"json_to_scenery: Can not open '{path}'.") from None
    return loads(text)


def _as_object(source) -> Object:
    if isinstance(source, Object):
        return source
    if isinstance(source, (dict, list)):
        return Object(source)
    raise TypeError("expected a parsed JSON value or an Object")


# ---- sceneries ------------------------------------------------------------------

@dataclass
class PlenoscopeInScenery:
    """plenoscope::PlenoscopeInScenery: the light-field sensor's frame,
    configuration and geometry, and its lixels as sensors 0..n-1."""
    frame: Frame
    config: factories.LightFieldSensorConfig
    light_field_sensor_geometry: factories.LightFieldSensorGeometry
    light_field_channels: list = field(default_factory=list)


class JsonScenery(Scenery):
    """merlict::Scenery as the JSON reader fills it, plus the plenoscopes
    of plenoscope::PlenoscopeScenery.  `sensors` are the frames with a
    "sensor_id", in the order the reader met them (SensorMap.cpp:8-14);
    `sensor_map` finds them by id."""

    def __init__(self):
        super().__init__()
        self.sensor_map = ResourceMap("sensor")
        self.plenoscopes: list[PlenoscopeInScenery] = []
        self.current_working_directory = ""

    def add_sensor(self, id: int, frame: Frame) -> Sensor:
        s = Sensor(id, frame)
        self.sensor_map.add(int(id), s)
        self.sensors.append(s)
        return s


def set_frame(f: Frame, o: Object):
    """json.cpp:180-192: name, pos, and rot as Tait-Bryan angles or as
    rot_axis and rot_angle (neither: no rotation)."""
    name = o.st("name")
    pos = o.vec3("pos")
    if o.key("rot"):
        rot = o.rot3("rot")
    elif o.key("rot_axis"):
        axis = o.vec3("rot_axis")
        rot = Rot3(axis=axis, angle=o.f8("rot_angle"))
    else:
        rot = ROT3_UNITY
    f.set_name_pos_rot(name, pos, rot)


def set_surface(s: SurfaceEntity, scenery: Scenery, o: Object):
    """json.cpp:194-207: colours and reflection/refraction functions by name."""
    su = o.obj("surface")
    if su.key("inner_color"):
        s.inner_color = scenery.colors.get(su.st("inner_color"))
    if su.key("outer_color"):
        s.outer_color = scenery.colors.get(su.st("outer_color"))
    if su.key("inner_reflection"):
        s.inner_reflection = scenery.functions.get(su.st("inner_reflection"))
    if su.key("outer_reflection"):
        s.outer_reflection = scenery.functions.get(su.st("outer_reflection"))
    if su.key("inner_refraction"):
        s.inner_refraction = scenery.functions.get(su.st("inner_refraction"))
    if su.key("outer_refraction"):
        s.outer_refraction = scenery.functions.get(su.st("outer_refraction"))


def add_Frame(mother, scenery, o):
    return mother.add(_new(Frame, o))


def _new(cls, o: Object):
    f = cls()
    set_frame(f, o)
    return f


def add_Sphere(mother, scenery, o):
    s = mother.add(_new(Sphere, o))
    s.set_radius(o.f8("radius"))
    set_surface(s, scenery, o)
    return s


def add_Annulus(mother, scenery, o):
    a = mother.add(_new(Annulus, o))
    a.set_outer_inner_radius(o.f8("outer_radius"), o.f8("inner_radius"))
    set_surface(a, scenery, o)
    return a


def add_Cylinder(mother, scenery, o):
    """json.cpp:321-343: "rot" with "radius" and "length", or "start_pos"
    and "end_pos" with "radius"."""
    c = Cylinder()
    mother.add(c)
    if o.key("rot"):
        set_frame(c, o)
        c.set_radius_and_length(o.f8("radius"), o.f8("length"))
    elif o.key("start_pos"):
        c.set_name_pos_rot(o.st("name"), (0.0, 0.0, 0.0), Rot3(0.0, 0.0, 0.0))
        c.set_cylinder(o.f8("radius"), o.vec3("start_pos"), o.vec3("end_pos"))
    else:
        raise ValueError("Expected Cylinder to have either 'pos', 'rot', 'radius', and "
                         "'length', or to have 'start_pos', 'end_pos', and 'radius'. But "
                         f"actually it has: {o.str()}")
    set_surface(c, scenery, o)
    return c


def add_Triangle(mother, scenery, o):
    t = mother.add(_new(Triangle, o))
    t.set_corners_in_xy_plane(o.f8("Ax"), o.f8("Ay"), o.f8("Bx"), o.f8("By"),
                              o.f8("Cx"), o.f8("Cy"))
    set_surface(t, scenery, o)
    return t


def add_Disc(mother, scenery, o):
    d = mother.add(_new(Disc, o))
    d.set_radius(o.f8("radius"))
    set_surface(d, scenery, o)
    return d


def add_Plane(mother, scenery, o):
    p = mother.add(_new(Plane, o))
    p.set_x_y_width(o.f8("x_width"), o.f8("y_width"))
    set_surface(p, scenery, o)
    return p


def add_HexPlane(mother, scenery, o):
    p = mother.add(_new(HexPlane, o))
    p.set_outer_hex_radius(o.f8("outer_radius"))
    set_surface(p, scenery, o)
    return p


def add_BiConvexLensHex(mother, scenery, o):
    """json.cpp:383-396: the surface first, so the caps inherit it."""
    lens = mother.add(_new(BiConvexLensHexBound, o))
    set_surface(lens, scenery, o)
    lens.set_curvature_radius_and_outer_hex_radius(o.f8("curvature_radius"), o.f8("outer_radius"))
    return lens


def add_SphereCapWithHexagonalBound(mother, scenery, o):
    cap = mother.add(_new(SphereCapWithHexagonalBound, o))
    cap.set_curvature_radius_and_outer_hex_radius(o.f8("curvature_radius"), o.f8("outer_radius"))
    set_surface(cap, scenery, o)
    return cap


def add_SphereCapWithRectangularBound(mother, scenery, o):
    cap = mother.add(_new(SphereCapWithRectangularBound, o))
    cap.set_curvature_radius_and_x_y_width(o.f8("curvature_radius"), o.f8("x_width"),
                                           o.f8("y_width"))
    set_surface(cap, scenery, o)
    return cap


def add_SegmentedReflector(mother, scenery, o):
    """json.cpp:428-449: segmented_imaging_reflector::Factory on a surface
    entity whose surface the facets adopt."""
    cfg = factories.ReflectorConfig(
        focal_length=o.f8("focal_length"),
        DaviesCotton_over_parabolic_mixing_factor=o.f8("DaviesCotton_over_parabolic_mixing_factor"),
        max_outer_aperture_radius=o.f8("max_outer_aperture_radius"),
        min_inner_aperture_radius=o.f8("min_inner_aperture_radius"),
        outer_aperture_shape_hex=o.b1("outer_aperture_shape_hex"),
        facet_inner_hex_radius=o.f8("facet_inner_hex_radius"),
        gap_between_facets=o.f8("gap_between_facets"))
    reflector = mother.add(_new(SurfaceEntity, o))
    set_surface(reflector, scenery, o)
    factories.segmented_reflector(reflector, cfg)
    return reflector


def read_binary_stl(path: str):
    """stereo_litography::BinaryReader (stereo_litography.cpp:142-275): an
    80-byte header that must not start with 'solid' (ASCII STL is refused),
    a uint32 facet count, then per facet 12 float32 (normal, A, B, C) and a
    uint16 attribute count.  Returns float64 arrays (n,3) normal, a, b, c."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError:
        raise RuntimeError(f"BinaryReader: Unable to open file: '{path}'") from None
    if data[:5] == b"solid":
        raise ValueError(f"BinaryReader: Unable to read file: '{path}' Expected binary file, "
                         "but actual header implies ascii format.")
    (count,) = struct.unpack_from("<I", data, 80) if len(data) >= 84 else (0,)
    rec = np.dtype([("v", "<f4", (12,)), ("attr", "<u2")])
    have = max(0, (len(data) - 84) // rec.itemsize)
    facets = np.frombuffer(data, dtype=rec, count=min(count, have), offset=84)
    v = facets["v"].astype(np.float64)
    if v.shape[0] < count:
        # merlict reads past the end as zeros (a failed read leaves the
        # buffer as constructed)
        v = np.concatenate([v, np.zeros((count - v.shape[0], 12))])
    return v[:, 0:3], v[:, 3:6], v[:, 6:9], v[:, 9:12]


def add_stl_to_and_inherit_surface_from_surfac_entity(path: str, proto: SurfaceEntity,
                                                      scale: float):
    """stereo_litography.cpp:10-31: one triangle per facet, vertices scaled,
    each adopting the surface of `proto`."""
    n, a, b, c = read_binary_stl(path)
    for i in range(n.shape[0]):
        tri = proto.add(Triangle(f"triangle_{i}", (0.0, 0.0, 0.0), ROT3_UNITY))
        tri.set_normal_and_3_vertecies(tuple(n[i]), tuple(a[i] * scale), tuple(b[i] * scale),
                                       tuple(c[i] * scale))
        tri.adopt_surface(proto)


def add_StereoLitography(mother, scenery, o):
    """json.cpp:301-318: triangles from a binary STL file, its path relative
    to the directory of the scenery file."""
    obj = mother.add(_new(SurfaceEntity, o))
    set_surface(obj, scenery, o)
    scale = o.f8("scale")
    path = ospath_join(scenery.current_working_directory, o.st("path"))
    add_stl_to_and_inherit_surface_from_surfac_entity(path, obj, scale)
    return obj


def ospath_dirname(path: str) -> str:
    """ospath::Path::dirname (merlict/ospath.cpp:24-32): up to the last '/'
    or '\\'."""
    k = max(path.rfind("/"), path.rfind("\\"))
    return path[:k] if k != -1 else ""


def ospath_join(path1: str, path2: str) -> str:
    """ospath::join (merlict/ospath.cpp:10-21)."""
    out = path1 if path1.endswith("/") else (path1 + "/" if path1 else "")
    return out + (path2[1:] if path2.rfind("/") == 0 else path2)


def basic_scenery() -> dict:
    """json.cpp:149-164."""
    return {
        "Frame": add_Frame,
        "Sphere": add_Sphere,
        "Annulus": add_Annulus,
        "Cylinder": add_Cylinder,
        "Triangle": add_Triangle,
        "Disc": add_Disc,
        "Plane": add_Plane,
        "HexPlane": add_HexPlane,
        "StereoLitography": add_StereoLitography,
        "BiConvexLensHex": add_BiConvexLensHex,
        "SphereCapWithHexagonalBound": add_SphereCapWithHexagonalBound,
        "SphereCapWithRectangularBound": add_SphereCapWithRectangularBound,
        "SegmentedReflector": add_SegmentedReflector,
    }


def make_children(mother: Frame, scenery: JsonScenery, o: Object):
    """json.cpp:209-228: each child of a known type, its sensor_id, then its
    own children; children of unknown types are skipped."""
    j2s = basic_scenery()
    for cidx in range(o.size()):
        jchild = o.obj(cidx)
        t = jchild.st("type")
        if t in j2s:
            child = j2s[t](mother, scenery, jchild)
            if jchild.key("sensor_id"):
                scenery.add_sensor(jchild.u8("sensor_id"), child)
            make_children(child, scenery, jchild.obj("children"))


def add_colors(colors: ResourceMap, o: Object):
    """json.cpp:230-236."""
    for cidx in range(o.size()):
        jcolor = o.obj(cidx)
        colors.add(jcolor.st("name"), jcolor.color("rgb"))


def json_to_vec_of_vecs(avsv: Object) -> list:
    """json.cpp:238-252: a list of [argument, value] pairs."""
    out = []
    for i in range(avsv.size()):
        point = avsv.obj(i)
        if point.size() != 2:
            raise ValueError("Expected argument_versus_value in linear_interpolation to be a "
                             "list of length-two-lists.")
        out.append([point.f8(0), point.f8(1)])
    return out


def add_functions(functions: ResourceMap, o: Object):
    """json.cpp:254-262."""
    for fidx in range(o.size()):
        jfun = o.obj(fidx)
        name = jfun.st("name")
        functions.add(name, Func1(json_to_vec_of_vecs(jfun.obj("argument_versus_value"))))


def json_to_linear_interpol_function(avsv) -> Func1:
    """json.cpp:264-268."""
    return Func1(json_to_vec_of_vecs(_as_object(avsv)))


def append_to_frame_in_scenery(mother: Frame, scenery: JsonScenery, source):
    """json.cpp:270-288: functions, colours, then the children.  `source`
    is a path (which also sets the directory STL paths are relative to) or
    a parsed JSON value."""
    if isinstance(source, (str, os.PathLike)):
        scenery.current_working_directory = ospath_dirname(os.fspath(source))
        source = load(os.fspath(source))
    o = _as_object(source)
    add_functions(scenery.functions, o.obj("functions"))
    add_colors(scenery.colors, o.obj("colors"))
    make_children(mother, scenery, o.obj("children"))


# ---- the plenoscope extension, json_to_plenoscope.h ---------------------------------

def _light_field_sensor_config(scenery: Scenery, o: Object):
    return factories.LightFieldSensorConfig(
        expected_imaging_system_focal_length=o.f8("expected_imaging_system_focal_length"),
        expected_imaging_system_max_aperture_radius=o.f8("expected_imaging_system_aperture_radius"),
        max_FoV_diameter=deg2rad(o.f8("max_FoV_diameter_deg")),
        pixel_FoV_hex_flat2flat=deg2rad(o.f8("hex_pixel_FoV_flat2flat_deg")),
        num_paxel_on_pixel_diagonal=o.u8("num_paxel_on_pixel_diagonal"),
        housing_overhead=o.f8("housing_overhead"),
        lens_refraction=scenery.functions.get(o.st("lens_refraction_vs_wavelength")),
        bin_reflection=scenery.functions.get(o.st("bin_reflection_vs_wavelength")))


def _add_plenoscope(mother, scenery, o, build):
    frame = mother.add(_new(Frame, o))
    cfg = _light_field_sensor_config(scenery, o)
    channels: list = []
    geometry = build(frame, scenery, cfg, channels)
    scenery.plenoscopes.append(PlenoscopeInScenery(frame, cfg, geometry, channels))
    return frame


def add_light_field_sensor(mother, scenery, o):
    """json_to_plenoscope.h:14-47."""
    return _add_plenoscope(mother, scenery, o, factories.light_field_sensor)


def add_light_field_sensor_demonstration(mother, scenery, o):
    """json_to_plenoscope.h:49-82."""
    return _add_plenoscope(mother, scenery, o, factories.demonstration_light_field_sensor)


def plenoscope_make_children(mother: Frame, scenery: JsonScenery, o: Object):
    """json_to_plenoscope.h:84-120: the basic types plus the light-field
    sensors; "sensor_id" is not read here."""
    j2s = basic_scenery()
    for cidx in range(o.size()):
        jchild = o.obj(cidx)
        t = jchild.st("type")
        if t in j2s:
            plenoscope_make_children(j2s[t](mother, scenery, jchild), scenery,
                                     jchild.obj("children"))
        elif t == "LightFieldSensor":
            plenoscope_make_children(add_light_field_sensor(mother, scenery, jchild), scenery,
                                     jchild.obj("children"))
        elif t == "LightFieldSensor_for_demonstration":
            plenoscope_make_children(add_light_field_sensor_demonstration(mother, scenery, jchild),
                                     scenery, jchild.obj("children"))


def plenoscope_append_to_frame_in_scenery(mother: Frame, scenery: JsonScenery, source):
    """json_to_plenoscope.h:122-138.  Unlike merlict's reader, a path does
    not set the directory for STL paths (they stay relative to the current
    directory)."""
    if isinstance(source, (str, os.PathLike)):
        source = load(os.fspath(source))
    o = _as_object(source)
    add_functions(scenery.functions, o.obj("functions"))
    add_colors(scenery.colors, o.obj("colors"))
    plenoscope_make_children(mother, scenery, o.obj("children"))


def load_scenery(source, plenoscope: bool = False) -> JsonScenery:
    """A scenery from a JSON file or value, with its tree initialised
    (Frame::init_tree_based_on_mother_child_relations), as merlict's
    propagation programs set it up (merlict_tests/apps/propagate.cpp:51-57,
    plenoscope_propagation.cpp:102-107)."""
    sc = JsonScenery()
    if plenoscope:
        plenoscope_append_to_frame_in_scenery(sc.root, sc, source)
    else:
        append_to_frame_in_scenery(sc.root, sc, source)
    sc.init()
    return sc


# ---- propagation settings and photon sources, json.cpp:510-562 -----------------------

def to_PropagationConfig(o) -> PropagationConfig:
    o = _as_object(o)
    return PropagationConfig(max_num_interactions_per_photon=o.u8("max_num_interactions_per_photon"))


def load_PropagationConfig(path: str) -> PropagationConfig:
    return to_PropagationConfig(load(path))


def transform_photons(o: Object, batch: dict) -> dict:
    """json.cpp:519-526: every photon moved by "rot" then "pos"."""
    T = t_from_rot_pos(o.rot3("rot"), o.vec3("pos"))
    return _photons.transform_photons(batch, T)


def to_parallel_disc(o: Object) -> dict:
    return _photons.parallel_towards_z_from_xy_disc(o.f8("disc_radius"), o.u8("num_photons"),
                                                    Mt19937(0))


def to_pointsource(o: Object) -> dict:
    return _photons.point_like_towards_z_opening_angle_num_photons(
        o.f8("opening_angle"), o.u8("num_photons"), Mt19937(0))


def to_photons(o) -> dict:
    """json.cpp:547-560: a "point_source" or a "parallel_disc", each drawn
    from Mt19937(0), then moved by "pos" and "rot"."""
    o = _as_object(o)
    if o.key("point_source"):
        batch = to_pointsource(o.obj("point_source"))
    elif o.key("parallel_disc"):
        batch = to_parallel_disc(o.obj("parallel_disc"))
    else:
        raise UnkownTypeOfLightSource("Expected InternalPhotonSource from json to be either "
                                      "'point_source', or 'parallel_disc'.")
    return transform_photons(o, batch)


def load_photons(path: str) -> dict:
    return to_photons(load(path))


__all__ = [
    "MissingKey", "ListTooShort", "BadTriple", "UnkownTypeOfLightSource", "Object", "load",
    "loads", "JsonScenery", "PlenoscopeInScenery", "set_frame", "set_surface", "basic_scenery",
    "make_children", "add_colors", "add_functions", "json_to_vec_of_vecs",
    "json_to_linear_interpol_function", "append_to_frame_in_scenery",
    "plenoscope_append_to_frame_in_scenery", "load_scenery", "to_PropagationConfig",
    "load_PropagationConfig", "to_photons", "load_photons", "read_binary_stl",
]
