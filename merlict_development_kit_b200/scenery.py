"""Scene description: a frame tree with surfaces and primitives, initialised
and flattened into the engine's flat scene.

This mirrors merlict's scenery model (merlict/Frame.h, SurfaceEntity.h,
scenery/primitive/*) closely enough that a tree built here and one built
with merlict's own classes flatten to identical arrays: positions and
rotations compose in the same order (HomTra3.cpp:24-263), children are
grouped into octants the same way (Frame.cpp:190-255) and bounding spheres
are computed with the same rules (Frames.cpp:37-206).  Floating-point
operations follow merlict's order; libm's hypot is called for hypot, as
merlict does.
"""
from __future__ import annotations

import ctypes
import math
from typing import Sequence

import numpy as np

from . import abi

_libm = ctypes.CDLL("libm.so.6")
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]
_libm.hypot.restype = ctypes.c_double


def hypot(a: float, b: float) -> float:
    return _libm.hypot(a, b)


# ---- Vec3 as tuples, merlict/Vec3.cpp ---------------------------------------

def v_add(a, b):
    return (a[0] + b[0], a[1] + b[1], a[2] + b[2])


def v_sub(a, b):
    return (a[0] - b[0], a[1] - b[1], a[2] - b[2])


def v_mul(a, s):
    return (a[0] * s, a[1] * s, a[2] * s)


def v_div(a, s):
    return (a[0] / s, a[1] / s, a[2] / s)


def v_dot(self, v):
    return v[0] * self[0] + v[1] * self[1] + v[2] * self[2]


def v_norm(a):
    return math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2])


def v_cross(a, v):
    return (a[1] * v[2] - a[2] * v[1], a[2] * v[0] - a[0] * v[2], a[0] * v[1] - a[1] * v[0])


def v_octant(a):
    return 4 * (a[0] >= 0.0) + 2 * (a[1] >= 0.0) + 1 * (a[2] >= 0.0)


def c_acos(x: float) -> float:
    """acos with C's domain behaviour: NaN outside [-1, 1]."""
    return math.acos(x) if -1.0 <= x <= 1.0 else math.nan


def v_angle_in_between(a, b):
    an = v_div(a, v_norm(a))
    bn = v_div(b, v_norm(b))
    return c_acos(v_dot(an, bn))


MAX_DEVIATION_EQUAL_VEC3_SQUARE = 1e-14   # merlict/Vec3.h:45


ORIGIN = (0.0, 0.0, 0.0)
UNIT_X = (1.0, 0.0, 0.0)
UNIT_Y = (0.0, 1.0, 0.0)
UNIT_Z = (0.0, 0.0, 1.0)


def deg2rad(deg: float) -> float:
    return (math.pi * deg) / 180.0   # merlict/tools.cpp:9-11


# ---- Rot3 and HomTra3 -------------------------------------------------------

class Rot3:
    """Tait-Bryan xyz angles or an axis and an angle (merlict/Rot3.cpp)."""

    def __init__(self, rx=0.0, ry=0.0, rz=0.0, axis=None, angle=None):
        if axis is not None:
            if angle == 0.0:
                self.xyz = (0.0, 0.0, 0.0)
                self.axis = None
            else:
                self.xyz = None
                self.axis = v_div(axis, v_norm(axis))
                self.angle = float(angle)
        else:
            self.xyz = (float(rx), float(ry), float(rz))
            self.axis = None

    @staticmethod
    def from_axis(axis, angle) -> "Rot3":
        return Rot3(axis=axis, angle=angle)


ROT3_UNITY = Rot3(0.0, 0.0, 0.0)

IDENTITY = ((1.0, 0.0, 0.0, 0.0), (0.0, 1.0, 0.0, 0.0), (0.0, 0.0, 1.0, 0.0))


def t_mul(T, G):
    """HomTra3::operator*, HomTra3.cpp:241-263."""
    rows = []
    for r in range(3):
        t0, t1, t2, t3 = T[r]
        rows.append((
            t0 * G[0][0] + t1 * G[1][0] + t2 * G[2][0],
            t0 * G[0][1] + t1 * G[1][1] + t2 * G[2][1],
            t0 * G[0][2] + t1 * G[1][2] + t2 * G[2][2],
            t0 * G[0][3] + t1 * G[1][3] + t2 * G[2][3] + t3))
    return tuple(rows)


def t_rotation(R: Rot3):
    """The rotation part of HomTra3::set_transformation, HomTra3.cpp:48-91."""
    if R.xyz is not None:
        rx, ry, rz = R.xyz
        cosRx, cosRy, cosRz = math.cos(rx), math.cos(ry), math.cos(rz)
        sinRx, sinRy, sinRz = math.sin(rx), math.sin(ry), math.sin(rz)
        return (
            (cosRy * cosRz, cosRx * sinRz + sinRx * sinRy * cosRz,
             sinRx * sinRz - cosRx * sinRy * cosRz, 0.0),
            (-cosRy * sinRz, cosRx * cosRz - sinRx * sinRy * sinRz,
             sinRx * cosRz + cosRx * sinRy * sinRz, 0.0),
            (sinRy, -sinRx * cosRy, cosRx * cosRy, 0.0))
    axis = v_div(R.axis, v_norm(R.axis))
    rx, ry, rz = axis
    sinR = math.sin(R.angle)
    cosR = math.cos(R.angle)
    return (
        (cosR + rx * rx * (1. - cosR), rx * ry * (1. - cosR) - rz * sinR,
         rx * rz * (1. - cosR) + ry * sinR, 0.0),
        (ry * rx * (1. - cosR) + rz * sinR, cosR + ry * ry * (1. - cosR),
         ry * rz * (1. - cosR) - rx * sinR, 0.0),
        (rz * rx * (1. - cosR) - ry * sinR, rz * ry * (1. - cosR) + rx * sinR,
         cosR + rz * rz * (1. - cosR), 0.0))


def t_from_rot_pos(R: Rot3, pos):
    translation = ((1.0, 0.0, 0.0, pos[0]), (0.0, 1.0, 0.0, pos[1]), (0.0, 0.0, 1.0, pos[2]))
    return t_mul(translation, t_rotation(R))


def t_inverse(T):
    """HomTra3::inverse, HomTra3.cpp:266-301."""
    return (
        (T[0][0], T[1][0], T[2][0], -(T[0][0] * T[0][3] + T[1][0] * T[1][3] + T[2][0] * T[2][3])),
        (T[0][1], T[1][1], T[2][1], -(T[0][1] * T[0][3] + T[1][1] * T[1][3] + T[2][1] * T[2][3])),
        (T[0][2], T[1][2], T[2][2], -(T[0][2] * T[0][3] + T[1][2] * T[1][3] + T[2][2] * T[2][3])))


def t_orientation(T, v):
    return (v[0] * T[0][0] + v[1] * T[0][1] + v[2] * T[0][2],
            v[0] * T[1][0] + v[1] * T[1][1] + v[2] * T[1][2],
            v[0] * T[2][0] + v[1] * T[2][1] + v[2] * T[2][2])


# ---- property tables, merlict/function/Func1.cpp ----------------------------

def _ieee_div(a: float, b: float) -> float:
    """a / b with IEEE semantics for b == 0 (inf or nan, as in C++)."""
    with np.errstate(all="ignore"):
        return float(np.float64(a) / np.float64(b))


class Func1:
    """Piecewise-linear table over [x_first, x_last)."""

    def __init__(self, xy: Sequence[Sequence[float]]):
        rows = [(float(r[0]), float(r[1])) for r in xy]
        if not rows:
            raise ValueError("LinInterpol: Function is empty.")
        pts = []
        for i, (x, y) in enumerate(rows):
            # slope from the table as given, before sorting (Func1.cpp:42-48)
            slope = (_ieee_div(y - rows[i + 1][1], x - rows[i + 1][0])
                     if i != len(rows) - 1 else 0.0)
            pts.append((x, y, slope))
        pts.sort(key=lambda p: p[0])
        for a, b in zip(pts, pts[1:]):
            if a[0] == b[0]:
                raise ValueError(f"Func1 argument {a[0]} is not unique")
        self.points = pts

    @property
    def limits(self):
        return (self.points[0][0], self.points[-1][0])

    def evaluate(self, x: float) -> float:
        lo, hi = self.limits
        if x < lo or x >= hi:
            raise IndexError(f"Expected {lo} <= x < {hi}, but x={x}")
        k = 0
        while k + 1 < len(self.points) and self.points[k + 1][0] <= x:
            k += 1
        x0, y0, s = self.points[k]
        return s * x + y0 - s * x0

    def mean(self, num_samples: int) -> float:
        """merlict::function::mean (merlict/function/tools.cpp:27-33)."""
        lo, hi = self.limits
        inc = (hi - lo) / float(num_samples)
        arg = lo
        total = 0.0
        for _ in range(num_samples):
            total = total + self.evaluate(arg)
            arg = arg + inc
        return total / num_samples


def _func1_max(self) -> float:
    """Func1::max (Func1.cpp:149-153): the largest value in the table."""
    m = self.points[0][1]
    for p in self.points:
        if p[1] > m:
            m = p[1]
    return m


Func1.max = _func1_max

FUNCTION_DEFAULT_STEPS = 4096   # merlict/function/tools.h:12


def function_integral(f: Func1, steps: int = FUNCTION_DEFAULT_STEPS) -> Func1:
    """merlict::function::integral (merlict/function/tools.cpp:38-58): the
    running sum of f(x) step on `steps` points, the last one evaluated just
    inside the upper limit."""
    lo, hi = f.limits
    step = (hi - lo) / float(steps)
    F = [[lo, 0.0]]
    for i in range(1, steps):
        x = lo + i * step
        F.append([x, f.evaluate(x) * step + F[-1][1]])
    F.append([hi, f.evaluate(math.nextafter(hi, lo)) * step + F[-1][1]])
    return Func1(F)


def function_inverse(f: Func1, steps: int = FUNCTION_DEFAULT_STEPS) -> Func1:
    """merlict::function::inverse (merlict/function/tools.cpp:60-79): the
    table of (f(x), x) on `steps` points."""
    lo, hi = f.limits
    step = (hi - lo) / float(steps)
    inv = [[f.evaluate(lo), lo]]
    for i in range(1, steps):
        x = lo + i * step
        inv.append([f.evaluate(x), x])
    inv.append([f.evaluate(math.nextafter(hi, lo)), hi])
    return Func1(inv)


DEFAULT_REFLECTION = Func1([[200e-9, 0.0], [1200e-9, 0.0]])
DEFAULT_REFRACTION = Func1([[200e-9, 1.0], [1200e-9, 1.0]])
DEFAULT_ABSORPTION = Func1([[200e-9, math.inf], [1200e-9, math.inf]])


def constant(value: float, lo: float = 200e-9, hi: float = 1200e-9) -> Func1:
    return Func1([[lo, value], [hi, value]])


# ---- frames -----------------------------------------------------------------

FRAME_MAX_NUMBER_CHILDREN = 16
FRAME_MIN_STRUCTURE_SIZE = 1e-6


class Frame:
    """A node of the scene tree (merlict/Frame.h): position and rotation in
    its mother frame, children, bounding sphere."""

    primitive = abi.PRIM_NONE
    is_surface = False

    def __init__(self, name: str = "frame", pos=ORIGIN, rot: Rot3 = ROT3_UNITY):
        self.children: list[Frame] = []
        self.mother: Frame | None = None
        self.bounding_sphere_radius = 0.0
        self.T_world = IDENTITY
        self.set_name_pos_rot(name, pos, rot)

    def set_name_pos_rot(self, name, pos, rot):
        if not name or any(c.isspace() for c in name) or "/" in name:
            raise ValueError(f"invalid frame name '{name}'")
        self.name = name
        self.pos = (float(pos[0]), float(pos[1]), float(pos[2]))
        self.rot = rot
        self.T_mother = t_from_rot_pos(rot, self.pos)

    def add(self, child: "Frame") -> "Frame":
        self.children.append(child)
        child.mother = self
        return child

    def params(self):
        return [0.0] * abi.LEAF_PARAMS

    # -- Frame::init_tree_based_on_mother_child_relations, Frame.cpp:125-158
    def init_tree(self) -> "Frame":
        self._cluster_children()
        self._init_frame2world(None)
        self._update_bounding_sphere()
        return self

    def _cluster_children(self):
        stack = [self]
        while stack:
            f = stack.pop()
            f._cluster_own_children()
            stack.extend(reversed(f.children))

    def _cluster_own_children(self):
        if len(self.children) > FRAME_MAX_NUMBER_CHILDREN:
            sectors = [[] for _ in range(8)]
            for child in self.children:
                sectors[v_octant(child.pos)].append(child)
            self.children = []
            for k in range(8):
                sector = sectors[k]
                if positions_in_mother_too_close(sector):
                    for child in sector:
                        child.mother = self
                        self.children.append(child)
                elif len(sector) == 1:
                    sector[0].mother = self
                    self.children.append(sector[0])
                elif len(sector) > 1:
                    center = bounding_sphere_center(sector)
                    octant = Frame(f"oct_{k}", center, ROT3_UNITY)
                    self.add(octant)
                    for child in sector:
                        child.pos = v_sub(child.pos, center)
                        child.T_mother = t_from_rot_pos(child.rot, child.pos)
                        child.mother = octant
                        octant.children.append(child)

    def _init_frame2world(self, mother_T):
        stack = [(self, mother_T)]
        while stack:
            f, mT = stack.pop()
            f.T_world = t_mul(mT, f.T_mother) if mT is not None else f.T_mother
            for c in f.children:
                stack.append((c, f.T_world))

    def _update_bounding_sphere(self):
        order = []
        stack = [self]
        while stack:
            f = stack.pop()
            order.append(f)
            stack.extend(f.children)
        for f in reversed(order):
            if f.children:
                f.bounding_sphere_radius = bounding_sphere_radius(f.children, ORIGIN)

    @property
    def position_in_world(self):
        T = self.T_world
        return (T[0][3], T[1][3], T[2][3])


class SurfaceEntity(Frame):
    """merlict/SurfaceEntity.h: a frame with surface properties."""

    is_surface = True

    def __init__(self, name="surface", pos=ORIGIN, rot=ROT3_UNITY):
        super().__init__(name, pos, rot)
        self.outer_reflection = DEFAULT_REFLECTION
        self.inner_reflection = DEFAULT_REFLECTION
        self.outer_refraction = DEFAULT_REFRACTION
        self.inner_refraction = DEFAULT_REFRACTION
        self.outer_absorption = DEFAULT_ABSORPTION
        self.inner_absorption = DEFAULT_ABSORPTION
        self.allowed_frame: Frame | None = None

    def adopt_surface(self, proto: "SurfaceEntity"):
        for k in ("reflection", "refraction", "absorption"):
            setattr(self, "outer_" + k, getattr(proto, "outer_" + k))
            setattr(self, "inner_" + k, getattr(proto, "inner_" + k))

    def adopt_surface_inside_out(self, proto: "SurfaceEntity"):
        for k in ("reflection", "refraction", "absorption"):
            setattr(self, "outer_" + k, getattr(proto, "inner_" + k))
            setattr(self, "inner_" + k, getattr(proto, "outer_" + k))

    def boundary_layer_is_transparent(self) -> bool:
        return (self.outer_refraction is not DEFAULT_REFRACTION or
                self.inner_refraction is not DEFAULT_REFRACTION)


# ---- bounding spheres, merlict/Frames.cpp ------------------------------------

def position_mean_in_mother(frames):
    s = (0.0, 0.0, 0.0)
    for f in frames:
        s = v_add(s, f.pos)
    return v_div(s, float(len(frames)))


def position_spread_in_mother(frames):
    if len(frames) < 2:
        return 0.0
    mean = position_mean_in_mother(frames)
    u = (0.0, 0.0, 0.0)
    for f in frames:
        r = v_sub(f.pos, mean)
        u = v_add(u, (r[0] * r[0], r[1] * r[1], r[2] * r[2]))
    u = v_div(u, float(len(frames)))
    return math.sqrt(v_norm(u))


def positions_in_mother_too_close(frames):
    return len(frames) >= 2 and position_spread_in_mother(frames) < FRAME_MIN_STRUCTURE_SIZE


def bounding_sphere_radius(frames, center):
    radius = 0.0
    for f in frames:
        need = v_norm(v_sub(center, f.pos)) + f.bounding_sphere_radius
        if need > radius:
            radius = need
    return radius


def bounding_sphere_center_alternative(frames):
    if len(frames) == 1:
        return frames[0].pos
    start = end = None
    maximum = 0.0
    for i in range(len(frames)):
        for j in range(i, len(frames)):
            if i != j:
                dist = (v_norm(v_sub(frames[i].pos, frames[j].pos)) +
                        frames[i].bounding_sphere_radius + frames[j].bounding_sphere_radius)
                if dist > maximum:
                    maximum = dist
                    start, end = frames[i], frames[j]
    if start is None:
        nan = float("nan")
        return (nan, nan, nan)
    d = v_sub(end.pos, start.pos)
    d = v_div(d, v_norm(d))
    return v_add(start.pos, v_mul(d, 0.5 * maximum - start.bounding_sphere_radius))


def bounding_sphere_center(frames):
    center = position_mean_in_mother(frames)
    if len(frames) < FRAME_MAX_NUMBER_CHILDREN:
        alternative = bounding_sphere_center_alternative(frames)
        if bounding_sphere_radius(frames, center) > bounding_sphere_radius(frames, alternative):
            center = alternative
    return center


# ---- primitives, merlict/scenery/primitive ----------------------------------

COS_PI_6 = math.cos(math.pi / 6.0)


class SphereCapWithHexagonalBound(SurfaceEntity):
    primitive = abi.PRIM_SPHERE_CAP_HEX

    def set_curvature_radius_and_outer_hex_radius(self, curvature_radius, outer_hex_radius):
        self.curvature_radius = float(curvature_radius)
        outer = float(outer_hex_radius)
        if outer > self.curvature_radius:
            outer = self.curvature_radius
        if outer <= 0.0:
            raise ValueError("outer hex radius must be > 0")
        self.outer_hex_radius = outer
        self.hex_inner = outer * COS_PI_6
        R = self.curvature_radius
        self.bounding_sphere_radius = hypot(outer, R - math.sqrt(R * R - outer * outer))
        return self

    def params(self):
        return [self.curvature_radius, self.hex_inner] + [0.0] * 6


class SphereCapWithCylinderBound(SurfaceEntity):
    primitive = abi.PRIM_SPHERE_CAP_CYL

    def set_curvature_radius_and_outer_radius(self, curvature_radius, cap_radius):
        R = float(curvature_radius)
        r = float(cap_radius)
        if r > R:
            r = R
        self.curvature_radius = R
        self.radius_square = r * r
        self.bounding_sphere_radius = hypot(r, R - math.sqrt(R * R - r * r))
        return self

    def params(self):
        return [self.curvature_radius, self.radius_square] + [0.0] * 6


class SphereCapWithRectangularBound(SurfaceEntity):
    primitive = abi.PRIM_SPHERE_CAP_RECT

    def set_curvature_radius_and_x_y_width(self, curvature_radius, x_width, y_width):
        self.curvature_radius = float(curvature_radius)
        self.hx = 0.5 * float(x_width)
        self.hy = 0.5 * float(y_width)
        self.bounding_sphere_radius = hypot(self.hx, self.hy)
        return self

    def params(self):
        return [self.curvature_radius, self.hx, self.hy] + [0.0] * 5


class EllipticalCapWithHexagonalBound(SurfaceEntity):
    primitive = abi.PRIM_ELLIPTIC_CAP_HEX

    def set_focal_length_radii_ratio_hex_angle_hex_radius(self, focal_length, ratio,
                                                          hex_rotation, outer_hex_radius):
        mean = focal_length * 0.5
        self.X = mean * ratio
        self.Y = mean / ratio
        self.Z = 0.5 * (self.X + self.Y)
        self.iXX = 1.0 / (self.X * self.X)
        self.iYY = 1.0 / (self.Y * self.Y)
        self.iZZ = 1.0 / (self.Z * self.Z)
        outer = float(outer_hex_radius)
        if outer > self.Z:
            outer = self.Z
        self.hex_inner = outer * COS_PI_6
        Z = self.Z
        self.bounding_sphere_radius = hypot(outer, Z - math.sqrt(Z * Z - outer * outer))
        return self

    def params(self):
        return [self.X, self.Y, self.Z, self.iXX, self.iYY, self.iZZ, self.hex_inner, 0.0]


class Disc(SurfaceEntity):
    primitive = abi.PRIM_DISC

    def set_radius(self, radius):
        if radius <= 0.0:
            raise ValueError("radius must be > 0")
        self.radius_square = float(radius) * float(radius)
        self.bounding_sphere_radius = math.sqrt(self.radius_square)
        return self

    def params(self):
        return [self.radius_square] + [0.0] * 7


class HexPlane(SurfaceEntity):
    primitive = abi.PRIM_HEX_PLANE

    def set_outer_hex_radius(self, outer_hex_radius):
        if outer_hex_radius <= 0.0:
            raise ValueError("outer radius must be > 0")
        self.outer_radius = float(outer_hex_radius)
        self.hex_inner = self.outer_radius * COS_PI_6
        self.bounding_sphere_radius = self.outer_radius
        return self

    def params(self):
        return [self.hex_inner] + [0.0] * 7


class Plane(SurfaceEntity):
    primitive = abi.PRIM_PLANE

    def set_x_y_width(self, x_width, y_width):
        if x_width <= 0.0 or y_width <= 0.0:
            raise ValueError("widths must be > 0")
        self.hx = 0.5 * float(x_width)
        self.hy = 0.5 * float(y_width)
        self.bounding_sphere_radius = hypot(self.hx, self.hy)
        return self

    def params(self):
        return [self.hx, self.hy] + [0.0] * 6


class Annulus(SurfaceEntity):
    primitive = abi.PRIM_ANNULUS

    def set_outer_inner_radius(self, outer_radius, inner_radius):
        self.outer_r2 = float(outer_radius) * float(outer_radius)
        self.inner_r2 = float(inner_radius) * float(inner_radius)
        self.bounding_sphere_radius = math.sqrt(self.outer_r2)
        return self

    def params(self):
        return [self.outer_r2, self.inner_r2] + [0.0] * 6


class PlaneDualSphericalBound(SurfaceEntity):
    primitive = abi.PRIM_PLANE_DUAL_SPHERE

    def set_x_hight_and_y_width(self, hight, width):
        d = (width * width - hight * hight) / (2.0 * hight)
        self.circle_radius = d / 2.0 + hight / 2.0
        self.circ1 = (+d / 2.0, 0.0)
        self.circ2 = (-d / 2.0, 0.0)
        self.bounding_sphere_radius = width * 0.5
        return self

    def params(self):
        return [self.circ1[0], self.circ1[1], self.circ2[0], self.circ2[1],
                self.circle_radius, 0.0, 0.0, 0.0]


class Triangle(SurfaceEntity):
    primitive = abi.PRIM_TRIANGLE

    def set_corners_in_xy_plane(self, ax, ay, bx, by, cx, cy):
        """Triangle.cpp:9-22: every edge longer than zero."""
        self.A, self.B, self.C = ((float(ax), float(ay)), (float(bx), float(by)),
                                  (float(cx), float(cy)))

        def edge(p, q):
            return math.sqrt((p[0] - q[0]) * (p[0] - q[0]) + (p[1] - q[1]) * (p[1] - q[1]))
        for length, name in ((edge(self.A, self.B), "AB"), (edge(self.C, self.A), "AC"),
                             (edge(self.C, self.B), "CB")):
            if not length > 0.0:
                raise ValueError(f"Triangle: expected edge length of {name} > 0.0, "
                                 f"but actual {length}m")
        norms = [math.sqrt(p[0] * p[0] + p[1] * p[1]) for p in (self.A, self.B, self.C)]
        self.bounding_sphere_radius = max(norms)
        return self

    def set_normal_and_3_vertecies(self, normal, a, b, c):
        """Triangle.cpp:24-57: the frame at the centroid, rotated so that its
        z axis is the facet normal; the corners in that frame's xy plane."""
        pos = v_div(v_add(v_add(a, b), c), 3.0)
        a, b, c = v_sub(a, pos), v_sub(b, pos), v_sub(c, pos)
        d = v_sub(normal, UNIT_Z)
        if v_dot(d, d) > MAX_DEVIATION_EQUAL_VEC3_SQUARE:
            rot = Rot3(axis=v_cross(UNIT_Z, normal), angle=v_angle_in_between(UNIT_Z, normal))
            inv = t_inverse(t_from_rot_pos(rot, ORIGIN))
            a, b, c = t_orientation(inv, a), t_orientation(inv, b), t_orientation(inv, c)
        else:
            rot = ROT3_UNITY
        self.set_name_pos_rot(self.name, pos, rot)
        return self.set_corners_in_xy_plane(a[0], a[1], b[0], b[1], c[0], c[1])

    def params(self):
        return [self.A[0], self.A[1], self.B[0], self.B[1], self.C[0], self.C[1], 0.0, 0.0]


class Cylinder(SurfaceEntity):
    primitive = abi.PRIM_CYLINDER

    def set_radius_and_length(self, radius, length):
        """Cylinder.cpp:68-72."""
        self._set_radius(radius)
        if not length > 0.0:
            raise ValueError(f"The length of a cylinder must be larger than 0.0m, not {length}")
        self.length = float(length)
        self.bounding_sphere_radius = hypot(0.5 * self.length, self.radius)
        return self

    def _set_radius(self, radius):
        if not radius > 0.0:
            raise ValueError(f"The radius of a cylinder must be larger than 0.0m, not {radius}")
        self.radius = float(radius)

    def set_cylinder(self, radius, start, end):
        """Cylinder.cpp:17-67: position at the middle, z axis along end-start."""
        self._set_radius(radius)
        d = v_sub(start, end)
        if v_dot(d, d) <= MAX_DEVIATION_EQUAL_VEC3_SQUARE:
            raise ValueError("The start and end point of a cylinder must not be the same")
        axis = v_sub(end, start)
        pos = v_add(start, v_div(axis, 2.0))
        if axis[0] == 0.0 and axis[1] == 0.0 and abs(axis[2]) > 0.0:
            rot = Rot3(axis=UNIT_Z, angle=0.0)
        else:
            rot = Rot3(axis=v_cross(axis, UNIT_Z),
                       angle=-math.acos(v_dot(UNIT_Z, axis) / v_norm(axis)))
        self.radius = float(radius)
        self.length = v_norm(v_sub(end, start))
        self.set_name_pos_rot(self.name, pos, rot)
        self.bounding_sphere_radius = hypot(0.5 * self.length, self.radius)
        return self

    def params(self):
        return [self.radius, self.length] + [0.0] * 6


class Sphere(SurfaceEntity):
    primitive = abi.PRIM_SPHERE

    def set_radius(self, radius):
        if radius <= 0.0:
            raise ValueError("sphere radius must be > 0")
        self.radius = float(radius)
        self.bounding_sphere_radius = self.radius
        return self

    def params(self):
        return [self.radius] + [0.0] * 7


# ---- composite primitives ---------------------------------------------------

class BiConvexLensHexBound(SurfaceEntity):
    """Two hexagonal caps looking inwards plus six dual-sphere side walls
    (merlict/scenery/primitive/BiConvexLensHexBound.cpp:7-64).  Set the
    lens's surface (inner_refraction) before calling
    set_curvature_radius_and_outer_hex_radius."""

    def set_curvature_radius_and_outer_hex_radius(self, R, outer):
        cap_h = R - math.sqrt(R * R - outer * outer)
        front = self.add(SphereCapWithHexagonalBound("front_cap", (0.0, 0.0, -cap_h), ROT3_UNITY))
        rear = self.add(SphereCapWithHexagonalBound("rear_cap", (0.0, 0.0, cap_h),
                                                    Rot3(math.pi, 0.0, 0.0)))
        for cap in (front, rear):
            cap.adopt_surface_inside_out(self)
            cap.set_curvature_radius_and_outer_hex_radius(R, outer)
            cap.allowed_frame = self
        inner = outer * math.sqrt(3.0) / 2.0
        hight = 2.0 * (R - math.sqrt(R * R - outer * outer)
                       + math.sqrt(R * R - inner * inner) - R)
        for i in range(6):
            phi = float(i) * 1.0 / 3.0 * math.pi
            wall = self.add(PlaneDualSphericalBound(
                f"wall_{i}", (inner * math.sin(phi), inner * math.cos(phi), 0.0),
                Rot3(math.pi * 0.5, math.pi * 0.5, phi)))
            wall.set_x_hight_and_y_width(hight, outer)
        return self


class BiConvexLens(SurfaceEntity):
    """Two round caps (merlict/scenery/primitive/BiConvexLens.cpp:7-36)."""

    def set_curvature_radius_and_aperture_radius(self, R, aperture):
        cap_h = R - math.sqrt(R * R - aperture * aperture)
        front = self.add(SphereCapWithCylinderBound("front_cap", (0.0, 0.0, -cap_h), ROT3_UNITY))
        rear = self.add(SphereCapWithCylinderBound("rear_cap", (0.0, 0.0, cap_h),
                                                   Rot3(math.pi, 0.0, 0.0)))
        for cap in (front, rear):
            cap.adopt_surface_inside_out(self)
            cap.set_curvature_radius_and_outer_radius(R, aperture)
            cap.allowed_frame = self
        return self


class RectangularBox(SurfaceEntity):
    """Six planes adopting the box's surface (RectangularBox.cpp:7-54)."""

    def set_xyz_width(self, xw, yw, zw):
        z_off = (0.0, 0.0, 0.5 * zw)
        x_off = (0.5 * xw, 0.0, 0.0)
        y_off = (0.0, 0.5 * yw, 0.0)
        walls = [
            (z_off, Rot3(0.0, 0.0, 0.0), xw, yw),
            (v_mul(z_off, -1.0), Rot3(math.pi, 0.0, 0.0), xw, yw),
            (x_off, Rot3(0.0, -math.pi / 2.0, 0.0), zw, yw),
            (v_mul(x_off, -1.0), Rot3(0.0, math.pi / 2.0, 0.0), zw, yw),
            (y_off, Rot3(math.pi / 2.0, 0.0, 0.0), xw, zw),
            (v_mul(y_off, -1.0), Rot3(-math.pi / 2.0, 0.0, 0.0), xw, zw),
        ]
        for i, (pos, rot, a, b) in enumerate(walls):
            w = self.add(Plane(f"{self.name}_wall_{i}", pos, rot))
            w.set_x_y_width(a, b)
            w.adopt_surface(self)
        return self


# ---- hexagonal grids, merlict/scenery/geometry/HexGrid*.cpp ------------------

def hex_grid_annulus(outer_radius: float, inner_radius: float, spacing: float):
    unit_b = v_mul(UNIT_Y, spacing)
    unit_a = v_mul(v_add(v_mul(UNIT_Y, 0.5), v_div(v_mul(UNIT_X, math.sqrt(3.0)), 2.0)), spacing)
    n = int(2.0 * math.floor(outer_radius / spacing))
    grid = []
    for a in range(-n, n + 1):
        for b in range(-n, n + 1):
            cell = v_add(v_mul(unit_a, float(a)), v_mul(unit_b, float(b)))
            r = v_norm(cell)
            if r <= outer_radius and r >= inner_radius:
                grid.append(cell)
    return grid


HEX_UNIT_U = UNIT_Y
HEX_UNIT_V = v_add(v_mul(UNIT_X, +math.sin(2. / 3. * math.pi)), v_mul(UNIT_Y, math.cos(2. / 3. * math.pi)))
HEX_UNIT_W = v_add(v_mul(UNIT_X, -math.sin(2. / 3. * math.pi)), v_mul(UNIT_Y, math.cos(2. / 3. * math.pi)))


def hex_prism_inside(inner, v):
    u = v_dot(HEX_UNIT_U, v)
    vv = v_dot(HEX_UNIT_V, v)
    w = v_dot(HEX_UNIT_W, v)
    return u < inner and u > -inner and vv < inner and vv > -inner and w < inner and w > -inner


def hex_grid_flower(outer_grid_radius: float, facets_on_diagonal: int):
    """HexGridFlower.cpp:7-48: returns (cells, facet_spacing)."""
    if facets_on_diagonal % 2 == 0:
        facets_on_diagonal += 1
    inner_grid = outer_grid_radius * (math.sqrt(3.0) / 2.0)
    outer_facet = (2.0 * inner_grid) / (0.5 * (3.0 * float(facets_on_diagonal) + 1.0))
    spacing = 2.0 * (outer_facet * (math.sqrt(3.0) / 2.0))
    prism_inner = outer_grid_radius * COS_PI_6
    unit_b = v_mul(UNIT_X, spacing)
    unit_a = v_mul(v_add(v_mul(UNIT_X, 0.5), v_div(v_mul(UNIT_Y, math.sqrt(3.0)), 2.0)), spacing)
    n = int(2.0 * math.floor(outer_grid_radius / spacing))
    cells = []
    for a in range(-n, n + 1):
        for b in range(-n, n + 1):
            cell = v_add(v_mul(unit_a, float(a)), v_mul(unit_b, float(b)))
            if hex_prism_inside(prism_inner, cell):
                cells.append(cell)
    return cells, spacing


# ---- sensors and flattening ---------------------------------------------------

class Sensor:
    """merlict::sensor::Sensor: an id and the frame whose arrivals it collects."""

    def __init__(self, id: int, frame: Frame):
        self.id = int(id)
        self.frame = frame


class NoSuchKey(KeyError):
    """ResourceMap::NoSuchKey (merlict/scenery/ResourceMap.h)."""


class KeyAlreadyInUse(KeyError):
    """ResourceMap::KeyAlreadyInUse (merlict/scenery/ResourceMap.h)."""


class ResourceMap:
    """A map of named resources that refuses unknown and reused names
    (ColorMap.cpp:8-37, FunctionMap.cpp:8-35, SensorMap.cpp:8-47)."""

    def __init__(self, kind: str):
        self.kind = kind
        self.items: dict = {}

    def has(self, key) -> bool:
        return key in self.items

    def get(self, key):
        if key not in self.items:
            raise NoSuchKey(f"There is no {self.kind} called '{key}'.")
        return self.items[key]

    def add(self, key, value):
        if key in self.items:
            raise KeyAlreadyInUse(f"The {self.kind} key '{key}' is already in use.")
        self.items[key] = value
        return value


class Scenery:
    """A root frame plus the sensors, colors and functions of the scene
    (merlict/scenery/Scenery.h)."""

    def __init__(self):
        self.root = Frame("root", ORIGIN, Rot3(0.0, 0.0, 0.0))
        self.sensors: list[Sensor] = []
        self.colors = ResourceMap("color")
        self.functions = ResourceMap("function")

    def add_sensor(self, id: int, frame: Frame) -> Sensor:
        s = Sensor(id, frame)
        self.sensors.append(s)
        return s

    def init(self) -> "Scenery":
        frames = [s.frame for s in self.sensors]
        if len(set(map(id, frames))) != len(frames):
            raise ValueError("two sensors share the same frame")
        self.root.init_tree()
        return self

    def flatten(self) -> abi.FlatScene:
        return flatten(self.root, self.sensors)


def flatten(root: Frame, sensors: Sequence[Sensor] = ()) -> abi.FlatScene:
    """Flattens an initialised tree in the order merlict's CausalIntersection
    visits it (RayAndFrame.cpp:137-149)."""
    nodes = []
    node_sphere, node_skip, node_leaf = [], [], []
    leaf_node, leaf_T, leaf_prim, leaf_params, leaf_surface = [], [], [], [], []
    node_index = {}
    fn_ids = {}
    fn_offset = [0]
    fn_points = []

    def fid(f: Func1) -> int:
        k = id(f)
        if k not in fn_ids:
            fn_ids[k] = len(fn_offset) - 1
            for p in f.points:
                fn_points.append(p)
            fn_offset.append(len(fn_points))
        return fn_ids[k]

    d_refl, d_refr, d_abs = fid(DEFAULT_REFLECTION), fid(DEFAULT_REFRACTION), fid(DEFAULT_ABSORPTION)
    allowed_frames = []
    # iterative preorder with explicit skip fix-up
    pending = [(root, False)]
    while pending:
        f, closing = pending.pop()
        if closing:
            node_skip[node_index[id(f)]] = len(nodes)
            continue
        idx = len(nodes)
        nodes.append(f)
        node_index[id(f)] = idx
        p = f.position_in_world
        node_sphere.append((p[0], p[1], p[2], f.bounding_sphere_radius))
        node_skip.append(-1)
        if f.children:
            node_leaf.append(-1)
            pending.append((f, True))
            for c in reversed(f.children):
                pending.append((c, False))
        else:
            node_leaf.append(len(leaf_node))
            leaf_node.append(idx)
            T = f.T_world
            leaf_T.append(T[0] + T[1] + T[2])
            leaf_prim.append(f.primitive)
            leaf_params.append(f.params())
            if f.is_surface:
                flags = 0
                if f.boundary_layer_is_transparent():
                    flags |= abi.FLAG_TRANSPARENT
                if f.inner_refraction is DEFAULT_REFRACTION:
                    flags |= abi.FLAG_INNER_REFRACTION_DEFAULT
                if f.outer_refraction is DEFAULT_REFRACTION:
                    flags |= abi.FLAG_OUTER_REFRACTION_DEFAULT
                leaf_surface.append([fid(f.outer_reflection), fid(f.inner_reflection),
                                     fid(f.outer_refraction), fid(f.inner_refraction),
                                     fid(f.outer_absorption), fid(f.inner_absorption), -1, flags])
                allowed_frames.append(f.allowed_frame)
            else:
                leaf_surface.append([d_refl, d_refl, d_refr, d_refr, d_abs, d_abs, -1,
                                     abi.FLAG_INNER_REFRACTION_DEFAULT | abi.FLAG_OUTER_REFRACTION_DEFAULT])
                allowed_frames.append(None)
            node_skip[idx] = idx + 1
    for leaf, fr in enumerate(allowed_frames):
        if fr is not None:
            if id(fr) not in node_index:
                raise ValueError("a surface restricts propagation to a frame outside its tree")
            leaf_surface[leaf][abi.SURF_ALLOWED_NODE] = node_index[id(fr)]
    leaf_sensor = np.full(len(leaf_node), -1, np.int32)
    sensor_ids = np.zeros(len(sensors), np.int64)
    node_leaf_a = np.asarray(node_leaf, np.int32)
    for s_idx, s in enumerate(sensors):
        sensor_ids[s_idx] = s.id
        n = node_index.get(id(s.frame))
        if n is not None and node_leaf_a[n] >= 0:
            leaf_sensor[node_leaf_a[n]] = s_idx
    flat = abi.FlatScene(
        node_sphere=np.asarray(node_sphere, np.float64).reshape(-1, 4),
        node_skip=np.asarray(node_skip, np.int32),
        node_leaf=node_leaf_a,
        leaf_node=np.asarray(leaf_node, np.int32),
        leaf_frame2world=np.asarray(leaf_T, np.float64).reshape(-1, 12),
        leaf_primitive=np.asarray(leaf_prim, np.int32),
        leaf_params=np.asarray(leaf_params, np.float64).reshape(-1, abi.LEAF_PARAMS),
        leaf_surface=np.asarray(leaf_surface, np.int32).reshape(-1, abi.SURF_COLUMNS),
        leaf_sensor=leaf_sensor,
        function_offset=np.asarray(fn_offset, np.int32),
        function_points=np.asarray(fn_points, np.float64).reshape(-1, 3),
        default_refraction=d_refr,
        hex_unit_u=np.asarray(HEX_UNIT_U), hex_unit_v=np.asarray(HEX_UNIT_V),
        hex_unit_w=np.asarray(HEX_UNIT_W),
        num_sensors=len(sensors),
        sensor_ids=sensor_ids,
    )
    flat.validate()
    return flat
