"""Optical systems of the benchmark configurations, built with this
package's scenery model.

* segmented_reflector: the Davies-Cotton / parabolic mix of hexagonal
  spherical-cap facets of merlict's segmented_imaging_reflector
  (merlict/scenery/segmented_imaging_reflector/Geometry.cpp:14-191,
  Factory.cpp:14-27);
* light_field_sensor: merlict_portal_plenoscope's light-field sensor -- a
  lens array of BiConvexLensHexBound, bin walls, face plate, housing and a
  plane of hexagonal lixel sensors (light_field_sensor/Geometry.cpp:13-141,
  Factory.cpp:16-207);
* reflector_camera / light_field_telescope: the scenes of the benchmark
  configurations (a reflector with a hexagonal-pixel camera or a
  light-field sensor in its focal plane).

The layout rules and their floating-point order follow merlict's, so the
flattened scenes agree bit for bit with scenes built by merlict itself.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from .scenery import (ROT3_UNITY, UNIT_X, UNIT_Y, UNIT_Z, Annulus, BiConvexLensHexBound,
                      Cylinder, Disc, Frame, Func1, HexPlane, Plane, Rot3, Scenery, Sensor,
                      SphereCapWithHexagonalBound, SurfaceEntity, constant, deg2rad,
                      hex_grid_annulus, hex_grid_flower, hypot, v_add, v_angle_in_between,
                      v_cross, v_div, v_dot, v_mul, v_norm, v_sub)


# ---- segmented imaging reflector ---------------------------------------------

@dataclass
class ReflectorConfig:
    """segmented_imaging_reflector::Config (Config.cpp:7-17)."""
    focal_length: float = 4.889
    DaviesCotton_over_parabolic_mixing_factor: float = 0.5
    max_outer_aperture_radius: float = 2.1
    min_inner_aperture_radius: float = 0.2
    facet_inner_hex_radius: float = 0.30
    gap_between_facets: float = 0.01
    outer_aperture_shape_hex: bool = False


def hex_aperture_facets(outer: float, inner: float, spacing: float, max_outer_radius: float):
    """Facet centres inside a hexagonal outer aperture and outside an inner
    disc (Geometry.cpp:32-67)."""
    unit_b = v_mul(UNIT_Y, spacing)
    unit_a = v_mul(v_add(v_mul(UNIT_Y, 0.5), v_div(v_mul(UNIT_X, math.sqrt(3.0)), 2.0)), spacing)
    unit_u = UNIT_X
    unit_v = v_add(v_mul(UNIT_Y, math.sin(2.0 / 3.0 * math.pi)), v_mul(UNIT_X, math.cos(2.0 / 3.0 * math.pi)))
    unit_w = v_add(v_mul(UNIT_Y, -math.sin(2.0 / 3.0 * math.pi)), v_mul(UNIT_X, math.cos(2.0 / 3.0 * math.pi)))
    R = (math.sqrt(3.0) / 2.0) * outer
    N = int(2.0 * math.ceil(max_outer_radius / spacing))
    out = []
    for a in range(-N, N + 1):
        for b in range(-N, N + 1):
            c = v_add(v_mul(unit_a, float(a)), v_mul(unit_b, float(b)))
            u, v, w = v_dot(unit_u, c), v_dot(unit_v, c), v_dot(unit_w, c)
            if (u < R and u > -R and v < R and v > -R and w < R and w > -R and
                    hypot(c[0], c[1]) > inner):
                out.append(c)
    return out


class ReflectorGeometry:
    """Facet centres and orientations (Geometry.cpp:14-191)."""

    def __init__(self, cfg: ReflectorConfig):
        self.cfg = cfg
        f = cfg.focal_length
        self.focal_point = (0.0, 0.0, f)
        spacing = self.facet_spacing
        outer = cfg.max_outer_aperture_radius - spacing / 2.0
        inner = cfg.min_inner_aperture_radius + spacing / 2.0
        if cfg.outer_aperture_shape_hex:
            pos = hex_aperture_facets(outer, inner, spacing, cfg.max_outer_aperture_radius)
        else:
            pos = hex_grid_annulus(outer, inner, spacing)
        pos = [(p[0], p[1], self.z_pos(math.sqrt(p[0] * p[0] + p[1] * p[1] + 0.0 * 0.0)))
               for p in pos]
        # move the dish until the mean facet distance to the focal point is f
        it = 0
        while True:
            it += 1
            if it > 100:
                raise RuntimeError("Exceeded max number of 100 iterations.")
            total = 0.0
            for p in pos:
                total = total + v_norm(v_sub(p, self.focal_point))
            deviation = f - total / float(len(pos))
            step = -deviation * 0.5
            pos = [(p[0], p[1], p[2] + step) for p in pos]
            if not (abs(deviation) > f * 1e-6):
                break
        self.facet_positions = pos

    @property
    def facet_spacing(self) -> float:
        return self.cfg.facet_inner_hex_radius * 2.0 + self.cfg.gap_between_facets

    @property
    def facet_outer_hex_radius(self) -> float:
        return self.cfg.facet_inner_hex_radius * 2.0 / math.sqrt(3.0)

    def z_pos(self, dist: float) -> float:
        f = self.cfg.focal_length
        z_dc = f - math.sqrt(f * f - dist * dist)
        z_pa = 1.0 / (4.0 * f) * dist * dist
        w = self.cfg.DaviesCotton_over_parabolic_mixing_factor
        return w * z_dc + (1.0 - w) * z_pa

    def rotation_for_facet(self, pos) -> Rot3:
        to_focal = v_sub(self.focal_point, pos)
        axis = v_cross(to_focal, UNIT_Z)
        angle = v_angle_in_between(UNIT_Z, to_focal)
        return Rot3(axis=axis, angle=-(0.5 * angle))

    @property
    def num_facets(self) -> int:
        return len(self.facet_positions)

    @property
    def effective_area(self) -> float:
        r = self.cfg.facet_inner_hex_radius
        return self.num_facets * (r * r * 6.0 / math.sqrt(3.0))


def segmented_reflector(reflector: SurfaceEntity, cfg: ReflectorConfig) -> ReflectorGeometry:
    """Adds the facets to `reflector`, each adopting its surface."""
    g = ReflectorGeometry(cfg)
    for i, pos in enumerate(g.facet_positions):
        facet = reflector.add(SphereCapWithHexagonalBound(
            f"mirror_facet_{i}", pos, g.rotation_for_facet(pos)))
        facet.set_curvature_radius_and_outer_hex_radius(
            cfg.focal_length * 2.0, g.facet_outer_hex_radius)
        facet.adopt_surface(reflector)
    return g


# ---- light-field sensor -------------------------------------------------------

@dataclass
class LightFieldSensorConfig:
    """light_field_sensor::Config (merlict_portal_plenoscope/light_field_sensor/Config.cpp)."""
    expected_imaging_system_focal_length: float = 75.0
    expected_imaging_system_max_aperture_radius: float = 25.0
    max_FoV_diameter: float = deg2rad(6.5)
    pixel_FoV_hex_flat2flat: float = deg2rad(0.1)
    num_paxel_on_pixel_diagonal: int = 13
    housing_overhead: float = 1.2
    lens_refraction: Func1 | None = None
    bin_reflection: Func1 | None = None


def lens_maker_curvature_radius(focal_length: float, aperture_radius: float,
                                refractive_index: float) -> float:
    """lens_maker::get_curvature_radius, geometry/lens_maker.cpp:16-36."""
    R = focal_length
    deviation = 0.0
    it = 0
    n = refractive_index
    while True:
        it += 1
        if it > 1000:
            raise RuntimeError("lens maker: exceeded 1000 iterations")
        R = R - deviation * 0.1
        t = 2.0 * R - 2.0 * math.sqrt(R * R - aperture_radius * aperture_radius)
        f_inv = (n - 1.0) * (2.0 / R - ((n - 1.0) * t) / (n * R * R))
        deviation = 1.0 / f_inv - focal_length
        if not (abs(deviation) > 1e-6):
            break
    return R


class LightFieldSensorGeometry:
    """light_field_sensor::Geometry (Geometry.cpp:13-141)."""

    def __init__(self, cfg: LightFieldSensorConfig):
        self.cfg = cfg
        f = cfg.expected_imaging_system_focal_length
        self.pixel_lens_inner_aperture_radius = f * math.tan(cfg.pixel_FoV_hex_flat2flat / 2.0)
        self.pixel_lens_outer_aperture_radius = self.pixel_lens_inner_aperture_radius * 2.0 / math.sqrt(3.0)
        self.pixel_spacing = self.pixel_lens_inner_aperture_radius * 2.0
        self.max_outer_sensor_radius = f * math.tan(cfg.max_FoV_diameter / 2.0)
        # paxel template (set_up_paxel_per_pixel_template_grid)
        self.paxel_template, self.lixel_spacing = hex_grid_flower(
            self.pixel_lens_outer_aperture_radius, cfg.num_paxel_on_pixel_diagonal)
        # pixel grid
        self.pixel_grid = hex_grid_annulus(
            self.max_outer_sensor_radius - self.pixel_lens_outer_aperture_radius, 0.0,
            self.pixel_spacing)
        self.lixel_inner_radius = 0.5 * self.lixel_spacing
        self.lixel_outer_radius = self.lixel_inner_radius * 2.0 / math.sqrt(3.0)
        air = self.pixel_lens_inner_aperture_radius - 0.5 * self.lixel_inner_radius
        f_over_d = f / (2.0 * cfg.expected_imaging_system_max_aperture_radius)
        self.pixel_lens_focal_length = f_over_d * 2.0 * air
        self.pixel_plane_to_paxel_plane_distance = self.pixel_lens_focal_length
        r = 1.0 + self.pixel_plane_to_paxel_plane_distance / f
        self.paxel_grid_centers = [v_mul(p, r) for p in self.pixel_grid]
        self.lixel_positions = [v_add(c, p) for c in self.paxel_grid_centers
                                for p in self.paxel_template]
        mean_n = cfg.lens_refraction.mean(137)
        self.pixel_lens_curvature_radius = 1.20 * lens_maker_curvature_radius(
            self.pixel_lens_focal_length, self.pixel_lens_outer_aperture_radius, mean_n)
        self.outer_sensor_housing_radius = self.max_outer_sensor_radius * cfg.housing_overhead
        self.bin_hight = self.pixel_plane_to_paxel_plane_distance * 0.25
        self.lixel_z_orientation = 1.0 / 6.0 * math.pi

    @property
    def num_pixels(self) -> int:
        return len(self.pixel_grid)

    @property
    def num_lixels(self) -> int:
        return len(self.lixel_positions)


# merlict's named colours the factory registers (merlict/Color.cpp); they
# only matter for rendering, but their names take part in the scenery's
# colour map and so in its duplicate-name errors.
COLOR_WHITE, COLOR_GREEN, COLOR_GRAY, COLOR_RED = (255, 255, 255), (0, 255, 0), (128, 128, 128), (255, 0, 0)


def _lens_array(frame: Frame, scenery: Scenery, g: "LightFieldSensorGeometry"):
    """Factory::add_lens_array, Factory.cpp:16-37."""
    scenery.colors.add("lens_white", COLOR_WHITE)
    lens_array = frame.add(Frame("lens_array", (0.0, 0.0, 0.0), ROT3_UNITY))
    for i, pos in enumerate(g.pixel_grid):
        lens = lens_array.add(BiConvexLensHexBound(f"lens_{i}", pos, ROT3_UNITY))
        lens.inner_refraction = g.cfg.lens_refraction
        lens.set_curvature_radius_and_outer_hex_radius(
            g.pixel_lens_curvature_radius, g.pixel_lens_outer_aperture_radius)


def _pixel_bin(frame: Frame, g: "LightFieldSensorGeometry", name: str, pos):
    """Factory::add_pixel_bin_with_name_at_pos, Factory.cpp:58-85."""
    b = frame.add(Frame(name, pos, ROT3_UNITY))
    R = g.pixel_lens_inner_aperture_radius
    h = g.bin_hight
    for j in range(6):
        phi = float(j) * 1.0 / 3.0 * math.pi
        wall = b.add(Plane(f"{name}_{j}", (R * math.sin(phi), R * math.cos(phi), -0.5 * h),
                           Rot3(-math.pi * 0.5, 0.0, phi)))
        wall.set_x_y_width(g.pixel_lens_outer_aperture_radius, h)
        wall.outer_reflection = g.cfg.bin_reflection


def _pixel_bin_array(frame: Frame, scenery: Scenery, g: "LightFieldSensorGeometry"):
    """Factory::add_pixel_bin_array, Factory.cpp:39-56."""
    bins = frame.add(Frame("bin_array", (0.0, 0.0, g.pixel_plane_to_paxel_plane_distance),
                           ROT3_UNITY))
    scenery.colors.add("bin_wall_green", COLOR_GREEN)
    for i, pos in enumerate(g.paxel_grid_centers):
        _pixel_bin(bins, g, f"bin_{i}", pos)


def _frontplate(frame: Frame, scenery: Scenery, g: "LightFieldSensorGeometry"):
    """Factory::add_light_field_sensor_frontplate, Factory.cpp:87-124."""
    scenery.colors.add("housing_gray", COLOR_GRAY)
    face_pos = hex_grid_annulus(g.max_outer_sensor_radius + g.pixel_spacing,
                                g.max_outer_sensor_radius - g.pixel_lens_outer_aperture_radius,
                                g.pixel_spacing)
    face_plate = frame.add(Frame("face_plate", (0.0, 0.0, 0.0), ROT3_UNITY))
    for i, pos in enumerate(face_pos):
        face = face_plate.add(HexPlane(f"face_{i}", pos, ROT3_UNITY))
        face.set_outer_hex_radius(g.pixel_lens_outer_aperture_radius)
    ring = face_plate.add(Annulus("outer_front_ring", (0.0, 0.0, 0.0), ROT3_UNITY))
    ring.set_outer_inner_radius(g.outer_sensor_housing_radius, g.max_outer_sensor_radius)


def _lixel_sensor_plane(frame: Frame, scenery: Scenery, g: "LightFieldSensorGeometry", sensors):
    """Factory::add_lixel_sensor_plane, Factory.cpp:126-151: lixel i is
    sensor i."""
    scenery.colors.add("cell_red", COLOR_RED)
    lixels = frame.add(Frame("lixel_array", (0.0, 0.0, g.pixel_plane_to_paxel_plane_distance),
                             ROT3_UNITY))
    for i, pos in enumerate(g.lixel_positions):
        lix = lixels.add(HexPlane(f"lixel_{i}", pos, Rot3(0.0, 0.0, g.lixel_z_orientation)))
        lix.set_outer_hex_radius(g.lixel_outer_radius)
        sensors.append(Sensor(i, lix))


def _image_sensor_housing(frame: Frame, scenery: Scenery, g: "LightFieldSensorGeometry"):
    """Factory::add_image_sensor_housing, Factory.cpp:153-189."""
    scenery.colors.add("frontplate_gray", COLOR_GRAY)
    housing_height = .67 * g.outer_sensor_housing_radius
    housing = frame.add(Frame("sensor_housing", (0.0, 0.0, 0.0), ROT3_UNITY))
    top = housing.add(Disc("top", (0.0, 0.0, housing_height), ROT3_UNITY))
    top.set_radius(g.outer_sensor_housing_radius)
    cyl = housing.add(Cylinder("cylinder", (0.0, 0.0, 0.0), ROT3_UNITY))
    cyl.set_cylinder(g.outer_sensor_housing_radius, (0.0, 0.0, 0.0), (0.0, 0.0, housing_height))


def light_field_sensor(frame: Frame, scenery: Scenery, cfg: LightFieldSensorConfig,
                       sensors: list | None = None):
    """Factory::add_light_field_sensor_to_frame_in_scenery (Factory.cpp:191-207).
    The lixels become sensors 0..num_lixels-1, appended to `sensors`
    (default: the scenery's own sensors)."""
    g = LightFieldSensorGeometry(cfg)
    sensors = scenery.sensors if sensors is None else sensors
    front = frame.add(Frame("front", (0.0, 0.0, 0.0), ROT3_UNITY))
    _lens_array(front, scenery, g)
    _frontplate(front, scenery, g)
    _image_sensor_housing(frame, scenery, g)
    _pixel_bin_array(frame, scenery, g)
    _lixel_sensor_plane(frame, scenery, g, sensors)
    return g


def demonstration_light_field_sensor(frame: Frame, scenery: Scenery, cfg: LightFieldSensorConfig,
                                     sensors: list | None = None):
    """Factory::add_demonstration_light_field_sensor_to_frame_in_scenery
    (Factory.cpp:209-266): one lens, one bin and the lixels of one pixel
    (at 0.95 of their size)."""
    g = LightFieldSensorGeometry(cfg)
    sensors = scenery.sensors if sensors is None else sensors
    scenery.colors.add("lens_white", COLOR_WHITE)
    lens = frame.add(BiConvexLensHexBound("lens_0", (0.0, 0.0, 0.0), ROT3_UNITY))
    lens.inner_refraction = cfg.lens_refraction
    lens.set_curvature_radius_and_outer_hex_radius(
        g.pixel_lens_curvature_radius, g.pixel_lens_outer_aperture_radius)
    bins = frame.add(Frame("bin_array", (0.0, 0.0, g.pixel_plane_to_paxel_plane_distance),
                           ROT3_UNITY))
    scenery.colors.add("bin_wall_green", COLOR_GREEN)
    _pixel_bin(bins, g, "bin_0", (0.0, 0.0, 0.0))
    scenery.colors.add("light_field_sensor_cell_red", COLOR_RED)
    lixels = frame.add(Frame("lixel_array", (0.0, 0.0, g.pixel_plane_to_paxel_plane_distance),
                             ROT3_UNITY))
    for i, pos in enumerate(g.paxel_template):
        lix = lixels.add(HexPlane(f"lixel_{i}", pos, Rot3(0.0, 0.0, g.lixel_z_orientation)))
        lix.set_outer_hex_radius(0.95 * g.lixel_outer_radius)
        sensors.append(Sensor(i, lix))
    return g


# ---- benchmark scenes -----------------------------------------------------------

def reflector_camera(focal_length=4.9, davies_cotton=1.0, max_aperture_radius=2.1,
                     min_aperture_radius=0.0, facet_inner_hex_radius=0.3, gap=0.01,
                     reflectivity=0.9, num_pixels=1440, pixel_flat2flat=0.0095,
                     shield_radius=0.2) -> Scenery:
    """A segmented reflector with a flat camera of hexagonal pixels in its
    focal plane: the pixel centres are the `num_pixels` points of a
    hexagonal grid nearest the optical axis, each pixel a sensor."""
    sc = Scenery()
    reflector = sc.root.add(SurfaceEntity("reflector", (0.0, 0.0, 0.0), ROT3_UNITY))
    reflector.outer_reflection = constant(reflectivity)
    segmented_reflector(reflector, ReflectorConfig(
        focal_length, davies_cotton, max_aperture_radius, min_aperture_radius,
        facet_inner_hex_radius, gap))
    cam = sc.root.add(Frame("camera", (0.0, 0.0, focal_length), ROT3_UNITY))
    grid_radius = pixel_flat2flat * (math.sqrt(float(num_pixels)) + 2.0)
    cells = hex_grid_annulus(grid_radius, 0.0, pixel_flat2flat)
    order = sorted(range(len(cells)), key=lambda i: v_norm(cells[i]))
    if len(order) < num_pixels:
        raise RuntimeError("pixel grid too small")
    for i in range(num_pixels):
        # unrotated: flat sides face the grid neighbours, pixels tile without overlap
        pix = cam.add(HexPlane(f"pixel_{i}", cells[order[i]], ROT3_UNITY))
        pix.set_outer_hex_radius(pixel_flat2flat / math.sqrt(3.0))
        sc.add_sensor(i, pix)
    if shield_radius > 0.0:
        disc = sc.root.add(Disc("shield", (0.0, 0.0, focal_length + 1e-3), ROT3_UNITY))
        disc.set_radius(shield_radius)
    return sc.init()


def large_reflector_camera(focal_length=106.5, aperture_radius=35.5, davies_cotton=0.0,
                           facet_inner_hex_radius=0.45, gap=0.01, fov_deg=6.5,
                           pixel_fov_deg=0.06667, reflectivity=0.9) -> Scenery:
    """A large parabolic segmented reflector (hexagonal spherical-cap facets
    of curvature radius 2f = 213 m) with a flat camera of hexagonal pixels
    in its focal plane.  The pixel grid is the one merlict_portal_plenoscope
    lays out for its lens array (light_field_sensor/Geometry.cpp:13-77):
    spacing 2 f tan(pixel_fov/2) out to f tan(fov/2) -- 8,443 pixels for
    the default 0.06667 degree pixels and 6.5 degree field of view.  With
    0.9 m facets the reflector layout yields 5,388 facets on the 35.5 m
    aperture."""
    sc = Scenery()
    reflector = sc.root.add(SurfaceEntity("reflector", (0.0, 0.0, 0.0), ROT3_UNITY))
    reflector.outer_reflection = constant(reflectivity)
    segmented_reflector(reflector, ReflectorConfig(
        focal_length, davies_cotton, aperture_radius, 0.0, facet_inner_hex_radius, gap))
    inner = focal_length * math.tan(deg2rad(pixel_fov_deg) / 2.0)
    outer = inner * 2.0 / math.sqrt(3.0)
    max_radius = focal_length * math.tan(deg2rad(fov_deg) / 2.0)
    cells = hex_grid_annulus(max_radius - outer, 0.0, 2.0 * inner)
    cam = sc.root.add(Frame("camera", (0.0, 0.0, focal_length), ROT3_UNITY))
    for i, pos in enumerate(cells):
        pix = cam.add(HexPlane(f"pixel_{i}", pos, ROT3_UNITY))
        pix.set_outer_hex_radius(outer)
        sc.add_sensor(i, pix)
    return sc.init()


def light_field_telescope(focal_length=10.7, aperture_radius=5.35, fov_deg=6.5,
                          pixel_fov_deg=0.186, paxels_on_diagonal=9, housing_overhead=1.1,
                          reflectivity=0.9, davies_cotton=1.0, facet_inner_hex_radius=0.3,
                          gap=0.01) -> Scenery:
    """A segmented reflector with a light-field sensor in its focal plane;
    the lens refractive index falls from 1.52 at 200 nm to 1.46 at 1200 nm
    (1.50 at 300 nm, 1.47 at 700 nm)."""
    sc = Scenery()
    refl = constant(reflectivity)
    n_lens = Func1([[200e-9, 1.52], [300e-9, 1.50], [700e-9, 1.47], [1200e-9, 1.46]])
    reflector = sc.root.add(SurfaceEntity("reflector", (0.0, 0.0, 0.0), ROT3_UNITY))
    reflector.outer_reflection = refl
    segmented_reflector(reflector, ReflectorConfig(
        focal_length, davies_cotton, aperture_radius, 0.0, facet_inner_hex_radius, gap))
    cfg = LightFieldSensorConfig(
        expected_imaging_system_focal_length=focal_length,
        expected_imaging_system_max_aperture_radius=aperture_radius,
        max_FoV_diameter=deg2rad(fov_deg), pixel_FoV_hex_flat2flat=deg2rad(pixel_fov_deg),
        num_paxel_on_pixel_diagonal=paxels_on_diagonal, housing_overhead=housing_overhead,
        lens_refraction=n_lens, bin_reflection=refl)
    lfs = sc.root.add(Frame("light_field_sensor", (0.0, 0.0, focal_length), ROT3_UNITY))
    light_field_sensor(lfs, sc, cfg)
    return sc.init()
