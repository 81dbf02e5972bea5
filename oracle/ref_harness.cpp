// ref_harness.cpp -- TEST INFRASTRUCTURE, not product code.
//
// C entry points around the unmodified reference library (compiled from the
// reference sources by oracle/Makefile) for the parity tests, the golden
// fixture generator and the CPU baseline of the bench:
//
//  * ref_scene_build  builds a scene with the reference's own classes and
//    factories (segmented_imaging_reflector::Factory, light_field_sensor::
//    Factory, the test benches of merlict/tests/PhotonTest.cpp and
//    BiConvexLensTest.cpp) and runs Frame::init_tree_based_on_mother_child_
//    relations;
//  * ref_scene_flat   flattens it with merlict_b200::flatten (the product's
//    drop-in shim) into the layout of include/merlict_b200.h;
//  * ref_propagate    runs merlict's Propagator on given photons, either
//    photon by photon with a random::Generator that replays the engine's
//    Philox stream (or an explicit uniform stream), exactly as
//    merlict_multi_thread.cpp:12-26 drives it, or through the reference's
//    own propagate_photons_in_frame_with_config[_multi_thread] with its
//    Mt19937; then Sensors::assign_photons.  Per-photon results and
//    histories are read back through merlict's public accessors.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "merlict/merlict.h"
#include "merlict/scenery/segmented_imaging_reflector/segmented_imaging_reflector.h"
#include "merlict_corsika/PhotonFactory.h"
#include "merlict_corsika/event_tape.h"
#include "merlict_corsika/eventio.h"
#include "merlict_portal_plenoscope/calibration/LixelStatisticsFiller.h"
#include "merlict_multi_thread/merlict_multi_thread.h"
#include "merlict_portal_plenoscope/light_field_sensor/LightFieldSensor.h"
#include "merlict_json/json.h"
#include "merlict_portal_plenoscope/json_to_plenoscope.h"
#include "merlict_portal_plenoscope/PlenoscopeScenery.h"
#include "merlict_portal_plenoscope/night_sky_background/NightSkyBackground.h"
#include "merlict_signal_processing/PhotoElectricConverter.h"
#include "merlict_signal_processing/PhotonStream.h"
#include "merlict_signal_processing/PipelinePhoton.h"
#include "merlict_signal_processing/pulse_extraction.h"
#include "merlict_b200.h"
#include "merlict_b200_philox.h"
#include "merlict_b200_shim.h"

namespace ml = merlict;

namespace {

thread_local std::string last_error;

struct Handle {
    plenoscope::PlenoscopeScenery scenery;
    std::vector<ml::sensor::Sensor*> owned_sensors;
    ml::sensor::Sensors sensors;
    merlict_b200::FlatScene flat;
    bool flattened = false;
    std::vector<double> last_support;   // ray supports after the last propagation
    std::vector<std::unique_ptr<plenoscope::light_field_sensor::Geometry>> geometries;
    std::vector<std::unique_ptr<ml::function::Func1>> functions;
    const ml::function::Func1* fn(std::vector<std::vector<double>> xy) {
        functions.emplace_back(new ml::function::Func1(xy));
        return functions.back().get();
    }
    ~Handle() {
        for (ml::sensor::Sensor* s : owned_sensors) delete s;
    }
};

double param(const double* p, int n, int k, double fallback) {
    return k < n ? p[k] : fallback;
}

// ---- test benches of merlict/tests/PhotonTest.cpp ------------------------

void build_two_mirrors(Handle* h) {  // PhotonTest.cpp:27-82
    ml::Frame* table = h->scenery.root.add<ml::Plane>();
    table->set_name_pos_rot("optical_table", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    const ml::function::Func1* refl = h->fn({{200e-9, 1}, {1200e-9, 1}});
    ml::Plane* m1 = table->add<ml::Plane>();
    m1->set_name_pos_rot("mirror_1", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    m1->outer_reflection = refl; m1->inner_reflection = refl;
    m1->set_x_y_width(1.0, 1.0);
    ml::Plane* m2 = table->add<ml::Plane>();
    m2->set_name_pos_rot("mirror_2", ml::Vec3(0.0, 0.0, 1.0), ml::ROT3_UNITY);
    m2->outer_reflection = refl; m2->inner_reflection = refl;
    m2->set_x_y_width(1.0, 1.0);
}

void build_mirror_absorber(Handle* h) {  // PhotonTest.cpp:84-175
    ml::Frame* table = h->scenery.root.add<ml::Plane>();
    table->set_name_pos_rot("optical_table", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    const ml::function::Func1* refl = h->fn({{200e-9, 0.42}, {1200e-9, 0.42}});
    ml::Plane* mirror = table->add<ml::Plane>();
    mirror->set_name_pos_rot("mirror", ml::VEC3_ORIGIN,
                             ml::Rot3(0, ml::deg2rad(90), ml::deg2rad(45)));
    mirror->outer_reflection = refl; mirror->inner_reflection = refl;
    mirror->set_x_y_width(1.0, 1.0);
    ml::Plane* absorber = table->add<ml::Plane>();
    absorber->set_name_pos_rot("absorber", ml::Vec3(0, 2, 0), ml::Rot3(ml::deg2rad(90), 0, 0));
    absorber->set_x_y_width(1.0, 1.0);
    h->owned_sensors.push_back(new ml::sensor::Sensor(0, absorber));
}

void build_water_box(Handle* h, bool absorbing) {  // PhotonTest.cpp:177-302
    const ml::function::Func1* water = h->fn({{200e-9, 1.33}, {1200e-9, 1.33}});
    ml::RectangularBox* box = h->scenery.root.add<ml::RectangularBox>();
    box->set_name_pos_rot("box", ml::Vec3(0.0, 0.0, 1.0), ml::Rot3(0.0, 0.0, 0.0));
    if (absorbing) box->inner_absorption = h->fn({{200e-9, 1.0}, {1200e-9, 1.0}});
    box->inner_refraction = water;
    box->set_xyz_width(1.0, 1.0, 1.0);
    ml::Plane* absorber = h->scenery.root.add<ml::Plane>();
    absorber->set_name_pos_rot("absorber", ml::Vec3(0.0, 0.0, 3.0), ml::ROT3_UNITY);
    absorber->set_x_y_width(1.0, 1.0);
    h->owned_sensors.push_back(new ml::sensor::Sensor(0, absorber));
}

void build_biconvex_lens(Handle* h) {  // BiConvexLensTest.cpp:8-82
    ml::Frame* bench = h->scenery.root.add<ml::Frame>();
    bench->set_name_pos_rot("BiConvexLens_test_world", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    ml::lens_maker::Config cfg;
    cfg.focal_length = 1.0;
    cfg.aperture_radius = 0.125;
    cfg.refractive_index = 1.49;
    ml::BiConvexLens* lens = bench->add<ml::BiConvexLens>();
    lens->set_name_pos_rot("little_lens", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    lens->inner_refraction = h->fn({{200e-9, 1.49}, {1200e-9, 1.49}});
    lens->set_curvature_radius_and_aperture_radius(
        ml::lens_maker::get_curvature_radius(cfg), cfg.aperture_radius);
    ml::Disc* sensor = bench->add<ml::Disc>();
    sensor->set_name_pos_rot("sensor_disc", ml::Vec3(0.0, 0.0, -1.0), ml::ROT3_UNITY);
    sensor->set_radius(cfg.aperture_radius);
    h->owned_sensors.push_back(new ml::sensor::Sensor(0, sensor));
}

void build_sphere(Handle* h) {  // SphereIntersectionTest.cpp:6-33
    ml::Sphere* s = h->scenery.root.add<ml::Sphere>();
    s->set_name_pos_rot("my_sphere", ml::Vec3(0, 0, 0), ml::Rot3(0, 0, 0));
    s->set_radius(1.0);
}

// One leaf of every primitive kind, in several poses, with mirrors, glass,
// absorbers, an absorbing medium and sensors; more than 16 children at the
// root so that octant clustering (Frame.cpp:190-255) is exercised.
void build_primitive_zoo(Handle* h) {
    const ml::function::Func1* mirror = h->fn({{200e-9, 0.8}, {400e-9, 0.9}, {1200e-9, 0.7}});
    const ml::function::Func1* half = h->fn({{200e-9, 0.5}, {1200e-9, 0.5}});
    const ml::function::Func1* glass = h->fn({{200e-9, 1.52}, {500e-9, 1.49}, {1200e-9, 1.46}});
    const ml::function::Func1* water = h->fn({{200e-9, 1.33}, {1200e-9, 1.33}});
    const ml::function::Func1* murky = h->fn({{200e-9, 0.7}, {1200e-9, 2.0}});
    ml::Frame& root = h->scenery.root;
    unsigned sensor_id = 0;
    auto sense = [&](const ml::Frame* f) {
        h->owned_sensors.push_back(new ml::sensor::Sensor(sensor_id++, f));
    };
    const double deg = M_PI/180.0;

    ml::Annulus* annulus = root.add<ml::Annulus>();
    annulus->set_name_pos_rot("annulus", ml::Vec3(1.5, 0.2, -0.3), ml::Rot3(0.3, -0.2, 0.1));
    annulus->set_outer_inner_radius(0.6, 0.25);
    annulus->outer_reflection = mirror;
    sense(annulus);

    ml::BiConvexLensHexBound* lens = root.add<ml::BiConvexLensHexBound>();
    lens->set_name_pos_rot("hexlens", ml::Vec3(-1.2, 0.8, 0.4), ml::Rot3(10*deg, 5*deg, 0.0));
    lens->inner_refraction = glass;
    lens->set_curvature_radius_and_outer_hex_radius(1.2, 0.45);

    ml::BiConvexLens* lens2 = root.add<ml::BiConvexLens>();
    lens2->set_name_pos_rot("roundlens", ml::Vec3(0.2, -1.5, 0.9), ml::Rot3(-20*deg, 0.0, 30*deg));
    lens2->inner_refraction = glass;
    lens2->set_curvature_radius_and_aperture_radius(0.9, 0.35);

    ml::Cylinder* cyl = root.add<ml::Cylinder>();
    cyl->set_name_pos_rot("cylinder", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    cyl->set_cylinder(0.3, ml::Vec3(-0.5, -0.4, -1.2), ml::Vec3(0.6, 0.2, -0.6));
    cyl->inner_reflection = half;
    cyl->outer_reflection = mirror;

    ml::Disc* disc = root.add<ml::Disc>();
    disc->set_name_pos_rot("disc", ml::Vec3(0.0, 0.0, 2.2), ml::Rot3(0.0, 15*deg, 0.0));
    disc->set_radius(0.7);
    sense(disc);

    ml::EllipticalCapWithHexagonalBound* ell = root.add<ml::EllipticalCapWithHexagonalBound>();
    ell->set_name_pos_rot("ellipse", ml::Vec3(0.9, 1.3, -1.4), ml::Rot3(0.1, 0.2, 0.3));
    ell->set_focalLength_radiiRatio_hexAngel_hexRadius(3.0, 1.2, 0.0, 0.5);
    ell->outer_reflection = mirror;

    ml::HexPlane* hex = root.add<ml::HexPlane>();
    hex->set_name_pos_rot("hexplane", ml::Vec3(-1.6, -1.0, -0.8), ml::Rot3(0.0, 0.0, 30*deg));
    hex->set_outer_hex_radius(0.5);
    sense(hex);

    ml::Plane* plane = root.add<ml::Plane>();
    plane->set_name_pos_rot("plane", ml::Vec3(0.5, 0.5, 3.0), ml::Rot3(5*deg, -7*deg, 0.0));
    plane->set_x_y_width(2.5, 1.5);
    plane->inner_reflection = half;
    sense(plane);

    ml::PlaneDualSphericalBound* dual = root.add<ml::PlaneDualSphericalBound>();
    dual->set_name_pos_rot("dualsphere", ml::Vec3(1.8, -1.2, 0.5), ml::Rot3(M_PI*0.5, M_PI*0.5, 0.4));
    dual->set_x_hight_and_y_width(0.3, 0.6);
    dual->outer_reflection = half;

    ml::RectangularBox* box = root.add<ml::RectangularBox>();
    box->set_name_pos_rot("waterbox", ml::Vec3(-0.4, 1.8, -0.2), ml::Rot3(0.2, 0.1, -0.3));
    box->inner_refraction = water;
    box->inner_absorption = murky;
    box->set_xyz_width(0.6, 0.5, 0.4);

    ml::Sphere* sphere = root.add<ml::Sphere>();
    sphere->set_name_pos_rot("sphere", ml::Vec3(0.0, 0.0, 0.0), ml::ROT3_UNITY);
    sphere->set_radius(0.35);
    sphere->inner_refraction = glass;

    ml::SphereCapWithCylinderBound* capc = root.add<ml::SphereCapWithCylinderBound>();
    capc->set_name_pos_rot("cap_cyl", ml::Vec3(-0.3, -0.2, -2.2), ml::Rot3(0.05, -0.04, 0.0));
    capc->set_curvature_radius_and_outer_radius(3.0, 0.8);
    capc->outer_reflection = mirror;

    ml::SphereCapWithHexagonalBound* caph = root.add<ml::SphereCapWithHexagonalBound>();
    caph->set_name_pos_rot("cap_hex", ml::Vec3(1.4, -0.6, -2.0), ml::Rot3(0.0, 0.1, 0.2));
    caph->set_curvature_radius_and_outer_hex_radius(4.0, 0.6);
    caph->outer_reflection = mirror;
    caph->inner_reflection = half;

    ml::SphereCapWithRectangularBound* capr = root.add<ml::SphereCapWithRectangularBound>();
    capr->set_name_pos_rot("cap_rect", ml::Vec3(-1.5, 0.3, -1.9), ml::Rot3(-0.1, 0.0, 0.0));
    capr->set_curvature_radius_and_x_y_width(2.5, 0.9, 0.6);
    capr->outer_reflection = mirror;

    ml::Triangle* tri = root.add<ml::Triangle>();
    tri->set_name_pos_rot("triangle", ml::Vec3(0.0, -1.0, 1.6), ml::Rot3(0.4, 0.0, 0.0));
    tri->set_corners_in_xy_plane(-0.5, -0.3, 0.6, -0.2, 0.1, 0.7);
    sense(tri);

    ml::Triangle* tri2 = root.add<ml::Triangle>();
    tri2->set_name_pos_rot("triangle_n", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    tri2->set_normal_and_3_vertecies(
        ml::Vec3(0.3, 0.2, 1.0),
        ml::Vec3(1.2, 1.1, 1.4), ml::Vec3(1.9, 1.0, 1.3), ml::Vec3(1.5, 1.7, 1.2));
    tri2->outer_reflection = half;

    ml::Frame* empty = root.add<ml::Frame>();
    empty->set_name_pos_rot("empty_frame", ml::Vec3(0.3, 0.3, 0.3), ml::ROT3_UNITY);

    // a small grid of hexagonal pixels as a nested frame
    ml::Frame* cam = root.add<ml::Frame>();
    cam->set_name_pos_rot("camera", ml::Vec3(0.0, 0.0, -2.9), ml::Rot3(0.0, 0.0, 0.1));
    ml::HexGridAnnulus grid(0.9, 0.25);
    const std::vector<ml::Vec3> cells = grid.get_grid();
    for (size_t i = 0; i < cells.size(); i++) {
        ml::HexPlane* pix = cam->add<ml::HexPlane>();
        pix->set_name_pos_rot("pixel_" + std::to_string(i), cells[i], ml::ROT3_UNITY);
        pix->set_outer_hex_radius(0.25/std::sqrt(3.0));
        sense(pix);
    }
}

// ---- optical systems of the benchmark configurations ---------------------

// Segmented imaging reflector (segmented_imaging_reflector::Factory) and a
// flat camera of hexagonal pixels at the focal plane, plus an optional
// shield disc just above the camera.
// p: f, DC mixing, max aperture radius, min aperture radius, facet inner
//    hex radius, gap, reflectivity, number of pixels, pixel flat-to-flat,
//    shield radius (0: none)
void build_reflector_camera(Handle* h, const double* p, int n) {
    const double f = param(p, n, 0, 4.9);
    ml::segmented_imaging_reflector::Config c;
    c.focal_length = f;
    c.DaviesCotton_over_parabolic_mixing_factor = param(p, n, 1, 1.0);
    c.max_outer_aperture_radius = param(p, n, 2, 2.1);
    c.min_inner_aperture_radius = param(p, n, 3, 0.0);
    c.facet_inner_hex_radius = param(p, n, 4, 0.3);
    c.gap_between_facets = param(p, n, 5, 0.01);
    const double reflectivity = param(p, n, 6, 0.9);
    const unsigned num_pixels = static_cast<unsigned>(param(p, n, 7, 1440));
    const double pixel_f2f = param(p, n, 8, 0.0095);
    const double shield = param(p, n, 9, 0.0);

    ml::SurfaceEntity* reflector = h->scenery.root.add<ml::SurfaceEntity>();
    reflector->set_name_pos_rot("reflector", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    reflector->outer_reflection = h->fn({{200e-9, reflectivity}, {1200e-9, reflectivity}});
    ml::segmented_imaging_reflector::Factory fab(c);
    fab.add_to_SurfaceEntity(reflector);

    ml::Frame* cam = h->scenery.root.add<ml::Frame>();
    cam->set_name_pos_rot("camera", ml::Vec3(0.0, 0.0, f), ml::ROT3_UNITY);
    // pixel centres: the hexagonal grid closest to the optical axis
    const double grid_radius = pixel_f2f*(std::sqrt(static_cast<double>(num_pixels)) + 2.0);
    ml::HexGridAnnulus grid(grid_radius, pixel_f2f);
    std::vector<ml::Vec3> cells = grid.get_grid();
    std::vector<size_t> order(cells.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return cells[a].norm() < cells[b].norm();
    });
    if (order.size() < num_pixels) throw std::runtime_error("pixel grid too small");
    for (unsigned i = 0; i < num_pixels; i++) {
        ml::HexPlane* pix = cam->add<ml::HexPlane>();
        // unrotated: the hexagons' flat sides face the grid's neighbours, so
        // the pixels tile the focal plane without overlap
        pix->set_name_pos_rot("pixel_" + std::to_string(i), cells[order[i]], ml::ROT3_UNITY);
        pix->set_outer_hex_radius(pixel_f2f/std::sqrt(3.0));
        h->owned_sensors.push_back(new ml::sensor::Sensor(i, pix));
    }
    if (shield > 0.0) {
        ml::Disc* disc = h->scenery.root.add<ml::Disc>();
        disc->set_name_pos_rot("shield", ml::Vec3(0.0, 0.0, f + 1e-3), ml::ROT3_UNITY);
        disc->set_radius(shield);
    }
}

// A large parabolic segmented reflector with a flat camera of hexagonal
// pixels in its focal plane; the pixel grid is the one
// light_field_sensor/Geometry.cpp:13-77 lays out for its lens array
// (spacing 2 f tan(pixel FoV / 2) out to f tan(FoV / 2)).
// p: f, max aperture radius, DC mixing, facet inner hex radius, gap, FoV
//    diameter [deg], pixel FoV [deg], reflectivity
void build_large_reflector(Handle* h, const double* p, int n) {
    const double f = param(p, n, 0, 106.5);
    ml::segmented_imaging_reflector::Config c;
    c.focal_length = f;
    c.DaviesCotton_over_parabolic_mixing_factor = param(p, n, 2, 0.0);
    c.max_outer_aperture_radius = param(p, n, 1, 35.5);
    c.min_inner_aperture_radius = 0.0;
    c.facet_inner_hex_radius = param(p, n, 3, 0.45);
    c.gap_between_facets = param(p, n, 4, 0.01);
    const double fov = ml::deg2rad(param(p, n, 5, 6.5));
    const double pixel_fov = ml::deg2rad(param(p, n, 6, 0.06667));
    const double reflectivity = param(p, n, 7, 0.9);

    ml::SurfaceEntity* reflector = h->scenery.root.add<ml::SurfaceEntity>();
    reflector->set_name_pos_rot("reflector", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    reflector->outer_reflection = h->fn({{200e-9, reflectivity}, {1200e-9, reflectivity}});
    ml::segmented_imaging_reflector::Factory fab(c);
    fab.add_to_SurfaceEntity(reflector);

    const double inner = f*std::tan(pixel_fov/2.0);
    const double outer = inner*2.0/std::sqrt(3.0);
    const double max_radius = f*std::tan(fov/2.0);
    ml::HexGridAnnulus grid(max_radius - outer, 0.0, 2.0*inner);
    const std::vector<ml::Vec3> cells = grid.get_grid();
    ml::Frame* cam = h->scenery.root.add<ml::Frame>();
    cam->set_name_pos_rot("camera", ml::Vec3(0.0, 0.0, f), ml::ROT3_UNITY);
    for (size_t i = 0; i < cells.size(); i++) {
        ml::HexPlane* pix = cam->add<ml::HexPlane>();
        pix->set_name_pos_rot("pixel_" + std::to_string(i), cells[i], ml::ROT3_UNITY);
        pix->set_outer_hex_radius(outer);
        h->owned_sensors.push_back(new ml::sensor::Sensor(static_cast<unsigned>(i), pix));
    }
}

// Segmented reflector plus the light-field sensor of
// merlict_portal_plenoscope/light_field_sensor/Factory.cpp:235-249 at the
// focal plane.
// p: f, max aperture radius, FoV diameter [deg], pixel FoV [deg], paxels on
//    the pixel diagonal, housing overhead, reflectivity, DC mixing, facet
//    inner hex radius, gap
void build_light_field_sensor(Handle* h, const double* p, int n) {
    const double f = param(p, n, 0, 10.7);
    const double R = param(p, n, 1, 5.35);
    ml::segmented_imaging_reflector::Config c;
    c.focal_length = f;
    c.DaviesCotton_over_parabolic_mixing_factor = param(p, n, 7, 1.0);
    c.max_outer_aperture_radius = R;
    c.min_inner_aperture_radius = 0.0;
    c.facet_inner_hex_radius = param(p, n, 8, 0.3);
    c.gap_between_facets = param(p, n, 9, 0.01);
    const double reflectivity = param(p, n, 6, 0.9);
    const ml::function::Func1* refl = h->fn({{200e-9, reflectivity}, {1200e-9, reflectivity}});
    const ml::function::Func1* n_lens =
        h->fn({{200e-9, 1.52}, {300e-9, 1.50}, {700e-9, 1.47}, {1200e-9, 1.46}});

    ml::SurfaceEntity* reflector = h->scenery.root.add<ml::SurfaceEntity>();
    reflector->set_name_pos_rot("reflector", ml::VEC3_ORIGIN, ml::ROT3_UNITY);
    reflector->outer_reflection = refl;
    ml::segmented_imaging_reflector::Factory fab(c);
    fab.add_to_SurfaceEntity(reflector);

    plenoscope::light_field_sensor::Config lc;
    lc.expected_imaging_system_focal_length = f;
    lc.expected_imaging_system_max_aperture_radius = R;
    lc.max_FoV_diameter = ml::deg2rad(param(p, n, 2, 6.5));
    lc.pixel_FoV_hex_flat2flat = ml::deg2rad(param(p, n, 3, 0.186));
    lc.num_paxel_on_pixel_diagonal = static_cast<unsigned>(param(p, n, 4, 9));
    lc.housing_overhead = param(p, n, 5, 1.1);
    lc.lens_refraction = n_lens;
    lc.bin_reflection = refl;
    h->geometries.emplace_back(new plenoscope::light_field_sensor::Geometry(lc));
    plenoscope::light_field_sensor::Geometry* geometry = h->geometries.back().get();
    ml::Frame* lfs = h->scenery.root.add<ml::Frame>();
    lfs->set_name_pos_rot("light_field_sensor", ml::Vec3(0, 0, f), ml::ROT3_UNITY);
    plenoscope::light_field_sensor::Factory factory(geometry);
    factory.add_light_field_sensor_to_frame_in_scenery(lfs, &h->scenery);
    ml::sensor::Sensors* lixels = factory.get_sub_pixels();
    for (ml::sensor::Sensor* s : lixels->by_occurence) h->owned_sensors.push_back(s);
    delete lixels;   // the Sensor objects are kept in owned_sensors
}

// ---- a random::Generator that replays a given stream ---------------------

class ReplayGenerator : public ml::random::Generator {
 public:
    int mode = 0;               // 0: Philox stream, 1: explicit uniforms
    uint64_t philox_seed = 0;
    uint64_t stream = 0;
    const double* uniforms = nullptr;
    uint32_t stride = 0;
    uint32_t used = 0;
    bool exhausted = false;
    double uniform() override {
        const uint32_t k = used++;
        if (mode == 0) return mlgpu_philox_uniform(philox_seed, stream, k);
        if (k >= stride) { exhausted = true; return 0.5; }
        return uniforms[static_cast<size_t>(stream)*stride + k];
    }
    uint64_t create_seed() override { return 0; }
    double normal(const double mean, const double std_dev) override {
        (void)std_dev; return mean;
    }
};

template <typename Tag, typename Tag::type Member>
struct Accessor { friend typename Tag::type member_of(Tag) { return Member; } };
struct InteractionHistory {
    typedef std::vector<ml::Interaction> ml::RayForPropagation::*type;
    friend type member_of(InteractionHistory);
};
template struct Accessor<InteractionHistory, &ml::RayForPropagation::interaction_history>;

// The reference's photons for a batch of host planes (FP64), photon i with
// simulation_truth_id i.
std::vector<ml::Photon> make_photons(const mlgpu_photons* ph, uint64_t n) {
    std::vector<ml::Photon> photons;
    photons.reserve(n);
    for (uint64_t i = 0; i < n; i++) {
        const ml::Vec3 s(((const double*)ph->support_x)[i], ((const double*)ph->support_y)[i],
                         ((const double*)ph->support_z)[i]);
        const ml::Vec3 d(((const double*)ph->direction_x)[i], ((const double*)ph->direction_y)[i],
                         ((const double*)ph->direction_z)[i]);
        ml::Photon p(s, d, ((const double*)ph->wavelength)[i]);
        p.simulation_truth_id = static_cast<int32_t>(i);
        photons.push_back(p);
    }
    return photons;
}

// The ray support each photon holds after propagation (ref_last_supports).
void keep_supports(Handle* h, const std::vector<ml::Photon>& photons) {
    h->last_support.resize(3*photons.size());
    for (size_t i = 0; i < photons.size(); i++) {
        const ml::Vec3 s = photons[i].support();
        h->last_support[3*i] = s.x;
        h->last_support[3*i + 1] = s.y;
        h->last_support[3*i + 2] = s.z;
    }
}

// Per-photon results of propagated photons whose arrivals the scene's
// sensors hold (after Sensors::assign_photons), read through merlict's
// public accessors; used[i] = uniforms photon i drew (0 when unknown).
void write_results(Handle* h, const std::vector<ml::Photon>& photons,
                   const std::vector<uint32_t>& used, uint32_t max_interactions,
                   mlgpu_results* out) {
    const uint64_t n = photons.size();
    const merlict_b200::FlatScene* flat = nullptr;
    if (!h->flattened) {
        h->flat = merlict_b200::flatten(&h->scenery.root, &h->sensors);
        h->flattened = true;
    }
    flat = &h->flat;
    std::map<const ml::Frame*, int32_t> leaf_of;
    for (size_t l = 0; l < flat->leaf_node.size(); l++)
        leaf_of[flat->node_frame[flat->leaf_node[l]]] = static_cast<int32_t>(l);
    auto leaf_id = [&](const ml::SurfaceEntity* o) -> int32_t {
        if (o == &ml::VOID_SURFACE_ENTITY) return MLGPU_LEAF_VOID;
        auto it = leaf_of.find(o);
        return it == leaf_of.end() ? MLGPU_LEAF_PHOTON_SOURCE : it->second;
    };
    // arrivals by photon id (simulation_truth_id == photon index)
    std::vector<int32_t> sensor_of(n, -1);
    std::vector<const ml::sensor::PhotonArrival*> arrival_of(n, nullptr);
    for (size_t s = 0; s < h->sensors.by_occurence.size(); s++)
        for (const ml::sensor::PhotonArrival& a : h->sensors.by_occurence[s]->photon_arrival_history) {
            sensor_of[a.simulation_truth_id] = static_cast<int32_t>(s);
            arrival_of[a.simulation_truth_id] = &a;
        }
    const uint32_t len = max_interactions + 1;
    for (uint64_t i = 0; i < n; i++) {
        const ml::Photon& p = photons[i];
        const ml::Intersection& fin = p.final_intersection();
        const int32_t leaf = p.num_interactions() > 1 ? leaf_id(fin.object())
                                                      : MLGPU_LEAF_PHOTON_SOURCE;
        out->sensor[i] = sensor_of[i];
        double x = fin.position_in_object_frame().x;
        double y = fin.position_in_object_frame().y;
        double t, tx, ty;
        if (arrival_of[i]) {
            t = arrival_of[i]->arrival_time;
            tx = arrival_of[i]->theta_x;
            ty = arrival_of[i]->theta_y;
            x = arrival_of[i]->x_intersect;
            y = arrival_of[i]->y_intersect;
        } else {
            // merlict evaluates the time of flight only for photons given
            // to a sensor (Sensor.cpp:14-30).  For a photon that ended in
            // the void it would dereference the refraction table of
            // VOID_SURFACE_ENTITY, which is built before the default
            // tables in SurfaceEntity.cpp:9-27 and holds null pointers.
            t = NAN;
            const ml::Vec3 inc = p.final_intersection_incident_direction_wrt_frame();
            tx = -1.0*inc.x; ty = -1.0*inc.y;
        }
        if (out->x) ((double*)out->x)[i] = x;
        if (out->y) ((double*)out->y)[i] = y;
        if (out->time) out->time[i] = t;
        if (out->theta_x) ((double*)out->theta_x)[i] = tx;
        if (out->theta_y) ((double*)out->theta_y)[i] = ty;
        if (out->final_leaf) out->final_leaf[i] = leaf;
        if (out->info) {
            const uint32_t u = used[i] > 255 ? 255 : used[i];
            out->info[i] = static_cast<uint32_t>(p.final_interaction()) |
                (p.num_interactions() << 8) | (u << 16);
        }
        if (out->final_position) {
            const ml::Vec3 w = fin.position_in_root_frame();
            out->final_position[3*i] = w.x;
            out->final_position[3*i + 1] = w.y;
            out->final_position[3*i + 2] = w.z;
        }
        if (out->final_direction) {
            out->final_direction[3*i] = p.direction().x;
            out->final_direction[3*i + 1] = p.direction().y;
            out->final_direction[3*i + 2] = p.direction().z;
        }
        if (out->history) {
            const std::vector<ml::Interaction>& kinds = p.*member_of(InteractionHistory());
            for (uint32_t k = 0; k < len; k++) {
                mlgpu_history_entry* e = &out->history[i*len + k];
                std::memset(e, 0, sizeof(*e));
                e->leaf = MLGPU_LEAF_PHOTON_SOURCE;
                if (k >= p.num_interactions()) continue;
                const ml::Intersection& is = p.intersection_at(k);
                const ml::Vec3 pos = is.position_in_object_frame();
                const ml::Vec3 nrm = is.surface_normal_in_object_frame();
                e->position[0] = pos.x; e->position[1] = pos.y; e->position[2] = pos.z;
                e->normal[0] = nrm.x; e->normal[1] = nrm.y; e->normal[2] = nrm.z;
                e->distance = is.distance_to_ray_support();
                e->leaf = k == 0 ? MLGPU_LEAF_PHOTON_SOURCE : leaf_id(is.object());
                e->interaction = static_cast<uint8_t>(kinds[k]);
                e->from_outside_to_inside = is.from_outside_to_inside() ? 1 : 0;
            }
        }
    }
}

}  // namespace

extern "C" {

const char* ref_last_error(void) { return last_error.c_str(); }

void* ref_scene_build(const char* kind, const double* params, int num_params) {
    try {
        std::unique_ptr<Handle> h(new Handle);
        const std::string k(kind);
        if (k == "two_mirrors") build_two_mirrors(h.get());
        else if (k == "mirror_absorber") build_mirror_absorber(h.get());
        else if (k == "water_box") build_water_box(h.get(), false);
        else if (k == "absorbing_box") build_water_box(h.get(), true);
        else if (k == "biconvex_lens") build_biconvex_lens(h.get());
        else if (k == "sphere") build_sphere(h.get());
        else if (k == "primitive_zoo") build_primitive_zoo(h.get());
        else if (k == "reflector_camera") build_reflector_camera(h.get(), params, num_params);
        else if (k == "light_field_sensor") build_light_field_sensor(h.get(), params, num_params);
        else if (k == "large_reflector") build_large_reflector(h.get(), params, num_params);
        else throw std::invalid_argument("unknown scene kind '" + k + "'");
        h->sensors.init(h->owned_sensors);
        h->scenery.root.init_tree_based_on_mother_child_relations();
        return h.release();
    } catch (const std::exception& e) {
        last_error = e.what();
        return nullptr;
    }
}

void ref_scene_free(void* handle) { delete static_cast<Handle*>(handle); }

int ref_scene_flat(void* handle, mlgpu_flat_scene* out) {
    Handle* h = static_cast<Handle*>(handle);
    try {
        if (!h->flattened) {
            h->flat = merlict_b200::flatten(&h->scenery.root, &h->sensors);
            h->flattened = true;
        }
        *out = h->flat.view();
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return 1;
    }
}

int ref_scene_num_sensors(void* handle) {
    return static_cast<int>(static_cast<Handle*>(handle)->sensors.size());
}

// mode 0: per-photon Propagator on the Philox stream (seed) -- "replay"
// mode 1: per-photon Propagator on explicit uniforms[n][stride]
// mode 2: reference propagate_photons_in_frame_with_config, Mt19937(seed)
// mode 3: reference ..._multi_thread, Mt19937(seed) seeding per photon
// Results are written to `out` (host pointers, double precision); the time
// of propagate + Sensors::assign_photons goes to *seconds.
int ref_propagate(void* handle, const mlgpu_photons* ph, uint64_t n,
                  uint32_t max_interactions, int mode, uint64_t seed,
                  const double* uniforms, uint32_t stride, int num_threads,
                  mlgpu_results* out, double* seconds) {
    Handle* h = static_cast<Handle*>(handle);
    try {
        std::vector<ml::Photon> photons = make_photons(ph, n);
        ml::PropagationConfig cfg;
        cfg.max_num_interactions_per_photon = max_interactions;
        std::vector<uint32_t> used(n, 0);
        h->sensors.clear_history();

        const auto t0 = std::chrono::steady_clock::now();
        if (mode == 0 || mode == 1) {
            auto work = [&](uint64_t begin, uint64_t end) {
                for (uint64_t i = begin; i < end; i++) {
                    ReplayGenerator g;
                    g.mode = mode; g.philox_seed = seed; g.stream = i;
                    g.uniforms = uniforms; g.stride = stride;
                    ml::PropagationEnvironment env;
                    env.root_frame = &h->scenery.root;
                    env.config = &cfg;
                    env.prng = &g;
                    ml::Propagator(&photons[i], env);
                    used[i] = g.used;
                }
            };
            const int nt = num_threads > 1 ? num_threads : 1;
            std::vector<std::thread> pool;
            for (int t = 0; t < nt; t++)
                pool.emplace_back(work, n*t/nt, n*(t + 1)/nt);
            for (std::thread& t : pool) t.join();
        } else if (mode == 2) {
            ml::random::Mt19937 prng(seed);
            ml::propagate_photons_in_frame_with_config(&photons, &h->scenery.root, &cfg, &prng);
        } else if (mode == 3) {
            ml::random::Mt19937 prng(seed);
            ml::propagate_photons_in_frame_with_config_multi_thread(
                &photons, &h->scenery.root, &cfg, &prng);
        } else {
            throw std::invalid_argument("unknown mode");
        }
        h->sensors.assign_photons(&photons);
        const auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();

        keep_supports(h, photons);
        if (out) write_results(h, photons, used, max_interactions, out);
        return 0;
    } catch (const std::out_of_range& e) {
        last_error = e.what();
        return MLGPU_ERR_OUT_OF_RANGE;
    } catch (const std::invalid_argument& e) {
        last_error = e.what();
        return MLGPU_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MLGPU_ERR_RUNTIME;
    }
}

// merlict's EventIoPhotonFactory (merlict_corsika/PhotonFactory.cpp) on
// given bunches (8 floats each), bunch i drawing uniforms[i] for its
// weight's extra photon and getting id i.  Writes each photon's support,
// direction (as the Photon holds it), wavelength and id, in bunch order, up
// to `capacity` photons; *total = the number of photons made.
int ref_corsika_photons(const float* bunches, uint64_t n, const double* uniforms, double* sx,
                        double* sy, double* sz, double* dx, double* dy, double* dz, double* wl,
                        int32_t* ids, uint64_t capacity, uint64_t* total) {
    try {
        ReplayGenerator g;
        g.mode = 1;
        g.stride = 1;
        g.uniforms = uniforms;
        uint64_t k = 0;
        for (uint64_t i = 0; i < n; i++) {
            std::array<float, 8> row;
            for (int j = 0; j < 8; j++) row[j] = bunches[8*i + j];
            g.stream = i;
            g.used = 0;
            ml::EventIoPhotonFactory factory(row, static_cast<unsigned int>(i), &g);
            while (factory.has_still_photons_to_be_made()) {
                const ml::Photon p = factory.make_photon();
                if (k < capacity) {
                    const ml::Vec3 s = p.support(), d = p.direction();
                    sx[k] = s.x; sy[k] = s.y; sz[k] = s.z;
                    dx[k] = d.x; dy[k] = d.y; dz[k] = d.z;
                    wl[k] = p.wavelength;
                    ids[k] = p.simulation_truth_id;
                }
                k++;
            }
        }
        *total = k;
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MLGPU_ERR_INVALID_ARGUMENT;
    }
}

// plenoscope::calibration::LixelStatisticsFiller on given per-photon results
// (one block of n photons, in order): out[num_lixel][12] receives the
// LixelStatistic fields.  sensor < 0: the photon reached no sensor.
int ref_lixel_statistics(const int32_t* sensor, const float* cx, const float* cy, const float* x,
                         const float* y, const float* t, uint64_t n, uint64_t num_lixel,
                         uint64_t num_blocks, uint64_t photons_per_block, float* out) {
    try {
        std::vector<plenoscope::CalibrationPhotonResult> block(n);
        for (uint64_t i = 0; i < n; i++) {
            block[i].reached_sensor = sensor[i] >= 0;
            block[i].lixel_id = sensor[i] >= 0 ? static_cast<uint32_t>(sensor[i]) : 0u;
            block[i].x_tilt_vs_optical_axis = cx[i];
            block[i].y_tilt_vs_optical_axis = cy[i];
            block[i].x_pos_on_principal_aperture = x[i];
            block[i].y_pos_on_principal_aperture = y[i];
            block[i].time_of_flight = t[i];
        }
        plenoscope::calibration::LixelStatisticsFiller filler(num_lixel, num_blocks,
                                                              photons_per_block);
        filler.fill_in_block(block);
        const std::vector<plenoscope::calibration::LixelStatistic> st =
            filler.get_lixel_statistics();
        for (uint64_t l = 0; l < num_lixel; l++) {
            const plenoscope::calibration::LixelStatistic& a = st[l];
            const float v[12] = {a.efficiency, a.efficiency_std, a.cx_mean, a.cx_std, a.cy_mean,
                                 a.cy_std, a.x_mean, a.x_std, a.y_mean, a.y_std,
                                 a.time_delay_mean, a.time_delay_std};
            for (int k = 0; k < 12; k++) out[12*l + k] = v[k];
        }
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MLGPU_ERR_RUNTIME;
    }
}

// A scenery read by the reference's own JSON readers: merlict's
// (json.cpp:270-288; its sensors are the frames with a sensor_id, in the
// order read) or, with plenoscope != 0, the plenoscope extension
// (json_to_plenoscope.h:122-138; its sensors are the lixels of the one
// light-field sensor).
void* ref_scene_from_json(const char* path, int plenoscope) {
    try {
        std::unique_ptr<Handle> h(new Handle);
        if (plenoscope) {
            plenoscope::json::append_to_frame_in_scenery(&h->scenery.root, &h->scenery, path);
            if (h->scenery.plenoscopes.size() != 1)
                throw std::invalid_argument("expected exactly one plenoscope in the scenery");
            ml::sensor::Sensors* channels = h->scenery.plenoscopes.at(0).light_field_channels;
            for (ml::sensor::Sensor* s : channels->by_occurence) h->owned_sensors.push_back(s);
            delete channels;   // the Sensor objects are kept in owned_sensors
            h->scenery.plenoscopes.at(0).light_field_channels = nullptr;
            h->sensors.init(h->owned_sensors);
        } else {
            ml::json::append_to_frame_in_scenery(&h->scenery.root, &h->scenery, path);
            h->sensors.init(h->scenery.sensors.sensors);
        }
        h->scenery.root.init_tree_based_on_mother_child_relations();
        return h.release();
    } catch (const std::exception& e) {
        last_error = e.what();
        return nullptr;
    }
}

// The ids of the scene's sensors, by index.
int ref_scene_sensor_ids(void* handle, uint64_t* ids, int capacity) {
    Handle* h = static_cast<Handle*>(handle);
    const int n = static_cast<int>(h->sensors.by_occurence.size());
    for (int i = 0; i < n && i < capacity; i++) ids[i] = h->sensors.by_occurence[i]->id;
    return n;
}

// json::load_photons (json.cpp:543-562) as rows of photons2raw_matrix
// (id, support, direction, wavelength); returns the number of photons, or
// -1 on error.  Writes at most `capacity` rows.
int64_t ref_json_photons(const char* path, double* rows, uint64_t capacity) {
    try {
        std::vector<ml::Photon> photons = ml::json::load_photons(path);
        const std::vector<std::vector<double>> m = ml::photons2raw_matrix(&photons);
        for (uint64_t i = 0; i < m.size() && i < capacity; i++)
            for (int k = 0; k < 8; k++) rows[8*i + k] = m[i][k];
        return static_cast<int64_t>(m.size());
    } catch (const std::exception& e) {
        last_error = e.what();
        return -1;
    }
}

// raw_matrix2photons of tsvio::gen_table_from_file (merlict_tests/apps/
// propagate.cpp:63-64), back as raw rows.
int64_t ref_table_photons(const char* path, double* rows, uint64_t capacity) {
    try {
        std::vector<ml::Photon> photons =
            ml::raw_matrix2photons(ml::tsvio::gen_table_from_file(path));
        const std::vector<std::vector<double>> m = ml::photons2raw_matrix(&photons);
        for (uint64_t i = 0; i < m.size() && i < capacity; i++)
            for (int k = 0; k < 8; k++) rows[8*i + k] = m[i][k];
        return static_cast<int64_t>(m.size());
    } catch (const std::exception& e) {
        last_error = e.what();
        return -1;
    }
}

// json::load_PropagationConfig (json.cpp:510-517).
int ref_json_propagation_config(const char* path, uint64_t* max_num_interactions_per_photon) {
    try {
        const ml::PropagationConfig cfg = ml::json::load_PropagationConfig(path);
        *max_num_interactions_per_photon = cfg.max_num_interactions_per_photon;
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return 1;
    }
}

// merlict's Mt19937(seed).uniform(), n times (Mt19937.cpp:8-20).
void ref_mt19937_uniforms(uint64_t seed, uint64_t n, double* out) {
    ml::random::Mt19937 prng(seed);
    for (uint64_t i = 0; i < n; i++) out[i] = prng.uniform();
}

// ---- the signal chain after binning --------------------------------------
//
// ref_signal_chain runs merlict's own steps for one event, as
// plenoscope_propagation.cpp:201-247 chains them: get_photon_pipelines,
// night_sky_background::inject_nsb_into_photon_pipeline,
// PhotoElectricConverter::Converter per lixel and extract_pulses per lixel.
// mode 0 replays the engine's draw schedule (stage s of lixel i draws from
// Philox stream ((0xF0 | s) << 56) | (offset + i); the background stage
// moves on to the next lixel after 2 nsb_count[i] + 1 draws); mode 1 uses
// merlict's Mt19937(seed) for everything, in merlict's order.

namespace {

class SignalReplay : public ml::random::Generator {
 public:
    uint64_t key = 0, stream = 0, offset = 0;
    uint32_t k = 0;
    const uint32_t* budget_of = nullptr;   // background stage: draws per lixel
    uint64_t next_lixel = 0, left = 0;
    uint64_t stage = 0;

    static uint64_t stream_of(uint64_t stage, uint64_t offset, uint64_t lixel) {
        return ((0xF0ull | stage) << 56) | ((offset + lixel) & ((1ull << 56) - 1));
    }
    void select(uint64_t st, uint64_t lixel) {
        stage = st;
        stream = stream_of(st, offset, lixel);
        k = 0;
    }
    double uniform() override {
        if (budget_of) {
            while (left == 0) {
                select(stage, next_lixel);
                left = 2ull*budget_of[next_lixel] + 1ull;
                next_lixel++;
            }
            left--;
        }
        return mlgpu_philox_uniform(key, stream, k++);
    }
    uint64_t create_seed() override { return 0; }
    double normal(const double mean, const double std_dev) override {
        const double u1 = uniform();
        const double u2 = uniform();
        return mean + std_dev*(sqrt(-2.0*log(1.0 - u1))*cos(2.0*M_PI*u2));
    }
};

struct SignalResult {
    std::vector<uint64_t> offsets[3];        // photon pipelines, pulses, channels
    std::vector<double> pipe_time, pipe_wavelength, pulse_time;
    std::vector<int32_t> pipe_truth, pulse_truth, channel_truth;
    std::vector<uint8_t> channel_slice;
    double nsb_exposure_start_time = 0.0;
    double seconds = 0.0;
};

std::vector<std::vector<double>> xy_table(const double* xy, uint32_t n) {
    std::vector<std::vector<double>> t;
    for (uint32_t i = 0; i < n; i++) t.push_back({xy[2*i], xy[2*i + 1]});
    return t;
}

}  // namespace

// lfs: expected focal length, expected aperture radius, max FoV diameter
// [deg], pixel FoV flat2flat [deg], paxels on the pixel diagonal, housing
// overhead -- the light-field sensor whose geometry the background light
// uses (Light.cpp:8-24).  times: exposure, time slice, arrival time std.
void* ref_signal_chain(int mode, uint64_t seed, uint64_t offset, const int32_t* sensor,
                       const double* time, const double* wavelength, const int32_t* truth,
                       uint64_t n, uint32_t num_sensors, const float* lixel_efficiency,
                       const double* qe_xy, uint32_t num_qe, double dark_rate,
                       double probability_for_second_puls, const double* flux_xy,
                       uint32_t num_flux, const double* lfs, const double* times,
                       const uint32_t* nsb_count) {
    try {
        namespace sp = signal_processing;
        namespace nsb = plenoscope::night_sky_background;
        std::unique_ptr<SignalResult> r(new SignalResult);
        // the light-field sensor's geometry, for the background light
        ml::function::Func1 lens_n({{200e-9, 1.5}, {1200e-9, 1.5}});
        plenoscope::light_field_sensor::Config lc;
        lc.expected_imaging_system_focal_length = lfs[0];
        lc.expected_imaging_system_max_aperture_radius = lfs[1];
        lc.max_FoV_diameter = ml::deg2rad(lfs[2]);
        lc.pixel_FoV_hex_flat2flat = ml::deg2rad(lfs[3]);
        lc.num_paxel_on_pixel_diagonal = static_cast<unsigned int>(lfs[4]);
        lc.housing_overhead = lfs[5];
        lc.lens_refraction = &lens_n;
        lc.bin_reflection = &lens_n;
        plenoscope::light_field_sensor::Geometry geometry(lc);
        if (geometry.num_lixel() != num_sensors)
            throw std::invalid_argument("the light-field sensor's lixels differ from the sensors");
        const ml::function::Func1 flux(xy_table(flux_xy, num_flux));
        const nsb::Light light(&geometry, &flux);
        const ml::function::Func1 qe(xy_table(qe_xy, num_qe));
        sp::PhotoElectricConverter::Config pc;
        pc.quantum_efficiency_vs_wavelength = &qe;
        pc.dark_rate = dark_rate;
        pc.probability_for_second_puls = probability_for_second_puls;
        sp::PhotoElectricConverter::Converter converter(&pc);
        const std::vector<float> efficiency(lixel_efficiency, lixel_efficiency + num_sensors);
        const double exposure = times[0], slice = times[1], time_std = times[2];

        // the arrivals as merlict's sensors hold them (Sensor::assign_photon)
        std::unique_ptr<ml::Frame[]> frames(new ml::Frame[num_sensors]);
        std::vector<ml::sensor::Sensor> sensors;
        sensors.reserve(num_sensors);
        for (uint32_t i = 0; i < num_sensors; i++) sensors.emplace_back(i, &frames[i]);
        for (uint64_t i = 0; i < n; i++) {
            if (sensor[i] < 0) continue;
            ml::sensor::PhotonArrival a;
            a.simulation_truth_id = truth[i];
            a.wavelength = wavelength[i];
            a.arrival_time = time[i];
            sensors.at(sensor[i]).photon_arrival_history.push_back(a);
        }
        std::vector<ml::sensor::Sensor*> ptrs;
        for (ml::sensor::Sensor& s : sensors) ptrs.push_back(&s);
        ml::sensor::Sensors channels(ptrs);

        SignalReplay replay;
        replay.key = seed;
        replay.offset = offset;
        ml::random::Mt19937 mt(seed);
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::vector<sp::PipelinePhoton>> pipes = sp::get_photon_pipelines(&channels);
        if (mode == 0) {
            replay.budget_of = nsb_count;
            replay.stage = 1;
        }
        nsb::inject_nsb_into_photon_pipeline(&pipes, exposure, &efficiency, &light,
                                             &r->nsb_exposure_start_time,
                                             mode == 0 ? static_cast<ml::random::Generator*>(&replay)
                                                       : &mt);
        replay.budget_of = nullptr;
        std::vector<std::vector<sp::ElectricPulse>> electric;
        electric.reserve(pipes.size());
        for (uint64_t i = 0; i < pipes.size(); i++) {
            replay.select(2, i);
            electric.push_back(converter.get_pulse_pipeline_for_photon_pipeline(
                pipes[i], exposure, mode == 0 ? static_cast<ml::random::Generator*>(&replay) : &mt));
        }
        std::vector<std::vector<sp::ExtractedPulse>> extracted;
        if (mode == 0) {
            for (uint64_t i = 0; i < electric.size(); i++) {
                replay.select(3, i);
                extracted.push_back(sp::extract_pulses(electric[i], slice, time_std, &replay));
            }
        } else {
            extracted = sp::extract_pulses(electric, slice, time_std, &mt);
        }
        r->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

        for (int j = 0; j < 3; j++) r->offsets[j].push_back(0);
        for (const auto& p : pipes) {
            for (const sp::PipelinePhoton& ph : p) {
                r->pipe_time.push_back(ph.arrival_time);
                r->pipe_wavelength.push_back(ph.wavelength);
                r->pipe_truth.push_back(ph.simulation_truth_id);
            }
            r->offsets[0].push_back(r->pipe_time.size());
        }
        for (const auto& p : electric) {
            for (const sp::ElectricPulse& e : p) {
                r->pulse_time.push_back(e.arrival_time);
                r->pulse_truth.push_back(e.simulation_truth_id);
            }
            r->offsets[1].push_back(r->pulse_time.size());
        }
        for (const auto& p : extracted) {
            for (const sp::ExtractedPulse& e : p) {
                r->channel_slice.push_back(e.arrival_time_slice);
                r->channel_truth.push_back(e.simulation_truth_id);
            }
            r->offsets[2].push_back(r->channel_slice.size());
        }
        return r.release();
    } catch (const std::exception& e) {
        last_error = e.what();
        return nullptr;
    }
}

// The result's arrays: 0-2 offsets (pipelines, pulses, channels), 3 pipeline
// times, 4 pipeline wavelengths, 5 pipeline truth ids, 6 pulse times, 7 pulse
// truth ids, 8 channel slices, 9 channel truth ids.  Returns the element
// count; copies when `out` is not NULL.
uint64_t ref_signal_result(void* handle, int which, void* out) {
    SignalResult* r = static_cast<SignalResult*>(handle);
    auto put = [out](const auto& v) {
        if (out) std::memcpy(out, v.data(), v.size()*sizeof(v[0]));
        return static_cast<uint64_t>(v.size());
    };
    switch (which) {
        case 0: case 1: case 2: return put(r->offsets[which]);
        case 3: return put(r->pipe_time);
        case 4: return put(r->pipe_wavelength);
        case 5: return put(r->pipe_truth);
        case 6: return put(r->pulse_time);
        case 7: return put(r->pulse_truth);
        case 8: return put(r->channel_slice);
        case 9: return put(r->channel_truth);
        default: return 0;
    }
}

double ref_signal_start_time(void* handle) {
    return static_cast<SignalResult*>(handle)->nsb_exposure_start_time;
}

double ref_signal_seconds(void* handle) { return static_cast<SignalResult*>(handle)->seconds; }

void ref_signal_free(void* handle) { delete static_cast<SignalResult*>(handle); }

// PhotonStream::write and write_simulation_truth (PhotonStream.cpp:15-78)
// of channels given as offsets [num_channels + 1], slices and truth ids.
int ref_photon_stream_write(const char* path, const char* truth_path, const uint64_t* offsets,
                            const uint8_t* slices, const int32_t* truth, uint32_t num_channels,
                            float time_slice_duration) {
    try {
        std::vector<std::vector<signal_processing::ExtractedPulse>> channels(num_channels);
        for (uint32_t c = 0; c < num_channels; c++)
            for (uint64_t k = offsets[c]; k < offsets[c + 1]; k++)
                channels[c].emplace_back(slices[k], truth[k]);
        signal_processing::PhotonStream::write(channels, time_slice_duration, path);
        signal_processing::PhotonStream::write_simulation_truth(channels, truth_path);
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return 1;
    }
}

// ---- CORSIKA files ----------------------------------------------------------
// A whole file through merlict's readers: eventio::Run (kind 0) or
// event_tape::Run (kind 1), every event's header, telescope offsets (EventIO)
// and bunches kept for ref_corsika_file_result.

namespace {
struct CorsikaFile {
    std::vector<float> run_header, tel_pos, event_headers, offsets, bunches;
    std::vector<uint64_t> offset_start{0}, bunch_start{0};
    std::string input_card;
};
}  // namespace

void* ref_corsika_file_read(const char* path, int kind) {
    try {
        std::unique_ptr<CorsikaFile> r(new CorsikaFile);
        auto add_bunches = [&](const std::vector<std::array<float, 8>>& b) {
            for (const auto& row : b) r->bunches.insert(r->bunches.end(), row.begin(), row.end());
            r->bunch_start.push_back(r->bunches.size()/8);
        };
        if (kind == 0) {
            eventio::Run run(path);
            r->run_header.assign(run.header.raw.begin(), run.header.raw.end());
            r->input_card = run.header.input_card;
            for (const eventio::TelPos& t : run.header.tel_pos)
                r->tel_pos.insert(r->tel_pos.end(), {t.x, t.y, t.z, t.r});
            while (run.has_still_events_left()) {
                eventio::Event e = run.next_event();
                r->event_headers.insert(r->event_headers.end(), e.header.raw.begin(),
                                        e.header.raw.end());
                for (const eventio::TelOffset& o : e.header.telescope_offsets)
                    r->offsets.insert(r->offsets.end(), {o.toff, o.xoff, o.yoff, o.weight});
                r->offset_start.push_back(r->offsets.size()/4);
                add_bunches(e.photons);
            }
        } else {
            event_tape::Run run(path);
            r->run_header.assign(run.header.begin(), run.header.end());
            while (run.has_still_events_left()) {
                event_tape::Event e = run.next_event();
                r->event_headers.insert(r->event_headers.end(), e.header.begin(), e.header.end());
                add_bunches(e.photons);
            }
        }
        return r.release();
    } catch (const std::exception& e) {
        last_error = e.what();
        return nullptr;
    }
}

// 0 run header, 1 telescope positions, 2 event headers, 3 telescope offsets,
// 4 offsets per event (uint64 starts), 5 bunches, 6 bunch starts (uint64),
// 7 input card (bytes).  Returns the element count; copies when out != NULL.
uint64_t ref_corsika_file_result(void* handle, int which, void* out) {
    CorsikaFile* r = static_cast<CorsikaFile*>(handle);
    auto put = [out](const auto& v) {
        if (out && !v.empty()) std::memcpy(out, v.data(), v.size()*sizeof(v[0]));
        return static_cast<uint64_t>(v.size());
    };
    switch (which) {
        case 0: return put(r->run_header);
        case 1: return put(r->tel_pos);
        case 2: return put(r->event_headers);
        case 3: return put(r->offsets);
        case 4: return put(r->offset_start);
        case 5: return put(r->bunches);
        case 6: return put(r->bunch_start);
        case 7: return put(r->input_card);
        default: return 0;
    }
}

void ref_corsika_file_free(void* handle) { delete static_cast<CorsikaFile*>(handle); }

int ref_hardware_concurrency(void) {
    return static_cast<int>(std::thread::hardware_concurrency());
}

// The ray supports (x, y, z per photon) the photons held after the last
// ref_propagate (or shim_propagate) on this scene; returns the photon count,
// copies when out != NULL.
uint64_t ref_last_supports(void* handle, double* out) {
    const Handle* h = static_cast<const Handle*>(handle);
    if (out && !h->last_support.empty())
        std::memcpy(out, h->last_support.data(), h->last_support.size()*sizeof(double));
    return h->last_support.size()/3;
}

// The drop-in's history rebuild (merlict_b200::rebuild_histories) without
// the engine: fresh photons from the planes get the given histories (rows
// of max_interactions + 1 entries, as mlgpu_results.history holds them),
// infos and final directions, then merlict's own Sensors::assign_photons
// runs on them; their results (and supports) are written as ref_propagate
// writes them.  Fed with ref_propagate's own export of the same photons,
// the results must come back unchanged.
int ref_rebuild_photons(void* handle, const mlgpu_photons* ph, uint64_t n,
                        uint32_t max_interactions, const mlgpu_history_entry* history,
                        const uint32_t* info, const double* final_direction,
                        mlgpu_results* out) {
    Handle* h = static_cast<Handle*>(handle);
    try {
        std::vector<ml::Photon> photons = make_photons(ph, n);
        if (!h->flattened) {
            h->flat = merlict_b200::flatten(&h->scenery.root, &h->sensors);
            h->flattened = true;
        }
        merlict_b200::rebuild_histories(&photons, h->flat, history, info, final_direction,
                                        max_interactions);
        h->sensors.clear_history();
        h->sensors.assign_photons(&photons);
        keep_supports(h, photons);
        if (out) write_results(h, photons, std::vector<uint32_t>(n, 0), max_interactions, out);
        return 0;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MLGPU_ERR_RUNTIME;
    }
}

#ifdef MLGPU_WITH_SHIM
// The product's C++ drop-in (merlict_b200_shim.h) on a scene built here, the
// way a merlict application would call it in place of the reference's own
// functions:
//   mode 0  merlict_b200::propagate_photons_in_frame_with_config, then
//           merlict's own Sensors::assign_photons on the rebuilt photons;
//   mode 1  merlict_b200::propagate_photons_in_frame_with_config_multi_thread,
//           then Sensors::assign_photons;
//   mode 2  merlict_b200::propagate_and_assign_photons (arrivals written
//           straight into the sensors; the photons keep no history).
// The generator is merlict's Mt19937(mt_seed); *philox_seed receives the
// seed the drop-in drew from it (Generator::create_seed), with which
// ref_propagate's mode 0 replays the same streams.  Results as for
// ref_propagate (info without the uniform count); in mode 2 only the
// arrival fields (sensor, x, y, time, theta_x, theta_y) are meaningful.
// A std:: exception from the drop-in returns the status of its type.
int shim_propagate(void* handle, const mlgpu_photons* ph, uint64_t n,
                   uint32_t max_interactions, int mode, uint64_t mt_seed,
                   uint64_t* philox_seed, mlgpu_results* out) {
    Handle* h = static_cast<Handle*>(handle);
    struct Recording : ml::random::Mt19937 {
        explicit Recording(uint64_t seed) : ml::random::Mt19937(seed) {}
        uint64_t drawn = 0;
        uint64_t create_seed() override {
            drawn = ml::random::Mt19937::create_seed();
            return drawn;
        }
    };
    try {
        std::vector<ml::Photon> photons = make_photons(ph, n);
        ml::PropagationConfig cfg;
        cfg.max_num_interactions_per_photon = max_interactions;
        Recording prng(mt_seed);
        h->sensors.clear_history();
        if (mode == 0) {
            merlict_b200::propagate_photons_in_frame_with_config(
                &photons, &h->scenery.root, &cfg, &prng);
            h->sensors.assign_photons(&photons);
        } else if (mode == 1) {
            merlict_b200::propagate_photons_in_frame_with_config_multi_thread(
                &photons, &h->scenery.root, &cfg, &prng);
            h->sensors.assign_photons(&photons);
        } else if (mode == 2) {
            merlict_b200::propagate_and_assign_photons(
                &photons, &h->scenery.root, &cfg, &prng, &h->sensors);
        } else {
            throw std::invalid_argument("unknown mode");
        }
        if (philox_seed) *philox_seed = prng.drawn;
        keep_supports(h, photons);
        if (out) write_results(h, photons, std::vector<uint32_t>(n, 0), max_interactions, out);
        return 0;
    } catch (const std::out_of_range& e) {
        last_error = e.what();
        return MLGPU_ERR_OUT_OF_RANGE;
    } catch (const std::invalid_argument& e) {
        last_error = e.what();
        return MLGPU_ERR_INVALID_ARGUMENT;
    } catch (const std::exception& e) {
        last_error = e.what();
        return MLGPU_ERR_RUNTIME;
    }
}
#endif

}  // extern "C"
