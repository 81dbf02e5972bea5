// merlict_b200_flatten.cpp -- merlict frame tree -> mlgpu_flat_scene
// (declared in merlict_b200_shim.h).
//
// The flattener reads primitive parameters that merlict keeps in protected
// or private members.  It does so without editing merlict, through member
// pointers formed in explicit template instantiations (access checking does
// not apply to the template arguments of an explicit instantiation).
#include "merlict_b200_shim.h"

#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <sstream>
#include <stdexcept>

namespace merlict_b200 {
namespace {

namespace ml = merlict;

template <typename Tag, typename Tag::type Member>
struct Accessor {
    friend typename Tag::type member_of(Tag) { return Member; }
};

#define MLGPU_MEMBER(TAG, CLASS, TYPE, NAME)                        \
    struct TAG {                                                    \
        typedef TYPE CLASS::*type;                                  \
        friend type member_of(TAG);                                 \
    };                                                              \
    template struct Accessor<TAG, &CLASS::NAME>

MLGPU_MEMBER(HexInner, ml::HexagonalPrismZ, double, inner_radius);
MLGPU_MEMBER(CylRadiusSquare, ml::CylinderPrismZ, double, radius_square);
MLGPU_MEMBER(DualCirc1, ml::DualSphericalPrismZ, ml::Vec2, circ1);
MLGPU_MEMBER(DualCirc2, ml::DualSphericalPrismZ, ml::Vec2, circ2);
MLGPU_MEMBER(CapHexBounds, ml::SphereCapWithHexagonalBound, ml::HexagonalPrismZ, hexBounds);
MLGPU_MEMBER(CapHexR, ml::SphereCapWithHexagonalBound, double, curvature_radius);
MLGPU_MEMBER(CapCylBounds, ml::SphereCapWithCylinderBound, ml::CylinderPrismZ, CylBounds);
MLGPU_MEMBER(CapCylR, ml::SphereCapWithCylinderBound, double, curvature_radius);
MLGPU_MEMBER(CapRectBounds, ml::SphereCapWithRectangularBound, ml::RectangularPrismZ, rect_bounds);
MLGPU_MEMBER(CapRectR, ml::SphereCapWithRectangularBound, double, curvature_radius);
MLGPU_MEMBER(EllHexBounds, ml::EllipticalCapWithHexagonalBound, ml::HexagonalPrismZ, hexBounds);
MLGPU_MEMBER(EllX, ml::EllipticalCapWithHexagonalBound, double, X_curvature_radius);
MLGPU_MEMBER(EllY, ml::EllipticalCapWithHexagonalBound, double, Y_curvature_radius);
MLGPU_MEMBER(EllZ, ml::EllipticalCapWithHexagonalBound, double, Z_curvature_radius);
MLGPU_MEMBER(EllIXX, ml::EllipticalCapWithHexagonalBound, double, iXX);
MLGPU_MEMBER(EllIYY, ml::EllipticalCapWithHexagonalBound, double, iYY);
MLGPU_MEMBER(EllIZZ, ml::EllipticalCapWithHexagonalBound, double, iZZ);
MLGPU_MEMBER(DiscBounds, ml::Disc, ml::CylinderPrismZ, cylinder_bounds);
MLGPU_MEMBER(HexPlaneBounds, ml::HexPlane, ml::HexagonalPrismZ, hex_bounds);
MLGPU_MEMBER(PlaneBounds, ml::Plane, ml::RectangularPrismZ, RectBounds);
MLGPU_MEMBER(AnnulusOuter, ml::Annulus, ml::CylinderPrismZ, outer_bound);
MLGPU_MEMBER(AnnulusInner, ml::Annulus, ml::CylinderPrismZ, inner_bound);
MLGPU_MEMBER(DualBounds, ml::PlaneDualSphericalBound, ml::DualSphericalPrismZ, dual_sphere_bounds);
MLGPU_MEMBER(TriA, ml::Triangle, ml::Vec2, A);
MLGPU_MEMBER(TriB, ml::Triangle, ml::Vec2, B);
MLGPU_MEMBER(TriC, ml::Triangle, ml::Vec2, C);
MLGPU_MEMBER(CylinderRadius, ml::Cylinder, double, Radius);
MLGPU_MEMBER(CylinderLength, ml::Cylinder, double, Length);
MLGPU_MEMBER(SphereRadius, ml::Sphere, double, radius);

template <typename Tag, typename Object>
auto get(const Object& o, Tag tag) -> decltype(o.*member_of(tag)) {
    return o.*member_of(tag);
}

struct LeafDescription {
    int32_t primitive = MLGPU_PRIM_NONE;
    double params[MLGPU_LEAF_PARAMS] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// Primitive kind and parameters of a leaf frame, in the units and with the
// derived quantities the leaf's calculate_intersection_with uses.
LeafDescription describe_leaf(const ml::Frame* f) {
    LeafDescription d;
    double* p = d.params;
    if (auto o = dynamic_cast<const ml::SphereCapWithHexagonalBound*>(f)) {
        d.primitive = MLGPU_PRIM_SPHERE_CAP_HEX;
        p[0] = get(*o, CapHexR());
        p[1] = get(get(*o, CapHexBounds()), HexInner());
    } else if (auto o = dynamic_cast<const ml::SphereCapWithCylinderBound*>(f)) {
        d.primitive = MLGPU_PRIM_SPHERE_CAP_CYL;
        p[0] = get(*o, CapCylR());
        p[1] = get(get(*o, CapCylBounds()), CylRadiusSquare());
    } else if (auto o = dynamic_cast<const ml::SphereCapWithRectangularBound*>(f)) {
        d.primitive = MLGPU_PRIM_SPHERE_CAP_RECT;
        p[0] = get(*o, CapRectR());
        p[1] = get(*o, CapRectBounds()).get_half_x_width();
        p[2] = get(*o, CapRectBounds()).get_half_y_width();
    } else if (auto o = dynamic_cast<const ml::EllipticalCapWithHexagonalBound*>(f)) {
        d.primitive = MLGPU_PRIM_ELLIPTIC_CAP_HEX;
        p[0] = get(*o, EllX());
        p[1] = get(*o, EllY());
        p[2] = get(*o, EllZ());
        p[3] = get(*o, EllIXX());
        p[4] = get(*o, EllIYY());
        p[5] = get(*o, EllIZZ());
        p[6] = get(get(*o, EllHexBounds()), HexInner());
    } else if (auto o = dynamic_cast<const ml::Disc*>(f)) {
        d.primitive = MLGPU_PRIM_DISC;
        p[0] = get(get(*o, DiscBounds()), CylRadiusSquare());
    } else if (auto o = dynamic_cast<const ml::HexPlane*>(f)) {
        d.primitive = MLGPU_PRIM_HEX_PLANE;
        p[0] = get(get(*o, HexPlaneBounds()), HexInner());
    } else if (auto o = dynamic_cast<const ml::Plane*>(f)) {
        d.primitive = MLGPU_PRIM_PLANE;
        p[0] = get(*o, PlaneBounds()).get_half_x_width();
        p[1] = get(*o, PlaneBounds()).get_half_y_width();
    } else if (auto o = dynamic_cast<const ml::Annulus*>(f)) {
        d.primitive = MLGPU_PRIM_ANNULUS;
        p[0] = get(get(*o, AnnulusOuter()), CylRadiusSquare());
        p[1] = get(get(*o, AnnulusInner()), CylRadiusSquare());
    } else if (auto o = dynamic_cast<const ml::PlaneDualSphericalBound*>(f)) {
        d.primitive = MLGPU_PRIM_PLANE_DUAL_SPHERE;
        const ml::DualSphericalPrismZ& b = get(*o, DualBounds());
        p[0] = get(b, DualCirc1()).x;
        p[1] = get(b, DualCirc1()).y;
        p[2] = get(b, DualCirc2()).x;
        p[3] = get(b, DualCirc2()).y;
        p[4] = b.get_circle_radius();
    } else if (auto o = dynamic_cast<const ml::Triangle*>(f)) {
        d.primitive = MLGPU_PRIM_TRIANGLE;
        p[0] = get(*o, TriA()).x; p[1] = get(*o, TriA()).y;
        p[2] = get(*o, TriB()).x; p[3] = get(*o, TriB()).y;
        p[4] = get(*o, TriC()).x; p[5] = get(*o, TriC()).y;
    } else if (auto o = dynamic_cast<const ml::Cylinder*>(f)) {
        d.primitive = MLGPU_PRIM_CYLINDER;
        p[0] = get(*o, CylinderRadius());
        p[1] = get(*o, CylinderLength());
    } else if (auto o = dynamic_cast<const ml::Sphere*>(f)) {
        d.primitive = MLGPU_PRIM_SPHERE;
        p[0] = get(*o, SphereRadius());
    } else {
        // A Frame or SurfaceEntity without children and without its own
        // calculate_intersection_with: merlict never reports a hit on it.
        d.primitive = MLGPU_PRIM_NONE;
    }
    return d;
}

}  // namespace

mlgpu_flat_scene FlatScene::view() const {
    mlgpu_flat_scene v;
    std::memset(&v, 0, sizeof(v));
    v.num_nodes = static_cast<int32_t>(node_skip.size());
    v.node_sphere = node_sphere.data();
    v.node_skip = node_skip.data();
    v.node_leaf = node_leaf.data();
    v.num_leaves = static_cast<int32_t>(leaf_node.size());
    v.leaf_node = leaf_node.data();
    v.leaf_frame2world = leaf_frame2world.data();
    v.leaf_primitive = leaf_primitive.data();
    v.leaf_params = leaf_params.data();
    v.leaf_surface = leaf_surface.data();
    v.leaf_sensor = leaf_sensor.data();
    v.num_functions = static_cast<int32_t>(function_offset.size()) - 1;
    v.function_offset = function_offset.data();
    v.function_points = function_points.data();
    v.default_refraction = default_refraction;
    for (int k = 0; k < 3; k++) {
        v.hex_unit_u[k] = hex_unit_u[k];
        v.hex_unit_v[k] = hex_unit_v[k];
        v.hex_unit_w[k] = hex_unit_w[k];
    }
    v.num_sensors = num_sensors;
    return v;
}

int32_t FlatScene::node_index(const ml::Frame* frame) const {
    auto it = node_of_frame.find(frame);
    return it == node_of_frame.end() ? -1 : it->second;
}

FlatScene flatten(const ml::Frame* world, const ml::sensor::Sensors* sensors) {
    FlatScene fs;
    std::map<const ml::function::Func1*, int32_t> function_id;
    fs.function_offset.push_back(0);
    auto func = [&](const ml::function::Func1* f) -> int32_t {
        auto it = function_id.find(f);
        if (it != function_id.end()) return it->second;
        const int32_t id = static_cast<int32_t>(fs.function_offset.size()) - 1;
        for (const ml::function::Point& pt : f->func) {
            fs.function_points.push_back(pt.x);
            fs.function_points.push_back(pt.y);
            fs.function_points.push_back(pt.slope);
        }
        fs.function_offset.push_back(
            static_cast<int32_t>(fs.function_points.size() / 3));
        function_id[f] = id;
        return id;
    };
    const int32_t def_refl = func(ml::SurfaceEntity::DEFAULT_REFLECTION);
    const int32_t def_refr = func(ml::SurfaceEntity::DEFAULT_REFRACTION);
    const int32_t def_abs = func(ml::SurfaceEntity::DEFAULT_ABSORPTION);
    fs.default_refraction = def_refr;

    const ml::Vec3 u = ml::VEC3_UNIT_U, v = ml::VEC3_UNIT_V, w = ml::VEC3_UNIT_W;
    fs.hex_unit_u[0] = u.x; fs.hex_unit_u[1] = u.y; fs.hex_unit_u[2] = u.z;
    fs.hex_unit_v[0] = v.x; fs.hex_unit_v[1] = v.y; fs.hex_unit_v[2] = v.z;
    fs.hex_unit_w[0] = w.x; fs.hex_unit_w[1] = w.y; fs.hex_unit_w[2] = w.z;

    std::vector<const ml::Frame*> allowed_of_leaf;
    std::function<void(const ml::Frame*)> visit = [&](const ml::Frame* f) {
        const int32_t idx = static_cast<int32_t>(fs.node_skip.size());
        const ml::Vec3 c = f->position_in_world();
        fs.node_sphere.push_back(c.x);
        fs.node_sphere.push_back(c.y);
        fs.node_sphere.push_back(c.z);
        fs.node_sphere.push_back(f->get_bounding_sphere_radius());
        fs.node_skip.push_back(-1);
        fs.node_frame.push_back(f);
        fs.node_of_frame[f] = idx;
        if (f->has_children()) {
            fs.node_leaf.push_back(-1);
            for (const ml::Frame* child : *f->get_children()) visit(child);
        } else {
            const int32_t leaf = static_cast<int32_t>(fs.leaf_node.size());
            fs.node_leaf.push_back(leaf);
            fs.leaf_node.push_back(idx);
            const ml::HomTra3* T = f->frame2world();
            const ml::Vec3 col[4] = {T->rot_x(), T->rot_y(), T->rot_z(), T->translation()};
            for (int r = 0; r < 3; r++)
                for (int k = 0; k < 4; k++)
                    fs.leaf_frame2world.push_back(
                        r == 0 ? col[k].x : (r == 1 ? col[k].y : col[k].z));
            const LeafDescription d = describe_leaf(f);
            fs.leaf_primitive.push_back(d.primitive);
            for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) fs.leaf_params.push_back(d.params[k]);
            int32_t surf[MLGPU_SURF_COLUMNS] = {def_refl, def_refl, def_refr, def_refr,
                                                def_abs, def_abs, -1, 0};
            const ml::Frame* allowed = nullptr;
            const ml::SurfaceEntity* se = dynamic_cast<const ml::SurfaceEntity*>(f);
            if (se) {
                surf[MLGPU_SURF_OUTER_REFLECTION] = func(se->outer_reflection);
                surf[MLGPU_SURF_INNER_REFLECTION] = func(se->inner_reflection);
                surf[MLGPU_SURF_OUTER_REFRACTION] = func(se->outer_refraction);
                surf[MLGPU_SURF_INNER_REFRACTION] = func(se->inner_refraction);
                surf[MLGPU_SURF_OUTER_ABSORPTION] = func(se->outer_absorption);
                surf[MLGPU_SURF_INNER_ABSORPTION] = func(se->inner_absorption);
                int32_t flags = 0;
                if (se->boundary_layer_is_transparent()) flags |= MLGPU_FLAG_TRANSPARENT;
                if (se->inner_refraction == ml::SurfaceEntity::DEFAULT_REFRACTION)
                    flags |= MLGPU_FLAG_INNER_REFRACTION_DEFAULT;
                if (se->outer_refraction == ml::SurfaceEntity::DEFAULT_REFRACTION)
                    flags |= MLGPU_FLAG_OUTER_REFRACTION_DEFAULT;
                surf[MLGPU_SURF_FLAGS] = flags;
                if (se->has_restrictions_on_frames_to_propagate_to())
                    allowed = se->allowed_frame_to_propagate_to();
            } else {
                surf[MLGPU_SURF_FLAGS] = MLGPU_FLAG_INNER_REFRACTION_DEFAULT |
                    MLGPU_FLAG_OUTER_REFRACTION_DEFAULT;
            }
            for (int k = 0; k < MLGPU_SURF_COLUMNS; k++) fs.leaf_surface.push_back(surf[k]);
            fs.leaf_sensor.push_back(-1);
            fs.leaf_entity.push_back(se);
            allowed_of_leaf.push_back(allowed);
        }
        fs.node_skip[idx] = static_cast<int32_t>(fs.node_skip.size());
    };
    visit(world->root());

    for (size_t leaf = 0; leaf < allowed_of_leaf.size(); leaf++) {
        if (!allowed_of_leaf[leaf]) continue;
        const int32_t node = fs.node_index(allowed_of_leaf[leaf]);
        if (node < 0) {
            std::stringstream info;
            info << "merlict_b200::flatten: the frame '"
                 << fs.node_frame[fs.leaf_node[leaf]]->path_in_tree()
                 << "' restricts propagation to a frame outside its tree.";
            throw std::invalid_argument(info.str());
        }
        fs.leaf_surface[leaf*MLGPU_SURF_COLUMNS + MLGPU_SURF_ALLOWED_NODE] = node;
    }

    if (sensors) {
        fs.num_sensors = static_cast<int32_t>(sensors->by_occurence.size());
        for (size_t s = 0; s < sensors->by_occurence.size(); s++) {
            ml::sensor::Sensor* sensor = sensors->by_occurence[s];
            fs.sensor_of_index.push_back(sensor);
            const int32_t node = fs.node_index(sensor->frame);
            if (node < 0) continue;
            const int32_t leaf = fs.node_leaf[node];
            if (leaf >= 0) fs.leaf_sensor[leaf] = static_cast<int32_t>(s);
        }
    }
    return fs;
}

}  // namespace merlict_b200
