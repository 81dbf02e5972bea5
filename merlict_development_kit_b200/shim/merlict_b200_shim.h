// merlict_b200_shim.h -- drop-in for merlict's propagation entry points.
//
// A merlict build that links this file and libmerlict_b200.so can replace
//
//   merlict::propagate_photons_in_frame_with_config(...)     Photons.h:12-16
//   merlict::propagate_photons_in_frame_with_config_multi_thread(...)
//                                      merlict_multi_thread.h:12-16
//
// by the functions of the same signature below (namespace merlict_b200).
// The first call for a `world` frame flattens its initialised tree
// (Frame::init_tree_based_on_mother_child_relations must have run) and
// uploads it; later calls reuse the device copy.  The photons' histories
// are rebuilt on the host so that sensor::Sensors::assign_photons and every
// other reader of Photon works unchanged.  Errors raised by the engine come
// back as the std:: exception the reference would have thrown.
#ifndef MERLICT_B200_SHIM_H_
#define MERLICT_B200_SHIM_H_

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "merlict/merlict.h"
#include "merlict_b200.h"

namespace merlict_b200 {

// Host image of an mlgpu_flat_scene built from a merlict frame tree.  It
// owns the arrays; view() hands out pointers into them.
class FlatScene {
 public:
    std::vector<double> node_sphere;
    std::vector<int32_t> node_skip;
    std::vector<int32_t> node_leaf;
    std::vector<int32_t> leaf_node;
    std::vector<double> leaf_frame2world;
    std::vector<int32_t> leaf_primitive;
    std::vector<double> leaf_params;
    std::vector<int32_t> leaf_surface;
    std::vector<int32_t> leaf_sensor;
    std::vector<int32_t> function_offset;
    std::vector<double> function_points;
    int32_t default_refraction = 0;
    double hex_unit_u[3];
    double hex_unit_v[3];
    double hex_unit_w[3];
    int32_t num_sensors = 0;

    // bookkeeping for writing results back into merlict objects
    std::vector<const merlict::Frame*> node_frame;
    std::vector<const merlict::SurfaceEntity*> leaf_entity;
    std::vector<merlict::sensor::Sensor*> sensor_of_index;
    std::map<const merlict::Frame*, int32_t> node_of_frame;

    mlgpu_flat_scene view() const;
    int32_t node_index(const merlict::Frame* frame) const;
};

// Walks the tree of `world` (from world->root()) in the order
// CausalIntersection visits it (RayAndFrame.cpp:137-149).  `sensors` may be
// null; otherwise leaf_sensor maps each sensor's frame to its position in
// sensors->by_occurence.  Throws std::invalid_argument on a frame type it
// does not know.
FlatScene flatten(
    const merlict::Frame* world,
    const merlict::sensor::Sensors* sensors = nullptr);

// Same signature and meaning as merlict/Photons.h:12-16.  Draws one seed
// from `prng` per call for the device's counter-based generator.
void propagate_photons_in_frame_with_config(
    std::vector<merlict::Photon>* photons,
    const merlict::Frame* world,
    const merlict::PropagationConfig* settings,
    merlict::random::Generator* prng);

// Same signature as merlict_multi_thread.h:12-16; on the GPU both are one
// launch.
void propagate_photons_in_frame_with_config_multi_thread(
    std::vector<merlict::Photon>* photons,
    const merlict::Frame* world,
    const merlict::PropagationConfig* settings,
    merlict::random::Generator* prng);

// Fast path: propagate and append the arrivals straight to the sensors'
// photon_arrival_history (what Sensors::assign_photons would append),
// without rebuilding the photons' histories.
void propagate_and_assign_photons(
    const std::vector<merlict::Photon>* photons,
    const merlict::Frame* world,
    const merlict::PropagationConfig* settings,
    merlict::random::Generator* prng,
    merlict::sensor::Sensors* sensors);

// Throws the exception the reference raises for an engine status.
void throw_on_error(int status);

// Appends to each fresh photon (only its production interaction) the
// intersections and interactions the engine recorded for it --
// history[i*(max_interactions + 1) + k], k < info[i] >> 8 & 0xff -- through
// merlict's public RayForPropagation::push_back_intersection_and_interaction
// (RayForPropagation.h:49-51) and Intersection's constructor
// (Intersection.h:24-29), objects mapped back through flat.leaf_entity; and
// sets the photon's ray to the support and direction merlict's Propagator
// would have left (final_direction[3 i .. 3 i + 2]).  Throws
// std::runtime_error on a history that names no known leaf.
void rebuild_histories(
    std::vector<merlict::Photon>* photons,
    const FlatScene& flat,
    const mlgpu_history_entry* history,
    const uint32_t* info,
    const double* final_direction,
    uint32_t max_interactions);

}  // namespace merlict_b200

#endif  // MERLICT_B200_SHIM_H_
