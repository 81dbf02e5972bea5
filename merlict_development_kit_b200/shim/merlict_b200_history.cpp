// merlict_b200_history.cpp -- rebuilds merlict Photon objects from the
// engine's per-photon history (mlgpu_history_entry rows), so that every
// reader of a propagated Photon -- Sensors::assign_photons, time_of_flight,
// the final intersection's incident direction -- works unchanged.
//
// Host code only (no engine call), so that it can be checked on the CPU.
#include "merlict_b200_shim.h"

#include <stdexcept>

namespace merlict_b200 {
namespace {

namespace ml = merlict;

// merlict's Propagator moves the ray with Ray::set_support_and_direction
// (PhotonAndFrame.cpp:56-66, 104-118); these give the rebuilt photon the
// ray it would hold after merlict's own propagation.
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

MLGPU_MEMBER(RaySupport, ml::Ray, ml::Vec3, support_);
MLGPU_MEMBER(RayDirection, ml::Ray, ml::Vec3, direction_);

bool moves_on(uint8_t interaction) {
    return interaction == MLGPU_REFLECTION_ON_SURFACE ||
        interaction == MLGPU_FRESNEL_REFLECTION_ON_SURFACE ||
        interaction == MLGPU_REFRACTION_TO_INSIDE || interaction == MLGPU_REFRACTION_TO_OUTSIDE;
}

}  // namespace

void rebuild_histories(
    std::vector<ml::Photon>* photons,
    const FlatScene& flat,
    const mlgpu_history_entry* history,
    const uint32_t* info,
    const double* final_direction,
    uint32_t max_interactions
) {
    const size_t len = static_cast<size_t>(max_interactions) + 1;
    const int32_t num_leaves = static_cast<int32_t>(flat.leaf_entity.size());
    for (size_t i = 0; i < photons->size(); i++) {
        ml::Photon& photon = (*photons)[i];
        const uint32_t n_int = (info[i] >> 8) & 0xff;
        if (n_int < 1 || n_int > len)
            throw std::runtime_error("merlict_b200: engine history length out of range");
        const mlgpu_history_entry* h = &history[i*len];
        // entry 0 is the production the Photon's constructor already holds
        // (RayForPropagation.cpp:52-64)
        std::vector<ml::Intersection> rebuilt;
        rebuilt.reserve(n_int);
        for (uint32_t k = 1; k < n_int; k++) {
            if (h[k].leaf >= num_leaves || h[k].leaf < MLGPU_LEAF_VOID)
                throw std::runtime_error("merlict_b200: engine history names an unknown leaf");
            const ml::SurfaceEntity* object = h[k].leaf >= 0
                ? flat.leaf_entity[h[k].leaf] : &ml::VOID_SURFACE_ENTITY;
            const ml::Vec3 normal(h[k].normal[0], h[k].normal[1], h[k].normal[2]);
            // any incident direction with the recorded sign against the
            // normal gives the recorded side (Intersection.cpp:133-139)
            const ml::Vec3 incident = normal*(h[k].from_outside_to_inside ? -1.0 : 1.0);
            rebuilt.emplace_back(
                object,
                ml::Vec3(h[k].position[0], h[k].position[1], h[k].position[2]),
                normal, h[k].distance, incident);
        }
        for (uint32_t k = 1; k < n_int; k++)
            photon.push_back_intersection_and_interaction(
                rebuilt[k - 1], static_cast<ml::Interaction>(h[k].interaction));
        if (n_int > 1) {
            // The ray starts where its last step started: at the last
            // intersection when that step reflected or refracted, else at the
            // one before (every earlier step moved the ray on).
            const ml::Intersection* start = nullptr;
            if (moves_on(h[n_int - 1].interaction)) start = &rebuilt[n_int - 2];
            else if (n_int > 2) start = &rebuilt[n_int - 3];
            ml::Ray& ray = photon;
            if (start) ray.*member_of(RaySupport()) = start->position_in_root_frame();
            ray.*member_of(RayDirection()) = ml::Vec3(
                final_direction[3*i], final_direction[3*i + 1], final_direction[3*i + 2]);
        }
    }
}

}  // namespace merlict_b200
