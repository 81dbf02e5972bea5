// merlict_b200_shim.cpp -- the drop-in propagation entry points declared
// in merlict_b200_shim.h: they flatten and upload a scene once per world
// frame (merlict_b200_flatten.cpp), call the engine's C ABI and rebuild the
// photons' histories (merlict_b200_history.cpp).
#include "merlict_b200_shim.h"

#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

namespace merlict_b200 {
namespace ml = merlict;

void throw_on_error(int status) {
    if (status == MLGPU_OK) return;
    char message[1024];
    mlgpu_last_error(message, sizeof(message));
    switch (status) {
    case MLGPU_ERR_INVALID_ARGUMENT: throw std::invalid_argument(message);
    case MLGPU_ERR_OUT_OF_RANGE: throw std::out_of_range(message);
    default: throw std::runtime_error(message);
    }
}

namespace {

struct DeviceScene {
    FlatScene flat;
    mlgpu_scene* scene = nullptr;
};

std::mutex cache_mutex;
std::map<std::pair<const ml::Frame*, const ml::sensor::Sensors*>, DeviceScene*> cache;

DeviceScene* scene_for(const ml::Frame* world, const ml::sensor::Sensors* sensors) {
    std::lock_guard<std::mutex> lock(cache_mutex);
    // the engine's structs must be the ones this file was compiled against
    if (mlgpu_abi_version() != MLGPU_ABI_VERSION)
        throw std::runtime_error(
            "merlict_b200: libmerlict_b200.so has ABI version " +
            std::to_string(mlgpu_abi_version()) + ", this drop-in was built for " +
            std::to_string(MLGPU_ABI_VERSION) + "; rebuild the drop-in");
    const auto key = std::make_pair(world->root(), sensors);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    DeviceScene* ds = new DeviceScene;
    ds->flat = flatten(world, sensors);
    const mlgpu_flat_scene view = ds->flat.view();
    const int status = mlgpu_scene_create(&view, &ds->scene);
    if (status != MLGPU_OK) {
        delete ds;
        throw_on_error(status);
    }
    cache[key] = ds;
    return ds;
}

struct PhotonPlanes {
    std::vector<double> sx, sy, sz, dx, dy, dz, wavelength;
    std::vector<int32_t> id;
    mlgpu_photons view;
    explicit PhotonPlanes(const std::vector<ml::Photon>& photons) {
        const size_t n = photons.size();
        sx.resize(n); sy.resize(n); sz.resize(n);
        dx.resize(n); dy.resize(n); dz.resize(n);
        wavelength.resize(n); id.resize(n);
        for (size_t i = 0; i < n; i++) {
            const ml::Photon& p = photons[i];
            if (p.num_interactions() != 1)
                throw std::invalid_argument(
                    "merlict_b200: photons must be fresh (only their production "
                    "interaction) when handed to the GPU engine.");
            sx[i] = p.support().x; sy[i] = p.support().y; sz[i] = p.support().z;
            dx[i] = p.direction().x; dy[i] = p.direction().y; dz[i] = p.direction().z;
            wavelength[i] = p.wavelength;
            id[i] = p.simulation_truth_id;
        }
        view.dtype = MLGPU_F64;
        view.support_x = sx.data(); view.support_y = sy.data(); view.support_z = sz.data();
        view.direction_x = dx.data(); view.direction_y = dy.data(); view.direction_z = dz.data();
        view.wavelength = wavelength.data();
        view.simulation_truth_id = id.data();
    }
};

mlgpu_settings settings_for(const DeviceScene* ds, const ml::Frame* world,
                            const ml::PropagationConfig* cfg) {
    mlgpu_settings st;
    std::memset(&st, 0, sizeof(st));
    st.max_num_interactions_per_photon = cfg->max_num_interactions_per_photon;
    st.start_node = ds->flat.node_index(world);
    st.tracer = MLGPU_TRACER_FP64;
    return st;
}

mlgpu_rng rng_for(ml::random::Generator* prng) {
    mlgpu_rng rng;
    std::memset(&rng, 0, sizeof(rng));
    rng.mode = MLGPU_RNG_PHILOX;
    rng.seed = prng->create_seed();
    return rng;
}

}  // namespace

void propagate_photons_in_frame_with_config(
    std::vector<ml::Photon>* photons,
    const ml::Frame* world,
    const ml::PropagationConfig* settings,
    ml::random::Generator* prng
) {
    if (photons->empty()) return;
    DeviceScene* ds = scene_for(world, nullptr);
    PhotonPlanes planes(*photons);
    const mlgpu_settings st = settings_for(ds, world, settings);
    const mlgpu_rng rng = rng_for(prng);
    const size_t n = photons->size();
    const size_t len = st.max_num_interactions_per_photon + 1;
    std::vector<mlgpu_history_entry> history(n*len);
    std::vector<int32_t> sensor(n);
    std::vector<uint32_t> info(n);
    std::vector<double> final_direction(3*n);
    mlgpu_results res;
    std::memset(&res, 0, sizeof(res));
    res.dtype = MLGPU_F64;
    res.sensor = sensor.data();
    res.info = info.data();
    res.final_direction = final_direction.data();
    res.history = history.data();
    throw_on_error(mlgpu_propagate_host(ds->scene, &planes.view, n, &st, &rng, &res));

    rebuild_histories(photons, ds->flat, history.data(), info.data(), final_direction.data(),
                      st.max_num_interactions_per_photon);
}

void propagate_photons_in_frame_with_config_multi_thread(
    std::vector<ml::Photon>* photons,
    const ml::Frame* world,
    const ml::PropagationConfig* settings,
    ml::random::Generator* prng
) {
    // qualified: argument-dependent lookup would also find merlict's own
    merlict_b200::propagate_photons_in_frame_with_config(photons, world, settings, prng);
}

void propagate_and_assign_photons(
    const std::vector<ml::Photon>* photons,
    const ml::Frame* world,
    const ml::PropagationConfig* settings,
    ml::random::Generator* prng,
    ml::sensor::Sensors* sensors
) {
    if (photons->empty()) return;
    DeviceScene* ds = scene_for(world, sensors);
    PhotonPlanes planes(*photons);
    const mlgpu_settings st = settings_for(ds, world, settings);
    const mlgpu_rng rng = rng_for(prng);
    const size_t n = photons->size();
    std::vector<int32_t> sensor(n);
    std::vector<double> x(n), y(n), t(n), tx(n), ty(n);
    mlgpu_results res;
    std::memset(&res, 0, sizeof(res));
    res.dtype = MLGPU_F64;
    res.sensor = sensor.data();
    res.x = x.data(); res.y = y.data(); res.time = t.data();
    res.theta_x = tx.data(); res.theta_y = ty.data();
    throw_on_error(mlgpu_propagate_host(ds->scene, &planes.view, n, &st, &rng, &res));
    // Sensors::assign_photons order: photon by photon (Sensors.cpp:31-37).
    for (size_t i = 0; i < n; i++) {
        if (sensor[i] < 0) continue;
        ds->flat.sensor_of_index[sensor[i]]->photon_arrival_history.emplace_back(
            (*photons)[i].simulation_truth_id, (*photons)[i].wavelength,
            t[i], x[i], y[i], tx[i], ty[i]);
    }
}

}  // namespace merlict_b200
