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
    // page-locked staging of the host-buffer calls (grown as needed, kept
    // for the scene's lifetime), and the lock that serialises calls on the
    // scene (the engine's scene is not re-entrant)
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    std::mutex call;
};

// `bytes` of the scene's page-locked staging (its contents are not kept).
void* staging(DeviceScene* ds, size_t bytes) {
    if (bytes > ds->pinned_bytes) {
        void* old = ds->pinned;
        ds->pinned = nullptr;
        ds->pinned_bytes = 0;
        throw_on_error(mlgpu_host_free(old));
        const size_t grown = bytes + bytes/4;
        void* p = nullptr;
        throw_on_error(mlgpu_host_alloc(grown, &p));
        ds->pinned = p;
        ds->pinned_bytes = grown;
    }
    return ds->pinned;
}

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

// The photons' planes, written into `d` (7 n doubles: support x, y, z,
// direction x, y, z, wavelength) and `id` (n ints).
mlgpu_photons fill_planes(const std::vector<ml::Photon>& photons, double* d, int32_t* id) {
    const size_t n = photons.size();
    double* sx = d; double* sy = d + n; double* sz = d + 2*n;
    double* dx = d + 3*n; double* dy = d + 4*n; double* dz = d + 5*n;
    double* wavelength = d + 6*n;
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
    mlgpu_photons view;
    std::memset(&view, 0, sizeof(view));
    view.dtype = MLGPU_F64;
    view.support_x = sx; view.support_y = sy; view.support_z = sz;
    view.direction_x = dx; view.direction_y = dy; view.direction_z = dz;
    view.wavelength = wavelength;
    view.simulation_truth_id = id;
    return view;
}

struct PhotonPlanes {
    std::vector<double> planes;
    std::vector<int32_t> id;
    mlgpu_photons view;
    explicit PhotonPlanes(const std::vector<ml::Photon>& photons)
        : planes(7*photons.size()), id(photons.size()) {
        view = fill_planes(photons, planes.data(), id.data());
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
    std::lock_guard<std::mutex> lock(ds->call);
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
    std::lock_guard<std::mutex> lock(ds->call);
    const size_t n = photons->size();
    // inputs and results in page-locked staging, so that the engine moves
    // the batch in pieces whose copies overlap the tracing: 7 n doubles of
    // planes, 5 n doubles of results (x, y, t, theta x, theta y), n ids, n
    // sensors
    double* mem = static_cast<double*>(staging(ds, n*(12*sizeof(double) + 2*sizeof(int32_t))));
    double* out = mem + 7*n;
    int32_t* ids = reinterpret_cast<int32_t*>(out + 5*n);
    int32_t* sensor = ids + n;
    const mlgpu_photons view = fill_planes(*photons, mem, ids);
    const mlgpu_settings st = settings_for(ds, world, settings);
    const mlgpu_rng rng = rng_for(prng);
    const double* x = out;
    const double* y = out + n;
    const double* t = out + 2*n;
    const double* tx = out + 3*n;
    const double* ty = out + 4*n;
    mlgpu_results res;
    std::memset(&res, 0, sizeof(res));
    res.dtype = MLGPU_F64;
    res.sensor = sensor;
    res.x = out; res.y = out + n; res.time = out + 2*n;
    res.theta_x = out + 3*n; res.theta_y = out + 4*n;
    throw_on_error(mlgpu_propagate_host(ds->scene, &view, n, &st, &rng, &res));
    // Sensors::assign_photons order: photon by photon (Sensors.cpp:31-37).
    for (size_t i = 0; i < n; i++) {
        if (sensor[i] < 0) continue;
        ds->flat.sensor_of_index[sensor[i]]->photon_arrival_history.emplace_back(
            (*photons)[i].simulation_truth_id, (*photons)[i].wavelength,
            t[i], x[i], y[i], tx[i], ty[i]);
    }
}

}  // namespace merlict_b200
