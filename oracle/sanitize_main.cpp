// sanitize_main.cpp -- TEST INFRASTRUCTURE, not product code.
//
// The host code of the C++ drop-in -- the frame-tree flattener
// (merlict_b200_flatten.cpp) and the history rebuild
// (merlict_b200_history.cpp) -- built with AddressSanitizer and
// UndefinedBehaviorSanitizer (oracle/Makefile target `sanitize`) and run
// over the test scenes.  For each scene: build it with the reference's own
// classes, flatten it, propagate photons with merlict's Propagator on the
// engine's Philox streams, export every photon's history, rebuild fresh
// photons from that export (merlict_b200::rebuild_histories), let merlict's
// Sensors::assign_photons bin them, export again: both exports must be equal
// bit for bit.  Exit status 0: every scene round-tripped and no sanitizer
// fired (a sanitizer report aborts the program).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "merlict_b200.h"

extern "C" {
const char* ref_last_error(void);
void* ref_scene_build(const char* kind, const double* params, int num_params);
void ref_scene_free(void* handle);
int ref_scene_flat(void* handle, mlgpu_flat_scene* out);
int ref_propagate(void* handle, const mlgpu_photons* ph, uint64_t n, uint32_t max_interactions,
                  int mode, uint64_t seed, const double* uniforms, uint32_t stride,
                  int num_threads, mlgpu_results* out, double* seconds);
int ref_rebuild_photons(void* handle, const mlgpu_photons* ph, uint64_t n,
                        uint32_t max_interactions, const mlgpu_history_entry* history,
                        const uint32_t* info, const double* final_direction,
                        mlgpu_results* out);
uint64_t ref_last_supports(void* handle, double* out);
}

namespace {

struct Export {
    std::vector<int32_t> sensor, final_leaf;
    std::vector<double> x, y, time, tx, ty, final_position, final_direction, support;
    std::vector<uint32_t> info;
    std::vector<mlgpu_history_entry> history;
    mlgpu_results res;
    Export(uint64_t n, uint32_t max_int)
        : sensor(n), final_leaf(n), x(n), y(n), time(n), tx(n), ty(n),
          final_position(3*n), final_direction(3*n), support(3*n), info(n),
          history(n*(max_int + 1)) {
        std::memset(&res, 0, sizeof(res));
        res.dtype = MLGPU_F64;
        res.sensor = sensor.data(); res.final_leaf = final_leaf.data();
        res.x = x.data(); res.y = y.data(); res.time = time.data();
        res.theta_x = tx.data(); res.theta_y = ty.data(); res.info = info.data();
        res.final_position = final_position.data();
        res.final_direction = final_direction.data();
        res.history = history.data();
    }
};

bool same_bits(const void* a, const void* b, size_t bytes) { return std::memcmp(a, b, bytes) == 0; }

template <typename T>
bool same(const std::vector<T>& a, const std::vector<T>& b) {
    return a.size() == b.size() && same_bits(a.data(), b.data(), a.size()*sizeof(T));
}

// A small deterministic generator (SplitMix64) for the photon batch.
struct SplitMix {
    uint64_t s;
    double uniform() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30))*0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27))*0x94d049bb133111ebull;
        z ^= z >> 31;
        return static_cast<double>(z >> 11)*0x1.0p-53;
    }
};

// Photons from a sphere of 1.5 times the scene's bounding radius around its
// centre, aimed at random points inside the bounding sphere; or, with
// disc_radius > 0, from a disc of that radius at `height` going down within
// `zenith` radians of -z (the camera scenes' light).
void photons_for(const mlgpu_flat_scene& f, uint64_t n, uint64_t seed,
                 std::vector<std::vector<double>>* planes, double disc_radius = 0.0,
                 double height = 0.0, double zenith = 0.0) {
    const double cx = f.node_sphere[0], cy = f.node_sphere[1], cz = f.node_sphere[2];
    const double r = f.node_sphere[3] > 0.0 ? f.node_sphere[3] : 1.0;
    SplitMix g{seed};
    planes->assign(7, std::vector<double>(n));
    auto on_sphere = [&g](double* v) {
        const double z = 2.0*g.uniform() - 1.0, phi = 2.0*M_PI*g.uniform();
        const double q = std::sqrt(1.0 - z*z);
        v[0] = q*std::cos(phi); v[1] = q*std::sin(phi); v[2] = z;
    };
    for (uint64_t i = 0; i < n && disc_radius > 0.0; i++) {
        const double r_ = disc_radius*std::sqrt(g.uniform()), phi = 2.0*M_PI*g.uniform();
        const double cz_ = 1.0 - g.uniform()*(1.0 - std::cos(zenith)), az = 2.0*M_PI*g.uniform();
        const double sz_ = std::sqrt(1.0 - cz_*cz_);
        (*planes)[0][i] = r_*std::cos(phi);
        (*planes)[1][i] = r_*std::sin(phi);
        (*planes)[2][i] = height;
        (*planes)[3][i] = sz_*std::cos(az);
        (*planes)[4][i] = sz_*std::sin(az);
        (*planes)[5][i] = -cz_;
        (*planes)[6][i] = 300e-9 + 400e-9*g.uniform();
    }
    for (uint64_t i = 0; i < n && !(disc_radius > 0.0); i++) {
        double a[3], b[3];
        on_sphere(a);
        on_sphere(b);
        const double s[3] = {cx + 1.5*r*a[0], cy + 1.5*r*a[1], cz + 1.5*r*a[2]};
        const double u = 0.7*r*std::cbrt(g.uniform());
        const double t[3] = {cx + u*b[0], cy + u*b[1], cz + u*b[2]};
        double d[3] = {t[0] - s[0], t[1] - s[1], t[2] - s[2]};
        const double dn = std::sqrt(d[0]*d[0] + d[1]*d[1] + d[2]*d[2]);
        for (int k = 0; k < 3; k++) {
            (*planes)[k][i] = s[k];
            (*planes)[3 + k][i] = d[k]/dn;
        }
        (*planes)[6][i] = 300e-9 + 400e-9*g.uniform();
    }
}

int run_scene(const char* kind, const std::vector<double>& params, uint64_t n,
              uint32_t max_int, const std::vector<double>& disc = {}) {
    void* h = ref_scene_build(kind, params.data(), static_cast<int>(params.size()));
    if (!h) {
        std::fprintf(stderr, "%s: build failed: %s\n", kind, ref_last_error());
        return 1;
    }
    mlgpu_flat_scene flat;
    if (ref_scene_flat(h, &flat) != 0) {
        std::fprintf(stderr, "%s: flatten failed: %s\n", kind, ref_last_error());
        ref_scene_free(h);
        return 1;
    }
    std::vector<std::vector<double>> planes;
    if (disc.size() == 3) photons_for(flat, n, 12345, &planes, disc[0], disc[1], disc[2]);
    else photons_for(flat, n, 12345, &planes);
    mlgpu_photons ph;
    std::memset(&ph, 0, sizeof(ph));
    ph.dtype = MLGPU_F64;
    ph.support_x = planes[0].data(); ph.support_y = planes[1].data();
    ph.support_z = planes[2].data(); ph.direction_x = planes[3].data();
    ph.direction_y = planes[4].data(); ph.direction_z = planes[5].data();
    ph.wavelength = planes[6].data();

    Export a(n, max_int), b(n, max_int);
    double sec = 0.0;
    int st = ref_propagate(h, &ph, n, max_int, 0, 77, nullptr, 0, 1, &a.res, &sec);
    if (st == 0) ref_last_supports(h, a.support.data());
    if (st == 0)
        st = ref_rebuild_photons(h, &ph, n, max_int, a.history.data(), a.info.data(),
                                 a.final_direction.data(), &b.res);
    if (st == 0) ref_last_supports(h, b.support.data());
    if (st != 0) {
        std::fprintf(stderr, "%s: status %d: %s\n", kind, st, ref_last_error());
        ref_scene_free(h);
        return 1;
    }
    for (uint64_t i = 0; i < n; i++) a.info[i] &= 0xffffu;   // no uniform counts on rebuild
    const bool ok = same(a.sensor, b.sensor) && same(a.final_leaf, b.final_leaf) &&
        same(a.x, b.x) && same(a.y, b.y) && same(a.time, b.time) && same(a.tx, b.tx) &&
        same(a.ty, b.ty) && same(a.info, b.info) && same(a.final_position, b.final_position) &&
        same(a.final_direction, b.final_direction) && same(a.support, b.support) &&
        same(a.history, b.history);
    uint64_t on_sensor = 0, steps = 0;
    for (uint64_t i = 0; i < n; i++) {
        on_sensor += a.sensor[i] >= 0;
        steps += (a.info[i] >> 8) & 0xff;
    }
    std::printf("%-20s nodes %6d leaves %6d photons %llu on sensors %llu mean interactions "
                "%.2f round trip %s\n", kind, flat.num_nodes, flat.num_leaves,
                static_cast<unsigned long long>(n), static_cast<unsigned long long>(on_sensor),
                static_cast<double>(steps)/static_cast<double>(n), ok ? "ok" : "DIFFERS");
    ref_scene_free(h);
    return ok ? 0 : 1;
}

}  // namespace

int main() {
    int bad = 0;
    bad += run_scene("two_mirrors", {}, 2000, 50);
    bad += run_scene("mirror_absorber", {}, 2000, 5);
    bad += run_scene("water_box", {}, 2000, 10);
    bad += run_scene("absorbing_box", {}, 2000, 10);
    bad += run_scene("biconvex_lens", {}, 2000, 10);
    bad += run_scene("sphere", {}, 2000, 10);
    bad += run_scene("primitive_zoo", {}, 5000, 10);
    const double deg = M_PI/180.0;
    bad += run_scene("reflector_camera", {4.9, 1.0, 2.1, 0.0, 0.3, 0.01, 0.9, 1440, 0.0095, 0.2},
                     5000, 5, {2.0, 10.0, 1.5*deg});
    bad += run_scene("light_field_sensor", {10.7, 5.35, 1.0, 0.186, 9, 1.1, 0.9}, 5000, 10,
                     {5.55, 21.4, 0.5*deg});
    bad += run_scene("large_reflector", {106.5, 35.5, 0.0, 0.45, 0.01, 1.0, 0.06667, 0.9}, 5000,
                     5, {36.0, 110.0, 0.5*deg});
    std::printf("%s\n", bad ? "FAILED" : "all scenes round-tripped");
    return bad ? 1 : 0;
}
