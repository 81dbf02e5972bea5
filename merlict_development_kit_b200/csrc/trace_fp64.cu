// trace_fp64.cu -- the plain FP64 tracer: one thread per photon, merlict's
// propagation state machine (merlict/PhotonAndFrame.cpp:13-124) with the
// frame-tree search of CausalIntersection (merlict/RayAndFrame.cpp:126-173)
// done as a stackless walk over the preorder node array.
//
// This translation unit is compiled with --fmad=false and without fast-math
// so that every add, multiply, divide and square root rounds exactly as in
// the reference's x86-64 build (no FMA contraction there either): given the
// same uniforms, photons end on the same surface with bit-identical
// positions, directions and times.  The only libm call on the path, exp()
// in the absorption test (PhotonAndFrame.cpp:32-38), may differ by one ulp
// from glibc; it is exactly 1 for merlict's default infinite absorption.
#include <cstdint>

#include "mlgpu_internal.h"
#include "merlict_b200_philox.h"

namespace mlgpu {
namespace {

struct v3 { double x, y, z; };

__device__ __forceinline__ v3 mk(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
// Vec3::operator*(Vec3), merlict/Vec3.cpp:35-37
__device__ __forceinline__ double dot(v3 self, v3 v) { return v.x*self.x + v.y*self.y + v.z*self.z; }
__device__ __forceinline__ v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 scale(v3 a, double s) { return mk(a.x*s, a.y*s, a.z*s); }
__device__ __forceinline__ v3 divide(v3 a, double s) { return mk(a.x/s, a.y/s, a.z/s); }
__device__ __forceinline__ double norm(v3 a) { return sqrt(a.x*a.x + a.y*a.y + a.z*a.z); }
__device__ __forceinline__ v3 normalized(v3 a) { return divide(a, norm(a)); }

// HomTra3 (merlict/HomTra3.cpp:154-216); T holds the three rows.
__device__ __forceinline__ v3 orientation(const double* t, v3 v) {
    return mk(v.x*t[0] + v.y*t[1] + v.z*t[2],
              v.x*t[4] + v.y*t[5] + v.z*t[6],
              v.x*t[8] + v.y*t[9] + v.z*t[10]);
}
__device__ __forceinline__ v3 orientation_inverse(const double* t, v3 v) {
    return mk(v.x*t[0] + v.y*t[4] + v.z*t[8],
              v.x*t[1] + v.y*t[5] + v.z*t[9],
              v.x*t[2] + v.y*t[6] + v.z*t[10]);
}
__device__ __forceinline__ v3 position(const double* t, v3 p) {
    return mk(p.x*t[0] + p.y*t[1] + p.z*t[2] + t[3],
              p.x*t[4] + p.y*t[5] + p.z*t[6] + t[7],
              p.x*t[8] + p.y*t[9] + p.z*t[10] + t[11]);
}
// position_inverse with the translation term precomputed on the host
__device__ __forceinline__ v3 position_inverse(const double* t, const double* ti, v3 p) {
    return mk(p.x*t[0] + p.y*t[4] + p.z*t[8] - ti[0],
              p.x*t[1] + p.y*t[5] + p.z*t[9] - ti[1],
              p.x*t[2] + p.y*t[6] + p.z*t[10] - ti[2]);
}

__device__ __constant__ double IDENTITY[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};

// Vec3::mirror, merlict/Vec3.cpp:59-113, operation order kept
__device__ __forceinline__ v3 mirror(v3 n, v3 r) {
    const double x = n.x, y = n.y, z = n.z;
    return mk(
        (1. - 2.*x*x) * r.x + - 2.*x*y * r.y + - 2.*x*z * r.z,
        - 2.*x*y * r.x + (1. - 2.*y*y) * r.y + - 2.*y*z * r.z,
        - 2.*x*z * r.x + - 2.*y*z * r.y + (1. - 2.*z*z) * r.z);
}

// Vec3 != (MAX_DEVIATION_EQUAL_VEC3_SQUARE, merlict/Vec3.h:45)
__device__ __forceinline__ bool differs(v3 a, v3 b) {
    const v3 d = sub(a, b);
    return dot(d, d) > 1e-14;
}

struct Isec {
    v3 pos;
    v3 normal;
    double dist;
    int32_t leaf;      // < 0: none
    bool outside;
};

// Func1::evaluate (merlict/function/Func1.cpp:66-71,118-130) with the range
// check of Limits::assert_contains (Limits.cpp:37-46); out-of-range raises
// MLGPU_ERR_OUT_OF_RANGE in *err and returns 0.
__device__ double func_eval(const DevScene& sc, int32_t f, double x, int* err) {
    const int32_t b = __ldg(sc.fn_offset + f);
    const int32_t n = __ldg(sc.fn_offset + f + 1) - b;
    const double* p = sc.fn_points + 3*(size_t)b;
    if (x < __ldg(p) || x >= __ldg(p + 3*(n - 1))) {
        if (!*err) *err = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    int32_t first = 0, count = n;
    while (count > 0) {
        const int32_t step = count >> 1;
        const int32_t it = first + step;
        if (!(__ldg(p + 3*it) > x)) { first = it + 1; count -= step + 1; }
        else { count = step; }
    }
    if (first == 0 || (first == n && x > __ldg(p + 3*(n - 1)))) {
        if (!*err) *err = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    const double* p0 = p + 3*(first - 1);
    const double slope = __ldg(p0 + 2);
    return slope*x + __ldg(p0 + 1) - slope*__ldg(p0);
}

// HexagonalPrismZ::is_inside, HexagonalPrismZ.cpp:14-30
__device__ __forceinline__ bool hex_inside(const DevScene& sc, double inner, v3 v) {
    const double u = dot(mk(sc.hex_u[0], sc.hex_u[1], sc.hex_u[2]), v);
    const double vv = dot(mk(sc.hex_v[0], sc.hex_v[1], sc.hex_v[2]), v);
    const double w = dot(mk(sc.hex_w[0], sc.hex_w[1], sc.hex_w[2]), v);
    return u < inner && u > -inner && vv < inner && vv > -inner && w < inner && w > -inner;
}

__device__ __forceinline__ bool cap_bound_inside(const DevScene& sc, int32_t prim,
                                                 const double* pr, v3 v) {
    switch (prim) {
    case MLGPU_PRIM_SPHERE_CAP_HEX: return hex_inside(sc, pr[1], v);
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: return hex_inside(sc, pr[6], v);
    case MLGPU_PRIM_SPHERE_CAP_CYL: return v.x*v.x + v.y*v.y < pr[1];
    case MLGPU_PRIM_SPHERE_CAP_RECT: return fabs(v.x) < pr[1] && fabs(v.y) < pr[2];
    default: return false;
    }
}

__device__ __forceinline__ v3 cap_normal(int32_t prim, const double* pr, v3 p) {
    if (prim == MLGPU_PRIM_ELLIPTIC_CAP_HEX) {
        // EllipticalCapRayIntersectionEquation.cpp:83-99 (y-term with iAA)
        const double ix = p.x, iy = p.y;
        const double f = pr[2] * 0.5 * sqrt(1.0 - (ix*ix)*pr[3] - (iy*iy)*pr[4]);
        const v3 n = mk(f*(-2.0*ix*pr[3]), f*(-2.0*iy*pr[3]), 1.0);
        return divide(n, norm(n));
    }
    const v3 n = sub(mk(0.0, 0.0, pr[0]), p);   // SphericalCapRayIntersectionEquation.cpp:51-57
    return divide(n, norm(n));
}

// QuadraticEquation, merlict/scenery/geometry/QuadraticEquation.cpp:12-30
__device__ __forceinline__ bool quadratic(double P, double Q, double* plus, double* minus) {
    const double p_over_2 = 0.5*P;
    const double inner = p_over_2*p_over_2 - Q;
    if (!(inner >= 0.0)) return false;
    const double sq = sqrt(inner);
    *minus = -p_over_2 - sq;
    *plus = -p_over_2 + sq;
    return true;
}

__device__ __forceinline__ void set_isec(Isec* r, int32_t leaf, v3 p, v3 n, double d, v3 inc) {
    r->leaf = leaf; r->pos = p; r->normal = n; r->dist = d;
    r->outside = dot(n, inc) < 0.0;
}

// SurfaceWithOuterPrismBound::add_causeal_intersection, SurfaceWithOuterPrismBound.cpp:7-70
__device__ void add_causal(const DevScene& sc, int32_t leaf, int32_t prim, const double* pr,
                           double r2, double plus, double minus, v3 s, v3 d, Isec* out) {
    const v3 pi = add(s, scale(d, plus));
    const v3 mi = add(s, scale(d, minus));
    const bool p_in = cap_bound_inside(sc, prim, pr, pi);
    const bool m_in = cap_bound_inside(sc, prim, pr, mi);
    const bool p_causal = plus > 0.0 && dot(pi, pi) <= r2;
    const bool m_causal = minus > 0.0 && dot(mi, mi) <= r2;
    double sol = minus;
    bool ok = false;
    if (p_in && m_in) {
        if (p_causal && m_causal) { sol = (minus >= plus) ? plus : minus; ok = true; }
        else if (p_causal) { sol = plus; ok = true; }
        else if (m_causal) { sol = minus; ok = true; }
    } else if (p_in && p_causal) {
        sol = plus; ok = true;
    } else if (m_in && m_causal) {
        sol = minus; ok = true;
    }
    if (ok) {
        const v3 p = add(s, scale(d, sol));
        if (differs(s, p)) set_isec(out, leaf, p, cap_normal(prim, pr, p), sol, d);
    }
}

__device__ __forceinline__ double tri_sign(v3 p1, double p2x, double p2y, double p3x, double p3y) {
    return (p1.x - p3x) * (p2y - p3y) - (p2x - p3x) * (p1.y - p3y);
}

// calculate_intersection_with of the leaf primitives
// (merlict/scenery/primitive), ray given in the leaf's frame.
__device__ void intersect_leaf(const DevScene& sc, int32_t leaf, int32_t prim,
                               const double* pr, double r2, v3 s, v3 d, Isec* out) {
    out->leaf = -1;
    switch (prim) {
    case MLGPU_PRIM_SPHERE_CAP_HEX:
    case MLGPU_PRIM_SPHERE_CAP_CYL:
    case MLGPU_PRIM_SPHERE_CAP_RECT: {
        const double R = pr[0];
        const double dd = dot(d, d), ss = dot(s, s), sd = dot(s, d);
        const double Rdz = R*d.z, Rsz = R*s.z;
        const double P = 2.0 * (sd - Rdz) / dd;
        const double Q = (ss - 2.0*Rsz) / dd;
        double plus, minus;
        if (quadratic(P, Q, &plus, &minus))
            add_causal(sc, leaf, prim, pr, r2, plus, minus, s, d, out);
        break;
    }
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: {
        const double C = pr[2], iAA = pr[3], iBB = pr[4], iCC = pr[5];
        const double a = (d.x*d.x)*iAA + (d.y*d.y)*iBB + (d.z*d.z)*iCC;
        const double b = 2.0*((s.x*d.x)*iAA + (s.y*d.y)*iBB + d.z*(s.z - C)*iCC);
        const double c = (s.x*s.x)*iAA + (s.y*s.y)*iBB + (s.z*s.z - 2.0*s.z*C)*iCC;
        double plus, minus;
        if (quadratic(b/a, c/a, &plus, &minus))
            add_causal(sc, leaf, prim, pr, r2, plus, minus, s, d, out);
        break;
    }
    case MLGPU_PRIM_DISC:
    case MLGPU_PRIM_HEX_PLANE:
    case MLGPU_PRIM_PLANE:
    case MLGPU_PRIM_ANNULUS:
    case MLGPU_PRIM_PLANE_DUAL_SPHERE:
    case MLGPU_PRIM_TRIANGLE: {
        // XyPlaneRayIntersectionEquation.cpp:6-40
        const bool parallel = d.z == 0. && (d.x != 0. || d.y != 0.);
        if (parallel) break;
        const double v = -s.z / d.z;
        if (!(v > 0.0)) break;
        const v3 p = add(s, scale(d, v));
        bool inside = false;
        switch (prim) {
        case MLGPU_PRIM_DISC: inside = p.x*p.x + p.y*p.y < pr[0]; break;
        case MLGPU_PRIM_HEX_PLANE: inside = hex_inside(sc, pr[0], p); break;
        case MLGPU_PRIM_PLANE: inside = fabs(p.x) < pr[0] && fabs(p.y) < pr[1]; break;
        case MLGPU_PRIM_ANNULUS:
            inside = (p.x*p.x + p.y*p.y < pr[0]) && !(p.x*p.x + p.y*p.y < pr[1]);
            break;
        case MLGPU_PRIM_PLANE_DUAL_SPHERE: {
            const double ax = pr[0] - p.x, ay = pr[1] - p.y;
            const double bx = pr[2] - p.x, by = pr[3] - p.y;
            const double r = pr[4];
            inside = (ax*ax + ay*ay <= r*r) && (bx*bx + by*by <= r*r);
            break;
        }
        default: {  // triangle, Triangle.cpp:92-103
            const bool bA = tri_sign(p, pr[0], pr[1], pr[2], pr[3]) < 0.0;
            const bool bB = tri_sign(p, pr[2], pr[3], pr[4], pr[5]) < 0.0;
            const bool bC = tri_sign(p, pr[4], pr[5], pr[0], pr[1]) < 0.0;
            inside = (bA == bB) && (bB == bC);
            break;
        }
        }
        if (inside && differs(s, p)) set_isec(out, leaf, p, mk(0.0, 0.0, 1.0), v, d);
        break;
    }
    case MLGPU_PRIM_CYLINDER: {
        // ZaxisCylinderRayIntersectionEquation.cpp:6-86, Cylinder.cpp:121-150
        const double radius = pr[0], length = pr[1];
        const double dx2 = d.x*d.x, dy2 = d.y*d.y;
        const double sxdx = s.x*d.x, sydy = s.y*d.y;
        const double sx2 = s.x*s.x, sy2 = s.y*s.y;
        const double r2c = radius*radius;
        const double dnom = dx2 + dy2;
        const double p = 2.0*(sxdx + sydy) / dnom;
        const double q = (sx2 + sy2 - r2c) / dnom;
        double plus, minus, v = 0.0;
        bool causal = false;
        if (quadratic(p, q, &plus, &minus)) {
            if (minus < 0.0 && plus >= 0.0) { causal = true; v = plus; }
            if (plus >= 0.0 && minus >= 0.0) { causal = true; v = minus; }
        }
        if (!causal) break;
        const v3 pt = add(s, scale(d, v));
        if (fabs(pt.z) <= length/2.0 && differs(s, pt)) {
            const v3 n = mk(pt.x, pt.y, 0.0);
            set_isec(out, leaf, pt, divide(n, norm(n)), v, d);
        }
        break;
    }
    case MLGPU_PRIM_SPHERE: {
        // Sphere.cpp:50-104
        const double radius = pr[0];
        const double sd = dot(s, d), dd = dot(d, d), ss = dot(s, s);
        const double r2s = radius*radius;
        double vP, vM;
        if (!quadratic(2*(sd / dd), ss/dd - r2s, &vP, &vM)) break;
        double v;
        if (vP >= 0.0 && vM >= 0.0) v = vM;
        else if (!(vP < 0.0 && vM < 0.0)) v = vP;
        else break;
        const v3 p = add(s, scale(d, v));
        if (differs(s, p)) set_isec(out, leaf, p, divide(p, norm(p)), v, d);
        break;
    }
    default:
        break;
    }
}

// ray_intersects_frames_bounding_sphere, merlict/RayAndFrame.cpp:16-107
__device__ __forceinline__ bool sphere_cull(double4 nd, v3 s, v3 d) {
    const v3 c = mk(nd.x, nd.y, nd.z);
    const double alpha = dot(d, c) - dot(s, d);
    const v3 q = add(s, scale(d, alpha));
    const v3 sc = sub(c, q);
    if (dot(sc, sc) > nd.w) return false;
    if (alpha < 0.0) {
        const v3 w = sub(c, s);
        return dot(w, w) <= nd.w;
    }
    return true;
}

// CausalIntersection (merlict/RayAndFrame.cpp:126-173) over the subtree of
// `root`: nodes failing the bounding-sphere test are skipped with their
// subtree, leaves are intersected in visiting order and the first minimum
// distance wins.
__device__ Isec first_intersection(const DevScene& sc, int32_t root, v3 s, v3 d) {
    Isec best;
    best.leaf = -1;
    bool have = false;
    int32_t i = root;
    const int32_t end = __ldg(&sc.node_meta[root].x);
    while (i < end) {
        const double2* np = reinterpret_cast<const double2*>(sc.node + i);
        const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
        const double4 nd = make_double4(n01.x, n01.y, n23.x, n23.y);
        const int2 meta = __ldg(&sc.node_meta[i]);
        if (!sphere_cull(nd, s, d)) { i = meta.x; continue; }
        if (meta.y >= 0) {
            const LeafRec* L = sc.leaf + meta.y;
            double T[12], ti[3], pr[MLGPU_LEAF_PARAMS];
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = __ldg(&L->T[k]);
#pragma unroll
            for (int k = 0; k < 3; k++) ti[k] = __ldg(&L->tinv[k]);
#pragma unroll
            for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) pr[k] = __ldg(&L->params[k]);
            const int32_t prim = __ldg(&L->primitive);
            const v3 so = position_inverse(T, ti, s);
            const v3 dobj = orientation_inverse(T, d);
            Isec cand;
            intersect_leaf(sc, meta.y, prim, pr, nd.w, so, dobj, &cand);
            if (cand.leaf >= 0 && (!have || cand.dist < best.dist)) {
                best = cand;
                have = true;
            }
        }
        i++;
    }
    if (!have) {
        best.leaf = MLGPU_LEAF_VOID;
        best.pos = add(s, scale(d, 1e4));
        best.normal = d;
        best.dist = 1e4;
        best.outside = dot(d, d) < 0.0;
    }
    return best;
}

template <typename T>
__device__ __forceinline__ double load_in(const void* p, uint64_t i) {
    return (double)__ldg(static_cast<const T*>(p) + i);
}

__device__ __forceinline__ void store_hist(mlgpu_history_entry* h, const Isec& is, int kind) {
    h->position[0] = is.pos.x; h->position[1] = is.pos.y; h->position[2] = is.pos.z;
    h->normal[0] = is.normal.x; h->normal[1] = is.normal.y; h->normal[2] = is.normal.z;
    h->distance = is.dist;
    h->leaf = is.leaf;
    h->interaction = (uint8_t)kind;
    h->from_outside_to_inside = (uint8_t)is.outside;
    h->pad[0] = 0; h->pad[1] = 0;
}

template <typename In, typename Out>
__global__ void __launch_bounds__(128)
trace_fp64_kernel(const TraceArgs a) {
    const DevScene& sc = a.scene;
    const uint64_t i = (uint64_t)blockIdx.x*blockDim.x + threadIdx.x;
    if (i >= a.num_photons) return;
    const uint32_t max_int = a.max_interactions;
    mlgpu_history_entry* hist =
        a.results.history ? a.results.history + i*(uint64_t)(max_int + 1) : nullptr;

    const double lambda = load_in<In>(a.photons.wavelength, i);
    const v3 s0 = mk(load_in<In>(a.photons.sx, i), load_in<In>(a.photons.sy, i),
                     load_in<In>(a.photons.sz, i));
    v3 s = s0;
    // Ray::set_support_and_direction normalises (Ray.cpp:16-20)
    v3 d = normalized(mk(load_in<In>(a.photons.dx, i), load_in<In>(a.photons.dy, i),
                         load_in<In>(a.photons.dz, i)));
    Isec last;
    last.leaf = MLGPU_LEAF_PHOTON_SOURCE; last.pos = s; last.normal = d; last.dist = 0.0;
    last.outside = dot(d, d) < 0.0;
    if (hist) store_hist(&hist[0], last, MLGPU_PRODUCTION);
    v3 last_world = position(IDENTITY, s0);
    v3 second_last_world = last_world;
    uint32_t n_int = 1;
    int interaction = MLGPU_PRODUCTION;
    int32_t root = a.start_node;
    double tof = 0.0;
    int tof_error = 0;
    int err = 0;
    uint32_t k_draw = 0;
    const uint64_t stream = a.rng.photon_offset + i;

    auto draw = [&]() -> double {
        const uint32_t k = k_draw++;
        if (a.rng.mode == MLGPU_RNG_REPLAY) {
            if (k >= a.rng.stride) { if (!err) err = MLGPU_ERR_RUNTIME; return 0.5; }
            return __ldg(a.rng.uniforms + i*(uint64_t)a.rng.stride + k);
        }
        return mlgpu_philox_uniform(a.rng.seed, stream, k);
    };

    while (n_int <= max_int) {
        const Isec is = first_intersection(sc, root, s, d);
        const bool hit = is.leaf >= 0;
        const LeafRec* L = hit ? sc.leaf + is.leaf : nullptr;
        double T[12];
        if (hit) {
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = __ldg(&L->T[k]);
        } else {
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = IDENTITY[k];
        }
        int32_t fn[6] = {0, 0, 0, 0, 0, 0};
        int32_t flags = 0, allowed = -1;
        if (hit) {
#pragma unroll
            for (int k = 0; k < 6; k++) fn[k] = __ldg(&L->fn[k]);
            flags = __ldg(&L->flags);
            allowed = __ldg(&L->allowed_node);
        }
        bool absorbed = false;
        if (hit) {
            const double depth = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_ABSORPTION
                                                              : MLGPU_SURF_INNER_ABSORPTION], lambda, &err);
            const double survival = exp(-is.dist/depth);
            absorbed = draw() > survival;
        }
        int kind;
        bool moved = false;
        v3 new_s = s, new_d = d;
        if (!hit || absorbed) {
            kind = MLGPU_ABSORPTION_IN_VOID;
        } else {
            const double refl = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFLECTION
                                                             : MLGPU_SURF_INNER_REFLECTION], lambda, &err);
            if (refl >= draw()) {
                kind = MLGPU_REFLECTION_ON_SURFACE;
                new_s = position(T, is.pos);
                new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                moved = true;
            } else if (!(flags & MLGPU_FLAG_TRANSPARENT)) {
                kind = MLGPU_ABSORPTION_ON_SURFACE;
            } else {
                // Fresnel, merlict/Fresnel.cpp:7-38
                const v3 inc = orientation_inverse(T, d);
                const v3 nrm = is.outside ? is.normal : scale(is.normal, -1.0);
                const double n_from = func_eval(sc, fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION
                                                                   : MLGPU_SURF_INNER_REFRACTION], lambda, &err);
                const double n_to = func_eval(sc, fn[is.outside ? MLGPU_SURF_INNER_REFRACTION
                                                                 : MLGPU_SURF_OUTER_REFRACTION], lambda, &err);
                const double cosI = dot(nrm, inc)*(-1.0);
                const double ratio = n_from/n_to;
                const double sinT2 = ratio*ratio*(1.0 - cosI*cosI);
                const double cosT = sqrt(1.0 - sinT2);
                double R;
                if (sinT2 > 1.0) {
                    R = 1.0;
                } else {
                    const double rOrth = (n_from*cosI - n_to*cosT) / (n_from*cosI + n_to*cosT);
                    const double rPar = (n_to*cosI - n_from*cosT) / (n_to*cosI + n_from*cosT);
                    R = (rOrth*rOrth + rPar*rPar) / 2.0;
                }
                if (R > draw()) {
                    kind = MLGPU_FRESNEL_REFLECTION_ON_SURFACE;
                    new_s = position(T, is.pos);
                    new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                    moved = true;
                } else {
                    kind = is.outside ? MLGPU_REFRACTION_TO_INSIDE : MLGPU_REFRACTION_TO_OUTSIDE;
                    const bool to_default = is.outside
                        ? (flags & MLGPU_FLAG_INNER_REFRACTION_DEFAULT) != 0
                        : (flags & MLGPU_FLAG_OUTER_REFRACTION_DEFAULT) != 0;
                    root = (allowed >= 0 && !to_default) ? allowed : 0;
                    const v3 refr = add(scale(inc, ratio), scale(nrm, ratio*cosI - cosT));
                    new_s = position(T, is.pos);
                    new_d = normalized(orientation(T, refr));
                    moved = true;
                }
            }
        }
        if (hist) store_hist(&hist[n_int], is, kind);
        {
            // time-of-flight term, merlict/Photon.cpp:37-56
            const int32_t f = hit
                ? fn[is.outside ? MLGPU_SURF_OUTER_REFRACTION : MLGPU_SURF_INNER_REFRACTION]
                : sc.default_refraction;
            int terr = 0;
            const double n = func_eval(sc, f, lambda, &terr);
            if (terr && !tof_error) tof_error = terr;
            tof += n*is.dist/299792458.0;
        }
        second_last_world = last_world;
        last_world = moved ? new_s : position(T, is.pos);
        n_int++;
        interaction = kind;
        last = is;
        if (!moved) break;
        s = new_s;
        d = new_d;
    }
    if (hist) {
        for (uint32_t k = n_int; k < max_int + 1; k++) {
            mlgpu_history_entry* h = &hist[k];
            h->position[0] = 0; h->position[1] = 0; h->position[2] = 0;
            h->normal[0] = 0; h->normal[1] = 0; h->normal[2] = 0;
            h->distance = 0; h->leaf = MLGPU_LEAF_PHOTON_SOURCE;
            h->interaction = 0; h->from_outside_to_inside = 0; h->pad[0] = 0; h->pad[1] = 0;
        }
    }
    const int32_t sensor = last.leaf >= 0 ? __ldg(&sc.leaf[last.leaf].sensor) : -1;
    if (sensor >= 0 && tof_error && !err) err = tof_error;

    // final_intersection_incident_direction_wrt_frame, RayForPropagation.cpp:114-136
    v3 inc = mk(0.0, 0.0, 0.0);
    if (n_int > 1) {
        const v3 w = normalized(sub(last_world, second_last_world));
        if (last.leaf >= 0) {
            double T[12];
#pragma unroll
            for (int k = 0; k < 12; k++) T[k] = __ldg(&sc.leaf[last.leaf].T[k]);
            inc = orientation_inverse(T, w);
        } else {
            inc = orientation_inverse(IDENTITY, w);
        }
    }
    const DevResults& r = a.results;
    r.sensor[i] = sensor;
    if (r.x) static_cast<Out*>(r.x)[i] = (Out)last.pos.x;
    if (r.y) static_cast<Out*>(r.y)[i] = (Out)last.pos.y;
    if (r.time) r.time[i] = tof;
    if (r.theta_x) static_cast<Out*>(r.theta_x)[i] = (Out)(-1.0*inc.x);
    if (r.theta_y) static_cast<Out*>(r.theta_y)[i] = (Out)(-1.0*inc.y);
    if (r.final_leaf) r.final_leaf[i] = last.leaf;
    if (r.info)
        r.info[i] = (uint32_t)interaction | (n_int << 8) |
            ((k_draw > 255u ? 255u : k_draw) << 16) | ((uint32_t)err << 24);
    if (r.final_position) {
        r.final_position[3*i] = last_world.x;
        r.final_position[3*i + 1] = last_world.y;
        r.final_position[3*i + 2] = last_world.z;
    }
    if (r.final_direction) {
        r.final_direction[3*i] = d.x;
        r.final_direction[3*i + 1] = d.y;
        r.final_direction[3*i + 2] = d.z;
    }
    if (err) atomicCAS(sc.error_word, 0u, (unsigned int)err);
}

}  // namespace

cudaError_t launch_trace_fp64(const TraceArgs& a, int block, cudaStream_t s) {
    if (a.num_photons == 0) return cudaSuccess;
    block = 128;
    const uint64_t grid = (a.num_photons + block - 1) / block;
    if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F64)
        trace_fp64_kernel<double, double><<<(unsigned)grid, block, 0, s>>>(a);
    else if (a.in_dtype == MLGPU_F32 && a.out_dtype == MLGPU_F64)
        trace_fp64_kernel<float, double><<<(unsigned)grid, block, 0, s>>>(a);
    else if (a.in_dtype == MLGPU_F64 && a.out_dtype == MLGPU_F32)
        trace_fp64_kernel<double, float><<<(unsigned)grid, block, 0, s>>>(a);
    else
        trace_fp64_kernel<float, float><<<(unsigned)grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace mlgpu
