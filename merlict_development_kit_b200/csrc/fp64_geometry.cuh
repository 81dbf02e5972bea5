// fp64_geometry.cuh -- merlict's per-photon geometry in double precision,
// shared by the FP64 tracers (trace_fp64.cu, wavefront_fp64.cu).  Include
// only from translation units compiled with --fmad=false: the operation
// order below is merlict's, and results are bit-identical to merlict's
// x86-64 build only without FMA contraction.
#ifndef MLGPU_FP64_GEOMETRY_CUH_
#define MLGPU_FP64_GEOMETRY_CUH_

#include <cstddef>
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace fp64 {
namespace {   // one copy per translation unit

struct v3 { double x, y, z; };

// Records a device-side error of a call in the scene's error word: the
// lowest non-zero status wins, so that a malformed photon
// (MLGPU_ERR_INVALID_ARGUMENT, which merlict throws from Photon's
// constructor before anything is propagated, Photon.cpp:20-28) is reported
// over the errors of photons traced beside it.
__device__ __forceinline__ void raise_error(unsigned int* word, unsigned int code) {
    unsigned int old = *reinterpret_cast<volatile unsigned int*>(word);
    while (old == 0u || old > code) {
        const unsigned int seen = atomicCAS(word, old, code);
        if (seen == old) break;
        old = seen;
    }
}

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

static __device__ __constant__ double IDENTITY[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};

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

// func_eval on one table of n (x, y, slope) points at `p`; the same
// arithmetic, so the same bits.
__device__ __forceinline__ double func_eval_points(const double* p, int32_t n, double x,
                                                   int* err) {
    if (x < p[0] || x >= p[3*(n - 1)]) {
        if (!*err) *err = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    int32_t first = 0, count = n;
    while (count > 0) {
        const int32_t step = count >> 1;
        const int32_t it = first + step;
        if (!(p[3*it] > x)) { first = it + 1; count -= step + 1; }
        else { count = step; }
    }
    if (first == 0 || (first == n && x > p[3*(n - 1)])) {
        if (!*err) *err = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    const double* p0 = p + 3*(first - 1);
    const double slope = p0[2];
    return slope*x + p0[1] - slope*p0[0];
}

// func_eval on tables at `pts` / `off` (a shared-memory copy, say).
__device__ double func_eval_tab(const double* pts, const int32_t* off, int32_t f, double x,
                                int* err) {
    const int32_t b = off[f];
    return func_eval_points(pts + 3*(size_t)b, off[f + 1] - b, x, err);
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

// ray_intersects_frames_bounding_sphere, merlict/RayAndFrame.cpp:16-107;
// sd = dot(s, d), which merlict recomputes for every frame (same value).
__device__ __forceinline__ bool sphere_cull(double4 nd, v3 s, v3 d, double sd) {
    const v3 c = mk(nd.x, nd.y, nd.z);
    const double alpha = dot(d, c) - sd;
    const v3 q = add(s, scale(d, alpha));
    const v3 sc = sub(c, q);
    if (dot(sc, sc) > nd.w) return false;
    if (alpha < 0.0) {
        const v3 w = sub(c, s);
        return dot(w, w) <= nd.w;
    }
    return true;
}

// Intersects one candidate leaf and keeps the closest hit.  Candidates of
// the frame-tree walk come in merlict's visiting order, so the strict "<"
// keeps the first minimum like min_element (RayAndFrame.cpp:160-173); for
// candidates in any other order, equal distances go to the leaf with the
// lower preorder index, which is the one merlict visits first.
__device__ __forceinline__ void test_candidate(const DevScene& sc, int32_t leaf, v3 s, v3 d,
                                               bool check_sphere, double sd, Isec* best,
                                               bool* have) {
    const LeafRec* L = sc.leaf + leaf;
    double T[12];
#pragma unroll
    for (int k = 0; k < 12; k++) T[k] = __ldg(&L->T[k]);
    const double r2 = __ldg(&L->r2);
    if (check_sphere && !sphere_cull(make_double4(T[3], T[7], T[11], r2), s, d, sd)) return;
    double ti[3], pr[MLGPU_LEAF_PARAMS];
#pragma unroll
    for (int k = 0; k < 3; k++) ti[k] = __ldg(&L->tinv[k]);
#pragma unroll
    for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) pr[k] = __ldg(&L->params[k]);
    const int32_t prim = __ldg(&L->primitive);
    Isec cand;
    intersect_leaf(sc, leaf, prim, pr, r2, position_inverse(T, ti, s),
                   orientation_inverse(T, d), &cand);
    if (cand.leaf >= 0 && (!*have || cand.dist < best->dist ||
                           (cand.dist == best->dist && cand.leaf < best->leaf))) {
        *best = cand;
        *have = true;
    }
}

// merlict's intersection of one leaf with a world ray; leaf < 0 if none.
// The leaf record in 16-byte loads: the first line (transform, inverse
// translation, primitive), the squared radius with the first parameter, and
// only as many further parameter pairs as the primitive has parameters --
// a warp whose lanes hold different leaves issues one request per lane and
// load, so every load left out counts.
static_assert(offsetof(LeafRec, tinv) == 96 && offsetof(LeafRec, primitive) == 120 &&
              offsetof(LeafRec, r2) == 128 && offsetof(LeafRec, params) == 136,
              "load_leaf reads the leaf record in 16-byte pieces");
__device__ __forceinline__ int primitive_params(int32_t prim) {
    switch (prim) {
    case MLGPU_PRIM_DISC: case MLGPU_PRIM_HEX_PLANE: case MLGPU_PRIM_SPHERE: return 1;
    case MLGPU_PRIM_SPHERE_CAP_HEX: case MLGPU_PRIM_SPHERE_CAP_CYL: case MLGPU_PRIM_PLANE:
    case MLGPU_PRIM_ANNULUS: case MLGPU_PRIM_CYLINDER: return 2;
    case MLGPU_PRIM_SPHERE_CAP_RECT: return 3;
    case MLGPU_PRIM_PLANE_DUAL_SPHERE: return 5;
    case MLGPU_PRIM_TRIANGLE: return 6;
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: return 7;
    default: return 0;
    }
}

__device__ __forceinline__ void load_leaf(const LeafRec* L, double* T, double* ti, double* pr,
                                          double* r2, int32_t* prim) {
    const double2* q = reinterpret_cast<const double2*>(L);
    double v[14];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double2 x = __ldg(q + k);
        v[2*k] = x.x;
        v[2*k + 1] = x.y;
    }
    const double2 tail = __ldg(q + 7);                     // tinv[2], primitive | sensor
    const double2 r2p0 = __ldg(q + 8);                     // r2, params[0]
#pragma unroll
    for (int k = 0; k < 12; k++) T[k] = v[k];
    ti[0] = v[12]; ti[1] = v[13]; ti[2] = tail.x;
    *prim = (int32_t)(uint32_t)(__double_as_longlong(tail.y) & 0xffffffffll);
    *r2 = r2p0.x;
    pr[0] = r2p0.y;
#pragma unroll
    for (int k = 1; k < MLGPU_LEAF_PARAMS; k++) pr[k] = 0.0;
    const int np = primitive_params(*prim);
    if (np > 1) { const double2 x = __ldg(q + 9); pr[1] = x.x; pr[2] = x.y; }
    if (np > 3) { const double2 x = __ldg(q + 10); pr[3] = x.x; pr[4] = x.y; }
    if (np > 5) { const double2 x = __ldg(q + 11); pr[5] = x.x; pr[6] = x.y; }
}

// load_leaf on the slot-ordered candidate records (DevScene::slot_rec):
// the same twelve pairs, the same selection by parameter count.
__device__ __forceinline__ void load_leaf_slot(const DevScene& sc, uint32_t j, double* T,
                                               double* ti, double* pr, double* r2,
                                               int32_t* prim) {
    const double2* q = sc.slot_rec + (size_t)(j >> 3)*96 + (j & 7);
    double v[14];
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const double2 x = __ldg(q + 8*k);
        v[2*k] = x.x;
        v[2*k + 1] = x.y;
    }
    const double2 tail = __ldg(q + 8*7);                   // tinv[2], primitive | sensor
    const double2 r2p0 = __ldg(q + 8*8);                   // r2, params[0]
#pragma unroll
    for (int k = 0; k < 12; k++) T[k] = v[k];
    ti[0] = v[12]; ti[1] = v[13]; ti[2] = tail.x;
    *prim = (int32_t)(uint32_t)(__double_as_longlong(tail.y) & 0xffffffffll);
    *r2 = r2p0.x;
    pr[0] = r2p0.y;
#pragma unroll
    for (int k = 1; k < MLGPU_LEAF_PARAMS; k++) pr[k] = 0.0;
    const int np = primitive_params(*prim);
    if (np > 1) { const double2 x = __ldg(q + 8*9); pr[1] = x.x; pr[2] = x.y; }
    if (np > 3) { const double2 x = __ldg(q + 8*10); pr[3] = x.x; pr[4] = x.y; }
    if (np > 5) { const double2 x = __ldg(q + 8*11); pr[5] = x.x; pr[6] = x.y; }
}

__device__ __forceinline__ Isec leaf_hit(const DevScene& sc, int32_t leaf, v3 s, v3 d) {
    double T[12], ti[3], pr[MLGPU_LEAF_PARAMS], r2;
    int32_t prim;
    load_leaf(sc.leaf + leaf, T, ti, pr, &r2, &prim);
    Isec h;
    intersect_leaf(sc, leaf, prim, pr, r2, position_inverse(T, ti, s), orientation_inverse(T, d),
                   &h);
    return h;
}

constexpr int kCandidates = 16;

__device__ __forceinline__ void set_void(Isec* is, v3 s, v3 d) {
    is->leaf = MLGPU_LEAF_VOID;
    is->pos = add(s, scale(d, 1e4));
    is->normal = d;
    is->dist = 1e4;
    is->outside = dot(d, d) < 0.0;
}

// CausalIntersection (merlict/RayAndFrame.cpp:126-173) over the subtree of
// `root`: nodes failing the bounding-sphere test are skipped with their
// subtree.  The walk only collects candidate leaves; they are intersected
// afterwards (or whenever the list is full), which keeps a warp's lanes
// together in the cheap walk instead of stalling on one lane's
// intersection.  The order, and so the result, is merlict's.
__device__ Isec first_intersection_tree(const DevScene& sc, int32_t root, v3 s, v3 d) {
    Isec best;
    best.leaf = -1;
    bool have = false;
    const double sd = dot(s, d);
    int32_t cand[kCandidates];
    int nc = 0;
    int32_t i = root;
    const int32_t end = __ldg(&sc.node_meta[root].x);
    while (i < end) {
        const double2* np = reinterpret_cast<const double2*>(sc.node + i);
        const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
        const int2 meta = __ldg(&sc.node_meta[i]);
        if (!sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, sd)) {
            i = meta.x;
            continue;
        }
        if (meta.y >= 0) {
            cand[nc++] = meta.y;
            if (nc == kCandidates) {
                for (int k = 0; k < nc; k++) test_candidate(sc, cand[k], s, d, false, sd, &best, &have);
                nc = 0;
            }
        }
        i++;
    }
    for (int k = 0; k < nc; k++) test_candidate(sc, cand[k], s, d, false, sd, &best, &have);
    if (!have) set_void(&best, s, d);
    return best;
}

// Candidates proposed by the BVH, each put through merlict's own test of
// the leaf's bounding sphere and merlict's intersection.  Returns false if
// the traversal stack would overflow (the caller then walks the frame tree).
__device__ bool first_intersection_bvh(const DevScene& sc, v3 s, v3 d, Isec* out) {
    Isec best;
    best.leaf = -1;
    bool have = false;
    const double sd = dot(s, d);
    {
        // merlict tests the root frame's own sphere first
        const double2* np = reinterpret_cast<const double2*>(sc.node);
        const double2 n01 = __ldg(np), n23 = __ldg(np + 1);
        if (!sphere_cull(make_double4(n01.x, n01.y, n23.x, n23.y), s, d, sd)) {
            set_void(out, s, d);
            return true;
        }
    }
    const float ox = (float)s.x, oy = (float)s.y, oz = (float)s.z;
    float fdx = (float)d.x, fdy = (float)d.y, fdz = (float)d.z;
    if (fabsf(fdx) < 1e-30f) fdx = copysignf(1e-30f, fdx);
    if (fabsf(fdy) < 1e-30f) fdy = copysignf(1e-30f, fdy);
    if (fabsf(fdz) < 1e-30f) fdz = copysignf(1e-30f, fdz);
    const float idx = 1.0f/fdx, idy = 1.0f/fdy, idz = 1.0f/fdz;
    const float eps = sc.bvh_eps + 4e-7f*(fabsf(ox) + fabsf(oy) + fabsf(oz));
    float tbest = INFINITY;
    int32_t stack[kBvhStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const int32_t ref = stack[--sp];
        if (ref < 0) {
            const int32_t start = (ref & 0x7fffffff) >> 3;
            const int32_t count = (ref & 7) + 1;
            for (int32_t j = 0; j < count; j++) {
                test_candidate(sc, __ldg(sc.bvh_leaf + start + j), s, d, true, sd, &best, &have);
                if (have) tbest = (float)best.dist*1.00001f + eps;
            }
            continue;
        }
        const float4* nq = reinterpret_cast<const float4*>(sc.bvh + ref);
        float tnear[kBvhWidth];
        int32_t cref[kBvhWidth];
        int nhit = 0;
#pragma unroll
        for (int g = 0; g < kBvhGroups; g++) {
            const float4 lx = __ldg(nq + g), ly = __ldg(nq + kBvhGroups + g);
            const float4 lz = __ldg(nq + 2*kBvhGroups + g), hx = __ldg(nq + 3*kBvhGroups + g);
            const float4 hy = __ldg(nq + 4*kBvhGroups + g), hz = __ldg(nq + 5*kBvhGroups + g);
            const int4 ch = __ldg(reinterpret_cast<const int4*>(nq + 6*kBvhGroups + g));
            const float lox[4] = {lx.x, lx.y, lx.z, lx.w}, loy[4] = {ly.x, ly.y, ly.z, ly.w};
            const float loz[4] = {lz.x, lz.y, lz.z, lz.w}, hix[4] = {hx.x, hx.y, hx.z, hx.w};
            const float hiy[4] = {hy.x, hy.y, hy.z, hy.w}, hiz[4] = {hz.x, hz.y, hz.z, hz.w};
            const int32_t child[4] = {ch.x, ch.y, ch.z, ch.w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const float ax = (lox[k] - eps - ox)*idx, bx = (hix[k] + eps - ox)*idx;
                const float ay = (loy[k] - eps - oy)*idy, by = (hiy[k] + eps - oy)*idy;
                const float az = (loz[k] - eps - oz)*idz, bz = (hiz[k] + eps - oz)*idz;
                const float tmin = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.0f));
                const float tmax = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), tbest));
                if (tmin <= tmax && child[k] != kBvhEmpty) {
                    tnear[nhit] = tmin;
                    cref[nhit] = child[k];
                    nhit++;
                }
            }
        }
        if (sp + nhit > kBvhStack) return false;
        // push far to near so that the nearest child is taken next
        for (int a = 0; a < nhit; a++) {
            int far = a;
            for (int b = a + 1; b < nhit; b++)
                if (tnear[b] > tnear[far]) far = b;
            const float tt = tnear[a]; tnear[a] = tnear[far]; tnear[far] = tt;
            const int32_t rr = cref[a]; cref[a] = cref[far]; cref[far] = rr;
            stack[sp++] = cref[a];
        }
    }
    if (!have) set_void(&best, s, d);
    *out = best;
    return true;
}


}  // namespace
}  // namespace fp64
}  // namespace mlgpu

#endif  // MLGPU_FP64_GEOMETRY_CUH_
