/*
 * merlict_oracle.c -- TEST INFRASTRUCTURE, not product code.
 *
 * CPU restatement, in plain C, of merlict's per-photon propagation and of
 * the sensor attribution that follows it, operating on the flattened scene
 * of include/merlict_b200.h.  It is the checker the CUDA tracer is compared
 * against (and the "port" CPU baseline); the product never links it.
 *
 * Parity pin: tests/test_oracle_golden.py compares this file, photon by
 * photon and bit for bit, with the reference library itself (built from
 * the reference sources by oracle/Makefile) on the scenes and uniform
 * streams stored in tests/golden/.
 *
 * Every function names the reference file:line it follows.  Arithmetic is
 * written in the reference's operation order so that, compiled without
 * floating-point contraction (-ffp-contract=off), results agree bit for bit.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "merlict_b200.h"
#include "merlict_b200_philox.h"

/* counters of the operations weighted by the FLOP model of the bench */
typedef struct oracle_counters {
    uint64_t nodes;        /* bounding-sphere tests, RayAndFrame.cpp:16-107 */
    uint64_t leaves;       /* leaf world->object transforms, HomTra3.cpp:170-216 */
    uint64_t caps;         /* cap quadratics, SphericalCapRayIntersectionEquation.cpp:19-37 */
    uint64_t cap_bounds;   /* causal cap-bound evaluations, SurfaceWithOuterPrismBound.cpp:13-68 */
    uint64_t planes;       /* plane-family hit + bound */
    uint64_t others;       /* cylinder, sphere, ellipsoid, triangle tests */
    uint64_t reflections;  /* PhotonAndFrame.cpp:56-66 */
    uint64_t fresnels;     /* PhotonAndFrame.cpp:75-118 */
    uint64_t segments;     /* time-of-flight segments, Photon.cpp:44-56 */
    uint64_t funcs;        /* Func1 evaluations */
    uint64_t steps;        /* propagation steps */
    /* steps by the number of leaves merlict intersects in them: [k] for k
     * leaves, [64] for 64 or more */
    uint64_t leaves_per_step[65];
} oracle_counters;

typedef struct { double x, y, z; } v3;

static v3 mk(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }

/* Vec3::operator*(Vec3), merlict/Vec3.cpp:35-37: v.x*x + v.y*y + v.z*z */
static double dot(v3 self, v3 v) { return v.x*self.x + v.y*self.y + v.z*self.z; }
static v3 add(v3 a, v3 b) { return mk(a.x+b.x, a.y+b.y, a.z+b.z); }   /* Vec3.cpp:47-49 */
static v3 sub(v3 a, v3 b) { return mk(a.x-b.x, a.y-b.y, a.z-b.z); }   /* Vec3.cpp:43-45 */
static v3 scale(v3 a, double s) { return mk(a.x*s, a.y*s, a.z*s); }   /* Vec3.cpp:39-41 */
static v3 divide(v3 a, double s) { return mk(a.x/s, a.y/s, a.z/s); }  /* Vec3.cpp:51-53 */
static double norm(v3 a) { return sqrt(a.x*a.x + a.y*a.y + a.z*a.z); } /* Vec3.cpp:23-25 */
static v3 normalized(v3 a) { return divide(a, norm(a)); }             /* Vec3.cpp:19-21 */

/* HomTra3, merlict/HomTra3.cpp:154-216; t holds the rows of T[3][4] */
static v3 orientation(const double* t, v3 v) {
    return mk(v.x*t[0] + v.y*t[1] + v.z*t[2],
              v.x*t[4] + v.y*t[5] + v.z*t[6],
              v.x*t[8] + v.y*t[9] + v.z*t[10]);
}
static v3 orientation_inverse(const double* t, v3 v) {
    return mk(v.x*t[0] + v.y*t[4] + v.z*t[8],
              v.x*t[1] + v.y*t[5] + v.z*t[9],
              v.x*t[2] + v.y*t[6] + v.z*t[10]);
}
static v3 position(const double* t, v3 p) {
    return mk(p.x*t[0] + p.y*t[1] + p.z*t[2] + t[3],
              p.x*t[4] + p.y*t[5] + p.z*t[6] + t[7],
              p.x*t[8] + p.y*t[9] + p.z*t[10] + t[11]);
}
static v3 position_inverse(const double* t, v3 p) {
    return mk(
        p.x*t[0] + p.y*t[4] + p.z*t[8] - (t[0]*t[3] + t[4]*t[7] + t[8]*t[11]),
        p.x*t[1] + p.y*t[5] + p.z*t[9] - (t[1]*t[3] + t[5]*t[7] + t[9]*t[11]),
        p.x*t[2] + p.y*t[6] + p.z*t[10] - (t[2]*t[3] + t[6]*t[7] + t[10]*t[11]));
}
static const double IDENTITY[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};

/* Vec3::mirror, merlict/Vec3.cpp:59-113 (operation order kept) */
static v3 mirror(v3 n, v3 r) {
    const double x = n.x, y = n.y, z = n.z;
    return mk(
        (1. - 2.*x*x) * r.x + - 2.*x*y * r.y + - 2.*x*z * r.z,
        - 2.*x*y * r.x + (1. - 2.*y*y) * r.y + - 2.*y*z * r.z,
        - 2.*x*z * r.x + - 2.*y*z * r.y + (1. - 2.*z*z) * r.z);
}

/* Vec3 != with MAX_DEVIATION_EQUAL_VEC3_SQUARE, Vec3.h:45, Vec3.cpp:121-127 */
static int differs(v3 a, v3 b) {
    const v3 d = sub(a, b);
    return dot(d, d) > 1e-14;
}

typedef struct {
    const mlgpu_flat_scene* s;
    int error;                 /* first MLGPU_ERR_* raised for this photon */
    oracle_counters* cnt;
} ctx;

/* Func1::evaluate, merlict/function/Func1.cpp:66-71,118-130 and
 * Limits::assert_contains, merlict/function/Limits.cpp:37-46 */
static double func_eval(ctx* c, int32_t f, double x) {
    const double* p = c->s->function_points + 3*(size_t)c->s->function_offset[f];
    const int32_t n = c->s->function_offset[f + 1] - c->s->function_offset[f];
    if (c->cnt) c->cnt->funcs++;
    if (x < p[0] || x >= p[3*(n - 1)]) {
        if (!c->error) c->error = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    /* std::upper_bound with comp_upp: first point with P.x > x */
    int32_t first = 0, count = n;
    while (count > 0) {
        const int32_t step = count/2;
        const int32_t it = first + step;
        if (!(p[3*it] > x)) { first = it + 1; count -= step + 1; }
        else { count = step; }
    }
    if (first == 0 || (first == n && x > p[3*(n - 1)])) {
        if (!c->error) c->error = MLGPU_ERR_OUT_OF_RANGE;
        return 0.0;
    }
    const double* p0 = p + 3*(first - 1);
    return p0[2]*x + p0[1] - p0[2]*p0[0];
}

typedef struct {
    int hit;          /* does_intersect(), Intersection.cpp:36-38 */
    int32_t leaf;
    v3 pos;           /* object frame */
    v3 normal;        /* object frame */
    double dist;
    int outside;      /* from_outside_to_inside, Intersection.cpp:133-139 */
} isec_t;

static void set_isec(isec_t* r, int32_t leaf, v3 p, v3 n, double d, v3 inc) {
    r->hit = 1; r->leaf = leaf; r->pos = p; r->normal = n; r->dist = d;
    r->outside = dot(n, inc) < 0.0;
}

/* hexagonal prism bound, HexagonalPrismZ.cpp:14-30 */
static int hex_inside(const mlgpu_flat_scene* s, double inner, v3 v) {
    const double u = dot(mk(s->hex_unit_u[0], s->hex_unit_u[1], s->hex_unit_u[2]), v);
    const double vv = dot(mk(s->hex_unit_v[0], s->hex_unit_v[1], s->hex_unit_v[2]), v);
    const double w = dot(mk(s->hex_unit_w[0], s->hex_unit_w[1], s->hex_unit_w[2]), v);
    return u < inner && u > -inner && vv < inner && vv > -inner &&
        w < inner && w > -inner;
}

/* the bound of a cap leaf, PrismZ::is_inside of its kind */
static int cap_bound_inside(const mlgpu_flat_scene* s, int32_t prim,
                            const double* pr, v3 v) {
    switch (prim) {
    case MLGPU_PRIM_SPHERE_CAP_HEX: return hex_inside(s, pr[1], v);
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: return hex_inside(s, pr[6], v);
    case MLGPU_PRIM_SPHERE_CAP_CYL: return v.x*v.x + v.y*v.y < pr[1];  /* CylinderPrismZ.cpp:13-15 */
    case MLGPU_PRIM_SPHERE_CAP_RECT:                                    /* RectangularPrismZ.cpp:41-43 */
        return fabs(v.x) < pr[1] && fabs(v.y) < pr[2];
    default: return 0;
    }
}

static v3 cap_normal(int32_t prim, const double* pr, v3 p) {
    if (prim == MLGPU_PRIM_ELLIPTIC_CAP_HEX) {
        /* EllipticalCapRayIntersectionEquation.cpp:83-99, y-term with iAA as in the reference */
        const double ix = p.x, iy = p.y;
        const double f = pr[2] * 0.5 * sqrt(1.0 - (ix*ix)*pr[3] - (iy*iy)*pr[4]);
        const v3 n = mk(f*(-2.0*ix*pr[3]), f*(-2.0*iy*pr[3]), 1.0);
        return divide(n, norm(n));
    }
    /* SphericalCapRayIntersectionEquation.cpp:51-57 */
    const v3 n = sub(mk(0.0, 0.0, pr[0]), p);
    return divide(n, norm(n));
}

/* SurfaceWithOuterPrismBound::add_causeal_intersection,
 * merlict/scenery/geometry/SurfaceWithOuterPrismBound.cpp:7-70 */
static void add_causal(ctx* c, int32_t leaf, int32_t prim, const double* pr,
                       double bsr, double plus, double minus, v3 s, v3 d,
                       isec_t* out) {
    const mlgpu_flat_scene* sc = c->s;
    const v3 pi = add(s, scale(d, plus));
    const v3 mi = add(s, scale(d, minus));
    const int p_in = cap_bound_inside(sc, prim, pr, pi);
    const int m_in = cap_bound_inside(sc, prim, pr, mi);
    const int p_causal = plus > 0.0 && dot(pi, pi) <= bsr*bsr;
    const int m_causal = minus > 0.0 && dot(mi, mi) <= bsr*bsr;
    double sol = minus;
    int ok = 0;
    if (c->cnt) c->cnt->cap_bounds++;
    if (p_in && m_in) {
        if (p_causal && m_causal) {
            sol = (minus >= plus) ? plus : minus;
            ok = 1;
        } else if (p_causal) {
            sol = plus; ok = 1;
        } else if (m_causal) {
            sol = minus; ok = 1;
        }
    } else if (p_in && p_causal) {
        sol = plus; ok = 1;
    } else if (m_in && m_causal) {
        sol = minus; ok = 1;
    }
    if (ok) {
        const v3 p = add(s, scale(d, sol));
        if (differs(s, p))
            set_isec(out, leaf, p, cap_normal(prim, pr, p), sol, d);
    }
}

/* QuadraticEquation, merlict/scenery/geometry/QuadraticEquation.cpp:12-30 */
static int quadratic(double P, double Q, double* plus, double* minus) {
    const double p_over_2 = 0.5*P;
    const double inner = p_over_2*p_over_2 - Q;
    if (!(inner >= 0.0)) return 0;
    const double sq = sqrt(inner);
    *minus = -p_over_2 - sq;
    *plus = -p_over_2 + sq;
    return 1;
}

/* XyPlaneRayIntersectionEquation.cpp:6-40 */
static int xy_plane(v3 s, v3 d, double* v) {
    const int parallel = d.z == 0. && (d.x != 0. || d.y != 0.);  /* Vec3.cpp:133-135 */
    if (parallel) return 0;
    *v = -s.z / d.z;
    return *v > 0.0;
}

/* Triangle::sign / is_inside_triangle, primitive/Triangle.cpp:92-103 */
static double tri_sign(v3 p1, double p2x, double p2y, double p3x, double p3y) {
    return (p1.x - p3x) * (p2y - p3y) - (p2x - p3x) * (p1.y - p3y);
}

/* Leaf's calculate_intersection_with (merlict/scenery/primitive/ *.cpp) on
 * the ray already transformed into the leaf's frame. */
static void intersect_leaf(ctx* c, int32_t leaf, v3 s, v3 d, double bsr,
                           isec_t* out) {
    const mlgpu_flat_scene* sc = c->s;
    const int32_t prim = sc->leaf_primitive[leaf];
    const double* pr = sc->leaf_params + (size_t)MLGPU_LEAF_PARAMS*leaf;
    out->hit = 0;
    switch (prim) {
    case MLGPU_PRIM_SPHERE_CAP_HEX:
    case MLGPU_PRIM_SPHERE_CAP_CYL:
    case MLGPU_PRIM_SPHERE_CAP_RECT: {
        /* SphericalCapRayIntersectionEquation.cpp:6-42 */
        const double R = pr[0];
        const double dd = dot(d, d), ss = dot(s, s), sd = dot(s, d);
        const double Rdz = R*d.z, Rsz = R*s.z;
        const double P = 2.0 * (sd - Rdz) / dd;
        const double Q = (ss - 2.0*Rsz) / dd;
        double plus, minus;
        if (c->cnt) c->cnt->caps++;
        if (quadratic(P, Q, &plus, &minus))
            add_causal(c, leaf, prim, pr, bsr, plus, minus, s, d, out);
        break;
    }
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: {
        /* EllipticalCapRayIntersectionEquation.cpp:7-72 */
        const double C = pr[2], iAA = pr[3], iBB = pr[4], iCC = pr[5];
        const double a = (d.x*d.x)*iAA + (d.y*d.y)*iBB + (d.z*d.z)*iCC;
        const double b = 2.0*((s.x*d.x)*iAA + (s.y*d.y)*iBB + d.z*(s.z - C)*iCC);
        const double cc = (s.x*s.x)*iAA + (s.y*s.y)*iBB + (s.z*s.z - 2.0*s.z*C)*iCC;
        double plus, minus;
        if (c->cnt) c->cnt->others++;
        if (quadratic(b/a, cc/a, &plus, &minus))
            add_causal(c, leaf, prim, pr, bsr, plus, minus, s, d, out);
        break;
    }
    case MLGPU_PRIM_DISC:
    case MLGPU_PRIM_HEX_PLANE:
    case MLGPU_PRIM_PLANE:
    case MLGPU_PRIM_ANNULUS:
    case MLGPU_PRIM_PLANE_DUAL_SPHERE:
    case MLGPU_PRIM_TRIANGLE: {
        /* Disc.cpp:31-50, HexPlane.cpp:28-47, Plane.cpp:40-59,
         * Annulus.cpp:38-60, PlaneDualSphericalBound.cpp:36-55,
         * Triangle.cpp:105-126 */
        double v;
        if (c->cnt) c->cnt->planes++;
        if (!xy_plane(s, d, &v)) break;
        const v3 p = add(s, scale(d, v));
        int inside = 0;
        switch (prim) {
        case MLGPU_PRIM_DISC: inside = p.x*p.x + p.y*p.y < pr[0]; break;
        case MLGPU_PRIM_HEX_PLANE: inside = hex_inside(sc, pr[0], p); break;
        case MLGPU_PRIM_PLANE: inside = fabs(p.x) < pr[0] && fabs(p.y) < pr[1]; break;
        case MLGPU_PRIM_ANNULUS:
            inside = (p.x*p.x + p.y*p.y < pr[0]) && !(p.x*p.x + p.y*p.y < pr[1]);
            break;
        case MLGPU_PRIM_PLANE_DUAL_SPHERE: {
            /* DualSphericalPrismZ.cpp:20-26, Vec2.cpp:72-75 */
            const double ax = pr[0] - p.x, ay = pr[1] - p.y;
            const double bx = pr[2] - p.x, by = pr[3] - p.y;
            const double r = pr[4];
            inside = (ax*ax + ay*ay <= r*r) && (bx*bx + by*by <= r*r);
            break;
        }
        case MLGPU_PRIM_TRIANGLE: {
            const int bA = tri_sign(p, pr[0], pr[1], pr[2], pr[3]) < 0.0;
            const int bB = tri_sign(p, pr[2], pr[3], pr[4], pr[5]) < 0.0;
            const int bC = tri_sign(p, pr[4], pr[5], pr[0], pr[1]) < 0.0;
            inside = (bA == bB) && (bB == bC);
            break;
        }
        }
        if (inside && differs(s, p))
            set_isec(out, leaf, p, mk(0.0, 0.0, 1.0), v, d);
        break;
    }
    case MLGPU_PRIM_CYLINDER: {
        /* ZaxisCylinderRayIntersectionEquation.cpp:6-86, Cylinder.cpp:121-150 */
        const double radius = pr[0], length = pr[1];
        const double dx2 = d.x*d.x, dy2 = d.y*d.y;
        const double sxdx = s.x*d.x, sydy = s.y*d.y;
        const double sx2 = s.x*s.x, sy2 = s.y*s.y;
        const double r2 = radius*radius;
        const double dnom = dx2 + dy2;
        const double p = 2.0*(sxdx + sydy) / dnom;
        const double q = (sx2 + sy2 - r2) / dnom;
        double plus, minus, v = 0.0;
        int causal = 0;
        if (c->cnt) c->cnt->others++;
        if (quadratic(p, q, &plus, &minus)) {
            if (minus < 0.0 && plus >= 0.0) { causal = 1; v = plus; }
            if (plus >= 0.0 && minus >= 0.0) { causal = 1; v = minus; }
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
        /* Sphere.cpp:50-104 */
        const double radius = pr[0];
        const double sd = dot(s, d), dd = dot(d, d), ss = dot(s, s);
        const double r2 = radius*radius;
        double vP, vM;
        if (c->cnt) c->cnt->others++;
        if (!quadratic(2*(sd / dd), ss/dd - r2, &vP, &vM)) break;
        double v;
        if (vP >= 0.0 && vM >= 0.0) v = vM;
        else if (!(vP < 0.0 && vM < 0.0)) v = vP;
        else break;
        const v3 p = add(s, scale(d, v));
        if (differs(s, p))
            set_isec(out, leaf, p, divide(p, norm(p)), v, d);
        break;
    }
    default:
        break;
    }
}

/* ray_intersects_frames_bounding_sphere, merlict/RayAndFrame.cpp:16-107,
 * with Ray::parameter_for_closest_distance_to_point, Ray.cpp:50-66 */
static int sphere_cull(const double* sph, v3 s, v3 d) {
    const v3 c = mk(sph[0], sph[1], sph[2]);
    const double r = sph[3];
    const double alpha = dot(d, c) - dot(s, d);
    const v3 q = add(s, scale(d, alpha));
    const v3 sc = sub(c, q);
    const double dist_square = dot(sc, sc);
    if (dist_square > r*r) return 0;
    if (alpha < 0.0) {
        const v3 w = sub(c, s);
        return dot(w, w) <= r*r;  /* Vec3.cpp:137-140 */
    }
    return 1;
}

/* CausalIntersection, merlict/RayAndFrame.cpp:126-173: depth-first search
 * over bounding spheres, leaves intersected in visiting order, first
 * minimum distance wins; no hit gives the void intersection at 1e4 m. */
static isec_t first_intersection(ctx* c, int32_t root, v3 s, v3 d) {
    const mlgpu_flat_scene* sc = c->s;
    isec_t best;
    best.hit = 0;
    int have = 0;
    int32_t i = root;
    const int32_t end = sc->node_skip[root];
    uint32_t tested = 0;
    while (i < end) {
        const double* sph = sc->node_sphere + 4*(size_t)i;
        if (c->cnt) c->cnt->nodes++;
        if (!sphere_cull(sph, s, d)) { i = sc->node_skip[i]; continue; }
        const int32_t leaf = sc->node_leaf[i];
        if (leaf >= 0) {
            const double* t = sc->leaf_frame2world + 12*(size_t)leaf;
            const v3 so = position_inverse(t, s);     /* Ray::transform_inverse, Ray.cpp:45-48 */
            const v3 dobj = orientation_inverse(t, d);
            isec_t cand;
            if (c->cnt) c->cnt->leaves++;
            tested++;
            intersect_leaf(c, leaf, so, dobj, sph[3], &cand);
            if (cand.hit && (!have || cand.dist < best.dist)) {
                best = cand;
                have = 1;
            }
        }
        i++;
    }
    if (c->cnt) c->cnt->leaves_per_step[tested < 64 ? tested : 64]++;
    if (!have) {
        best.hit = 0;
        best.leaf = MLGPU_LEAF_VOID;
        best.pos = add(s, scale(d, 1e4));
        best.normal = d;
        best.dist = 1e4;
        best.outside = dot(d, d) < 0.0;
    }
    return best;
}

typedef struct {
    const mlgpu_rng* rng;
    uint64_t stream;
    uint32_t k;
} draw_t;

static double draw(ctx* c, draw_t* r) {
    const uint32_t k = r->k++;
    if (r->rng->mode == MLGPU_RNG_REPLAY) {
        if (k >= r->rng->stride) {
            if (!c->error) c->error = MLGPU_ERR_RUNTIME;
            return 0.5;
        }
        return r->rng->uniforms[(size_t)r->stream*r->rng->stride + k];
    }
    return mlgpu_philox_uniform(r->rng->seed, r->rng->photon_offset + r->stream, k);
}

static const double* leaf_T(const mlgpu_flat_scene* s, int32_t leaf) {
    return leaf < 0 ? IDENTITY : s->leaf_frame2world + 12*(size_t)leaf;
}

/* Propagator::propagate and its branches, merlict/PhotonAndFrame.cpp:13-124,
 * followed by the per-photon part of Sensor::assign_photon
 * (merlict/sensor/Sensor.cpp:14-30). */
static void propagate_one(ctx* c, uint64_t i, const mlgpu_photons* ph,
                          const mlgpu_settings* st, const mlgpu_rng* rng,
                          const mlgpu_results* res) {
    const mlgpu_flat_scene* sc = c->s;
    const double lambda = ((const double*)ph->wavelength)[i];
    const uint32_t max_int = st->max_num_interactions_per_photon;
    mlgpu_history_entry* hist =
        res->history ? res->history + (size_t)i*(max_int + 1) : NULL;
    draw_t rd; rd.rng = rng; rd.stream = i; rd.k = 0;

    /* RayForPropagation ctor: Ray::set_support_and_direction normalises the
     * direction (Ray.cpp:16-20); the production entry has the photon source
     * as object, the direction as normal (RayForPropagation.cpp:52-64). */
    const v3 s0 = mk(((const double*)ph->support_x)[i],
                     ((const double*)ph->support_y)[i],
                     ((const double*)ph->support_z)[i]);
    v3 s = s0;
    v3 d = normalized(mk(((const double*)ph->direction_x)[i],
                         ((const double*)ph->direction_y)[i],
                         ((const double*)ph->direction_z)[i]));
    isec_t last;
    last.hit = 0; last.leaf = MLGPU_LEAF_PHOTON_SOURCE; last.pos = s;
    last.normal = d; last.dist = 0.0; last.outside = dot(d, d) < 0.0;
    if (hist) {
        mlgpu_history_entry* h = &hist[0];
        memset(h, 0, sizeof(*h));
        h->position[0] = s.x; h->position[1] = s.y; h->position[2] = s.z;
        h->normal[0] = d.x; h->normal[1] = d.y; h->normal[2] = d.z;
        h->distance = 0.0; h->leaf = MLGPU_LEAF_PHOTON_SOURCE;
        h->interaction = MLGPU_PRODUCTION; h->from_outside_to_inside = (uint8_t)last.outside;
    }
    /* root-frame positions of the last two history entries */
    v3 last_world = position(IDENTITY, s0);
    v3 second_last_world = last_world;
    uint32_t n_int = 1;
    int interaction = MLGPU_PRODUCTION;
    int32_t root = st->start_node;
    double tof = 0.0;
    int tof_error = 0;

    while (n_int <= max_int) {              /* PhotonAndFrame.cpp:13-21 */
        if (c->cnt) c->cnt->steps++;
        /* work_on_first_causal_intersection, :23-30 */
        const isec_t is = first_intersection(c, root, s, d);
        const int32_t* surf =
            is.hit ? sc->leaf_surface + (size_t)MLGPU_SURF_COLUMNS*is.leaf : NULL;
        const double* T = leaf_T(sc, is.leaf);
        int absorbed = 0;
        if (is.hit) {
            /* absorbed_in_medium_before_reaching_surface, :32-38 */
            const double depth = func_eval(c, surf[is.outside ? MLGPU_SURF_OUTER_ABSORPTION
                                                              : MLGPU_SURF_INNER_ABSORPTION], lambda);
            const double survival = exp(-is.dist/depth);
            absorbed = draw(c, &rd) > survival;
        }
        int kind;
        int moved = 0;
        v3 new_s = s, new_d = d;
        if (!is.hit || absorbed) {
            kind = MLGPU_ABSORPTION_IN_VOID;                    /* :50-54 */
        } else {
            /* interact_with_object, :40-48 */
            const double refl = func_eval(c, surf[is.outside ? MLGPU_SURF_OUTER_REFLECTION
                                                             : MLGPU_SURF_INNER_REFLECTION], lambda);
            if (refl >= draw(c, &rd)) {
                /* reflect_on_surface_and_propagate_on, :56-66, with
                 * Intersection::reflection_direction_in_root_frame, Intersection.cpp:74-79 */
                kind = MLGPU_REFLECTION_ON_SURFACE;
                new_s = position(T, is.pos);
                new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                moved = 1;
                if (c->cnt) c->cnt->reflections++;
            } else if (!(surf[MLGPU_SURF_FLAGS] & MLGPU_FLAG_TRANSPARENT)) {
                kind = MLGPU_ABSORPTION_ON_SURFACE;             /* :68-73, :120-124 */
            } else {
                /* fresnel_refraction_and_reflection, :75-87, Fresnel.cpp:7-38 */
                const v3 inc = orientation_inverse(T, d);
                const v3 nrm = is.outside ? is.normal : scale(is.normal, -1.0);
                const double n_from = func_eval(c, surf[is.outside ? MLGPU_SURF_OUTER_REFRACTION
                                                                   : MLGPU_SURF_INNER_REFRACTION], lambda);
                const double n_to = func_eval(c, surf[is.outside ? MLGPU_SURF_INNER_REFRACTION
                                                                 : MLGPU_SURF_OUTER_REFRACTION], lambda);
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
                if (c->cnt) c->cnt->fresnels++;
                if (R > draw(c, &rd)) {
                    kind = MLGPU_FRESNEL_REFLECTION_ON_SURFACE;
                    new_s = position(T, is.pos);
                    new_d = normalized(orientation(T, mirror(is.normal, orientation_inverse(T, d))));
                    moved = 1;
                } else {
                    /* pass_the_boundary_layer, :89-100, and
                     * propagate_on_after_boundary_layer, :102-118 */
                    kind = is.outside ? MLGPU_REFRACTION_TO_INSIDE : MLGPU_REFRACTION_TO_OUTSIDE;
                    const int to_default = is.outside
                        ? (surf[MLGPU_SURF_FLAGS] & MLGPU_FLAG_INNER_REFRACTION_DEFAULT) != 0
                        : (surf[MLGPU_SURF_FLAGS] & MLGPU_FLAG_OUTER_REFRACTION_DEFAULT) != 0;
                    const int32_t allowed = surf[MLGPU_SURF_ALLOWED_NODE];
                    root = (allowed >= 0 && !to_default) ? allowed : 0;
                    const v3 refr = add(scale(inc, ratio), scale(nrm, ratio*cosI - cosT));
                    new_s = position(T, is.pos);
                    new_d = normalized(orientation(T, refr));
                    moved = 1;
                }
            }
        }
        /* push_back_intersection_and_interaction, RayForPropagation.cpp:83-89 */
        if (hist) {
            mlgpu_history_entry* h = &hist[n_int];
            memset(h, 0, sizeof(*h));
            h->position[0] = is.pos.x; h->position[1] = is.pos.y; h->position[2] = is.pos.z;
            h->normal[0] = is.normal.x; h->normal[1] = is.normal.y; h->normal[2] = is.normal.z;
            h->distance = is.dist; h->leaf = is.leaf; h->interaction = (uint8_t)kind;
            h->from_outside_to_inside = (uint8_t)is.outside;
        }
        /* time-of-flight term of this entry, Photon.cpp:37-56:
         * refractive_index_coming_from * distance / c */
        {
            const int32_t f = is.hit
                ? surf[is.outside ? MLGPU_SURF_OUTER_REFRACTION : MLGPU_SURF_INNER_REFRACTION]
                : sc->default_refraction;
            const int saved = c->error;
            const double n = func_eval(c, f, lambda);
            if (c->error && !saved) { if (!tof_error) tof_error = c->error; c->error = 0; }
            tof += n*is.dist/299792458.0;
            if (c->cnt) c->cnt->segments++;
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
            memset(&hist[k], 0, sizeof(hist[k]));
            hist[k].leaf = MLGPU_LEAF_PHOTON_SOURCE;
        }
    }

    /* FindSensorByFrame on the final intersection's object, Sensors.cpp:20-29 */
    const int32_t sensor = last.leaf >= 0 ? sc->leaf_sensor[last.leaf] : -1;
    /* the time of flight is only evaluated for photons given to a sensor */
    if (sensor >= 0 && tof_error && !c->error) c->error = tof_error;

    /* final_intersection_incident_direction_wrt_frame, RayForPropagation.cpp:114-136 */
    v3 inc = mk(0.0, 0.0, 0.0);
    if (n_int > 1) {
        const v3 w = normalized(sub(last_world, second_last_world));
        inc = orientation_inverse(leaf_T(sc, last.leaf), w);
    }
    res->sensor[i] = sensor;
    if (res->x) ((double*)res->x)[i] = last.pos.x;
    if (res->y) ((double*)res->y)[i] = last.pos.y;
    if (res->time) res->time[i] = tof;
    if (res->theta_x) ((double*)res->theta_x)[i] = -1.0*inc.x;
    if (res->theta_y) ((double*)res->theta_y)[i] = -1.0*inc.y;
    if (res->final_leaf) res->final_leaf[i] = last.leaf;
    if (res->info)
        res->info[i] = (uint32_t)interaction | (n_int << 8) |
            ((rd.k > 255 ? 255u : rd.k) << 16) | ((uint32_t)c->error << 24);
    if (res->final_position) {
        res->final_position[3*i + 0] = last_world.x;
        res->final_position[3*i + 1] = last_world.y;
        res->final_position[3*i + 2] = last_world.z;
    }
    if (res->final_direction) {
        res->final_direction[3*i + 0] = d.x;
        res->final_direction[3*i + 1] = d.y;
        res->final_direction[3*i + 2] = d.z;
    }
}

/* Entry point for the checker: all pointers are host pointers, photons and
 * results in double precision.  Returns the first per-photon error code (0
 * if none).  `counters` may be NULL. */
int oracle_propagate(const mlgpu_flat_scene* scene,
                     const mlgpu_photons* photons, uint64_t num_photons,
                     const mlgpu_settings* settings, const mlgpu_rng* rng,
                     const mlgpu_results* results, oracle_counters* counters) {
    int first_error = 0;
    /* Photon::assert_wavelength_is_positive (merlict/Photon.cpp:20-28): the
     * caller builds every Photon before propagating, so a non-positive
     * wavelength fails the call before anything is traced. */
    for (uint64_t i = 0; i < num_photons; i++)
        if (((const double*)photons->wavelength)[i] <= 0.0) return MLGPU_ERR_INVALID_ARGUMENT;
    for (uint64_t i = 0; i < num_photons; i++) {
        ctx c;
        c.s = scene; c.error = 0; c.cnt = counters;
        propagate_one(&c, i, photons, settings, rng, results);
        if (c.error && !first_error) first_error = c.error;
    }
    return first_error;
}

/* Per-sensor counts and time histograms, the statistics a caller of
 * Sensors::assign_photons derives from the arrival lists. */
void oracle_bin_arrivals(const int32_t* sensor, const double* time, uint64_t n,
                         int32_t num_sensors, uint32_t* counts, uint32_t* time_hist,
                         uint32_t num_bins, double t_min, double t_max) {
    memset(counts, 0, sizeof(uint32_t)*(size_t)num_sensors);
    if (time_hist) memset(time_hist, 0, sizeof(uint32_t)*(size_t)num_sensors*num_bins);
    for (uint64_t i = 0; i < n; i++) {
        const int32_t s = sensor[i];
        if (s < 0 || s >= num_sensors) continue;
        counts[s]++;
        if (time_hist && num_bins) {
            const double f = (time[i] - t_min) / (t_max - t_min) * (double)num_bins;
            if (f >= 0.0 && f < (double)num_bins)
                time_hist[(size_t)s*num_bins + (uint32_t)f]++;
        }
    }
}

int oracle_sizeof_history_entry(void) { return (int)sizeof(mlgpu_history_entry); }
