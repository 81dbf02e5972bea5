// fp32_geometry.cuh -- single-precision intersection of a world ray with a
// leaf, for the batched FP32 tracer (wavefront_fp32.cu, wave_resolve.cuh).
//
// The bulk of the arithmetic is FP32; double precision is kept where the
// precision of the result needs it:
//  * the ray is moved, in FP64, to where it enters the leaf's bounding
//    sphere before it is turned into the leaf's frame, so that the FP32
//    local coordinates are small (a leaf-sized neighbourhood) and keep
//    ~1e-7 of the leaf size instead of ~1e-7 of the distance travelled;
//  * sphere caps (merlict/scenery/geometry/SphericalCapRayIntersectionEquation
//    .cpp) are solved in FP32 with the cancellation-free form
//    q = -(b + sign(b) sqrt(b^2 - 4ac))/2, roots q/a and c/q, then each root
//    gets one Newton step on the quadratic evaluated in FP64 -- the long
//    focal lengths of Cherenkov mirrors (R = 21 .. 213 m) make the textbook
//    form lose most of its digits in FP32 -- and the cap's hit point and
//    normal are evaluated in FP64 from the refined root.  The "pure FP32"
//    variant uses the textbook form without correction (precision study);
//  * distances along the ray are FP64.
// Bounds tests, normals and the plane family are FP32.
#ifndef MLGPU_FP32_GEOMETRY_CUH_
#define MLGPU_FP32_GEOMETRY_CUH_

#include <cstddef>
#include <cstdint>

#include "mlgpu_internal.h"

namespace mlgpu {
namespace fp32 {
namespace {   // one copy per translation unit

struct f3 { float x, y, z; };
struct d3 { double x, y, z; };

__device__ __forceinline__ f3 fmk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ d3 dmk(double x, double y, double z) { d3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ float fdot(f3 a, f3 b) { return a.x*b.x + a.y*b.y + a.z*b.z; }
__device__ __forceinline__ f3 fadd(f3 a, f3 b) { return fmk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ f3 fsub(f3 a, f3 b) { return fmk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ f3 fscale(f3 a, float s) { return fmk(a.x*s, a.y*s, a.z*s); }
__device__ __forceinline__ f3 fnormalized(f3 a) { return fscale(a, rsqrtf(fdot(a, a))); }

// R holds the rows of the leaf's rotation; object = R^T (world - origin)
__device__ __forceinline__ f3 to_local(const float* R, f3 v) {
    return fmk(R[0]*v.x + R[3]*v.y + R[6]*v.z,
               R[1]*v.x + R[4]*v.y + R[7]*v.z,
               R[2]*v.x + R[5]*v.y + R[8]*v.z);
}
__device__ __forceinline__ f3 to_world(const float* R, f3 v) {
    return fmk(R[0]*v.x + R[1]*v.y + R[2]*v.z,
               R[3]*v.x + R[4]*v.y + R[5]*v.z,
               R[6]*v.x + R[7]*v.y + R[8]*v.z);
}

struct Hit32 {
    int32_t leaf;      // < 0: none
    double v;          // distance along the world ray
    d3 p;              // intersection, leaf frame
    d3 n;              // surface normal, leaf frame
    bool outside;      // merlict's from_outside_to_inside
};

__device__ __forceinline__ d3 dwiden(f3 a) { return dmk(a.x, a.y, a.z); }

__device__ __forceinline__ bool hex_inside32(const DevScene& sc, float inner, f3 p) {
    const float u = (float)sc.hex_u[0]*p.x + (float)sc.hex_u[1]*p.y;
    const float v = (float)sc.hex_v[0]*p.x + (float)sc.hex_v[1]*p.y;
    const float w = (float)sc.hex_w[0]*p.x + (float)sc.hex_w[1]*p.y;
    return fabsf(u) < inner && fabsf(v) < inner && fabsf(w) < inner;
}

// Both roots of a t^2 + b t + c = 0 in FP32; `stable` selects the
// cancellation-free form.  Returns false without real roots.
__device__ __forceinline__ bool roots32(float a, float b, float c, bool stable, float* t1, float* t2) {
    const float disc = b*b - 4.0f*a*c;
    if (!(disc >= 0.0f)) return false;
    const float sq = sqrtf(disc);
    if (stable) {
        const float q = -0.5f*(b + copysignf(sq, b));
        *t1 = q/a;
        *t2 = (q != 0.0f) ? c/q : *t1;
    } else {
        const float p2 = 0.5f*b/a, qq = c/a;
        const float s2 = sqrtf(fmaxf(p2*p2 - qq, 0.0f));
        *t1 = -p2 - s2;
        *t2 = -p2 + s2;
    }
    return true;
}

// One Newton step on a t^2 + b t + c in FP64.
__device__ __forceinline__ double newton64(double a, double b, double c, double t) {
    const double f = (a*t + b)*t + c;
    const double df = 2.0*a*t + b;
    return df != 0.0 ? t - f/df : t;
}

// Intersection of the world ray (s, d) with leaf `leaf`, merlict's rules:
// causal solutions only, the self-intersection guard (a distance of more
// than 1e-7 m), strict bounds as in the reference.  `pure` selects the
// textbook single-precision form throughout (no rebasing, textbook roots,
// FP32 normals).  Without kNeedHit only the distance is wanted (the
// candidate pass): the Newton step of a spherical cap is then taken on the
// cap's sphere in world coordinates (the leaf's FP64 anchor), which needs
// none of the FP64 transform; with kNeedHit (the closest candidate's full
// hit) it is taken in the leaf frame of the FP64 transform, and the hit
// point and normal follow in FP64.
// The FP64 transform entry T[k] and parameter params[k] of a leaf: by leaf
// id from its record, or (kSlot) by candidate slot from the slot-ordered
// records (pairs 0-5 the transform, pair 8 onwards (r2, params[0]),
// (params[1], params[2]), ...).
template <bool kSlot>
__device__ __forceinline__ double leaf_T64(const DevScene& sc, int32_t id, int k) {
    if (kSlot) {
        const double2 x = __ldg(sc.slot_rec + (size_t)(id >> 3)*96 + (k >> 1)*8 + (id & 7));
        return (k & 1) ? x.y : x.x;
    }
    return __ldg(&sc.leaf[id].T[k]);
}
template <bool kSlot>
__device__ __forceinline__ double leaf_param64(const DevScene& sc, int32_t id, int k) {
    if (kSlot) {
        const int m = k + 1;
        const double2 x = __ldg(sc.slot_rec + (size_t)(id >> 3)*96 + (8 + (m >> 1))*8 + (id & 7));
        return (m & 1) ? x.y : x.x;
    }
    return __ldg(&sc.leaf[id].params[k]);
}

// 16-byte piece p of a leaf's LeafAnchor, by leaf id or (kSlot) by slot.
template <bool kSlot>
__device__ __forceinline__ double2 anchor_pair(const DevScene& sc, int32_t id, int p) {
    if (kSlot) {
        const uint4 x = __ldg(sc.slot_rec_f + (size_t)(id >> 3)*72 + (5 + p)*8 + (id & 7));
        return make_double2(__hiloint2double((int)x.y, (int)x.x),
                            __hiloint2double((int)x.w, (int)x.z));
    }
    return __ldg(reinterpret_cast<const double2*>(sc.leaf_anchor + id) + p);
}

// `leaf` is a leaf id, or with kSlot a candidate slot (the records then come
// from the slot-ordered copies, where the eight slots of a leaf range sit
// side by side, and Hit32::leaf holds the slot).
template <bool kNeedHit, bool kSlot = false>
__device__ Hit32 intersect32(const DevScene& sc, int32_t leaf, d3 s, d3 d, bool pure) {
    Hit32 h;
    h.leaf = -1;
    // R, params, r2 and primitive: the record's first 80 bytes in 16-byte loads
    static_assert(offsetof(LeafRecF, params) == 36 && offsetof(LeafRecF, r2) == 68 &&
                  offsetof(LeafRecF, primitive) == 72, "intersect32 reads LeafRecF in pieces");
    float v[20];
    double2 o01, o2R;   // the anchor: origin x, y; origin z, R
    if (kSlot) {
        const uint4* q = sc.slot_rec_f + (size_t)(leaf >> 3)*72 + (leaf & 7);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const uint4 x = __ldg(q + 8*k);
            v[4*k] = __uint_as_float(x.x); v[4*k + 1] = __uint_as_float(x.y);
            v[4*k + 2] = __uint_as_float(x.z); v[4*k + 3] = __uint_as_float(x.w);
        }
        o01 = anchor_pair<true>(sc, leaf, 0);
        o2R = anchor_pair<true>(sc, leaf, 1);
    } else {
        const float4* Lq = reinterpret_cast<const float4*>(sc.leaf_f + leaf);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const float4 x = __ldg(Lq + k);
            v[4*k] = x.x; v[4*k + 1] = x.y; v[4*k + 2] = x.z; v[4*k + 3] = x.w;
        }
        o01 = anchor_pair<false>(sc, leaf, 0);
        o2R = anchor_pair<false>(sc, leaf, 1);
    }
    const int32_t prim = __float_as_int(v[18]);
    if (prim == MLGPU_PRIM_NONE) return h;
    const d3 c = dmk(o01.x, o01.y, o2R.x);
    float R[9];
#pragma unroll
    for (int k = 0; k < 9; k++) R[k] = v[k];
    const float r2 = v[17];
    // rebase the ray (FP64) to where it enters the leaf's bounding sphere,
    // then go to the leaf frame (FP32).  A ray that starts inside the sphere
    // -- on the surface it just left, say -- is not moved, so its
    // self-intersection stays a root near zero.
    double t0 = 0.0;
    if (!pure) {
        const double tc = (c.x - s.x)*d.x + (c.y - s.y)*d.y + (c.z - s.z)*d.z;
        const double te = tc - sqrt((double)r2);
        if (te > 0.0) t0 = te;
    }
    const d3 rel = dmk(s.x + d.x*t0 - c.x, s.y + d.y*t0 - c.y, s.z + d.z*t0 - c.z);
    const f3 sl = to_local(R, fmk((float)rel.x, (float)rel.y, (float)rel.z));
    const f3 dl = to_local(R, fmk((float)d.x, (float)d.y, (float)d.z));
    float pr[MLGPU_LEAF_PARAMS];
#pragma unroll
    for (int k = 0; k < MLGPU_LEAF_PARAMS; k++) pr[k] = v[9 + k];
    const double v_min = 1e-7;   // merlict's self-intersection guard, |hit - support|^2 > 1e-14

    switch (prim) {
    case MLGPU_PRIM_DISC:
    case MLGPU_PRIM_HEX_PLANE:
    case MLGPU_PRIM_PLANE:
    case MLGPU_PRIM_ANNULUS:
    case MLGPU_PRIM_PLANE_DUAL_SPHERE:
    case MLGPU_PRIM_TRIANGLE: {
        if (dl.z == 0.0f) return h;
        const float vl = -sl.z/dl.z;
        const double v = t0 + (double)vl;
        if (!(v > v_min)) return h;
        const f3 p = fadd(sl, fscale(dl, vl));
        bool inside;
        switch (prim) {
        case MLGPU_PRIM_DISC: inside = p.x*p.x + p.y*p.y < pr[0]; break;
        case MLGPU_PRIM_HEX_PLANE: inside = hex_inside32(sc, pr[0], p); break;
        case MLGPU_PRIM_PLANE: inside = fabsf(p.x) < pr[0] && fabsf(p.y) < pr[1]; break;
        case MLGPU_PRIM_ANNULUS: {
            const float rr = p.x*p.x + p.y*p.y;
            inside = rr < pr[0] && !(rr < pr[1]);
            break;
        }
        case MLGPU_PRIM_PLANE_DUAL_SPHERE: {
            const float ax = pr[0] - p.x, ay = pr[1] - p.y, bx = pr[2] - p.x, by = pr[3] - p.y;
            inside = ax*ax + ay*ay <= pr[4]*pr[4] && bx*bx + by*by <= pr[4]*pr[4];
            break;
        }
        default: {
            const float sA = (p.x - pr[2])*(pr[1] - pr[3]) - (pr[0] - pr[2])*(p.y - pr[3]);
            const float sB = (p.x - pr[4])*(pr[3] - pr[5]) - (pr[2] - pr[4])*(p.y - pr[5]);
            const float sC = (p.x - pr[0])*(pr[5] - pr[1]) - (pr[4] - pr[0])*(p.y - pr[1]);
            inside = ((sA < 0.0f) == (sB < 0.0f)) && ((sB < 0.0f) == (sC < 0.0f));
            break;
        }
        }
        if (!inside) return h;
        h.leaf = leaf; h.v = v; h.p = dmk(p.x, p.y, 0.0); h.n = dmk(0.0, 0.0, 1.0);
        h.outside = dl.z < 0.0f;
        return h;
    }
    case MLGPU_PRIM_SPHERE_CAP_HEX:
    case MLGPU_PRIM_SPHERE_CAP_CYL:
    case MLGPU_PRIM_SPHERE_CAP_RECT:
    case MLGPU_PRIM_ELLIPTIC_CAP_HEX: {
        const bool ell = prim == MLGPU_PRIM_ELLIPTIC_CAP_HEX;
        float a, b, cc;
        if (ell) {
            const float C = pr[2], iA = pr[3], iB = pr[4], iC = pr[5];
            a = dl.x*dl.x*iA + dl.y*dl.y*iB + dl.z*dl.z*iC;
            b = 2.0f*(sl.x*dl.x*iA + sl.y*dl.y*iB + dl.z*(sl.z - C)*iC);
            cc = sl.x*sl.x*iA + sl.y*sl.y*iB + (sl.z*sl.z - 2.0f*sl.z*C)*iC;
        } else {
            const float Rc = pr[0];
            a = fdot(dl, dl);
            b = 2.0f*(fdot(sl, dl) - Rc*dl.z);
            cc = fdot(sl, sl) - 2.0f*Rc*sl.z;
        }
        float f1, f2;
        if (!roots32(a, b, cc, !pure, &f1, &f2)) return h;
        double t1 = f1, t2 = f2;
        d3 s64 = dwiden(sl), d64 = dwiden(dl);
        if (!pure && !kNeedHit && !ell) {
            // one Newton step each on |m + t d|^2 - R^2, m = rebased support
            // - sphere centre, in FP64 world coordinates
            const double2 c01 = anchor_pair<kSlot>(sc, leaf, 2);   // centre x, y
            const double2 c2p = anchor_pair<kSlot>(sc, leaf, 3);   // centre z, pad
            const d3 m = dmk(s.x + d.x*t0 - c01.x, s.y + d.y*t0 - c01.y, s.z + d.z*t0 - c2p.x);
            const double R = o2R.y;
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const double t = k == 0 ? t1 : t2;
                const d3 v = dmk(m.x + d.x*t, m.y + d.y*t, m.z + d.z*t);
                const double f = (v.x*v.x + v.y*v.y + v.z*v.z) - R*R;
                const double df = 2.0*(v.x*d.x + v.y*d.y + v.z*d.z);
                const double tn = df != 0.0 ? t - f/df : t;
                if (k == 0) t1 = tn; else t2 = tn;
            }
        } else if (!pure) {
            // one Newton step each on the quadratic in FP64, in the leaf frame
            // of the FP64 transform
            double Tr[9];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                Tr[3*k] = leaf_T64<kSlot>(sc, leaf, 4*k);
                Tr[3*k + 1] = leaf_T64<kSlot>(sc, leaf, 4*k + 1);
                Tr[3*k + 2] = leaf_T64<kSlot>(sc, leaf, 4*k + 2);
            }
            s64 = dmk(Tr[0]*rel.x + Tr[3]*rel.y + Tr[6]*rel.z,
                      Tr[1]*rel.x + Tr[4]*rel.y + Tr[7]*rel.z,
                      Tr[2]*rel.x + Tr[5]*rel.y + Tr[8]*rel.z);
            d64 = dmk(Tr[0]*d.x + Tr[3]*d.y + Tr[6]*d.z,
                      Tr[1]*d.x + Tr[4]*d.y + Tr[7]*d.z,
                      Tr[2]*d.x + Tr[5]*d.y + Tr[8]*d.z);
            double a64, b64, c64;
            if (ell) {
                const double C = pr[2], iA = pr[3], iB = pr[4], iC = pr[5];
                a64 = d64.x*d64.x*iA + d64.y*d64.y*iB + d64.z*d64.z*iC;
                b64 = 2.0*(s64.x*d64.x*iA + s64.y*d64.y*iB + d64.z*(s64.z - C)*iC);
                c64 = s64.x*s64.x*iA + s64.y*s64.y*iB + (s64.z*s64.z - 2.0*s64.z*C)*iC;
            } else {
                const double Rc = leaf_param64<kSlot>(sc, leaf, 0);
                a64 = d64.x*d64.x + d64.y*d64.y + d64.z*d64.z;
                b64 = 2.0*(s64.x*d64.x + s64.y*d64.y + s64.z*d64.z - Rc*d64.z);
                c64 = s64.x*s64.x + s64.y*s64.y + s64.z*s64.z - 2.0*Rc*s64.z;
            }
            t1 = newton64(a64, b64, c64, t1);
            t2 = newton64(a64, b64, c64, t2);
        }
        // merlict's causal choice between the two roots: the nearer one
        // that lies in front, inside the bound and inside the bounding
        // sphere (SurfaceWithOuterPrismBound.cpp:7-70)
        const double lo = fmin(t1, t2), hi = fmax(t1, t2);
        double best = 0.0;
        bool ok = false;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const double tl = k == 0 ? lo : hi;
            if (ok || !(t0 + tl > v_min)) continue;
            const f3 p = (!pure && !kNeedHit && !ell)
                ? fadd(sl, fscale(dl, (float)tl))
                : fmk((float)(s64.x + d64.x*tl), (float)(s64.y + d64.y*tl), (float)(s64.z + d64.z*tl));
            bool in;
            switch (prim) {
            case MLGPU_PRIM_SPHERE_CAP_HEX: in = hex_inside32(sc, pr[1], p); break;
            case MLGPU_PRIM_ELLIPTIC_CAP_HEX: in = hex_inside32(sc, pr[6], p); break;
            case MLGPU_PRIM_SPHERE_CAP_CYL: in = p.x*p.x + p.y*p.y < pr[1]; break;
            default: in = fabsf(p.x) < pr[1] && fabsf(p.y) < pr[2]; break;
            }
            if (in && fdot(p, p) <= r2) { best = tl; ok = true; }
        }
        if (!ok) return h;
        if (!kNeedHit) {
            h.leaf = leaf; h.v = t0 + best;
            return h;
        }
        if (pure) {
            const f3 p = fadd(sl, fscale(dl, (float)best));
            f3 n;
            if (ell) {
                const float f = pr[2]*0.5f*sqrtf(fmaxf(1.0f - p.x*p.x*pr[3] - p.y*p.y*pr[4], 0.0f));
                n = fnormalized(fmk(f*(-2.0f*p.x*pr[3]), f*(-2.0f*p.y*pr[3]), 1.0f));
            } else {
                n = fnormalized(fmk(-p.x, -p.y, pr[0] - p.z));
            }
            h.p = dwiden(p); h.n = dwiden(n);
            h.outside = fdot(n, dl) < 0.0f;
        } else {
            // hit point and normal in FP64: the normal's direction error
            // becomes a position error after the long lever arm to the
            // focal plane
            const d3 p = dmk(s64.x + d64.x*best, s64.y + d64.y*best, s64.z + d64.z*best);
            d3 n;
            if (ell) {
                const double iA = leaf_param64<kSlot>(sc, leaf, 3);
                const double iB = leaf_param64<kSlot>(sc, leaf, 4);
                const double C = leaf_param64<kSlot>(sc, leaf, 2);
                const double f = C*0.5*sqrt(fmax(1.0 - p.x*p.x*iA - p.y*p.y*iB, 0.0));
                n = dmk(f*(-2.0*p.x*iA), f*(-2.0*p.y*iA), 1.0);
            } else {
                n = dmk(-p.x, -p.y, leaf_param64<kSlot>(sc, leaf, 0) - p.z);
            }
            const double inv = 1.0/sqrt(n.x*n.x + n.y*n.y + n.z*n.z);
            n = dmk(n.x*inv, n.y*inv, n.z*inv);
            h.p = p; h.n = n;
            h.outside = n.x*d64.x + n.y*d64.y + n.z*d64.z < 0.0;
        }
        h.leaf = leaf; h.v = t0 + best;
        return h;
    }
    case MLGPU_PRIM_CYLINDER: {
        const float a = dl.x*dl.x + dl.y*dl.y;
        if (a == 0.0f) return h;
        const float b = 2.0f*(sl.x*dl.x + sl.y*dl.y);
        const float cc = sl.x*sl.x + sl.y*sl.y - pr[0]*pr[0];
        float t1, t2;
        if (!roots32(a, b, cc, !pure, &t1, &t2)) return h;
        const float lo = fminf(t1, t2), hi = fmaxf(t1, t2);
        // ZaxisCylinderRayIntersectionEquation.cpp:54-60: the nearer root in
        // front of the support, else the farther one
        float tl;
        if (t0 + (double)lo >= 0.0) tl = lo;
        else if (t0 + (double)hi >= 0.0) tl = hi;
        else return h;
        const double v = t0 + (double)tl;
        if (!(v > v_min)) return h;
        const f3 p = fadd(sl, fscale(dl, tl));
        if (!(fabsf(p.z) <= 0.5f*pr[1])) return h;
        const f3 n = fnormalized(fmk(p.x, p.y, 0.0f));
        h.leaf = leaf; h.v = v; h.p = dwiden(p); h.n = dwiden(n);
        h.outside = fdot(n, dl) < 0.0f;
        return h;
    }
    case MLGPU_PRIM_SPHERE: {
        const float a = fdot(dl, dl);
        const float b = 2.0f*fdot(sl, dl);
        const float cc = fdot(sl, sl) - pr[0]*pr[0];
        float t1, t2;
        if (!roots32(a, b, cc, !pure, &t1, &t2)) return h;
        const float lo = fminf(t1, t2), hi = fmaxf(t1, t2);
        float tl;
        if (t0 + (double)lo >= 0.0) tl = lo;           // Sphere.cpp:96-103
        else if (t0 + (double)hi >= 0.0) tl = hi;
        else return h;
        const double v = t0 + (double)tl;
        if (!(v > v_min)) return h;
        const f3 p = fadd(sl, fscale(dl, tl));
        const f3 n = fnormalized(p);
        h.leaf = leaf; h.v = v; h.p = dwiden(p); h.n = dwiden(n);
        h.outside = fdot(n, dl) < 0.0f;
        return h;
    }
    default:
        return h;
    }
}

}  // namespace
}  // namespace fp32
}  // namespace mlgpu

#endif  // MLGPU_FP32_GEOMETRY_CUH_
