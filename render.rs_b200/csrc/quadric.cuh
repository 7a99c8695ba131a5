// quadric.cuh — analytic RiSpec quadrics on the device, in f32.
//
// The reference's legacy primitives (src/geometry/sphere.rs, cylinder.rs,
// cone.rs, extra.rs; its Metal kernel isect_common.metal:95-330 runs the
// same tests in f32): the ray goes to object space with its direction
// normalised there, the roots are tested against the shape's z / angle
// cuts in the reference's order, and the hit distance is the world distance
// of the hit point from the ray origin. A scene's quadrics are few (a
// handful of spheres, disks and the like), so every query tests all of them
// before the BVH, as Scene::intersect scans its `objects` list before the
// TLAS (src/scene/mod.rs:105-146).
//
// The torus needs the real roots of a quartic, which an f32 closed form
// (Ferrari) cannot deliver reliably; its roots are isolated instead by
// sampling the polynomial for sign changes along the ray's chord through
// the torus' bounding sphere, refined by bisection and Newton steps.
#pragma once

#include "traverse.cuh"

namespace rt {

#define RT_Q_EPS 1e-6f  // EPSILON of src/math/mod.rs:9, the root cut-off
#define RT_Q_DEG (57.29577951308232f)

// Local hit point of an intersection query; the surface quantities come
// from the point afterwards (q_surface), only for the hit that is shaded.
struct QLocal {
    float3 p;
};
struct QSurface {
    float3 n;        // object-space normal
    float u, v;      // RiSpec parameterisation
    float dpdu, dpdv;
    bool front_set;  // the front face follows the world normal (sphere); else front
};

__device__ __forceinline__ bool q_theta_ok(float x, float y, float thetamax) {
    if (thetamax >= 360.0f) return true;
    float phi = atan2f(y, x) * RT_Q_DEG;
    if (phi < 0.0f) phi += 360.0f;
    return phi <= thetamax;
}
__device__ __forceinline__ float q_phi_u(float x, float y, float thetamax) {
    float phi = atan2f(y, x) * RT_Q_DEG;
    if (phi < 0.0f) phi += 360.0f;
    return fminf(fmaxf(phi / fmaxf(thetamax, 1e-9f), 0.0f), 1.0f);
}
__device__ __forceinline__ float q_clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }

// sphere.rs:39-103: near root, else the far root; a z or angle cut rejects
// without trying the other root.
__device__ __forceinline__ bool q_sphere(const float* pr, float3 o, float3 d, QLocal& h) {
    const float radius = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
    const float a = dot(d, d), b = 2.0f * dot(o, d), c = dot(o, o) - radius * radius;
    const float disc = b * b - 4.0f * a * c;
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc), t1 = (-b - sq) / (2.0f * a), t2 = (-b + sq) / (2.0f * a);
    const float t = t1 > RT_Q_EPS ? t1 : t2;
    if (!(t > RT_Q_EPS)) return false;
    const float3 p = o + d * t;
    if (p.z < zmin || p.z > zmax) return false;
    if (thetamax < 360.0f && !q_theta_ok(p.x, p.y, thetamax)) return false;
    h.p = p;
    return true;
}

// cylinder.rs:37-120: a z-cut miss of the near root retries the far root.
__device__ __forceinline__ bool q_cylinder(const float* pr, float3 o, float3 d, QLocal& h) {
    const float radius = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
    const float a = d.x * d.x + d.y * d.y, b = 2.0f * (o.x * d.x + o.y * d.y);
    const float c = o.x * o.x + o.y * o.y - radius * radius;
    if (fabsf(a) < RT_Q_EPS) return false;
    const float disc = b * b - 4.0f * a * c;
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc), t1 = (-b - sq) / (2.0f * a), t2 = (-b + sq) / (2.0f * a);
    float t = t1 > RT_Q_EPS ? t1 : t2;
    if (t <= RT_Q_EPS) return false;
    float3 p = o + d * t;
    if (p.z < zmin || p.z > zmax) {
        if (t == t1 && t2 > RT_Q_EPS) {
            t = t2;
            p = o + d * t;
            if (p.z < zmin || p.z > zmax) return false;
        } else {
            return false;
        }
    }
    if (thetamax < 360.0f && !q_theta_ok(p.x, p.y, thetamax)) return false;
    h.p = p;
    return true;
}

// cone.rs:36-142: x^2 + y^2 = k z^2, k = (radius / height)^2, 0 <= z <= height.
__device__ __forceinline__ void q_cone_finish(const float*, float3 p, QLocal& h) { h.p = p; }
__device__ __forceinline__ bool q_cone(const float* pr, float3 o, float3 d, QLocal& h) {
    const float height = pr[0], radius = pr[1], thetamax = pr[2];
    const float k = (radius / height) * (radius / height);
    const float a = d.x * d.x + d.y * d.y - k * d.z * d.z;
    const float b = 2.0f * (o.x * d.x + o.y * d.y - k * o.z * d.z);
    const float c = o.x * o.x + o.y * o.y - k * o.z * o.z;
    if (fabsf(a) < RT_Q_EPS) {
        if (fabsf(b) < RT_Q_EPS) return false;
        const float t = -c / b;
        if (t > RT_Q_EPS) {
            const float3 p = o + d * t;
            if (p.z >= 0.0f && p.z <= height) {
                q_cone_finish(pr, p, h);
                return true;
            }
        }
        return false;
    }
    const float disc = b * b - 4.0f * a * c;
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc);
    const float ts[2] = {(-b - sq) / (2.0f * a), (-b + sq) / (2.0f * a)};
    for (int i = 0; i < 2; i++) {
        const float t = ts[i];
        if (!(t > RT_Q_EPS)) continue;
        const float3 p = o + d * t;
        if (!(p.z >= 0.0f && p.z <= height)) continue;
        if (thetamax < 360.0f && !q_theta_ok(p.x, p.y, thetamax)) continue;
        q_cone_finish(pr, p, h);
        return true;
    }
    return false;
}

// Torus (extra.rs:243-303): the roots of the quartic in ascending order, the
// first past EPSILON inside both angle cuts. Roots are isolated on the chord
// of the bounding sphere (radius R + r) with the ray re-origined at the
// chord's start (smaller coefficients): 96 samples of the polynomial, each
// sign change bisected and then polished by two Newton steps.
__device__ __forceinline__ bool q_torus(const float* pr, float3 o, float3 d, QLocal& h) {
    const float R = pr[0], r = pr[1], phimin = pr[2], phimax = pr[3], thetamax = pr[4];
    const float bound = R + r;
    const float mid = -dot(o, d);  // d is unit length
    const float3 cp = o + d * mid;
    const float c2 = dot(cp, cp);
    if (c2 > bound * bound) return false;
    const float half = sqrtf(bound * bound - c2);
    const float t0 = fmaxf(mid - half, 0.0f), t1 = mid + half;
    if (t1 <= RT_Q_EPS) return false;
    const float3 so = o + d * t0;
    const float g = dot(d, d), hh = 2.0f * dot(so, d), i = dot(so, so) + R * R - r * r;
    const float j = d.x * d.x + d.y * d.y, k = 2.0f * (so.x * d.x + so.y * d.y), l = so.x * so.x + so.y * so.y;
    const float fr = 4.0f * R * R;
    const float a4 = g * g, a3 = 2.0f * g * hh, a2 = hh * hh + 2.0f * g * i - fr * j, a1 = 2.0f * hh * i - fr * k,
                a0 = i * i - fr * l;
    auto f = [&](float t) { return (((a4 * t + a3) * t + a2) * t + a1) * t + a0; };
    auto df = [&](float t) { return ((4.0f * a4 * t + 3.0f * a3) * t + 2.0f * a2) * t + a1; };
    const int STEPS = 96;
    const float span = t1 - t0, dt = span / (float)STEPS;
    float ta = 0.0f, fa = f(0.0f);
    for (int s = 1; s <= STEPS; s++) {
        const float tb = dt * (float)s, fb = f(tb);
        if ((fa < 0.0f) != (fb < 0.0f)) {
            float lo = ta, hi = tb, flo = fa;
            for (int it = 0; it < 20; it++) {
                const float m = 0.5f * (lo + hi), fm = f(m);
                if ((flo < 0.0f) != (fm < 0.0f)) {
                    hi = m;
                } else {
                    lo = m;
                    flo = fm;
                }
            }
            float t = 0.5f * (lo + hi);
            for (int it = 0; it < 2; it++) {
                const float dv = df(t);
                if (fabsf(dv) > 1e-30f) {
                    const float tn = t - f(t) / dv;
                    if (tn >= lo && tn <= hi) t = tn;
                }
            }
            const float tw = t + t0;
            if (tw > RT_Q_EPS) {
                const float3 p = o + d * tw;
                const float rxy = sqrtf(p.x * p.x + p.y * p.y);
                float vphi = atan2f(p.z, rxy - R) * RT_Q_DEG;
                while (vphi < phimin) vphi += 360.0f;
                while (vphi >= phimin + 360.0f) vphi -= 360.0f;
                const bool phi_ok = phimax - phimin >= 360.0f || vphi <= phimax;
                if (phi_ok && q_theta_ok(p.x, p.y, thetamax)) {
                    h.p = p;
                    return true;
                }
            }
        }
        ta = tb;
        fa = fb;
    }
    return false;
}

// extra.rs:347-381.
__device__ __forceinline__ bool q_disk(const float* pr, float3 o, float3 d, QLocal& h) {
    const float height = pr[0], radius = pr[1], thetamax = pr[2];
    if (fabsf(d.z) < RT_Q_EPS) return false;
    const float t = (height - o.z) / d.z;
    if (t <= RT_Q_EPS) return false;
    const float3 p = o + d * t;
    if (p.x * p.x + p.y * p.y > radius * radius) return false;
    if (!q_theta_ok(p.x, p.y, thetamax)) return false;
    h.p = p;
    return true;
}

// extra.rs:425-484 (paraboloid) and 526-632 (hyperboloid): up to two
// candidate roots in order, the first past EPSILON inside both cuts.
__device__ __forceinline__ int q_roots(float a, float b, float c, float* ts) {
    if (fabsf(a) < RT_Q_EPS) {
        if (fabsf(b) < RT_Q_EPS) return 0;
        ts[0] = -c / b;
        return 1;
    }
    const float disc = b * b - 4.0f * a * c;
    if (disc < 0.0f) return 0;
    const float sq = sqrtf(disc);
    ts[0] = (-b - sq) / (2.0f * a);
    ts[1] = (-b + sq) / (2.0f * a);
    return 2;
}
__device__ __forceinline__ bool q_paraboloid(const float* pr, float3 o, float3 d, QLocal& h) {
    const float rmax = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
    if (fabsf(zmax) < RT_Q_EPS) return false;
    const float k = rmax * rmax / zmax;
    float ts[2];
    const int nt = q_roots(d.x * d.x + d.y * d.y, 2.0f * (o.x * d.x + o.y * d.y) - k * d.z,
                           o.x * o.x + o.y * o.y - k * o.z, ts);
    for (int i = 0; i < nt; i++) {
        const float t = ts[i];
        if (t <= RT_Q_EPS) continue;
        const float3 p = o + d * t;
        if (p.z < zmin || p.z > zmax) continue;
        if (!q_theta_ok(p.x, p.y, thetamax)) continue;
        h.p = p;
        return true;
    }
    return false;
}
__device__ __forceinline__ bool q_hyperboloid(const float* pr, float3 o, float3 d, QLocal& h) {
    const float3 p1 = f3(pr[0], pr[1], pr[2]), p2 = f3(pr[3], pr[4], pr[5]);
    const float thetamax = pr[6];
    const float zlo = fminf(p1.z, p2.z), zhi = fmaxf(p1.z, p2.z);
    if (fabsf(p2.z - p1.z) < RT_Q_EPS) {
        // Flat annulus between the two radii (no st, extra.rs:540-567).
        if (fabsf(d.z) < RT_Q_EPS) return false;
        const float t = (p1.z - o.z) / d.z;
        if (t <= RT_Q_EPS) return false;
        const float3 p = o + d * t;
        const float r2 = p.x * p.x + p.y * p.y;
        const float ra = p1.x * p1.x + p1.y * p1.y, rb = p2.x * p2.x + p2.y * p2.y;
        if (r2 < fminf(ra, rb) || r2 > fmaxf(ra, rb)) return false;
        if (!q_theta_ok(p.x, p.y, thetamax)) return false;
        h.p = p;
        return true;
    }
    const float dz = p2.z - p1.z, iu = 1.0f / dz;
    const float sx = (p2.x - p1.x) * iu, sy = (p2.y - p1.y) * iu;
    const float cx = p1.x - p1.z * sx, cy = p1.y - p1.z * sy;
    const float pa = sx * sx + sy * sy, pb = 2.0f * (cx * sx + cy * sy), pc = cx * cx + cy * cy;
    float ts[2];
    const int nt = q_roots(d.x * d.x + d.y * d.y - pa * d.z * d.z,
                           2.0f * (o.x * d.x + o.y * d.y - pa * o.z * d.z) - pb * d.z,
                           o.x * o.x + o.y * o.y - pa * o.z * o.z - pb * o.z - pc, ts);
    for (int i = 0; i < nt; i++) {
        const float t = ts[i];
        if (t <= RT_Q_EPS) continue;
        const float3 p = o + d * t;
        if (p.z < zlo || p.z > zhi) continue;
        if (!q_theta_ok(p.x, p.y, thetamax)) continue;
        h.p = p;
        return true;
    }
    return false;
}

__device__ __forceinline__ bool q_local(const DevQuadric& q, float3 o, float3 d, QLocal& h) {
    switch (q.type) {
        case 0: return q_sphere(q.prm, o, d, h);
        case 1: return q_cylinder(q.prm, o, d, h);
        case 2: return q_cone(q.prm, o, d, h);
        case 3: return q_torus(q.prm, o, d, h);
        case 4: return q_disk(q.prm, o, d, h);
        case 5: return q_paraboloid(q.prm, o, d, h);
        case 6: return q_hyperboloid(q.prm, o, d, h);
    }
    return false;
}

// One quadric against a world ray: the world distance of its hit, or a
// negative value on a miss; `h` holds the local hit point.
__device__ __forceinline__ float q_world(const DevQuadric& q, float3 wo, float3 wd, QLocal& h) {
    const float3 lo = xf_point(q.w2o[0], q.w2o[1], q.w2o[2], wo);
    const float3 ld = normalize_ref(xf_vec(q.w2o[0], q.w2o[1], q.w2o[2], wd));
    if (!q_local(q, lo, ld, h)) return -1.0f;
    const float3 wp = xf_point(q.o2w[0], q.o2w[1], q.o2w[2], h.p);
    return length(wp - wo);
}

// The closest quadric hit below the world distance `limit`: its index (or
// ~0) and world distance.
__device__ __noinline__ uint32_t quadrics_closest(const DevScene& S, float3 o, float3 d, float limit, float& t_out) {
    uint32_t best = 0xFFFFFFFFu;
    for (uint32_t k = 0; k < S.n_quadrics; k++) {
        QLocal h;
        const float t = q_world(S.quadrics[k], o, d, h);
        if (t >= 0.0f && t < limit) {
            limit = t;
            best = k;
        }
    }
    t_out = limit;
    return best;
}

#define RT_Q_OFFSET 1e-4f  // RAY_OFFSET (src/raytracer/pt/mod.rs), the step past a crossing

// The closest quadric crossing that stops the ray when cutouts are decided
// inside the query (k_extend with cutouts): a crossing of a surface with
// presence p < 1 is passed with probability 1 - p (presence_passes on the
// ray's seed), and the search goes on from just past it, for at most 16
// crossings as the reference's skips. Returns the quadric (or ~0) and its
// world distance from o.
__device__ __noinline__ uint32_t quadrics_closest_stopping(const DevScene& S, float3 o, float3 d, float limit,
                                                           uint64_t seed, float& t_out) {
    float base = 0.0f;
    for (int seg = 0; seg < 16; seg++) {
        float t;
        const uint32_t k = quadrics_closest(S, o, d, limit - base, t);
        if (k == 0xFFFFFFFFu) break;
        const float pres = S.materials[S.quadrics[k].material].presence;
        if (!(pres < 1.0f && presence_passes(seed, RT_TRI_QUADRIC | k, 0xFFFFFFFFu ^ (uint32_t)seg, pres))) {
            t_out = base + t;
            return k;
        }
        o = o + d * (t + RT_Q_OFFSET);
        base += t + RT_Q_OFFSET;
    }
    t_out = limit;
    return 0xFFFFFFFFu;
}

// Shadow transmittance through the quadrics alone: the reference's segment
// loop (pt/mod.rs:1254-1306) restricted to them -- the closest crossing,
// (1 - presence) for a cutout and 0 for an opaque surface, then on from
// just past it -- for the world distance `dist` along the unit direction d.
// The mesh crossings multiply in separately (the product is the same in any
// order).
__device__ __noinline__ float quadrics_transmittance(const DevScene& S, float3 o, float3 d, float dist) {
    float vis = 1.0f;
    for (int seg = 0; seg < 16 && dist > 0.0f; seg++) {
        float t;
        const uint32_t k = quadrics_closest(S, o, d, dist, t);
        if (k == 0xFFFFFFFFu) break;
        const float pres = fminf(fmaxf(S.materials[S.quadrics[k].material].presence, 0.0f), 1.0f);
        if (pres >= 1.0f) return 0.0f;
        vis *= 1.0f - pres;
        if (vis < RT_TRANSMIT_CUTOFF) return 0.0f;
        o = o + d * (t + RT_Q_OFFSET);
        dist -= t + RT_Q_OFFSET;
    }
    return vis;
}

// Surface of a quadric at the object-space point p, as each shape's
// intersect finishes it (normal, RiSpec u / v and the st derivatives).
__device__ __forceinline__ QSurface q_surface(const DevQuadric& q, float3 p) {
    QSurface h;
    const float* pr = q.prm;
    h.front_set = false;
    const float ring = sqrtf(p.x * p.x + p.y * p.y);
    switch (q.type) {
        case 0: {  // sphere.rs:84-97
            const float radius = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
            const float zr = fmaxf(zmax - zmin, 1e-12f);
            const float rg = fmaxf(ring, 1e-6f * fmaxf(radius, 1e-12f));
            h.n = normalize_ref(p);
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01((p.z - zmin) / zr);
            h.dpdu = rg * thetamax / RT_Q_DEG;
            h.dpdv = zr * radius / rg;
            h.front_set = true;
            break;
        }
        case 1: {  // cylinder.rs:101-112
            const float radius = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
            const float zr = fmaxf(zmax - zmin, 1e-12f);
            h.n = normalize_ref(f3(p.x, p.y, 0.0f));
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01((p.z - zmin) / zr);
            h.dpdu = fmaxf(radius, 1e-12f) * thetamax / RT_Q_DEG;
            h.dpdv = zr;
            break;
        }
        case 2: {  // cone.rs:114-138
            const float height = pr[0], radius = pr[1], thetamax = pr[2];
            h.n = normalize_ref(f3(p.x / ring, p.y / ring, -radius / height));
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01(p.z / fmaxf(height, 1e-12f));
            h.dpdu = fmaxf(ring, 1e-6f * fmaxf(radius, 1e-12f)) * thetamax / RT_Q_DEG;
            h.dpdv = sqrtf(height * height + radius * radius);
            break;
        }
        case 3: {  // extra.rs:265-291
            const float R = pr[0], r = pr[1], phimin = pr[2], phimax = pr[3], thetamax = pr[4];
            const float rr = fmaxf(ring, 1e-12f), sc = 1.0f - R / rr;
            h.n = normalize_ref(f3(p.x * sc, p.y * sc, p.z));
            h.u = q_phi_u(p.x, p.y, thetamax);
            float vphi = atan2f(p.z, rr - R) * RT_Q_DEG;
            while (vphi < phimin) vphi += 360.0f;
            while (vphi >= phimin + 360.0f) vphi -= 360.0f;
            const float vr = fmaxf(phimax - phimin, 1e-9f);
            h.v = q_clamp01((vphi - phimin) / vr);
            h.dpdu = rr * thetamax / RT_Q_DEG;
            h.dpdv = fmaxf(r, 1e-12f) * vr / RT_Q_DEG;
            break;
        }
        case 4: {  // extra.rs:361-367
            const float radius = pr[1], thetamax = pr[2];
            h.n = f3(0.0f, 0.0f, 1.0f);
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01((radius - ring) / fmaxf(radius, 1e-12f));
            h.dpdu = fmaxf(ring, 1e-6f * fmaxf(radius, 1e-12f)) * thetamax / RT_Q_DEG;
            h.dpdv = radius;
            break;
        }
        case 5: {  // extra.rs:459-470
            const float rmax = pr[0], zmin = pr[1], zmax = pr[2], thetamax = pr[3];
            const float zr = fmaxf(zmax - zmin, 1e-12f);
            h.n = normalize_ref(f3(2.0f * p.x, 2.0f * p.y, -rmax * rmax / zmax));
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01((p.z - zmin) / zr);
            h.dpdu = fmaxf(ring, 1e-6f * fmaxf(rmax, 1e-12f)) * thetamax / RT_Q_DEG;
            h.dpdv = zr;
            break;
        }
        default: {  // extra.rs:540-567, 603-624
            const float3 p1 = f3(pr[0], pr[1], pr[2]), p2 = f3(pr[3], pr[4], pr[5]);
            const float thetamax = pr[6], dz = p2.z - p1.z;
            if (fabsf(dz) < RT_Q_EPS) {
                h.n = f3(0.0f, 0.0f, 1.0f);
                h.u = h.v = h.dpdu = h.dpdv = 0.0f;
                break;
            }
            const float iu = 1.0f / dz, sx = (p2.x - p1.x) * iu, sy = (p2.y - p1.y) * iu;
            const float cx = p1.x - p1.z * sx, cy = p1.y - p1.z * sy;
            const float pa = sx * sx + sy * sy, pb = 2.0f * (cx * sx + cy * sy);
            h.n = normalize_ref(f3(2.0f * p.x, 2.0f * p.y, -(2.0f * pa * p.z + pb)));
            h.u = q_phi_u(p.x, p.y, thetamax);
            h.v = q_clamp01((p.z - p1.z) / dz);
            h.dpdu = fmaxf(ring, 1e-12f) * thetamax / RT_Q_DEG;
            h.dpdv = fmaxf(length(p2 - p1), 1e-12f);
            break;
        }
    }
    return h;
}

// Shading geometry of a quadric hit at the world point wp reached along d:
// the world normal (not flipped, as the reference's quadrics report it),
// the front face, and st with its density (st units per world unit).
__device__ __forceinline__ void quadric_surface(const DevScene& S, uint32_t k, float3 wp, float3 d, float3& nw,
                                                bool& front, float* st) {
    const DevQuadric& q = S.quadrics[k];
    const QSurface h = q_surface(q, xf_point(q.w2o[0], q.w2o[1], q.w2o[2], wp));
    nw = normalize_ref(xf_normal(q.w2o[0], q.w2o[1], q.w2o[2], h.n));
    front = h.front_set ? dot(d, nw) < 0.0f : true;
    if (st) {
        st[0] = h.u;
        st[1] = h.v;
        st[2] = (h.dpdu > 0.0f || h.dpdv > 0.0f) ? rsqrtf(fmaxf(h.dpdu * h.dpdv, 1e-24f)) / q.scale : 0.0f;
    }
}

}  // namespace rt
