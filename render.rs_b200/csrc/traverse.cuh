// traverse.cuh — ray traversal of the two-level 8-wide BVH on sm_100a.
//
// Closest hit and any hit over the TLAS/BLAS pair, one ray per thread:
//  * node fetch: six 128-bit read-only loads (96-B node);
//  * child boxes decoded exactly (p + q * 2^e is an exact f32) and tested
//    with the robust slab test of Ize 2013 (t_far scaled by 1 + 2*gamma(3));
//  * triangles with the watertight test of Woop, Benthin and Wald 2013
//    (shear to ray space, edge functions, f64 fallback on exact zeros);
//  * traversal stack: the top 32 entries live in shared memory (one column
//    per thread, bank-conflict free), deeper entries spill to local memory
//    in halves; a stack deeper than the spill area sets an error bit.
// The reference's traversal is Bvh::traverse / any_hit (src/accel/bvh.rs:
// 141-245) over 2-wide nodes with Möller–Trumbore triangles
// (src/geometry/mesh.rs:117-142) and Instance::intersect (mesh.rs:308-381):
// same closest hit (parametric t along the unnormalised ray, instance
// transforms applied without renormalising), different arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rt_internal.h"

namespace rt {

// ---- small float3 helpers ---------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
// Normalise only above 1e-6, as the reference's Vec3::normalize
// (src/math/vector.rs:31-38).
__device__ __forceinline__ float3 normalize_ref(float3 a) {
    float l = length(a);
    return l > 1e-6f ? a / l : a;
}
__device__ __forceinline__ float maxc(float3 c) { return fmaxf(fmaxf(c.x, c.y), c.z); }
__device__ __forceinline__ float luminance(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
__device__ __forceinline__ float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }

// Row-major 3x4 affine applied to a point / a vector / a normal (transpose).
__device__ __forceinline__ float3 xf_point(const float4& r0, const float4& r1, const float4& r2, float3 p) {
    return f3(fmaf(r0.x, p.x, fmaf(r0.y, p.y, fmaf(r0.z, p.z, r0.w))),
              fmaf(r1.x, p.x, fmaf(r1.y, p.y, fmaf(r1.z, p.z, r1.w))),
              fmaf(r2.x, p.x, fmaf(r2.y, p.y, fmaf(r2.z, p.z, r2.w))));
}
__device__ __forceinline__ float3 xf_vec(const float4& r0, const float4& r1, const float4& r2, float3 v) {
    return f3(r0.x * v.x + r0.y * v.y + r0.z * v.z, r1.x * v.x + r1.y * v.y + r1.z * v.z,
              r2.x * v.x + r2.y * v.y + r2.z * v.z);
}
__device__ __forceinline__ float3 xf_normal(const float4& r0, const float4& r1, const float4& r2, float3 n) {
    return f3(r0.x * n.x + r1.x * n.y + r2.x * n.z, r0.y * n.x + r1.y * n.y + r2.y * n.z,
              r0.z * n.x + r1.z * n.y + r2.z * n.z);
}

// ---- motion blur ----------------------------------------------------------------
// World-to-object rows of instance `inst` for a ray at shutter time `time`
// (Instance::transforms_at, src/geometry/mesh.rs:295-304): a moving
// instance at t > 0 is placed by the component-wise lerp of its two
// object-to-world transforms, inverted here in f32 (adjugate over the
// determinant; identity when |det| < 1e-6, as Matrix4::inverse gives None).
// MOT false compiles the static path alone.
template <bool MOT>
__device__ __forceinline__ void inst_rows(const DevScene& S, uint32_t inst, float time, float4& x0, float4& x1,
                                          float4& x2) {
    if (MOT && S.inst_mot && time > 0.0f) {
        const uint32_t k = __ldg(S.inst_mot + inst);
        if (k != 0xFFFFFFFFu) {
            const DevInstMotion& M = S.inst_motion[k];
            float4 m[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                const float4 a = __ldg(&M.o2w0[r]), b = __ldg(&M.o2w1[r]);
                m[r] = make_float4(a.x + (b.x - a.x) * time, a.y + (b.y - a.y) * time, a.z + (b.z - a.z) * time,
                                   a.w + (b.w - a.w) * time);
            }
            const float3 a0 = xyz(m[0]), a1 = xyz(m[1]), a2 = xyz(m[2]);
            const float3 c0 = cross(a1, a2), c1 = cross(a2, a0), c2 = cross(a0, a1);
            const float det = dot(a0, c0);
            if (!(fabsf(det) >= 1e-6f)) {
                x0 = make_float4(1.0f, 0.0f, 0.0f, 0.0f);
                x1 = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
                x2 = make_float4(0.0f, 0.0f, 1.0f, 0.0f);
                return;
            }
            const float id = 1.0f / det;
            const float3 r0 = f3(c0.x, c1.x, c2.x) * id, r1 = f3(c0.y, c1.y, c2.y) * id,
                         r2 = f3(c0.z, c1.z, c2.z) * id;
            const float3 tr = f3(m[0].w, m[1].w, m[2].w);
            x0 = make_float4(r0.x, r0.y, r0.z, -dot(r0, tr));
            x1 = make_float4(r1.x, r1.y, r1.z, -dot(r1, tr));
            x2 = make_float4(r2.x, r2.y, r2.z, -dot(r2, tr));
            return;
        }
    }
    x0 = __ldg(S.inst_xf + 3 * (size_t)inst);
    x1 = __ldg(S.inst_xf + 3 * (size_t)inst + 1);
    x2 = __ldg(S.inst_xf + 3 * (size_t)inst + 2);
}

// Triangle `tri` (leaf order) at shutter time `time` (Mesh::vertex_at,
// mesh.rs:96-111): a deforming mesh's vertices lerp toward their
// shutter-close positions; the record's w fields are kept.
template <bool MOT>
__device__ __forceinline__ void tri_at(const DevScene& S, uint32_t tri, float time, float4& a, float4& b, float4& c) {
    const float4* tp = S.tris + 3 * (size_t)tri;
    a = __ldg(tp);
    b = __ldg(tp + 1);
    c = __ldg(tp + 2);
    if (MOT && time > 0.0f && __float_as_uint(b.w) == RT_DEFORM_MARK) {
        const float4* tq = S.tris1 + 3 * (size_t)tri;
        const float4 a1 = __ldg(tq), b1 = __ldg(tq + 1), c1 = __ldg(tq + 2);
        a = make_float4(a.x + (a1.x - a.x) * time, a.y + (a1.y - a.y) * time, a.z + (a1.z - a.z) * time, a.w);
        b = make_float4(b.x + (b1.x - b.x) * time, b.y + (b1.y - b.y) * time, b.z + (b1.z - b.z) * time, b.w);
        c = make_float4(c.x + (c1.x - c.x) * time, c.y + (c1.y - c.y) * time, c.z + (c1.z - c.z) * time, c.w);
    }
}

// ---- per-ray precomputation ------------------------------------------------------
struct RayPre {
    float3 o, d, inv;
    // Woop shear as three rows: A_x = (v - o) . rx, A_y = (v - o) . ry, A_z = (v - o) . rz
    float3 rx, ry, rz;
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__device__ __forceinline__ void ray_pre(RayPre& r, float3 o, float3 d) {
    r.o = o;
    r.d = d;
    auto safe = [](float x) { return fabsf(x) < 1e-30f ? copysignf(1e-30f, x) : x; };
    r.inv = f3(1.0f / safe(d.x), 1.0f / safe(d.y), 1.0f / safe(d.z));
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = (ax >= ay && ax >= az) ? 0 : (ay >= az ? 1 : 2);
    int kx = kz == 2 ? 0 : kz + 1;
    int ky = kx == 2 ? 0 : kx + 1;
    float dz = comp(d, kz);
    if (dz < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    float sx = comp(d, kx) / dz, sy = comp(d, ky) / dz, sz = 1.0f / dz;
    r.kx = kx;
    r.ky = ky;
    r.kz = kz;
    r.sx = sx;
    r.sy = sy;
    r.sz = sz;
    auto unit = [](int k) { return f3(k == 0 ? 1.f : 0.f, k == 1 ? 1.f : 0.f, k == 2 ? 1.f : 0.f); };
    r.rx = unit(kx) - unit(kz) * sx;
    r.ry = unit(ky) - unit(kz) * sy;
    r.rz = unit(kz) * sz;
}

// Watertight ray/triangle test. Returns true and writes t, b1, b2
// (barycentrics of v1, v2) when 0 < t < t_max.
__device__ __forceinline__ bool tri_watertight(const RayPre& r, float3 v0, float3 v1, float3 v2, float t_max,
                                               float& t_out, float& b1, float& b2) {
    float3 A = v0 - r.o, B = v1 - r.o, C = v2 - r.o;
    float ax = fmaf(-r.sx, comp(A, r.kz), comp(A, r.kx));
    float ay = fmaf(-r.sy, comp(A, r.kz), comp(A, r.ky));
    float bx = fmaf(-r.sx, comp(B, r.kz), comp(B, r.kx));
    float by = fmaf(-r.sy, comp(B, r.kz), comp(B, r.ky));
    float cx = fmaf(-r.sx, comp(C, r.kz), comp(C, r.kx));
    float cy = fmaf(-r.sy, comp(C, r.kz), comp(C, r.ky));
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float az = r.sz * comp(A, r.kz), bz = r.sz * comp(B, r.kz), cz = r.sz * comp(C, r.kz);
    float T = U * az + V * bz + W * cz;
    float t = T / det;
    if (!(t > 0.0f && t < t_max)) return false;
    t_out = t;
    float rdet = 1.0f / det;
    b1 = V * rdet;
    b2 = W * rdet;
    return true;
}

// ---- curve segments (src/geometry/curves.rs:107-188) ---------------------------------
// Rounded cone after Quilez: a sphere swept from pa (radius ra) to pb
// (radius rb). The ray is first advanced to its closest approach to pa
// (t0), so the quadratic's terms are on the scale of the segment rather
// than of the ray's length and keep their precision in f32; t is
// parametric along d (not normalised). Writes the outward normal when n is
// given.
// Roots closer than RT_SEG_EPS to the ray's origin count as behind it (the
// reference's bound is t > 1e-9 in f64, curves.rs:146, 182). The gap
// matters for thin segments: there the reference's surface normal is
// shorter than Vec3::normalize's 1e-6 threshold and stays unnormalised, so
// rays leaving a hair hit start on the surface itself (the 1e-4 offset
// along that normal vanishes); an f32 hit point is off the surface by about
// an ulp of its coordinates, and without the gap the ray would meet its own
// segment again at t ~ 1e-6 where the reference's f64 ray passes on.
// Offset origins (unit normals) sit 1e-4 away and are not affected.
#define RT_SEG_EPS 2e-5f
__device__ __forceinline__ bool seg_sphere(float3 o, float3 d, float dd, float3 c, float r, float t_lo, float t_hi,
                                           float& t) {
    const float3 oc = o - c;
    const float b = dot(oc, d), cc = dot(oc, oc) - r * r;
    const float disc = b * b - dd * cc;
    if (disc < 0.0f) return false;
    const float sq = sqrtf(disc);
    float tt = (-b - sq) / dd;
    if (tt <= t_lo) tt = (-b + sq) / dd;
    if (tt <= t_lo || tt >= t_hi) return false;
    t = tt;
    return true;
}
__device__ __forceinline__ bool seg_intersect(float3 o, float3 d, float4 a, float4 b, float4 c, float t_max, float& t_out,
                                              float3* n_out = nullptr) {
    const float3 pa = xyz(a), pb = xyz(b);
    const float ra = b.w, rb = c.x;
    const float dd = dot(d, d);
    const float t0 = dot(pa - o, d) / dd;
    const float3 os = o + d * t0;  // the ray's closest approach to pa
    const float lo = RT_SEG_EPS - t0, hi = t_max - t0;
    const float3 ba = pb - pa, oa = os - pa;
    const float m0 = dot(ba, ba);
    float ts;
    float3 n;
    if (m0 < 1e-24f) {
        // A point particle: the sphere of the larger radius.
        if (!seg_sphere(os, d, dd, pa, fmaxf(ra, rb), lo, hi, ts)) return false;
        n = os + d * ts - pa;
    } else {
        const float rr = ra - rb;
        const float m1 = dot(ba, oa), m2 = dot(ba, d), m3 = dot(d, oa), m5 = dot(oa, oa);
        const float d2 = m0 - rr * rr;
        const float k2 = d2 * dd - m2 * m2;
        const float k1 = d2 * m3 - m1 * m2 + m2 * rr * ra;
        const float k0 = d2 * m5 - m1 * m1 + m1 * rr * ra * 2.0f - m0 * ra * ra;
        bool body = false;
        if (fabsf(k2) > 1e-24f) {
            const float h = k1 * k1 - k0 * k2;
            if (h >= 0.0f) {
                const float tb = (-k1 - sqrtf(h)) / k2;
                const float y = m1 + tb * m2;
                if (tb > lo && tb < hi && y > 0.0f && y < d2) {
                    ts = tb;
                    n = (oa + d * tb) * d2 - ba * y;
                    body = true;
                }
            }
        }
        if (!body) {
            // Caps: the start sphere owns y <= 0, the end sphere y >= d2.
            bool any = false;
            float tc;
            float lim = hi;
            if (seg_sphere(os, d, dd, pa, ra, lo, lim, tc) && m1 + tc * m2 <= 0.0f) {
                any = true;
                ts = tc;
                lim = tc;
                n = os + d * tc - pa;
            }
            if (seg_sphere(os, d, dd, pb, rb, lo, lim, tc) && m1 + tc * m2 >= d2) {
                any = true;
                ts = tc;
                n = os + d * tc - pb;
            }
            if (!any) return false;
        }
    }
    const float t = t0 + ts;
    if (!(t > RT_SEG_EPS && t < t_max)) return false;
    t_out = t;
    if (n_out) *n_out = normalize_ref(n);
    return true;
}
__device__ __forceinline__ bool is_segment(float4 c) { return __float_as_uint(c.w) == RT_SEG_MARK; }

// ---- 8-wide node: decode and test all children --------------------------------------
__device__ __forceinline__ float q8(uint32_t word, int byte) {
    // Exact u8 -> f32 through the 2^23 mantissa trick.
    return __uint_as_float(0x4B000000u | ((word >> (8 * byte)) & 0xFFu)) - 8388608.0f;
}

struct NodeHits {
    float tn[8];
    uint32_t ref[8];
    uint32_t mask;
};

// ROBUST_SCALE = 1 + 2*gamma(3), gamma(n) = n*eps/(1 - n*eps), eps = 2^-24.
#define RT_ROBUST_SCALE 1.0000003576278687f

__device__ __forceinline__ void test_node(const uint4* __restrict__ nodes, uint32_t idx, const RayPre& r,
                                          float t_max, NodeHits& h) {
    const uint4* n = nodes + (size_t)idx * WIDE_NODE_WORDS;
    uint4 w0 = __ldg(n + 0), w1 = __ldg(n + 1), w2 = __ldg(n + 2), w3 = __ldg(n + 3);
    uint4 w4 = __ldg(n + 4), w5 = __ldg(n + 5);
    float sx = __uint_as_float((w0.w & 0xFFu) << 23);
    float sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
    float sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
    // Planes decode as fma(2^23 + q, s, p - 2^23 s): the byte q is spliced
    // into the mantissa of 2^23 with one byte permute. p = k s with
    // |k| <= 2^20 (the build keeps s >= 16 ulp of the node's coordinates), so
    // p - 2^23 s and the plane p + q s are exact f32 values.
    float px = __uint_as_float(w0.x) - 8388608.0f * sx;
    float py = __uint_as_float(w0.y) - 8388608.0f * sy;
    float pz = __uint_as_float(w0.z) - 8388608.0f * sz;
    const uint32_t nc = w0.w >> 24;
    h.ref[0] = w4.x; h.ref[1] = w4.y; h.ref[2] = w4.z; h.ref[3] = w4.w;
    h.ref[4] = w5.x; h.ref[5] = w5.y; h.ref[6] = w5.z; h.ref[7] = w5.w;
    h.mask = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        if (k >= (int)nc) break;
        uint32_t wlx = k < 4 ? w1.x : w1.y, wly = k < 4 ? w1.z : w1.w;
        uint32_t wlz = k < 4 ? w2.x : w2.y, whx = k < 4 ? w2.z : w2.w;
        uint32_t why = k < 4 ? w3.x : w3.y, whz = k < 4 ? w3.z : w3.w;
        const uint32_t sel = 0x7440u | (uint32_t)(k & 3);
        auto qf = [&](uint32_t w) { return __uint_as_float(__byte_perm(w, 0x4B000000u, sel)); };
        float lox = fmaf(qf(wlx), sx, px), hix = fmaf(qf(whx), sx, px);
        float loy = fmaf(qf(wly), sy, py), hiy = fmaf(qf(why), sy, py);
        float loz = fmaf(qf(wlz), sz, pz), hiz = fmaf(qf(whz), sz, pz);
        float t0x = (lox - r.o.x) * r.inv.x, t1x = (hix - r.o.x) * r.inv.x;
        float t0y = (loy - r.o.y) * r.inv.y, t1y = (hiy - r.o.y) * r.inv.y;
        float t0z = (loz - r.o.z) * r.inv.z, t1z = (hiz - r.o.z) * r.inv.z;
        float tnear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), 0.0f));
        float tfar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), t_max));
        tfar *= RT_ROBUST_SCALE;
        h.tn[k] = tnear;
        if (tnear <= tfar && h.ref[k] != REF_EMPTY) h.mask |= 1u << k;
    }
}

// ---- traversal stack: shared-memory top, local-memory spill ----------------------------
#ifndef RT_SH_STACK
#define RT_SH_STACK 32   // traversal stack entries kept in shared memory per thread (power of two)
#endif
#define RT_SPILL 96

struct TravStack {
    uint2* sh;       // this thread's column: entry k at sh[(k % 32) * stride]
    int stride;
    int sp, base;    // logical stack [0, sp); shared holds [base, sp)
    uint2 spill[RT_SPILL];
    bool overflow;

    __device__ __forceinline__ void init(uint2* col, int stride_) {
        sh = col;
        stride = stride_;
        sp = 0;
        base = 0;
        overflow = false;
    }
    __device__ __forceinline__ void push(uint32_t ref, float t) {
        if (sp - base == RT_SH_STACK) {
            if (base + RT_SH_STACK / 2 > RT_SPILL) {
                overflow = true;
                return;
            }
#pragma unroll 1
            for (int i = 0; i < RT_SH_STACK / 2; i++) spill[base + i] = sh[((base + i) & (RT_SH_STACK - 1)) * stride];
            base += RT_SH_STACK / 2;
        }
        sh[(sp & (RT_SH_STACK - 1)) * stride] = make_uint2(ref, __float_as_uint(t));
        sp++;
    }
    __device__ __forceinline__ uint2 pop() {
        if (sp == base && base > 0) {
            base -= RT_SH_STACK / 2;
#pragma unroll 1
            for (int i = 0; i < RT_SH_STACK / 2; i++) sh[((base + i) & (RT_SH_STACK - 1)) * stride] = spill[base + i];
        }
        sp--;
        return sh[(sp & (RT_SH_STACK - 1)) * stride];
    }
};

struct TraceHit {
    float t;
    uint32_t tri;    // leaf-order triangle index (global), ~0 on miss
    uint32_t inst;   // leaf-order instance index
    float b1, b2;    // barycentrics of v1, v2
};

// Error bits written to the device error word.
#define RT_DEVERR_STACK 1u
#define RT_DEVERR_ITER 2u
#define RT_MAX_TRAV_STEPS (1u << 22)   // default of DevScene::max_steps (rt_params.max_trav_steps)

// Resumable traversal state of one ray (registers), so persistent warps can
// advance rays a few steps at a time and refill lanes whose ray finished.
struct TravState {
    RayPre r;          // current ray (world, or the instance's object space)
    float3 o, d;       // world ray
    TraceHit hit;
    uint32_t cur;      // node / leaf reference being processed
    uint32_t cur_inst;
    uint32_t steps;
    int inst_sp;
    bool in_inst, found;
    float trans;       // shadow transmittance (TRANSMIT queries)
    float time;        // shutter time of the ray (motion blur; 0 in static scenes)
};

// Start a closest-hit / any-hit query; false when the scene is empty.
__device__ __forceinline__ bool trav_begin(const DevScene& S, TravState& ts, TravStack& st, float3 o, float3 d,
                                           float t_max, float time = 0.0f) {
    ts.time = time;
    ts.hit.t = t_max;
    ts.hit.tri = 0xFFFFFFFFu;
    ts.hit.inst = 0xFFFFFFFFu;
    ts.hit.b1 = ts.hit.b2 = 0.0f;
    ts.o = o;
    ts.d = d;
    ts.in_inst = false;
    ts.found = false;
    ts.inst_sp = 0;
    ts.cur_inst = 0;
    ts.steps = 0;
    ts.trans = 1.0f;
    st.sp = 0;
    st.base = 0;
    st.overflow = false;
    if (S.tlas_root == 0xFFFFFFFFu) return false;
    ray_pre(ts.r, o, d);
    ts.cur = S.tlas_root;
    return true;
}

// ---- phased traversal: node operations and leaf operations ---------------------------
// A lane's work splits into three operations so a warp can run all of its
// node tests together and then all of its leaf tests together (Aila & Laine
// 2009, "while-while"): lanes are then mostly in the same code.
//   op_node: test the 8 children of ts.cur, continue with the nearest, push
//            the rest; a leaf found is parked in `pending`.
//   op_pop:  next stack entry that can still hold a closer hit (leaving an
//            instance restores the world ray); false when the stack is empty.
//   op_leaf: the parked leaf — enter an instance (TLAS) or test triangles (BLAS).
struct PhaseState {
    TravState ts;
    uint32_t pending;  // parked leaf reference (bit 31 set), 0 = none
    bool need_pop;
};

__device__ __forceinline__ void phase_begin(PhaseState& ps) {
    ps.pending = 0;
    ps.need_pop = false;
    if (ps.ts.cur & REF_LEAF) {
        ps.pending = ps.ts.cur;
        ps.need_pop = true;
    }
}

// Returns false when the query is over (stack exhausted).
__device__ __forceinline__ bool op_pop(PhaseState& ps, TravStack& st) {
    TravState& ts = ps.ts;
    for (;;) {
        if (ts.in_inst && st.sp == ts.inst_sp) {
            ts.in_inst = false;
            ray_pre(ts.r, ts.o, ts.d);
        }
        if (st.sp == 0) return false;
        uint2 e = st.pop();
        if (__uint_as_float(e.y) < ts.hit.t) {
            ts.cur = e.x;
            ps.need_pop = false;
            if (e.x & REF_LEAF) {
                ps.pending = e.x;
                ps.need_pop = true;
            }
            return true;
        }
    }
}

// Returns true on a fatal condition (stack overflow): the query is over.
template <bool ANY>
__device__ __forceinline__ bool op_node(const DevScene& S, PhaseState& ps, TravStack& st, uint32_t* err) {
    TravState& ts = ps.ts;
    NodeHits h;
    test_node(S.nodes, ts.cur, ts.r, ts.hit.t, h);
    uint32_t m = h.mask;
    if (!m) {
        ps.need_pop = true;
        return false;
    }
    uint32_t next = 0;
    if (ANY) {
        int k0 = __ffs(m) - 1;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if (k == k0) next = h.ref[k];
            else if ((m >> k) & 1u) st.push(h.ref[k], h.tn[k]);
        }
    } else {
        while (__popc(m) > 1) {
            float bt = -1.0f;
            int bk = 0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (((m >> k) & 1u) && h.tn[k] > bt) {
                    bt = h.tn[k];
                    bk = k;
                }
            uint32_t rf = 0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (k == bk) rf = h.ref[k];
            st.push(rf, bt);
            m &= ~(1u << bk);
        }
#pragma unroll
        for (int k = 0; k < 8; k++)
            if ((m >> k) & 1u) next = h.ref[k];
    }
    if (st.overflow) {
        atomicOr(err, RT_DEVERR_STACK);
        return true;
    }
    ts.cur = next;
    if (next & REF_LEAF) {
        ps.pending = next;
        ps.need_pop = true;
    }
    return false;
}

// Returns true when the query is over (any-hit found, or a fatal condition).
// MOT: instances and triangles are placed at the ray's shutter time.
template <bool ANY, bool MOT = false>
__device__ __forceinline__ bool op_leaf(const DevScene& S, PhaseState& ps, TravStack& st, uint32_t* err) {
    TravState& ts = ps.ts;
    const uint32_t leaf = ps.pending;
    ps.pending = 0;
    uint32_t first = leaf & LEAF_FIRST_MASK;
    uint32_t count = ((leaf >> 27) & 15u) + 1u;
    if (!ts.in_inst) {
        for (uint32_t k = count - 1; k >= 1; k--) st.push(make_leaf_ref(first + k, 1), 0.0f);
        if (st.overflow) {
            atomicOr(err, RT_DEVERR_STACK);
            return true;
        }
        // TLAS item: (instance, child of its BLAS root); the child is a
        // node to descend from or a triangle leaf tested in this leaf phase.
        const uint2 item = __ldg(S.items + first);
        const uint32_t inst = item.x, root = item.y;
        ts.cur_inst = inst;
        float4 x0, x1, x2;
        inst_rows<MOT>(S, inst, ts.time, x0, x1, x2);
        ray_pre(ts.r, xf_point(x0, x1, x2, ts.o), xf_vec(x0, x1, x2, ts.d));
        ts.in_inst = true;
        ts.inst_sp = st.sp;
        ts.cur = root;
        ps.need_pop = true;
        if (root & REF_LEAF) ps.pending = root;
        else ps.need_pop = false;
        return false;
    }
    for (uint32_t k = 0; k < count; k++) {
        float4 a, b, c;
        tri_at<MOT>(S, first + k, ts.time, a, b, c);
        float t, b1 = 0.0f, b2 = 0.0f;
        const bool hit = (S.any_curves && is_segment(c)) ? seg_intersect(ts.r.o, ts.r.d, a, b, c, ts.hit.t, t)
                                                         : tri_watertight(ts.r, xyz(a), xyz(b), xyz(c), ts.hit.t, t, b1, b2);
        if (hit) {
            ts.hit.t = t;
            ts.hit.tri = first + k;
            ts.hit.inst = ts.cur_inst;
            ts.hit.b1 = b1;
            ts.hit.b2 = b2;
            ts.found = true;
            if (ANY) return true;
        }
    }
    ps.need_pop = true;
    return false;
}

// ---- warp-cooperative triangle leaves --------------------------------------------------
// In the leaf phase the lanes of a warp hold parked BLAS leaves of 1 to 16
// triangles each. Testing its own leaf, a lane idles while the warp's largest
// leaf finishes; instead the warp pools all parked triangles (at most
// 32 x 16) and tests them 32 at a time, each lane taking the next triangle
// of the pool with its owner's (object-space) ray fetched by shuffles. A
// ray's closest hit in its leaf is the minimum of the 64-bit key
// (t bits, triangle index) over its triangles, kept with a shared-memory
// atomicMin: the smallest t, and among equal t the first triangle in leaf
// order, which is the answer of the sequential loop.
struct LeafShared {
    unsigned long long key[32];  // best (t bits << 32 | triangle) per owner lane
    float2 bary[32];             // barycentrics of that triangle
    float trans[32];             // TRANSMIT: transmittance of this leaf's hits per owner
    uint16_t item[512];          // pool item -> (owner lane << 4) | index in its leaf
};

// Shadow transmittance (TRANSMIT): the reference walks a shadow ray's
// blockers in distance order, multiplying by (1 - presence) per cutout,
// returning zero at an opaque surface or once the product falls below 1e-4,
// for at most 16 segments (src/raytracer/pt/mod.rs:1241-1306). The product
// does not depend on the order, so here one traversal visits every surface
// the segment crosses (no t_max shrinking, like any-hit) and multiplies the
// factors, ending the query at an opaque hit or below 1e-4. The answers agree
// whenever the product falls below 1e-4 within 16 cutouts or fewer than 17
// are crossed, e.g. for every presence >= 0.44.
#define RT_TRANSMIT_CUTOFF 1e-4f

// Presence cutouts inside a closest-hit query (PRES): the reference
// (src/raytracer/pt/mod.rs:702-710) meets a hit of presence p < 1 and passes
// through it with probability 1 - p, tracing on from the hit point, for at
// most 16 such skips. Here the traversal makes the same decision for every
// cutout surface it meets and ignores the surfaces it passes through, so the
// closest hit returned is the first surface that stopped the ray, in one
// traversal. Each decision is an independent uniform per (ray, surface): a
// hash of the ray's seed (drawn from the path's random state) and the
// triangle and instance. The surfaces along the ray are then accepted with
// probability p each, as in the reference; the 16-skip cap is not kept (with
// p = 1/2 a ray reaches it with probability 2^-16).
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    return h ^ (h >> 16);
}
__device__ __forceinline__ bool presence_passes(uint64_t seed, uint32_t tri, uint32_t inst, float presence) {
    const uint32_t h = fmix32((uint32_t)seed ^ fmix32((uint32_t)(seed >> 32) ^ tri * 0x9E3779B9u) ^
                              inst * 0x27D4EB2Fu);
    return (float)(h >> 8) * (1.0f / 16777216.0f) >= presence;
}

// `mine`: this lane's parked leaf is a triangle leaf to test; `seed_own`:
// this lane's ray seed (PRES). Returns true when an any-hit query found a
// hit (the query is over).
// CURV: the scene has curve sets, whose leaves hold segments (seg_intersect).
// MOT: triangles are placed at the owner ray's shutter time.
template <bool ANY, bool TRANSMIT = false, bool PRES = false, bool CURV = false, bool MOT = false>
__device__ __forceinline__ bool leaf_coop(const DevScene& S, PhaseState& ps, bool mine, LeafShared& L,
                                          uint64_t seed_own = 0) {
    const uint32_t lane = threadIdx.x & 31u;
    TravState& ts = ps.ts;
    uint32_t first = 0, count = 0;
    if (mine) {
        first = ps.pending & LEAF_FIRST_MASK;
        count = ((ps.pending >> 27) & 15u) + 1u;
        ps.pending = 0;
        ps.need_pop = true;
    }
    uint32_t incl = count;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (lane >= (uint32_t)off) incl += v;
    }
    const uint32_t excl = incl - count, total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    for (uint32_t k = 0; k < count; k++) L.item[excl + k] = (uint16_t)((lane << 4) | k);
    L.key[lane] = ~0ull;
    L.trans[lane] = 1.0f;
    // TRANSMIT / PRES: the presence of the material of this lane's instance.
    const float pres_own =
        ((TRANSMIT || PRES) && mine) ? __ldg(&S.materials[__ldg(&S.inst[ts.cur_inst].z)].presence) : 1.0f;
    __syncwarp();
    // This lane's ray, as the owners of pool items read it.
    const float tmax_own = ts.hit.t;
    const uint32_t kpack = (uint32_t)ts.r.kx | ((uint32_t)ts.r.ky << 2) | ((uint32_t)ts.r.kz << 4);
    for (uint32_t base = 0; base < total; base += 32) {
        const uint32_t idx = base + lane;
        const bool has = idx < total;
        const uint32_t it = has ? L.item[idx] : 0u;
        const uint32_t owner = it >> 4;
        RayPre r;
        r.o.x = __shfl_sync(0xFFFFFFFFu, ts.r.o.x, owner);
        r.o.y = __shfl_sync(0xFFFFFFFFu, ts.r.o.y, owner);
        r.o.z = __shfl_sync(0xFFFFFFFFu, ts.r.o.z, owner);
        r.sx = __shfl_sync(0xFFFFFFFFu, ts.r.sx, owner);
        r.sy = __shfl_sync(0xFFFFFFFFu, ts.r.sy, owner);
        r.sz = __shfl_sync(0xFFFFFFFFu, ts.r.sz, owner);
        const uint32_t kp = __shfl_sync(0xFFFFFFFFu, kpack, owner);
        const uint32_t f = __shfl_sync(0xFFFFFFFFu, first, owner);
        float tmax = __shfl_sync(0xFFFFFFFFu, tmax_own, owner);
        r.kx = (int)(kp & 3u);
        r.ky = (int)((kp >> 2) & 3u);
        r.kz = (int)((kp >> 4) & 3u);
        if (CURV) {
            r.d.x = __shfl_sync(0xFFFFFFFFu, ts.r.d.x, owner);
            r.d.y = __shfl_sync(0xFFFFFFFFu, ts.r.d.y, owner);
            r.d.z = __shfl_sync(0xFFFFFFFFu, ts.r.d.z, owner);
        }
        const float pres = __shfl_sync(0xFFFFFFFFu, pres_own, owner);
        const float tm = MOT ? __shfl_sync(0xFFFFFFFFu, ts.time, owner) : 0.0f;
        uint64_t seed = 0;
        uint32_t inst_o = 0;
        if (PRES) {
            seed = ((uint64_t)__shfl_sync(0xFFFFFFFFu, (uint32_t)(seed_own >> 32), owner) << 32) |
                   __shfl_sync(0xFFFFFFFFu, (uint32_t)seed_own, owner);
            inst_o = __shfl_sync(0xFFFFFFFFu, ts.cur_inst, owner);
        }
        float t = 0.0f, b1 = 0.0f, b2 = 0.0f;
        unsigned long long key = ~0ull;
        float factor = 1.0f;
        if (has) {
            const unsigned long long best = L.key[owner];
            // Cull with the best hit so far, keeping hits at equal t (they
            // compete on the triangle index).
            if (!TRANSMIT && best != ~0ull)
                tmax = fminf(tmax, nextafterf(__uint_as_float((uint32_t)(best >> 32)), INFINITY));
            const uint32_t tri = f + (it & 15u);
            float4 a, b, c;
            tri_at<MOT>(S, tri, tm, a, b, c);
            const bool hit = (CURV && is_segment(c)) ? seg_intersect(r.o, r.d, a, b, c, tmax, t)
                                                     : tri_watertight(r, xyz(a), xyz(b), xyz(c), tmax, t, b1, b2);
            if (hit) {
                if (TRANSMIT) {
                    factor = pres >= 1.0f ? 0.0f : 1.0f - pres;
                } else if (!(PRES && pres < 1.0f && presence_passes(seed, tri, inst_o, pres))) {
                    key = ((unsigned long long)__float_as_uint(t) << 32) | tri;
                    atomicMin(&L.key[owner], key);
                }
            }
        }
        if (TRANSMIT) {
            // Pool items of one owner are consecutive lanes: a segmented
            // product scan (fixed order, so results are reproducible) leaves
            // each run's product on its last lane.
            const uint32_t seg = has ? owner : 32u + lane;
            float prod = factor;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const float v = __shfl_up_sync(0xFFFFFFFFu, prod, off);
                const uint32_t so = __shfl_up_sync(0xFFFFFFFFu, seg, off);
                if (lane >= (uint32_t)off && so == seg) prod *= v;
            }
            const uint32_t next_seg = __shfl_down_sync(0xFFFFFFFFu, seg, 1);
            if (has && (lane == 31u || next_seg != seg)) L.trans[owner] *= prod;
            __syncwarp();
        } else {
            __syncwarp();
            if (key != ~0ull && L.key[owner] == key) L.bary[owner] = make_float2(b1, b2);
            __syncwarp();
        }
    }
    if (TRANSMIT) {
        bool over = false;
        if (mine) {
            ts.trans *= L.trans[lane];
            if (!(ts.trans >= RT_TRANSMIT_CUTOFF)) {
                ts.trans = 0.0f;
                over = true;
            }
        }
        __syncwarp();
        return over;
    }
    bool hit_now = false;
    if (mine) {
        const unsigned long long best = L.key[lane];
        if (best != ~0ull) {
            const float2 bb = L.bary[lane];
            ts.hit.t = __uint_as_float((uint32_t)(best >> 32));
            ts.hit.tri = (uint32_t)best;
            ts.hit.inst = ts.cur_inst;
            ts.hit.b1 = bb.x;
            ts.hit.b2 = bb.y;
            ts.found = true;
            hit_now = true;
        }
    }
    __syncwarp();
    return ANY && hit_now;
}

}  // namespace rt
