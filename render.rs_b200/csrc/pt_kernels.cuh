// pt_kernels.cuh — wavefront path-tracing kernels.
//
// One slab = P path slots = k whole sample passes over the image
// (slot = s_local * npix + pixel). Per wave:
//   extend   closest hit for the queued slots, then push each slot onto the
//            queue of its hit's material class (miss, diffuse, conductor,
//            glass, mixed, emitter) with warp-aggregated atomics;
//   shade    classes in order, so warps see one BSDF: emission with MIS,
//            presence skip, NEE light pick + sample (shadow ray queued with
//            its contribution), BSDF sample, Russian roulette, next ray;
//   shadow   any hit (or the presence-attenuating closest-hit loop) and,
//            when visible, add the queued contribution to the slot's L.
// accumulate then clamps each sample (firefly) and adds it to the f64
// per-pixel accumulator in sample order, so the image is bitwise
// reproducible for a seed whatever order the queues were filled in.
//
// Reference: trace_full (src/raytracer/pt/mod.rs:449-990), sample_light
// (:1032-1209), transmittance (:1254-1306), render/render_sum (:71-133);
// the Metal wavefront it replaces is kernel_wf.metal:155-325.
#pragma once

#include "guide.cuh"
#include "pattern.cuh"
#include "quadric.cuh"
#include "media.cuh"
#include "hair.cuh"

namespace rt {

enum : uint32_t { CLS_MISS = N_MAT_CLASSES, N_QUEUES = N_MAT_CLASSES + 1 };

// Counter words (uint32) in Paths::cnt.
enum : uint32_t {
    CNT_EXT_IN = 0,
    CNT_EXT_OUT = 1,
    CNT_SHADOW = 2,
    CNT_CLASS = 3,                  // N_QUEUES words
    CNT_FETCH_EXT = CNT_CLASS + N_QUEUES,
    CNT_FETCH_SH = CNT_FETCH_EXT + 1,
    CNT_SSS = CNT_FETCH_SH + 1,     // subsurface walks queued this wave
    CNT_WORDS = 16
};

// Shadow-queue entries of scenes with media: the slot, bit 30 set when its
// surface / collision / walk-exit shadow ray (sh_*) is pending, bit 31 when
// its equiangular one (sh2_*) is; one entry per slot, so one thread adds
// both contributions in a fixed order.
#define SH_PRIMARY (1u << 30)
#define SH_EQUI (1u << 31)
#define SH_SLOT_MASK (SH_PRIMARY - 1u)

struct Paths {
    float* time;      // shutter time of the path (scenes with motion blur; else unused)
    float4* ray_o;    // origin xyz, w = roulette gain (see k_shade)
    float4* ray_d;    // direction xyz, w = tmax
    uint4* hit;       // t bits, tri (leaf order), inst (leaf order), b1|b2 half2
    float4* beta;     // throughput xyz, w = prev bsdf pdf
    float4* L;        // radiance xyz, w = travelled distance
    float4* prev;     // previous vertex xyz, w = flag bits
    uint4* rng;       // pcg state (lo, hi), inc (lo, hi)
    float4* sh_o;     // shadow origin xyz
    float4* sh_d;     // shadow direction xyz, w = remaining distance
    float4* sh_c;     // pending contribution xyz, w = 1 if it belongs to the diffuse AOV
    float4* aux_a;    // albedo xyz, depth
    float4* aux_n;    // normal xyz, id bits
    float4* aux_d;    // diffuse share xyz, hit flag
    float2* cone;     // ray cone (width, spread) when the scene has patterns, else null
    uint2* med;       // nested-media stack (media.cuh) when the scene has media, else null
    float4* sh2_o;    // equiangular shadow ray toward a point light (scenes with media):
    float4* sh2_d;    //   origin xyz + medium bits, direction xyz + distance,
    float4* sh2_c;    //   contribution xyz + diffuse-AOV flag
    uint32_t* q_sss;  // subsurface walks queued this wave (scenes with a walk), else null
    uint32_t* q_ext[2];
    uint32_t* q_cls;  // N_QUEUES x P
    uint32_t* q_sh;
    uint32_t* cnt;
    unsigned long long* stats;  // [0] extension rays, [1] shadow rays
    uint32_t* err;
    uint32_t P;
    // learned proposal (guided mode)
    float* g_rec;          // inference records, 16 floats (position, normal, wo)
    uint32_t* g_idx;       // slot -> inference record (~0 when not guided)
    uint32_t* g_cnt;       // number of inference records this wave
    const float* g_raw;    // decoded mixtures, 48 floats per inference record (guide.cuh)
    float* tr_rec;         // training vertices: [P][max_depth] x TR_FLOATS
    float* tb_rec;         // training batch, 16 floats per record
    uint32_t* tb_cnt;      // [0] records kept, [1] candidate records
    uint32_t* tb_blk;      // collection: kept records per block, then their offsets
    float* tr_keep;        // probability of keeping a candidate (device word)
    uint32_t tr_tag, tb_cap;
};

// Training vertex: p(3) n(3) wo(3) wi(3) beta(3) L at the next vertex(3),
// then the slab tag of its opening and of its closing (as uint bits). A
// record belongs to the current slab when both tags equal Paths::tr_tag,
// so stale records of earlier slabs never need clearing.
#define TR_FLOATS 20

struct PtConsts {
    uint32_t npix, width, max_depth, rr_start, aovs;
    uint32_t pres_in_trav;  // cutouts are decided inside k_extend's traversal; k_shade skips none
    float clamp;
    uint64_t sample0;  // first sample index of the slab
    uint32_t guided;
    uint32_t train;    // guided and still training: shading writes training vertices
    float alpha;       // one-sample MIS probability of sampling the guide
    GuideDev G;
    // Adaptive sampling (tol > 0): per pixel (luminance sum, luminance^2 sum,
    // samples counted), updated by k_accumulate, read by k_raygen.
    float adaptive_tol;
    double* lum_stats;
};

// flag bits in Paths::prev.w
#define FL_FROM_CAMERA 1u
#define FL_SKIP_SHIFT 1
#define FL_SKIP_MASK (31u << FL_SKIP_SHIFT)
#define FL_SPEC_SHIFT 6
#define FL_SPEC_NONE (3u << FL_SPEC_SHIFT)
#define FL_SPEC_TRUE (1u << FL_SPEC_SHIFT)
#define FL_SPEC_MASK (3u << FL_SPEC_SHIFT)
#define FL_AUX_SET (1u << 8)
#define FL_INACTIVE (1u << 9)   // adaptive sampling: the pixel had converged, no path was spawned
#define FL_SH2 (1u << 10)       // an equiangular shadow ray waits for the subsurface walk's queue entry
#define FL_DEPTH_SHIFT 16

#define RT_RAY_OFFSET 1e-4f
// Traversal kernels are latency-bound at a few warps per SM: asking the
// register allocator for 5 resident 128-thread blocks (at most 102 registers,
// no spills) raised closest hit from 219 to 246 Mrays/s on the 1M-triangle
// cloud; 6 blocks spills and no longer fits the 39 KB of shared memory a
// block holds with the 32-entry stack.
#ifndef RT_TRAV_MIN_BLOCKS
#define RT_TRAV_MIN_BLOCKS 5
#endif
#define RT_MAX_PRESENCE_SKIPS 16u

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated queue push of `val` into queue `q` (counter `c`).
__device__ __forceinline__ void push_queue(uint32_t* q, uint32_t* c, uint32_t val, bool active) {
    uint32_t m = __ballot_sync(0xFFFFFFFFu, active);
    if (!m) return;
    uint32_t leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(c, __popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (active) q[base + __popc(m & ((1u << lane_id()) - 1u))] = val;
}

// Hit point, world normal flipped against the ray (to_intersection,
// src/geometry/mesh.rs:427-439: front face from the unflipped normal),
// outgoing direction and material of a closest-hit record.
struct HitGeo {
    float3 p, nw, wo;
    float eucl;
    uint32_t mat;
    bool front;
    bool curve;  // a curve-set segment (hair shading applies)
};

// `time`: the path's shutter time (motion blur): moving instances and
// deforming meshes are taken at it (Instance::intersect, mesh.rs:308-381).
__device__ __forceinline__ void hit_geometry(const DevScene& S, float3 o, float3 d, uint4 hr, HitGeo& g,
                                             float time = 0.0f) {
    float t = __uint_as_float(hr.x);
    g.p = o + d * t;
    g.wo = -normalize_ref(d);
    g.eucl = length(g.p - o);
    g.curve = false;
    if (hr.y & RT_TRI_QUADRIC) {
        // Quadric: normal and front face as the shape reports them
        // (not flipped; shading flips toward wo as for every hit).
        const uint32_t k = hr.y & ~RT_TRI_QUADRIC;
        quadric_surface(S, k, g.p, d, g.nw, g.front, nullptr);
        g.mat = S.quadrics[k].material;
        return;
    }
    uint32_t il = hr.z;
    float4 x0, x1, x2, v0, v1, v2;
    inst_rows<true>(S, il, time, x0, x1, x2);
    uint4 info = __ldg(S.inst + il);
    tri_at<true>(S, hr.y, time, v0, v1, v2);
    float3 nl;
    MeshInfo mi = S.meshes[info.w];
    if (mi.attrs & MESH_CURVES) {
        // Curve segment (mesh.rs:323-344): the rounded cone's outward
        // normal at the hit, flipped against the ray as meshes are.
        float tt;
        nl = f3(0.0f, 0.0f, 1.0f);
        seg_intersect(xf_point(x0, x1, x2, o), xf_vec(x0, x1, x2, d), v0, v1, v2, INFINITY, tt, &nl);
        g.curve = true;
    } else if ((mi.attrs & MESH_NORMALS) && __float_as_uint(v1.w) != RT_DEFORM_MARK) {
        // Interpolated vertex normals (Mesh::local_normal, mesh.rs:200-220);
        // a deforming mesh takes the geometric normal at the shutter time.
        float b1 = __half2float(__ushort_as_half((unsigned short)(hr.w & 0xFFFFu)));
        float b2 = __half2float(__ushort_as_half((unsigned short)(hr.w >> 16)));
        uint32_t ot = __float_as_uint(v0.w);
        const uint32_t* ix = S.orig_idx + mi.idx_base + 3 * (size_t)ot;
        auto nrm = [&](uint32_t v) { return f3(S.normals[3 * v], S.normals[3 * v + 1], S.normals[3 * v + 2]); };
        nl = normalize_ref(nrm(ix[0]) * (1.0f - b1 - b2) + nrm(ix[1]) * b1 + nrm(ix[2]) * b2);
    } else {
        nl = normalize_ref(cross(xyz(v1) - xyz(v0), xyz(v2) - xyz(v0)));
    }
    float3 nw = normalize_ref(xf_normal(x0, x1, x2, nl));
    g.front = dot(nw, d) < 0.0f;
    g.nw = g.front ? nw : -nw;
    g.mat = info.z;
}

// World tangent of a curve hit (mesh.rs:342): the segment's axis (0, 0, 1
// for a point particle) through the instance's object-to-world transform,
// which is the inverse of the stored world-to-object rows: the adjugate's
// columns are their pairwise cross products.
__device__ __forceinline__ float3 curve_tangent(const DevScene& S, uint4 hr) {
    const float4* tp = S.tris + 3 * (size_t)hr.y;
    const float3 axis = xyz(__ldg(tp + 1)) - xyz(__ldg(tp));
    const float3 a = dot(axis, axis) > 1e-24f ? axis : f3(0.0f, 0.0f, 1.0f);
    const float4 x0 = __ldg(S.inst_xf + 3 * (size_t)hr.z), x1 = __ldg(S.inst_xf + 3 * (size_t)hr.z + 1),
                 x2 = __ldg(S.inst_xf + 3 * (size_t)hr.z + 2);
    const float3 r0 = xyz(x0), r1 = xyz(x1), r2 = xyz(x2);
    const float3 w = cross(r1, r2) * a.x + cross(r2, r0) * a.y + cross(r0, r1) * a.z;
    return normalize_ref(dot(r0, cross(r1, r2)) < 0.0f ? -w : w);
}

// (s, t), st density (st units per world unit) and the world-space st
// gradients at a closest hit: Mesh::st_at and st_gradients
// (src/geometry/mesh.rs:147-197) with the density carried to world scale
// by the instance's approx_scale and the gradients pulled back through the
// world-to-object transform (mesh.rs:357-371); zeros when the mesh has no st.
// With motion blur the hit's barycentrics come from the instance and the
// triangle at the path's shutter `time` (the reference's hit uv), while the
// density and the gradients keep the rest pose and the shutter-open
// transform, as Mesh::st_at / st_gradients and Instance::inverse do.
__device__ __forceinline__ HitSt hit_st(const DevScene& S, uint4 hr, float3 p, float time = 0.0f) {
    HitSt r{0.0f, 0.0f, 0.0f, f3(0.0f, 0.0f, 0.0f), f3(0.0f, 0.0f, 0.0f)};
    if (hr.y & RT_TRI_QUADRIC) {
        // The quadric's RiSpec (u, v) and density; no st gradients (the
        // reference's quadrics set none).
        float st[3];
        float3 nw;
        bool front;
        quadric_surface(S, hr.y & ~RT_TRI_QUADRIC, p, f3(0.0f, 0.0f, 1.0f), nw, front, st);
        r.s = st[0];
        r.t = st[1];
        r.dens = st[2];
        return r;
    }
    const uint4 info = __ldg(S.inst + hr.z);
    const MeshInfo mi = S.meshes[info.w];
    if (mi.attrs & MESH_CURVES) {
        // st = (0.5, v) with v the curve parameter along the segment, no
        // density (mesh.rs:323-344).
        const float4* tp = S.tris + 3 * (size_t)hr.y;
        const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float4 x0, x1, x2;
        inst_rows<true>(S, hr.z, time, x0, x1, x2);
        const float3 axis = xyz(b) - xyz(a);
        const float len2 = dot(axis, axis);
        const float along =
            len2 > 1e-24f ? fminf(fmaxf(dot(xf_point(x0, x1, x2, p) - xyz(a), axis) / len2, 0.0f), 1.0f) : 0.5f;
        r.s = 0.5f;
        r.t = c.y + (c.z - c.y) * along;
        return r;
    }
    if (!(mi.attrs & MESH_ST)) return r;
    const float4* tp = S.tris + 3 * (size_t)hr.y;
    const float4 v0 = __ldg(tp), v1 = __ldg(tp + 1), v2 = __ldg(tp + 2);
    const float4 x0 = __ldg(S.inst_xf + 3 * (size_t)hr.z), x1 = __ldg(S.inst_xf + 3 * (size_t)hr.z + 1),
                 x2 = __ldg(S.inst_xf + 3 * (size_t)hr.z + 2);
    const float3 e1 = xyz(v1) - xyz(v0), e2 = xyz(v2) - xyz(v0);
    const float3 nl = cross(e1, e2);
    const float n2 = dot(nl, nl);
    // Barycentrics of the hit point in f32 (the hit record's are half
    // precision, ~1e-3 of the triangle: too coarse for texture lookups).
    float b1 = __half2float(__ushort_as_half((unsigned short)(hr.w & 0xFFFFu)));
    float b2 = __half2float(__ushort_as_half((unsigned short)(hr.w >> 16)));
    if (time > 0.0f && S.motion) {
        // The hit's triangle and instance at the shutter time.
        float4 y0, y1, y2, w0, w1, w2;
        inst_rows<true>(S, hr.z, time, y0, y1, y2);
        tri_at<true>(S, hr.y, time, w0, w1, w2);
        const float3 f1 = xyz(w1) - xyz(w0), f2 = xyz(w2) - xyz(w0), fn = cross(f1, f2);
        const float m2 = dot(fn, fn);
        if (m2 > 0.0f) {
            const float3 q = xf_point(y0, y1, y2, p) - xyz(w0);
            b1 = dot(cross(q, f2), fn) / m2;
            b2 = dot(cross(f1, q), fn) / m2;
        }
    } else if (n2 > 0.0f) {
        const float3 q = f3(dot(xyz(x0), p) + x0.w, dot(xyz(x1), p) + x1.w, dot(xyz(x2), p) + x2.w) - xyz(v0);
        b1 = dot(cross(q, e2), nl) / n2;
        b2 = dot(cross(e1, q), nl) / n2;
    }
    const uint32_t* ix = S.orig_idx + mi.idx_base + 3 * (size_t)__float_as_uint(v0.w);
    const float2* st = reinterpret_cast<const float2*>(S.st);
    const float2 s0 = st[ix[0]], s1 = st[ix[1]], s2 = st[ix[2]];
    const float w = 1.0f - b1 - b2;
    r.s = s0.x * w + s1.x * b1 + s2.x * b2;
    r.t = s0.y * w + s1.y * b1 + s2.y * b2;
    const float st_area = 0.5f * fabsf((s1.x - s0.x) * (s2.y - s0.y) - (s2.x - s0.x) * (s1.y - s0.y));
    const float geo_area = 0.5f * length(nl);
    r.dens = (geo_area > 1e-18f ? sqrtf(st_area / geo_area) : 0.0f) / __ldg(S.inst_scale + info.y);
    if (n2 >= 1e-24f) {
        const float3 d1 = cross(e2, nl) / n2, d2 = cross(e1, nl) / -n2;
        const float3 gs = d1 * (s1.x - s0.x) + d2 * (s2.x - s0.x);
        const float3 gt = d1 * (s1.y - s0.y) + d2 * (s2.y - s0.y);
        r.gs = xf_normal(x0, x1, x2, gs);
        r.gt = xf_normal(x0, x1, x2, gt);
    }
    return r;
}

// ---- raygen: camera rays for all P slots ------------------------------------------
// render_pt prologue (kernel_pt.metal:2389-2434) / pt::camera_ray (mod.rs:340-356).
__device__ __forceinline__ float filter_offset(uint32_t kind, float width, float u) {
    if (kind == 1u) {
        float hw = width * 0.5f;
        return u < 0.5f ? (sqrtf(2.0f * u) - 1.0f) * hw : (1.0f - sqrtf(2.0f * (1.0f - u))) * hw;
    }
    if (kind == 2u) {
        // The second uniform is fract(u * 2654435761) as camera.rs:55 forms
        // it in f64. In f32 the product is a whole number for every
        // u > 2^-8 (its ulp there is >= 256), so u2 would be 0, the cosine 1
        // and every offset >= 0: a half-Gaussian shifted off the pixel
        // centre. One f64 multiply per camera ray keeps it centred.
        float u1 = fmaxf(u, 1e-12f);
        const double x = (double)u * 2654435761.0;
        float u2 = (float)(x - trunc(x));
        float g = sqrtf(-2.0f * logf(u1)) * cosf(2.0f * RT_PI * u2);
        return fminf(fmaxf(g * (width * 0.25f), -width * 0.5f), width * 0.5f);
    }
    return (u - 0.5f) * width;
}

// Adaptive sampling, as the reference's wavefront raygen
// (kernel_wf.metal:173-183): from sample 32 on, a pixel with at least 16
// samples stops spawning paths once the 95% confidence interval of its
// luminance, 1.96 sqrt(var / n), is below tol * max(mean, 0.05).
__device__ __forceinline__ bool pixel_converged(const PtConsts& C, uint32_t pixel, uint64_t sample) {
    if (sample < 32) return false;
    const double* st = C.lum_stats + 4 * (size_t)pixel;
    const double n = st[2];
    if (n < 16.0) return false;
    const double mean = st[0] / n;
    const double var = fmax(st[1] / n - mean * mean, 0.0);
    return 1.96 * sqrt(var / n) < (double)C.adaptive_tol * fmax(mean, 0.05);
}

__global__ void k_raygen(DevScene S, Paths P, PtConsts C) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool adaptive = C.adaptive_tol > 0.0f;
    uint32_t pixel = i % C.npix;
    uint64_t sample = C.sample0 + i / C.npix;
    if (adaptive) {
        // Converged pixels get no path; live ones are compacted into the queue.
        const bool live = i < P.P && !pixel_converged(C, pixel, sample);
        push_queue(P.q_ext[0], &P.cnt[CNT_EXT_IN], i, live);
        if (i >= P.P) return;
        if (!live) {
            P.L[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            P.prev[i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(FL_INACTIVE));
            return;
        }
    }
    if (i >= P.P) return;
    Pcg rng = pcg_for_pixel_sample(pixel, sample);
    uint32_t x = pixel % S.width, y = pixel / S.width;
    float fu = rng.next_f(), fv = rng.next_f();
    float px = (float)x + 0.5f + filter_offset(S.filter, S.filter_width, fu);
    float py = (float)y + 0.5f + filter_offset(S.filter, S.filter_width, fv);
    float uu = (px / (float)S.width) * 2.0f - 1.0f;
    float vv = 1.0f - (py / (float)S.height) * 2.0f;
    float3 eye = f3(S.eye[0], S.eye[1], S.eye[2]);
    float3 fwd = f3(S.fwd[0], S.fwd[1], S.fwd[2]);
    float3 rgt = f3(S.right[0], S.right[1], S.right[2]);
    float3 upv = f3(S.up[0], S.up[1], S.up[2]);
    float3 dir = fwd + rgt * (uu * S.half_w) + upv * (vv * S.half_h);
    float3 o = eye, d;
    if (S.projection == RT_PROJECTION_ORTHOGRAPHIC) {
        // Rays start on the screen window, parallel to forward (camera.rs:
        // 154-159). The lens samples are still drawn when the lens is open,
        // as pt::camera_ray draws them before generating the ray.
        if (S.lens_radius > 0.0f) {
            rng.next_f();
            rng.next_f();
        }
        o = eye + rgt * (uu * S.ortho_hw) + upv * (vv * S.ortho_hh);
        d = normalize_ref(fwd);
    } else if (S.lens_radius > 0.0f) {
        float lu = rng.next_f(), lv = rng.next_f();
        float r = S.lens_radius * sqrtf(lu), sp, cp;
        sincosf(2.0f * RT_PI * lv, &sp, &cp);
        float3 off = rgt * (r * cp) + upv * (r * sp);
        float3 focus = eye + dir * S.focal_distance;
        o = eye + off;
        d = normalize_ref(focus - o);
    } else {
        d = normalize_ref(dir);
    }
    if (S.motion) {
        // Shutter time after the filter and lens draws (pt/mod.rs:350-353,
        // kernel_pt.metal:2422-2434); camera motion moves the ray by
        // lerp(I, motion_inv, t), its direction renormalised.
        const float tm = rng.next_f();
        P.time[i] = tm;
        if (S.cam_moving && tm > 0.0f) {
            const float* M = S.cam_mot;
            float4 r[3];
#pragma unroll
            for (int k = 0; k < 3; k++)
                r[k] = make_float4((k == 0 ? 1.0f : 0.0f) + (M[4 * k] - (k == 0 ? 1.0f : 0.0f)) * tm,
                                   (k == 1 ? 1.0f : 0.0f) + (M[4 * k + 1] - (k == 1 ? 1.0f : 0.0f)) * tm,
                                   (k == 2 ? 1.0f : 0.0f) + (M[4 * k + 2] - (k == 2 ? 1.0f : 0.0f)) * tm,
                                   M[4 * k + 3] * tm);
            o = xf_point(r[0], r[1], r[2], o);
            d = normalize_ref(xf_vec(r[0], r[1], r[2], d));
        }
    }
    P.ray_o[i] = make_float4(o.x, o.y, o.z, 1.0f);
    P.ray_d[i] = make_float4(d.x, d.y, d.z, INFINITY);
    P.beta[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.L[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.prev[i] = make_float4(o.x, o.y, o.z, __uint_as_float(FL_FROM_CAMERA | FL_SPEC_NONE));
    if (P.med) P.med[i] = make_uint2(0u, 0u);  // camera rays start in the atmosphere
    // Ray cone: width 0, spread one pixel's angle (kernel_pt.metal:2283-2284).
    if (P.cone) P.cone[i] = make_float2(0.0f, 2.0f * S.half_h / (float)S.height);
    P.rng[i] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), (uint32_t)rng.inc,
                          (uint32_t)(rng.inc >> 32));
    if (C.aovs) {
        P.aux_a[i] = make_float4(0, 0, 0, 0);
        P.aux_n[i] = make_float4(0, 0, 0, 0);
        P.aux_d[i] = make_float4(0, 0, 0, 0);
    }
    if (!adaptive) {
        P.q_ext[0][i] = i;
        if (i == 0) P.cnt[CNT_EXT_IN] = P.P;
    }
}

// ---- learned proposal: network inputs for this wave's guided vertices ------------------
// Vertices of diffuse, conductor and mixed materials (below guide_depth when
// it is set) get a record (position, shading normal facing wo, wo); the shade
// kernel reads the network output through g_idx. Glass, emitters, misses and
// deeper vertices keep plain BSDF sampling.
__global__ void __launch_bounds__(128) k_guide_gather(DevScene S, Paths P, uint32_t guide_depth) {
    uint32_t counts[N_QUEUES];
    uint32_t total = 0;
#pragma unroll
    for (uint32_t c = 0; c < N_QUEUES; c++) {
        counts[c] = P.cnt[CNT_CLASS + c];
        total += counts[c];
    }
    uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j0 = blockIdx.x * blockDim.x; j0 < total; j0 += stride) {
        uint32_t j = j0 + threadIdx.x;
        bool active = j < total, want = false;
        uint32_t slot = 0;
        float rec[9];
        if (active) {
            uint32_t c = CLS_MISS, off = j;
            if (off >= counts[CLS_MISS]) {
                off -= counts[CLS_MISS];
                for (uint32_t k = 0; k < N_MAT_CLASSES; k++) {
                    if (off < counts[k]) {
                        c = k;
                        break;
                    }
                    off -= counts[k];
                }
            }
            slot = P.q_cls[(size_t)c * P.P + off];
            want = c == MAT_DIFFUSE || c == MAT_CONDUCTOR || c == MAT_MIXED;
            if (want && guide_depth) want = (__float_as_uint(P.prev[slot].w) >> FL_DEPTH_SHIFT) < guide_depth;
            if (want) {
                HitGeo hg;
                hit_geometry(S, xyz(P.ray_o[slot]), xyz(P.ray_d[slot]), P.hit[slot], hg,
                             S.motion ? P.time[slot] : 0.0f);
                float3 n = dot(hg.nw, hg.wo) >= 0.0f ? hg.nw : -hg.nw;
                rec[0] = hg.p.x; rec[1] = hg.p.y; rec[2] = hg.p.z;
                rec[3] = n.x; rec[4] = n.y; rec[5] = n.z;
                rec[6] = hg.wo.x; rec[7] = hg.wo.y; rec[8] = hg.wo.z;
            } else {
                P.g_idx[slot] = 0xFFFFFFFFu;
            }
        }
        uint32_t m = __ballot_sync(0xFFFFFFFFu, want);
        if (m) {
            uint32_t leader = __ffs(m) - 1, base = 0;
            if (lane_id() == leader) base = atomicAdd(P.g_cnt, __popc(m));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (want) {
                uint32_t idx = base + __popc(m & ((1u << lane_id()) - 1u));
                P.g_idx[slot] = idx;
                float4* r = reinterpret_cast<float4*>(P.g_rec + (size_t)idx * 16);
                r[0] = make_float4(rec[0], rec[1], rec[2], rec[3]);
                r[1] = make_float4(rec[4], rec[5], rec[6], rec[7]);
                r[2] = make_float4(rec[8], 0.f, 0.f, 0.f);
                r[3] = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    }
}

// ---- learned proposal: training batch from the slab's closed vertices -------------------
// weight = lum(L_end - L_vertex) / lum(beta_vertex) estimates
// lum(f cos Li) / pdf for the direction the path actually took (capped at 50).
// Every path of the slab recorded its vertices; a candidate (a closed record
// of positive weight) is kept with probability *tr_keep, decided by a hash of
// (slot, depth, slab tag), so the batch is a spatially uniform subsample.
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    // integer finaliser ("lowbias32", C. Wellons, hash-prospector)
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// Collection of the slab's closed training vertices, one thread per (slot,
// depth): the records of a path are consecutive, so the threads of a warp
// read neighbouring records of a few paths. A path opened records
// 0 .. depth-1 (its final bounce count); threads past that touch nothing.
// Whether a vertex is a candidate and whether it is kept depend only on the
// vertex (the keep draw hashes (slot, depth, slab tag)), and the kept records
// are written in (slot, depth) order -- per-block counts, an exclusive scan
// of the counts, then each record at its block's offset plus its rank in the
// block -- so the batches the Adam steps take are the same on every run.
__device__ __forceinline__ bool collect_vertex(const Paths& P, const PtConsts& C, float keep, uint64_t id, bool& cand,
                                               float& wt, const float*& rec) {
    const uint32_t slot = (uint32_t)(id / C.max_depth), d = (uint32_t)(id % C.max_depth);
    cand = false;
    wt = 0.0f;
    rec = nullptr;
    if (slot >= P.P || d >= (__float_as_uint(P.prev[slot].w) >> FL_DEPTH_SHIFT)) return false;
    const float* r = P.tr_rec + ((size_t)slot * C.max_depth + d) * TR_FLOATS;
    float2 tags = *reinterpret_cast<const float2*>(r + 18);
    if (__float_as_uint(tags.x) != P.tr_tag || __float_as_uint(tags.y) != P.tr_tag) return false;
    const float4 Le = P.L[slot];
    float3 dl = f3(Le.x - r[15], Le.y - r[16], Le.z - r[17]);
    float w = luminance(dl) / fmaxf(luminance(f3(r[12], r[13], r[14])), 1e-8f);
    cand = w > 0.0f && isfinite(w);
    uint32_t h = hash32((slot * C.max_depth + d) ^ hash32(P.tr_tag));
    wt = w;
    rec = r;
    return cand && (float)(h >> 8) * (1.0f / 16777216.0f) < keep;
}

#define COLLECT_BLOCK 256

// Pass 1: kept records per block (P.tb_blk), candidates counted into
// tb_cnt[1] (an integer sum: the same in any order).
__global__ void __launch_bounds__(COLLECT_BLOCK) k_guide_collect_count(Paths P, PtConsts C) {
    __shared__ uint32_t warp_kept[COLLECT_BLOCK / 32];
    const float keep = *P.tr_keep;
    const uint64_t id = (uint64_t)blockIdx.x * COLLECT_BLOCK + threadIdx.x;
    bool cand;
    float wt;
    const float* rec;
    const bool kept = collect_vertex(P, C, keep, id, cand, wt, rec);
    const uint32_t km = __ballot_sync(0xFFFFFFFFu, kept), cm = __ballot_sync(0xFFFFFFFFu, cand);
    if (lane_id() == 0) {
        warp_kept[threadIdx.x >> 5] = __popc(km);
        if (cm) atomicAdd(P.tb_cnt + 1, (uint32_t)__popc(cm));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < COLLECT_BLOCK / 32; w++) t += warp_kept[w];
        P.tb_blk[blockIdx.x] = t;
    }
}

// Pass 2: exclusive scan of the nb block counts in place (one block), total
// kept into tb_cnt[0].
__global__ void __launch_bounds__(1024) k_guide_collect_scan(uint32_t* blk, uint32_t nb, uint32_t* tb_cnt) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x, per = (nb + 1023) / 1024, b0 = t * per, b1 = min(nb, b0 + per);
    uint32_t sum = 0;
    for (uint32_t b = b0; b < b1; b++) sum += blk[b];
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        const uint32_t v = t >= off ? part[t - off] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;  // exclusive prefix of this thread's chunk
    for (uint32_t b = b0; b < b1; b++) {
        const uint32_t c = blk[b];
        blk[b] = run;
        run += c;
    }
    if (t == 1023) tb_cnt[0] = part[1023];
}

// Pass 3: each kept record to its block's offset plus its rank in the block.
__global__ void __launch_bounds__(COLLECT_BLOCK) k_guide_collect_write(Paths P, PtConsts C) {
    __shared__ uint32_t warp_off[COLLECT_BLOCK / 32];
    const float keep = *P.tr_keep;
    const uint64_t id = (uint64_t)blockIdx.x * COLLECT_BLOCK + threadIdx.x;
    bool cand;
    float wt;
    const float* rec;
    const bool kept = collect_vertex(P, C, keep, id, cand, wt, rec);
    const uint32_t km = __ballot_sync(0xFFFFFFFFu, kept);
    if (lane_id() == 0) warp_off[threadIdx.x >> 5] = __popc(km);
    __syncthreads();
    if (!kept) return;
    uint32_t base = P.tb_blk[blockIdx.x];
    for (uint32_t w = 0; w < (threadIdx.x >> 5); w++) base += warp_off[w];
    const uint32_t idx = base + __popc(km & ((1u << lane_id()) - 1u));
    if (idx < P.tb_cap) {
        float4* o = reinterpret_cast<float4*>(P.tb_rec + (size_t)idx * 16);
        const float4* ri = reinterpret_cast<const float4*>(rec);
        o[0] = ri[0];
        o[1] = ri[1];
        o[2] = ri[2];
        o[3] = make_float4(fminf(wt, 50.0f), 0.0f, 0.0f, 0.0f);
    }
}

// Keep probability for this slab's collection: aim the expected batch at 95%
// of the training capacity, given the previous slab's number of candidates
// (scaled by the ratio of the slabs' sample passes).
__global__ void k_guide_keep(const uint32_t* tb_cnt, float scale, uint32_t cap, float* keep) {
    float cand = (float)tb_cnt[1] * scale;
    *keep = cand > 0.0f ? fminf(1.0f, 0.95f * (float)cap / cand) : 1.0f;
}

// ---- persistent ray pump ----------------------------------------------------------------
// Each warp keeps 32 rays in flight. A lane whose ray finishes is refilled
// from the global work counter as soon as half the warp is idle (one
// warp-aggregated atomic per refill), so a few long rays no longer hold a
// warp's other lanes hostage (Aila & Laine 2009, "persistent while-while").
// load(j, o, d, tmax, seed, time) reads work item j (seed: the ray's
// presence seed, see leaf_coop; time: its shutter time, read with MOT);
// finish(done, j, ts) is called by
// the whole warp whenever some lane finished, with `done` true on those lanes.
// Within a warp the work alternates between a node phase (every lane that
// has no parked leaf tests nodes until it parks one or finishes) and a leaf
// phase (every lane with a parked leaf processes it), so lanes mostly run
// the same code path.
// A node phase ends once at most RT_NODE_PHASE_EXIT lanes still want node
// steps (and some lane has a parked leaf): the other lanes would idle while
// the last few walk down to their leaves, so they take their leaf phase now
// and the stragglers continue in the next node phase. Idle lanes are refilled
// once at most S.refill_at lanes hold a ray (RT_REFILL_SPARSE, or
// RT_REFILL_DENSE in scenes of densely overlapping instances: rt_internal.h).
// On the 1M-triangle cloud (B200), against running every node phase to the
// end with refills at 16: closest hit 286 -> 422 Mrays/s, any hit 420 -> 678,
// a 1920x1080 16-spp frame 154 -> 119 ms; thresholds 12-16 were within 2% of
// each other.
#ifndef RT_NODE_PHASE_EXIT
#define RT_NODE_PHASE_EXIT 14
#endif
// A node-phase step pops the next entry and tests it at once when it is a
// node (RT_FUSED_POP), instead of spending a whole warp step on the pop
// while other lanes test nodes: closest hit 422 -> 484 Mrays/s, the
// 1080p cloud frame 119 -> 105 ms. Entering instance leaves inside the node
// phase (RT_INST_IN_NODE_PHASE, with RT_FUSED_POP) made the forest frame 3-8%
// slower, so instance leaves wait for the leaf phase.
#ifndef RT_FUSED_POP
#define RT_FUSED_POP 1
#endif
#ifndef RT_INST_IN_NODE_PHASE
#define RT_INST_IN_NODE_PHASE 0
#endif
template <bool ANY, bool TRANSMIT = false, bool PRES = false, bool CURV = false, bool MOT = false, class Load,
          class Finish>
__device__ __forceinline__ void ray_pump(const DevScene& S, uint32_t n, uint32_t* fetch, uint32_t* err,
                                         TravStack& st, LeafShared& leaf, Load load, Finish finish) {
    PhaseState ps;
    bool active = false, exhausted = false;
    uint32_t item = 0, steps = 0;
    uint64_t ray_seed = 0;  // PRES: the current ray's presence seed
    const uint32_t lane = lane_id(), lt = (1u << lane) - 1u;
    for (;;) {
        uint32_t act = __ballot_sync(0xFFFFFFFFu, active);
        if (!exhausted && __popc(act) <= S.refill_at) {
            uint32_t idle = ~act;
            uint32_t leader = __ffs(idle) - 1, base = 0;
            if (lane == leader) base = atomicAdd(fetch, __popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (base >= n || n - base <= (uint32_t)__popc(idle)) exhausted = true;
            bool fresh = false;
            if (!active) {
                uint32_t j = base + __popc(idle & lt);
                if (base < n && j < n) {
                    item = j;
                    float3 o, d;
                    float tmax, time = 0.0f;
                    uint64_t seed = 0;
                    load(j, o, d, tmax, seed, time);
                    active = trav_begin(S, ps.ts, st, o, d, tmax, MOT ? time : 0.0f);
                    if (PRES) ray_seed = seed;
                    if (active) {
                        phase_begin(ps);
                        steps = 0;
                    } else {
                        fresh = true;  // empty scene: a miss, finished at once
                    }
                }
            }
            if (__any_sync(0xFFFFFFFFu, fresh)) finish(fresh, item, ps.ts);
            act = __ballot_sync(0xFFFFFFFFu, active);
        }
        if (act == 0) {
            if (exhausted) break;
            continue;
        }
        // Node phase.
        for (;;) {
            bool want = active && (ps.pending == 0 || (RT_FUSED_POP && RT_INST_IN_NODE_PHASE && !ps.ts.in_inst));
            const uint32_t wm = __ballot_sync(0xFFFFFFFFu, want);
            if (!wm) break;
            if (RT_NODE_PHASE_EXIT > 0 && __popc(wm) <= RT_NODE_PHASE_EXIT &&
                __any_sync(0xFFFFFFFFu, active && ps.pending != 0))
                break;
            bool done_now = false;
            if (want) {
                if (++steps > S.max_steps) {
                    atomicOr(err, RT_DEVERR_ITER);
                    done_now = true;
                } else if (RT_FUSED_POP) {
                    // One step: enter a parked instance leaf, or pop; then
                    // test the node that is current, if any.
                    if (RT_INST_IN_NODE_PHASE && ps.pending && !ps.ts.in_inst)
                        done_now = op_leaf<ANY, MOT>(S, ps, st, err);
                    else if (ps.need_pop)
                        done_now = !op_pop(ps, st);
                    if (!done_now && ps.pending == 0 && !ps.need_pop) done_now = op_node<ANY>(S, ps, st, err);
                } else if (ps.need_pop) {
                    done_now = !op_pop(ps, st);
                } else {
                    done_now = op_node<ANY>(S, ps, st, err);
                }
            }
            if (__any_sync(0xFFFFFFFFu, done_now)) finish(done_now, item, ps.ts);
            if (done_now) active = false;
        }
        // Leaf phase: instance leaves (TLAS) per lane, then the warp's
        // triangle leaves together (leaf_coop).
        bool done_now = false;
        if (active && ps.pending && !ps.ts.in_inst) done_now = op_leaf<ANY, MOT>(S, ps, st, err);
        const bool tri_leaf = active && !done_now && ps.pending && ps.ts.in_inst;
        if (__any_sync(0xFFFFFFFFu, tri_leaf))
            done_now |= leaf_coop<ANY, TRANSMIT, PRES, CURV, MOT>(S, ps, tri_leaf, leaf, ray_seed);
        if (__any_sync(0xFFFFFFFFu, done_now)) finish(done_now, item, ps.ts);
        if (done_now) active = false;
    }
}

// ---- extend ---------------------------------------------------------------------------
// `pres`: cutout surfaces are passed through inside the traversal
// (leaf_coop, PRES) instead of by the shade kernel's skip waves.
// QUAD: the scene has quadrics or curve sets; MOT: motion blur (rays carry
// their path's shutter time; launched with QUAD).
template <int BLOCK, bool PRES, bool QUAD = false, bool MOT = false>
__global__ void __launch_bounds__(BLOCK, RT_TRAV_MIN_BLOCKS) k_extend(DevScene S, Paths P, uint32_t qsel) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    __shared__ LeafShared leaf_sh[BLOCK / 32];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    const uint32_t* q = P.q_ext[qsel];
    const uint32_t n = P.cnt[CNT_EXT_IN];
    unsigned long long rays = 0;
    uint32_t slot = 0;
    uint32_t qk = 0xFFFFFFFFu;  // closest quadric of this lane's ray (scene/mod.rs:105-146), ~0 for none
    float qt = 0.0f;            // its parametric distance
    auto load = [&](uint32_t j, float3& o, float3& d, float& tmax, uint64_t& seed, float& time) {
        slot = q[j];
        float4 o4 = P.ray_o[slot], d4 = P.ray_d[slot];
        o = xyz(o4);
        d = xyz(d4);
        tmax = d4.w;
        if (MOT) time = P.time[slot];
        if (PRES) {
            // The path's random state at this bounce, hashed: a seed no
            // other ray of the render shares.
            const uint4 rs = P.rng[slot];
            seed = splitmix(((uint64_t)rs.x | ((uint64_t)rs.y << 32)) ^
                            (((uint64_t)rs.z | ((uint64_t)rs.w << 32)) * 0x9E3779B97F4A7C15ull));
        }
        qk = 0xFFFFFFFFu;
        if (QUAD) {
            // Quadrics first; the BVH then only looks for closer surfaces.
            const float dl = fmaxf(length(d), 1e-30f);
            float tw;
            qk = PRES ? quadrics_closest_stopping(S, o, d / dl, tmax * dl, seed, tw)
                      : quadrics_closest(S, o, d / dl, tmax * dl, tw);
            if (qk != 0xFFFFFFFFu) tmax = qt = tw / dl;
        }
    };
    auto finish = [&](bool done, uint32_t, const TravState& ts) {
        uint32_t cls = CLS_MISS;
        if (done) {
            const TraceHit& h = ts.hit;
            uint32_t uv = (uint32_t)__half_as_ushort(__float2half_rn(h.b1)) |
                          ((uint32_t)__half_as_ushort(__float2half_rn(h.b2)) << 16);
            if (ts.found) {
                P.hit[slot] = make_uint4(__float_as_uint(h.t), h.tri, h.inst, uv);
                cls = __ldg(&S.materials[__ldg(&S.inst[h.inst].z)].mclass);
            } else if (qk != 0xFFFFFFFFu) {
                P.hit[slot] = make_uint4(__float_as_uint(qt), RT_TRI_QUADRIC | qk, 0xFFFFFFFFu, 0u);
                cls = __ldg(&S.materials[S.quadrics[qk].material].mclass);
            } else {
                P.hit[slot] = make_uint4(__float_as_uint(h.t), 0xFFFFFFFFu, h.inst, uv);
            }
            rays++;
        }
        // Bucket by material class: one atomic per (warp, class).
        for (uint32_t c = 0; c < N_QUEUES; c++)
            push_queue(P.q_cls + (size_t)c * P.P, &P.cnt[CNT_CLASS + c], slot, done && cls == c);
    };
    ray_pump<false, false, PRES, QUAD, MOT>(S, n, &P.cnt[CNT_FETCH_EXT], P.err, st, leaf_sh[threadIdx.x >> 5], load,
                                            finish);
    if (rays) atomicAdd(&P.stats[0], rays);
}

// ---- shade ------------------------------------------------------------------------------
struct NeeOut {
    float3 o, d, c;
    float tmax;
};

// NEE for one light (mod.rs:1032-1209): returns true with a shadow ray and
// its unoccluded contribution (already divided by the pick pmf). eval(wi,
// pdf) gives the scattering value toward wi with any cosine applied and the
// pdf of the direction-sampling strategy it is MIS-weighted against; n only
// offsets the shadow ray's origin (zero at a medium collision).
template <class Eval>
__device__ __forceinline__ bool nee_light_eval(const DevScene& S, const DevLight& L, float3 p, float3 n, Eval eval,
                                               float pick, Pcg& rng, NeeOut& out) {
    float3 Le = f3(L.radiance[0], L.radiance[1], L.radiance[2]);
    auto shadow_to = [&](float3 target) {
        float3 dir = target - p;
        float dist = length(dir);
        out.o = p + n * RT_RAY_OFFSET;
        out.d = normalize_ref(dir);
        out.tmax = dist - 1e-3f;
    };
    float3 lp = f3(L.p[0], L.p[1], L.p[2]);
    switch (L.type) {
        case 0: {  // point
            float3 to = lp - p;
            float dist2 = fmaxf(dot(to, to), 1e-12f);
            float3 wi = normalize_ref(to);
            float bp;
            float3 f = eval(wi, bp);
            if (maxc(f) <= 0.0f) return false;
            // Light::radiance_toward (light.rs:155-167): a profile reshapes
            // the output toward the emission direction -wi.
            const float prof = L.ies == 0xFFFFFFFFu ? 1.0f : ies_factor(S, S.ies[L.ies], -wi);
            out.c = f * Le * prof / (dist2 * pick);
            shadow_to(lp);
            return true;
        }
        case 1: {  // distant (soft when the angular radius > 1e-5)
            float3 base = -f3(L.e1[0], L.e1[1], L.e1[2]);
            float3 wi = base;
            if (L.radius > 1e-5f) {
                float u = rng.next_f(), v = rng.next_f();
                float ct = 1.0f - u * (1.0f - L.cos_max);
                float stt = sqrtf(fmaxf(1.0f - ct * ct, 0.0f)), sp, cp;
                sincosf(2.0f * RT_PI * v, &sp, &cp);
                Frame lf(base);
                wi = lf.to_world(f3(stt * cp, stt * sp, ct));
            }
            float bp;
            float3 f = eval(wi, bp);
            if (maxc(f) <= 0.0f) return false;
            out.c = f * Le / pick;
            out.o = p + n * RT_RAY_OFFSET;
            out.d = wi;
            out.tmax = 1e8f;
            return true;
        }
        case 2:    // rect
        case 4: {  // disk
            float u = rng.next_f(), v = rng.next_f();
            float3 e1 = f3(L.e1[0], L.e1[1], L.e1[2]), e2 = f3(L.e2[0], L.e2[1], L.e2[2]);
            float3 sp;
            if (L.type == 2) {
                sp = lp + e1 * u + e2 * v;
            } else {
                float r = sqrtf(u), s, c;
                sincosf(2.0f * RT_PI * v, &s, &c);
                sp = lp + e1 * (r * c) + e2 * (r * s);
            }
            float3 to = sp - p;
            float dist2 = fmaxf(dot(to, to), 1e-12f);
            float3 wi = normalize_ref(to);
            float cos_l = fabsf(dot(wi, f3(L.n[0], L.n[1], L.n[2])));
            if (cos_l < 1e-9f || L.area <= 0.0f) return false;
            float bp;
            float3 f = eval(wi, bp);
            if (maxc(f) <= 0.0f) return false;
            float pdf_sa = pick * dist2 / (cos_l * L.area);
            out.c = f * Le * (power_heuristic(pdf_sa, bp) / pdf_sa);
            shadow_to(sp);
            return true;
        }
        case 5: {  // dome (mod.rs:1139-1172): the map's importance sampling, or a uniform sphere
            float u = rng.next_f(), v = rng.next_f();
            float3 wi, rad = Le;
            float pdf_dir = 0.25f / RT_PI;
            if ((uint32_t)(&L - S.lights) == S.env_light) {  // this dome carries the map
                float3 tex;
                wi = env_sample(S, u, v, &tex, &pdf_dir);
                rad = tex * Le;
                if (pdf_dir <= 0.0f) return false;
            } else {
                float z = 1.0f - 2.0f * u;
                float r = sqrtf(fmaxf(1.0f - z * z, 0.0f)), s, c;
                sincosf(2.0f * RT_PI * v, &s, &c);
                wi = f3(r * c, r * s, z);
            }
            float bp;
            float3 f = eval(wi, bp);
            if (maxc(f) <= 0.0f) return false;
            float pdf_sa = pick * pdf_dir;
            out.c = f * rad * (power_heuristic(pdf_sa, bp) / pdf_sa);
            out.o = p + n * RT_RAY_OFFSET;
            out.d = wi;
            out.tmax = 1e8f;
            return true;
        }
        case 3: {  // sphere
            float3 tc = lp - p;
            float dist2 = dot(tc, tc);
            float r2 = L.radius * L.radius;
            if (dist2 <= r2 * 1.0001f) return false;
            float sin2 = fminf(r2 / dist2, 1.0f);
            float cos_max = sqrtf(fmaxf(1.0f - sin2, 0.0f));
            float u = rng.next_f(), v = rng.next_f();
            float ct = 1.0f - u * (1.0f - cos_max);
            float stt = sqrtf(fmaxf(1.0f - ct * ct, 0.0f)), s, c;
            sincosf(2.0f * RT_PI * v, &s, &c);
            Frame lf(normalize_ref(tc));
            float3 wi = lf.to_world(f3(stt * c, stt * s, ct));
            float bp;
            float3 f = eval(wi, bp);
            if (maxc(f) <= 0.0f) return false;
            float dist = sqrtf(dist2) * ct - sqrtf(fmaxf(r2 - dist2 * stt * stt, 0.0f));
            float pdf_sa = pick / fmaxf(2.0f * RT_PI * (1.0f - cos_max), 1e-12f);
            out.c = f * Le * (power_heuristic(pdf_sa, bp) / pdf_sa);
            shadow_to(p + wi * dist);
            return true;
        }
    }
    return false;
}

// NEE from a surface: the BSDF value with cosine, MIS-weighted against the
// BSDF pdf, or under guiding the one-sample mixture alpha * q + (1 - alpha)
// * p_bsdf.
__device__ __forceinline__ bool nee_light(const DevScene& S, const DevLight& L, float3 p, float3 n, const Frame& fr,
                                          float3 wo_l, float eta, const DevMaterial& m, float pick, Pcg& rng,
                                          NeeOut& out, const MixtureRef* mix = nullptr, float alpha = 0.0f) {
    auto eval = [&](float3 wi, float& pdf) -> float3 {
        float3 wl = fr.to_local(wi);
        if (wl.z <= 0.0f) {
            pdf = 0.0f;
            return f3(0, 0, 0);
        }
        float3 f = bsdf_eval(m, wo_l, wl, eta, pdf) * wl.z;
        if (mix) pdf = alpha * mixture_pdf(*mix, wi) + (1.0f - alpha) * pdf;
        return f;
    };
    return nee_light_eval(S, L, p, n, eval, pick, rng, out);
}

// Hair at a curve hit (pt/mod.rs:737-781): NEE through the hair lobes
// (n, the viewer-facing normal, offsets the shadow ray), then a
// hair-sampled direction with its weight f / pdf (no cosine: f is per solid
// angle). Returns false when sampling fails and the path ends. Out of line:
// only hair hits call it, and the shade kernel keeps its registers.
__device__ __noinline__ bool shade_hair(const DevScene& S, const DevHair& hp, uint4 hr, float3 p, float3 n, float3 wo,
                                        Pcg& rng, NeeOut& ne, bool& nee_ok, float3& wi, float3& weight, float& pdf) {
    const FiberFrame ff(curve_tangent(S, hr), n, wo);
    HairEval g;
    hair_prepare(hp, ff.to_local(wo), ff.h, g);
    nee_ok = false;
    if (S.n_lights > 0) {
        uint32_t li;
        float pmf;
        if (light_sample(S, p, rng.next_f(), li, pmf)) {
            auto eval = [&](float3 w, float& pd) -> float3 { return hair_f_pdf(hp, g, ff.to_local(w), pd); };
            nee_ok = nee_light_eval(S, S.lights[li], p, n, eval, pmf, rng, ne);
        }
    }
    float3 wf, f;
    if (!hair_sample(hp, g, rng, wf, f, pdf)) return false;
    wi = normalize_ref(ff.to_world(wf));
    weight = f / pdf;
    return true;
}

// mod.rs:1000-1023 solid-angle pdf of an area light toward a hit.
__device__ __forceinline__ float light_pdf_sa(const DevLight& L, float3 origin, float3 hp) {
    if (L.type == 2 || L.type == 4) {
        float3 d = hp - origin;
        float dist2 = dot(d, d);
        float cos_l = fabsf(dot(normalize_ref(d), f3(L.n[0], L.n[1], L.n[2])));
        if (cos_l < 1e-9f || L.area <= 0.0f) return 0.0f;
        return dist2 / (cos_l * L.area);
    }
    if (L.type == 3) {
        float3 c = f3(L.p[0], L.p[1], L.p[2]) - origin;
        float sin2 = fminf(L.radius * L.radius / dot(c, c), 1.0f);
        float cos_max = sqrtf(fmaxf(1.0f - sin2, 0.0f));
        float sa = 2.0f * RT_PI * (1.0f - cos_max);
        return sa < 1e-12f ? 0.0f : 1.0f / sa;
    }
    return 0.0f;
}

#ifndef RT_SHADE_MIN_BLOCKS
#define RT_SHADE_MIN_BLOCKS 1
#endif
// PAT: the scene has patterns (ray cones tracked, patterned materials
// resolved per hit). The plain instance keeps its material reads on the
// global material table and the register count of a kernel without them.
// MED: the scene has participating media (medium segments, hull crossings,
// nested-media stacks, equiangular shadow rays).
template <bool PAT, bool MED = false>
__global__ void __launch_bounds__(128, RT_SHADE_MIN_BLOCKS) k_shade(DevScene S, Paths P, PtConsts C, uint32_t qout) {
    uint32_t counts[N_QUEUES];
    uint32_t total = 0;
#pragma unroll
    for (uint32_t c = 0; c < N_QUEUES; c++) {
        counts[c] = P.cnt[CNT_CLASS + c];
        total += counts[c];
    }
    uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j0 = blockIdx.x * blockDim.x; j0 < total; j0 += stride) {
        uint32_t j = j0 + threadIdx.x;
        bool active = j < total;
        uint32_t slot = 0;
        if (active) {
            // Queues are consumed class by class: miss first, then materials.
            uint32_t c = CLS_MISS, off = j;
            if (off < counts[CLS_MISS]) {
                c = CLS_MISS;
            } else {
                off -= counts[CLS_MISS];
                for (uint32_t k = 0; k < N_MAT_CLASSES; k++) {
                    if (off < counts[k]) {
                        c = k;
                        break;
                    }
                    off -= counts[k];
                }
            }
            slot = P.q_cls[(size_t)c * P.P + off];
        }
        bool extend = false, shadow = false, shadow2 = false, walk = false;
        if (active) {
            float4 o4 = P.ray_o[slot], d4 = P.ray_d[slot];
            uint4 hr = P.hit[slot];
            float4 beta4 = P.beta[slot], L4 = P.L[slot], prev4 = P.prev[slot];
            uint4 rs = P.rng[slot];
            Pcg rng;
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            rng.inc = (uint64_t)rs.z | ((uint64_t)rs.w << 32);
            uint32_t flags = __float_as_uint(prev4.w);
            float3 beta = xyz(beta4), Lr = xyz(L4);
            float3 o = xyz(o4), d = xyz(d4);
            float travel = L4.w;
            bool spec_true = (flags & FL_SPEC_MASK) == FL_SPEC_TRUE;
            float4 auxd = C.aovs ? P.aux_d[slot] : make_float4(0, 0, 0, 0);
            auto emit = [&](float3 c) {
                Lr = Lr + c;
                if (C.aovs && !spec_true) {
                    auxd.x += c.x;
                    auxd.y += c.y;
                    auxd.z += c.z;
                }
            };
            // Training: close the previous vertex's record with the radiance
            // gathered so far (its own emission and NEE included).
            auto tr_close = [&]() {
                if (!C.train) return;
                uint32_t d0 = flags >> FL_DEPTH_SHIFT;
                if (d0 == 0 || d0 > C.max_depth) return;
                float* r = P.tr_rec + ((size_t)slot * C.max_depth + (d0 - 1)) * TR_FLOATS;
                if (__float_as_uint(r[18]) == P.tr_tag && __float_as_uint(r[19]) != P.tr_tag) {
                    r[15] = Lr.x;
                    r[16] = Lr.y;
                    r[17] = Lr.z;
                    r[19] = __uint_as_float(P.tr_tag);
                }
            };
            uint2 mstk = make_uint2(0u, 0u);
            uint32_t cur_med = RT_MEDIUM_NONE;
            bool consumed = false;  // the medium segment ended this step (collision or absorbed path)
            if (MED) {
                mstk = P.med[slot];
                cur_med = mstack_top(mstk, S.atmosphere);
            }
            if (MED && cur_med != RT_MEDIUM_NONE) {
                // Medium interaction along this segment, before any surface
                // (pt/mod.rs:490-640). One light pick per segment serves both
                // the equiangular and the collision NEE, so their MIS weights
                // cancel its pmf.
                const DevMedium& med = S.media[cur_med];
                const float3 dn = normalize_ref(d);
                const float t_limit = hr.y != 0xFFFFFFFFu ? __uint_as_float(hr.x) * length(d) : 1e8f;
                const float t_seg = fminf(t_limit, med.max_distance);
                uint32_t pli = 0;
                float ppmf = 0.0f;
                const bool seg_pick = light_sample(S, o + dn * fminf(t_seg * 0.5f, 50.0f), rng.next_f(), pli, ppmf);
                const bool point = seg_pick && S.lights[pli].type == 0;
                const float3 lp = point ? f3(S.lights[pli].p[0], S.lights[pli].p[1], S.lights[pli].p[2]) : f3(0, 0, 0);
                if (point && t_seg > 1e-6f) {
                    // Equiangular single-scatter NEE toward the point light
                    // (Kulla-Fajardo); its shadow ray goes out as sh2.
                    const DevLight& Lp = S.lights[pli];
                    float pdf_eq;
                    const float t_eq = equiangular_sample(o, dn, t_seg, lp, rng.next_f(), pdf_eq);
                    if (pdf_eq > 1e-12f) {
                        const float3 pe = o + dn * t_eq;
                        const float rho = med_density(med, pe);
                        if (rho > 0.0f) {
                            const float3 tr = med_transmittance(med, o, dn, t_eq, rng);
                            const float3 to_l = lp - pe;
                            const float dist2 = fmaxf(dot(to_l, to_l), 1e-12f);
                            const float3 wi = normalize_ref(to_l);
                            const float ph = hg_phase(med.g, dot(dn, wi));
                            const float prof = Lp.ies == 0xFFFFFFFFu ? 1.0f : ies_factor(S, S.ies[Lp.ies], -wi);
                            const float pdf_d = distance_pdf_approx(med, t_eq, t_seg);
                            const float w_eq = pdf_eq / (pdf_eq + pdf_d);
                            const float3 c = beta * (med_sigma_s(med) * rho) * tr *
                                             f3(Lp.radiance[0], Lp.radiance[1], Lp.radiance[2]) *
                                             (prof * ph * w_eq / (dist2 * pdf_eq * ppmf));
                            if (maxc(c) > 0.0f) {
                                P.sh2_o[slot] = make_float4(pe.x, pe.y, pe.z, __uint_as_float(cur_med));
                                P.sh2_d[slot] = make_float4(wi.x, wi.y, wi.z, sqrtf(dist2) - 1e-3f);
                                P.sh2_c[slot] = make_float4(c.x, c.y, c.z, spec_true ? 0.0f : 1.0f);
                                shadow2 = true;
                            }
                        }
                    }
                }
                const MedEvent ev = med_sample(med, o, dn, t_limit, beta, rng);
                beta = beta * ev.w;
                if (ev.scatter) {
                    consumed = true;
                    const float3 pm = o + dn * ev.t;
                    if (C.aovs && !(flags & FL_AUX_SET)) {
                        flags |= FL_AUX_SET;
                        const float3 stt = med_sigma_t(med);
                        P.aux_a[slot] = make_float4(med.sigma_s[0] / fmaxf(stt.x, 1e-9f), med.sigma_s[1] / fmaxf(stt.y, 1e-9f),
                                                    med.sigma_s[2] / fmaxf(stt.z, 1e-9f), travel + ev.t);
                        P.aux_n[slot] = make_float4(-dn.x, -dn.y, -dn.z, __uint_as_float(0u));
                        auxd.w = 1.0f;
                    }
                    if ((flags & FL_SPEC_MASK) == FL_SPEC_NONE) flags &= ~FL_SPEC_MASK;
                    const float3 em = f3(med.emission[0], med.emission[1], med.emission[2]);
                    if (maxc(em) > 0.0f) emit(beta * em);
                    const float3 wo = -dn;
                    const float g = med.g;
                    if (seg_pick) {
                        // Collision NEE; point lights carry the MIS weight that
                        // pairs it with the equiangular strategy.
                        float w_dist = 1.0f;
                        if (point) {
                            const float pdf_d = distance_pdf_approx(med, ev.t, t_seg);
                            w_dist = pdf_d / (pdf_d + equiangular_pdf(o, dn, t_seg, lp, ev.t));
                        }
                        auto eval = [&](float3 wi, float& pdf) -> float3 {
                            const float ph = hg_phase(g, -dot(wo, wi));
                            pdf = ph;
                            return f3(ph, ph, ph);
                        };
                        NeeOut ne;
                        if (nee_light_eval(S, S.lights[pli], pm, f3(0.0f, 0.0f, 0.0f), eval, ppmf, rng, ne)) {
                            const float3 c = beta * ne.c * w_dist;
                            if (maxc(c) > 0.0f) {
                                P.sh_o[slot] = make_float4(ne.o.x, ne.o.y, ne.o.z, __uint_as_float(cur_med));
                                P.sh_d[slot] = make_float4(ne.d.x, ne.d.y, ne.d.z, ne.tmax);
                                P.sh_c[slot] = make_float4(c.x, c.y, c.z, spec_true ? 0.0f : 1.0f);
                                shadow = true;
                            }
                        }
                    }
                    // Continue along a phase-function sample (phase / pdf = 1).
                    const float u1 = rng.next_f(), u2 = rng.next_f();
                    float pdf;
                    const float3 wi = hg_sample(g, wo, u1, u2, pdf);
                    beta4.w = pdf;
                    prev4 = make_float4(pm.x, pm.y, pm.z, 0.0f);
                    flags &= ~FL_FROM_CAMERA;
                    if (PAT) {
                        float2 cn = P.cone[slot];
                        cn.y += 0.4f;
                        P.cone[slot] = cn;
                    }
                    const uint32_t depth = (flags >> FL_DEPTH_SHIFT) + 1;
                    flags = (flags & 0xFFFFu) | (depth << FL_DEPTH_SHIFT);
                    bool alive = true;
                    if (depth >= C.rr_start) {
                        const float q = fminf(maxc(beta) * o4.w, 0.95f);
                        if (q <= 0.0f || rng.next_f() > q) alive = false;
                        else beta = beta / q;
                    }
                    if (alive && depth < C.max_depth) {
                        P.ray_o[slot] = make_float4(pm.x, pm.y, pm.z, o4.w);
                        P.ray_d[slot] = make_float4(wi.x, wi.y, wi.z, INFINITY);
                        extend = true;
                    }
                } else if (maxc(beta) <= 0.0f) {
                    consumed = true;  // absorbed on the way
                }
            }
            if (consumed) {
                // handled above
            } else if (hr.y == 0xFFFFFFFFu) {
                tr_close();
                if (S.dome != 0xFFFFFFFFu) {
                    // Miss: the dome light, MIS-weighted against its NEE
                    // sampling unless seen from the camera (mod.rs:643-655).
                    const DevLight& D = S.lights[S.dome];
                    const bool mapped = S.dome == S.env_light;
                    float wgt = 1.0f;
                    if (!(flags & FL_FROM_CAMERA))
                        wgt = power_heuristic(beta4.w, light_pmf(S, xyz(prev4), S.dome) *
                                                           (mapped ? env_pdf(S, d) : 0.25f / RT_PI));
                    float3 rad = f3(D.radiance[0], D.radiance[1], D.radiance[2]);
                    if (mapped) rad = env_eval(S, d) * rad;
                    emit(beta * rad * wgt);
                } else {
                    emit(beta * f3(S.background[0], S.background[1], S.background[2]));
                }
            } else {
                HitGeo hg;
                const float tm = S.motion ? P.time[slot] : 0.0f;
                hit_geometry(S, o, d, hr, hg, tm);
                const float3 p = hg.p, wo = hg.wo;
                float3 nw = hg.nw;
                const bool front = hg.front;
                const float eucl = hg.eucl;
                // Volume hull: the crossing only toggles the medium
                // (pt/mod.rs:662-680): no AOV, no cone growth, no bounce.
                const bool hull_skip = MED && S.materials[hg.mat].hull != 0.0f &&
                                       ((flags & FL_SKIP_MASK) >> FL_SKIP_SHIFT) < RT_MAX_PRESENCE_SKIPS;
                travel += eucl;
                // Ray cone at this hit and the material's pattern outputs
                // (pt/mod.rs:687-689; footprint = cone width x st density).
                float2 cone = make_float2(0.0f, 0.0f);
                DevMaterial mres;
                const DevMaterial* mptr = S.materials + hg.mat;
                if (PAT) {
                    cone = P.cone[slot];
                    if (!hull_skip) cone.x += eucl * cone.y;
                    const DevMatPat mp = S.mat_pat[hg.mat];
                    if (mp.bind_n) {
                        const HitSt hs = hit_st(S, hr, p, tm);
                        mres = *mptr;
                        resolve_material(S, mp, hs, p, nw, d, cone.x, mres);
                        mptr = &mres;
                    }
                }
                const DevMaterial& m = *mptr;
                if (C.aovs && !(flags & FL_AUX_SET) && !hull_skip) {
                    flags |= FL_AUX_SET;
                    float3 an = dot(nw, wo) >= 0.0f ? nw : -nw;
                    P.aux_a[slot] = make_float4(m.albedo[0], m.albedo[1], m.albedo[2], travel);
                    P.aux_n[slot] = make_float4(an.x, an.y, an.z, __uint_as_float(m.id));
                    auxd.w = 1.0f;
                }
                uint32_t skips = (flags & FL_SKIP_MASK) >> FL_SKIP_SHIFT;
                bool done = false;
                if (hull_skip) {
                    flags = (flags & ~FL_SKIP_MASK) | ((skips + 1) << FL_SKIP_SHIFT);
                    if (front) mstack_push(mstk, S.materials[hg.mat].interior);
                    else mstack_pop(mstk);
                    const float3 no = p + normalize_ref(d) * RT_RAY_OFFSET;
                    P.ray_o[slot] = make_float4(no.x, no.y, no.z, o4.w);
                    P.ray_d[slot] = make_float4(d.x, d.y, d.z, INFINITY);
                    extend = true;
                    done = true;
                }
                if (!done && !C.pres_in_trav && m.presence < 1.0f && rng.next_f() >= m.presence &&
                    skips < RT_MAX_PRESENCE_SKIPS) {
                    // Presence cutout: pass straight through, no bounce.
                    flags = (flags & ~FL_SKIP_MASK) | ((skips + 1) << FL_SKIP_SHIFT);
                    travel += eucl;
                    float3 no = p + normalize_ref(d) * RT_RAY_OFFSET;
                    P.ray_o[slot] = make_float4(no.x, no.y, no.z, o4.w);
                    P.ray_d[slot] = make_float4(d.x, d.y, d.z, INFINITY);
                    extend = true;
                    done = true;
                }
                if (!done) {
                    tr_close();
                    float3 n = dot(nw, wo) >= 0.0f ? nw : -nw;
                    float eta = front ? m.ior : 1.0f / m.ior;
                    float3 em = f3(m.emission[0], m.emission[1], m.emission[2]);
                    if (maxc(em) > 0.0f) {
                        float wgt = 1.0f;
                        if (!(flags & FL_FROM_CAMERA) && m.area_light >= 0) {
                            float3 po = xyz(prev4);
                            float pick = light_pmf(S, po, (uint32_t)m.area_light);
                            float pl = light_pdf_sa(S.lights[m.area_light], po, p) * pick;
                            wgt = power_heuristic(beta4.w, pl);
                        }
                        emit(beta * em * wgt);
                    }
                    // Hair fibers scatter over the whole sphere with their own
                    // BSDF (pt/mod.rs:737-781), on curve hits only.
                    const bool fiber = hg.curve && m.hair != 0xFFFFFFFFu;
                    if (fiber) {
                        NeeOut ne;
                        bool nee_ok;
                        float3 wi, wgt;
                        float pv;
                        const bool ok = shade_hair(S, S.hair[m.hair], hr, p, n, wo, rng, ne, nee_ok, wi, wgt, pv);
                        if (nee_ok) {
                            const float3 c = beta * ne.c;
                            if (maxc(c) > 0.0f) {
                                P.sh_o[slot] = make_float4(ne.o.x, ne.o.y, ne.o.z, MED ? __uint_as_float(cur_med) : 0.0f);
                                P.sh_d[slot] = make_float4(ne.d.x, ne.d.y, ne.d.z, ne.tmax);
                                P.sh_c[slot] = make_float4(c.x, c.y, c.z, spec_true ? 0.0f : 1.0f);
                                shadow = true;
                            }
                        }
                        if (ok) {
                            beta = beta * wgt;
                            if ((flags & FL_SPEC_MASK) == FL_SPEC_NONE) flags &= ~FL_SPEC_MASK;
                            flags &= ~FL_FROM_CAMERA;
                            beta4.w = pv;
                            prev4 = make_float4(p.x, p.y, p.z, 0.0f);
                            if (PAT) cone.y += 0.4f;
                            const float3 side = dot(wi, nw) >= 0.0f ? nw : -nw;
                            const float3 no = p + side * RT_RAY_OFFSET;
                            const uint32_t depth = (flags >> FL_DEPTH_SHIFT) + 1;
                            flags = (flags & 0xFFFFu) | (depth << FL_DEPTH_SHIFT);
                            bool alive = true;
                            if (depth >= C.rr_start) {
                                const float q = fminf(maxc(beta) * o4.w, 0.95f);
                                if (q <= 0.0f || rng.next_f() > q) alive = false;
                                else beta = beta / q;
                            }
                            if (alive && depth < C.max_depth) {
                                P.ray_o[slot] = make_float4(no.x, no.y, no.z, o4.w);
                                P.ray_d[slot] = make_float4(wi.x, wi.y, wi.z, INFINITY);
                                extend = true;
                            }
                        }
                    }
                    // Subsurface scattering (pt/mod.rs:794-892): with probability
                    // sss_gain the path enters a random walk inside the object
                    // (k_sss), starting from a cosine direction around -n.
                    if (!fiber && m.sss_gain > 0.0f && rng.next_f() < m.sss_gain) {
                        if ((flags & FL_SPEC_MASK) == FL_SPEC_NONE) flags &= ~FL_SPEC_MASK;
                        const Frame ef(-n);
                        const float e1 = rng.next_f(), e2 = rng.next_f();
                        const float er = sqrtf(e1);
                        float es, ec;
                        sincosf(2.0f * RT_PI * e2, &es, &ec);
                        const float3 wd = normalize_ref(ef.to_world(f3(er * ec, er * es, sqrtf(fmaxf(1.0f - e1, 0.0f)))));
                        const float3 wp = p - n * RT_RAY_OFFSET;
                        P.ray_o[slot] = make_float4(wp.x, wp.y, wp.z, o4.w);
                        P.ray_d[slot] = make_float4(wd.x, wd.y, wd.z, INFINITY);
                        P.hit[slot] = make_uint4(hg.mat, 0u, 0u, 0u);
                        walk = true;
                    }
                    if (!walk && !fiber) {
                        Frame fr(n);
                        float3 wo_l = fr.to_local(wo);
                        // Learned proposal at this vertex (guided mode only).
                        MixtureRef mix{nullptr};
                        bool guided = false;
                        if (C.guided) {
                            uint32_t gi = P.g_idx[slot];
                            if (gi != 0xFFFFFFFFu) {
                                mix.p = reinterpret_cast<const float4*>(P.g_raw + (size_t)gi * G_OUT);
                                guided = true;
                            }
                        }
                        if (S.n_lights > 0 && m.has_lobes != 0.0f) {
                            uint32_t li;
                            float pmf;
                            if (light_sample(S, p, rng.next_f(), li, pmf)) {
                                NeeOut ne;
                                if (nee_light(S, S.lights[li], p, n, fr, wo_l, eta, m, pmf, rng, ne,
                                              guided ? &mix : nullptr, C.alpha)) {
                                    float3 c = beta * ne.c;
                                    if (maxc(c) > 0.0f) {
                                        P.sh_o[slot] = make_float4(ne.o.x, ne.o.y, ne.o.z, MED ? __uint_as_float(cur_med) : 0.0f);
                                        P.sh_d[slot] = make_float4(ne.d.x, ne.d.y, ne.d.z, ne.tmax);
                                        P.sh_c[slot] = make_float4(c.x, c.y, c.z, spec_true ? 0.0f : 1.0f);
                                        shadow = true;
                                    }
                                }
                            }
                        }
                        BsdfSample bs;
                        bool sampled;
                        float pdf_path = 0.0f;
                        if (guided) {
                            // One-sample MIS: the guide with probability alpha, else the
                            // BSDF; the path pdf is the mixture of both full pdfs.
                            if (rng.next_f() < C.alpha) {
                                float u0 = rng.next_f(), u1 = rng.next_f(), u2 = rng.next_f();
                                bs.wi = fr.to_local(mixture_sample(mix, u0, u1, u2));
                                bs.f = bsdf_eval(m, wo_l, bs.wi, eta, bs.pdf);
                                bs.transmitted = bs.wi.z < 0.0f;
                                bs.specular = false;
                                sampled = maxc(bs.f) > 0.0f;
                            } else {
                                sampled = bsdf_sample(m, wo_l, eta, rng, bs);
                            }
                            if (sampled) {
                                pdf_path = C.alpha * mixture_pdf(mix, fr.to_world(bs.wi)) + (1.0f - C.alpha) * bs.pdf;
                                sampled = pdf_path > 0.0f;
                            }
                        } else {
                            sampled = bsdf_sample(m, wo_l, eta, rng, bs);
                            pdf_path = bs.pdf;
                        }
                        // Roulette gain: Russian roulette acts on the throughput the
                        // path would carry had every bounce been BSDF-sampled,
                        // beta * prod(pdf_path / p_bsdf). Guiding concentrates paths
                        // on directions of high incident radiance and gives them a
                        // low beta for it; roulette on beta alone would kill those
                        // paths at the next bounce and cancel the gain. Without
                        // guiding the gain stays exactly 1 (the reference's rule,
                        // pt/mod.rs:980-987).
                        float rr_gain = o4.w;
                        if (guided && sampled)
                            rr_gain = fminf(fmaxf(rr_gain * (pdf_path / fmaxf(bs.pdf, 1e-20f)), 1e-20f), 1e20f);
                        if (sampled) {
                            float3 wi = fr.to_world(bs.wi);
                            const float3 beta_in = beta;
                            if (MED && bs.transmitted && m.interior != RT_MEDIUM_NONE) {  // pt/mod.rs:969-975
                                if (front) mstack_push(mstk, m.interior);
                                else mstack_pop(mstk);
                            }
                            beta = beta * bs.f * (fabsf(bs.wi.z) / pdf_path);
                            if (C.train) {
                                // Training vertex: closed with the radiance at the next vertex.
                                uint32_t d0 = flags >> FL_DEPTH_SHIFT;
                                if (d0 < C.max_depth) {
                                    float* r = P.tr_rec + ((size_t)slot * C.max_depth + d0) * TR_FLOATS;
                                    float3 wn = normalize_ref(wi);
                                    r[0] = p.x; r[1] = p.y; r[2] = p.z;
                                    r[3] = n.x; r[4] = n.y; r[5] = n.z;
                                    r[6] = wo.x; r[7] = wo.y; r[8] = wo.z;
                                    r[9] = wn.x; r[10] = wn.y; r[11] = wn.z;
                                    r[12] = beta_in.x; r[13] = beta_in.y; r[14] = beta_in.z;
                                    r[18] = __uint_as_float(P.tr_tag);
                                    r[19] = 0.0f;
                                }
                            }
                            if ((flags & FL_SPEC_MASK) == FL_SPEC_NONE)
                                flags = (flags & ~FL_SPEC_MASK) | (bs.specular ? FL_SPEC_TRUE : 0u);
                            flags &= ~FL_FROM_CAMERA;
                            beta4.w = pdf_path;
                            // Widen the cone after rough bounces (pt/mod.rs:965-967).
                            if (PAT) cone.y += fminf(1.0f / (1.0f + pdf_path), 0.4f);
                            prev4 = make_float4(p.x, p.y, p.z, 0.0f);
                            float off = bs.transmitted ? -RT_RAY_OFFSET : RT_RAY_OFFSET;
                            float3 no = p + n * off;
                            float3 nd = normalize_ref(wi);
                            uint32_t depth = (flags >> FL_DEPTH_SHIFT) + 1;
                            flags = (flags & 0xFFFFu) | (depth << FL_DEPTH_SHIFT);
                            bool alive = true;
                            if (depth >= C.rr_start) {
                                float q = fminf(maxc(beta) * rr_gain, 0.95f);
                                if (q <= 0.0f || rng.next_f() > q) alive = false;
                                else beta = beta / q;
                            }
                            if (alive && depth < C.max_depth) {
                                P.ray_o[slot] = make_float4(no.x, no.y, no.z, rr_gain);
                                P.ray_d[slot] = make_float4(nd.x, nd.y, nd.z, INFINITY);
                                extend = true;
                            }
                        }
                    }  // !walk
                }
                if (PAT) P.cone[slot] = cone;
            }
            if (MED) P.med[slot] = mstk;
            // A walk queues its equiangular shadow ray with its own (k_sss).
            if (walk && shadow2) flags |= FL_SH2;
            P.beta[slot] = make_float4(beta.x, beta.y, beta.z, beta4.w);
            P.L[slot] = make_float4(Lr.x, Lr.y, Lr.z, travel);
            P.prev[slot] = make_float4(prev4.x, prev4.y, prev4.z, __uint_as_float(flags));
            P.rng[slot] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), rs.z, rs.w);
            if (C.aovs) P.aux_d[slot] = auxd;
        }
        push_queue(P.q_ext[qout], &P.cnt[CNT_EXT_OUT], slot, extend);
        if (MED)
            push_queue(P.q_sh, &P.cnt[CNT_SHADOW], slot | (shadow ? SH_PRIMARY : 0u) | (shadow2 ? SH_EQUI : 0u),
                       (shadow || shadow2) && !walk);
        else
            push_queue(P.q_sh, &P.cnt[CNT_SHADOW], slot, shadow);
        if (P.q_sss) push_queue(P.q_sss, &P.cnt[CNT_SSS], slot, walk);
    }
}

// ---- shadow -------------------------------------------------------------------------------
template <int BLOCK, bool QUAD = false, bool MOT = false>
__global__ void __launch_bounds__(BLOCK, RT_TRAV_MIN_BLOCKS) k_shadow(DevScene S, Paths P, PtConsts C) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    __shared__ LeafShared leaf_sh[BLOCK / 32];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    uint32_t n = P.cnt[CNT_SHADOW];
    unsigned long long rays = 0;
    auto add = [&](uint32_t slot, float vis) {
        float4 c = P.sh_c[slot];
        float4 L = P.L[slot];
        P.L[slot] = make_float4(L.x + c.x * vis, L.y + c.y * vis, L.z + c.z * vis, L.w);
        if (C.aovs && c.w != 0.0f) {
            float4 a = P.aux_d[slot];
            P.aux_d[slot] = make_float4(a.x + c.x * vis, a.y + c.y * vis, a.z + c.z * vis, a.w);
        }
    };
    if (!S.any_presence) {
        // Opaque scenes: one any-hit query per shadow ray, through the pump.
        uint32_t slot = 0;
        bool qblock = false;  // a quadric blocks this lane's shadow ray
        auto load = [&](uint32_t j, float3& o, float3& d, float& tmax, uint64_t& seed, float& time) {
            slot = P.q_sh[j];
            float4 o4 = P.sh_o[slot], d4 = P.sh_d[slot];
            o = xyz(o4);
            d = xyz(d4);
            tmax = d4.w;
            if (MOT) time = P.time[slot];
            qblock = false;
            if (QUAD) {
                const float dl = fmaxf(length(d), 1e-30f);
                float tw;
                qblock = quadrics_closest(S, o, d / dl, tmax * dl, tw) != 0xFFFFFFFFu;
                if (qblock) tmax = -1.0f;  // nothing left for the BVH to find
            }
        };
        auto finish = [&](bool done, uint32_t, const TravState& ts) {
            if (!done) return;
            rays++;
            if (!ts.found && !qblock) add(slot, 1.0f);
        };
        ray_pump<true, false, false, QUAD, MOT>(S, n, &P.cnt[CNT_FETCH_SH], P.err, st, leaf_sh[threadIdx.x >> 5], load,
                                                finish);
        if (rays) atomicAdd(&P.stats[1], rays);
        return;
    }
    // Scenes with presence cutouts: transmittance queries through the pump
    // (traverse.cuh: one traversal per shadow ray, cutouts attenuate, opaque
    // surfaces block).
    uint32_t slot = 0;
    float qvis = 1.0f;  // transmittance of this lane's shadow ray through the quadrics
    auto load = [&](uint32_t j, float3& o, float3& d, float& tmax, uint64_t& seed, float& time) {
        slot = P.q_sh[j];
        float4 o4 = P.sh_o[slot], d4 = P.sh_d[slot];
        o = xyz(o4);
        d = xyz(d4);
        tmax = d4.w;
        if (MOT) time = P.time[slot];
        qvis = 1.0f;
        if (QUAD) {
            const float dl = fmaxf(length(d), 1e-30f);
            qvis = quadrics_transmittance(S, o, d / dl, tmax * dl);
            if (qvis == 0.0f) tmax = -1.0f;  // nothing left for the BVH to find
        }
    };
    auto finish = [&](bool done, uint32_t, const TravState& ts) {
        if (!done) return;
        rays++;
        const float vis = ts.trans * qvis;
        if (vis > 0.0f) add(slot, vis);
    };
    ray_pump<true, true, false, QUAD, MOT>(S, n, &P.cnt[CNT_FETCH_SH], P.err, st, leaf_sh[threadIdx.x >> 5], load,
                                           finish);
    if (rays) atomicAdd(&P.stats[1], rays);
}

// Between waves: the next extend queue becomes the current one.
// ---- subsurface walks ------------------------------------------------------------------
// One thread per walk queued by k_shade (pt/mod.rs:794-892): isotropic
// scattering through the material's homogeneous Burley-fit medium, one
// closest-hit query per step (trace_closest), roulette after step 8, at most
// 256 steps. The walk leaves diffusely where it first reaches a surface:
// NEE there for a white Lambert lobe, then a cosine direction becomes the
// path's next ray. Walks that escape or run out of steps end the path.
// MOT: the scene has motion blur (walks take the path's shutter time).
template <int BLOCK, bool MED, bool MOT = false>
__global__ void __launch_bounds__(BLOCK) k_sss(DevScene S, Paths P, PtConsts C, uint32_t qout) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    const uint32_t n = P.cnt[CNT_SSS];
    unsigned long long rays = 0;
    const uint32_t stride = gridDim.x * BLOCK;
    for (uint32_t j0 = blockIdx.x * BLOCK; j0 < n; j0 += stride) {
        const uint32_t j = j0 + threadIdx.x;
        uint32_t slot = 0;
        bool extend = false, shadow = false, shadow2 = false;
        if (j < n) {
            slot = P.q_sss[j];
            const float4 o4 = P.ray_o[slot], d4 = P.ray_d[slot];
            const float4 beta4 = P.beta[slot];
            float4 prev4 = P.prev[slot];
            const uint4 rs = P.rng[slot];
            Pcg rng;
            rng.state = (uint64_t)rs.x | ((uint64_t)rs.y << 32);
            rng.inc = (uint64_t)rs.z | ((uint64_t)rs.w << 32);
            uint32_t flags = __float_as_uint(prev4.w);
            float3 beta = xyz(beta4);
            float pdf_prev = beta4.w;
            const DevMaterial& m = S.materials[P.hit[slot].x];
            const float3 sst = f3(m.sss_st[0], m.sss_st[1], m.sss_st[2]);
            const float3 sss = f3(m.sss_ss[0], m.sss_ss[1], m.sss_ss[2]);
            const uint32_t cur_med = MED ? mstack_top(P.med[slot], S.atmosphere) : RT_MEDIUM_NONE;
            const float tm = MOT ? P.time[slot] : 0.0f;
            float3 wo = xyz(o4), wd = xyz(d4);
            bool exited = false;
            for (int step = 0; step < 256; step++) {
                uint4 hr;
                rays++;
                if (!trace_closest<MOT>(S, st, wo, wd, INFINITY, P.err, hr, tm)) break;  // escaped through a crack
                const MedEvent ev = homog_sample(sst, sss, __uint_as_float(hr.x), beta, rng);
                beta = beta * ev.w;
                if (ev.scatter) {
                    wo = wo + wd * ev.t;
                    const float u = rng.next_f(), v = rng.next_f();
                    const float z = 1.0f - 2.0f * u, r = sqrtf(fmaxf(1.0f - z * z, 0.0f));
                    float sp, cp;
                    sincosf(2.0f * RT_PI * v, &sp, &cp);
                    wd = f3(r * cp, r * sp, z);
                    const float q = fminf(maxc(beta), 0.95f);
                    if (q <= 0.0f || (step > 8 && rng.next_f() > q)) break;
                    if (step > 8) beta = beta / q;
                    continue;
                }
                // Exit on the outside: normal along the walk's direction.
                HitGeo hg;
                hit_geometry(S, wo, wd, hr, hg, tm);
                const float3 out_n = dot(hg.nw, wd) > 0.0f ? hg.nw : -hg.nw;
                const Frame xf(out_n);
                const float3 xp = hg.p;
                uint32_t li;
                float pmf;
                if (light_sample(S, xp, rng.next_f(), li, pmf)) {
                    auto eval = [&](float3 wi, float& pdf) -> float3 {
                        const float3 wl = xf.to_local(wi);
                        pdf = wl.z > 0.0f ? wl.z * (1.0f / RT_PI) : 0.0f;
                        return f3(pdf, pdf, pdf);
                    };
                    NeeOut ne;
                    if (nee_light_eval(S, S.lights[li], xp, out_n, eval, pmf, rng, ne)) {
                        const float3 c = beta * ne.c;
                        if (maxc(c) > 0.0f) {
                            const bool spec_true = (flags & FL_SPEC_MASK) == FL_SPEC_TRUE;
                            P.sh_o[slot] = make_float4(ne.o.x, ne.o.y, ne.o.z, MED ? __uint_as_float(cur_med) : 0.0f);
                            P.sh_d[slot] = make_float4(ne.d.x, ne.d.y, ne.d.z, ne.tmax);
                            P.sh_c[slot] = make_float4(c.x, c.y, c.z, spec_true ? 0.0f : 1.0f);
                            shadow = true;
                        }
                    }
                }
                const float x1 = rng.next_f(), x2 = rng.next_f();
                const float xr = sqrtf(x1);
                float xs, xc;
                sincosf(2.0f * RT_PI * x2, &xs, &xc);
                const float3 local = f3(xr * xc, xr * xs, sqrtf(fmaxf(1.0f - x1, 0.0f)));
                const float3 wi = normalize_ref(xf.to_world(local));
                pdf_prev = fmaxf(local.z, 1e-9f) * (1.0f / RT_PI);
                prev4 = make_float4(xp.x, xp.y, xp.z, 0.0f);
                flags &= ~FL_FROM_CAMERA;
                if (P.cone) {
                    float2 cn = P.cone[slot];
                    cn.y += 0.4f;
                    P.cone[slot] = cn;
                }
                wo = xp + out_n * RT_RAY_OFFSET;
                wd = wi;
                exited = true;
                break;
            }
            if (exited) {
                const uint32_t depth = (flags >> FL_DEPTH_SHIFT) + 1;
                flags = (flags & 0xFFFFu) | (depth << FL_DEPTH_SHIFT);
                bool alive = true;
                if (depth >= C.rr_start) {
                    const float q = fminf(maxc(beta) * o4.w, 0.95f);
                    if (q <= 0.0f || rng.next_f() > q) alive = false;
                    else beta = beta / q;
                }
                if (alive && depth < C.max_depth) {
                    P.ray_o[slot] = make_float4(wo.x, wo.y, wo.z, o4.w);
                    P.ray_d[slot] = make_float4(wd.x, wd.y, wd.z, INFINITY);
                    extend = true;
                }
            }
            shadow2 = MED && (flags & FL_SH2);
            flags &= ~FL_SH2;
            P.beta[slot] = make_float4(beta.x, beta.y, beta.z, pdf_prev);
            P.prev[slot] = make_float4(prev4.x, prev4.y, prev4.z, __uint_as_float(flags));
            P.rng[slot] = make_uint4((uint32_t)rng.state, (uint32_t)(rng.state >> 32), rs.z, rs.w);
        }
        push_queue(P.q_ext[qout], &P.cnt[CNT_EXT_OUT], slot, extend);
        if (MED)
            push_queue(P.q_sh, &P.cnt[CNT_SHADOW], slot | (shadow ? SH_PRIMARY : 0u) | (shadow2 ? SH_EQUI : 0u),
                       shadow || shadow2);
        else
            push_queue(P.q_sh, &P.cnt[CNT_SHADOW], slot, shadow);
    }
    if (rays) atomicAdd(&P.stats[0], rays);
}

// ---- shadow rays through media -------------------------------------------------------
// Transmittance of one shadow ray (pt/mod.rs:1244-1306): segment by segment
// to the closest hit, each segment taking its medium's transmittance
// (closed form, or ratio tracking from rng); volume hulls push and pop the
// medium (the ray starts in `medium`, the atmosphere below it), cutouts
// attenuate by 1 - presence, anything else blocks; at most 16 segments.
// EXTRA: motion blur (the ray's shutter time) and pattern-driven presence.
template <bool EXTRA>
__device__ __forceinline__ float3 shadow_walk(const DevScene& S, TravStack& st, float3 o, float3 d, float remaining,
                                              uint32_t medium, Pcg& rng, uint32_t* err, unsigned long long& rays,
                                              float time) {
    uint2 ms = make_uint2(0u, 0u);
    if (medium != RT_MEDIUM_NONE && medium != S.atmosphere) mstack_push(ms, medium);
    float3 vis = f3(1.0f, 1.0f, 1.0f);
    for (int k = 0; k < RT_MAX_PRESENCE_SKIPS; k++) {
        rays++;
        uint4 hr;
        const bool found = remaining > 0.0f && trace_closest<EXTRA>(S, st, o, d, remaining, err, hr, time);
        const float t = found ? __uint_as_float(hr.x) : remaining;
        const uint32_t cur = mstack_top(ms, S.atmosphere);
        if (cur != RT_MEDIUM_NONE) {
            vis = vis * med_transmittance(S.media[cur], o, d, fmaxf(t, 0.0f), rng);
            if (maxc(vis) < 1e-4f) return f3(0.0f, 0.0f, 0.0f);
        }
        if (!found) return vis;
        const uint32_t mat = (hr.y & RT_TRI_QUADRIC) ? S.quadrics[hr.y & ~RT_TRI_QUADRIC].material
                                                     : __ldg(&S.inst[hr.z].z);
        const DevMaterial& m = S.materials[mat];
        if (m.hull != 0.0f) {
            HitGeo hg;
            hit_geometry(S, o, d, hr, hg, time);
            if (hg.front) mstack_push(ms, m.interior);
            else mstack_pop(ms);
        } else {
            float presence = m.presence;
            if (EXTRA && S.presence_pat && S.mat_pat[mat].bind_n) {
                // Pattern-driven cutout: the blocker's material with its
                // patterns at the hit, footprint 0 (pt/mod.rs:1290,
                // kernel_pt.metal:1369).
                HitGeo hg;
                hit_geometry(S, o, d, hr, hg, time);
                const HitSt hs = hit_st(S, hr, hg.p, time);
                DevMaterial mres = m;
                resolve_material(S, S.mat_pat[mat], hs, hg.p, hg.nw, d, 0.0f, mres);
                presence = mres.presence;
            }
            if (presence >= 1.0f) return f3(0.0f, 0.0f, 0.0f);
            vis = vis * (1.0f - presence);
            if (maxc(vis) < 1e-4f) return f3(0.0f, 0.0f, 0.0f);
        }
        o = o + d * (t + RT_RAY_OFFSET);
        remaining -= t + RT_RAY_OFFSET;
    }
    return vis;
}

// Scenes with media: one thread per queued slot walks its shadow rays (the
// surface / collision / walk-exit one, then the equiangular one) and adds
// both contributions in that order. Ratio tracking draws from a stream
// derived from the path's state, so the image stays reproducible.
// Without MED (scenes whose cutouts are pattern-driven, no media) each
// queue entry is a plain slot with one shadow ray and no medium. EXTRA:
// motion blur or pattern-driven presence (kept out of the common variant,
// whose registers they would raise).
template <int BLOCK, bool MED = true, bool EXTRA = false>
__global__ void __launch_bounds__(BLOCK) k_shadow_walk(DevScene S, Paths P, PtConsts C) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    const uint32_t n = P.cnt[CNT_SHADOW];
    unsigned long long rays = 0;
    for (uint32_t j = blockIdx.x * BLOCK + threadIdx.x; j < n; j += gridDim.x * BLOCK) {
        const uint32_t e = MED ? P.q_sh[j] : (P.q_sh[j] | SH_PRIMARY);
        const uint32_t slot = e & SH_SLOT_MASK;
        const uint4 rs = P.rng[slot];
        Pcg rng;
        rng.state = splitmix(((uint64_t)rs.x | ((uint64_t)rs.y << 32)) ^ 0xD1B54A32D192ED03ull);
        rng.inc = (splitmix((uint64_t)rs.z | ((uint64_t)rs.w << 32)) << 1) | 1ull;
        float3 add = f3(0.0f, 0.0f, 0.0f), add_aux = f3(0.0f, 0.0f, 0.0f);
        for (int r = 0; r < (MED ? 2 : 1); r++) {
            if (!(e & (r == 0 ? SH_PRIMARY : SH_EQUI))) continue;
            const float4 o4 = r == 0 ? P.sh_o[slot] : P.sh2_o[slot];
            const float4 d4 = r == 0 ? P.sh_d[slot] : P.sh2_d[slot];
            const float4 c4 = r == 0 ? P.sh_c[slot] : P.sh2_c[slot];
            const float3 vis = shadow_walk<EXTRA>(S, st, xyz(o4), xyz(d4), d4.w,
                                                  MED ? __float_as_uint(o4.w) : RT_MEDIUM_NONE, rng, P.err, rays,
                                                  EXTRA && S.motion ? P.time[slot] : 0.0f);
            const float3 c = xyz(c4) * vis;
            add = add + c;
            if (c4.w != 0.0f) add_aux = add_aux + c;
        }
        const float4 L = P.L[slot];
        P.L[slot] = make_float4(L.x + add.x, L.y + add.y, L.z + add.z, L.w);
        if (C.aovs) {
            const float4 a = P.aux_d[slot];
            P.aux_d[slot] = make_float4(a.x + add_aux.x, a.y + add_aux.y, a.z + add_aux.z, a.w);
        }
    }
    if (rays) atomicAdd(&P.stats[1], rays);
}

__global__ void k_wave_prep(uint32_t* cnt) {
    uint32_t t = threadIdx.x;
    if (t == 0) {
        cnt[CNT_EXT_IN] = cnt[CNT_EXT_OUT];
        cnt[CNT_EXT_OUT] = 0;
        cnt[CNT_SHADOW] = 0;
        cnt[CNT_FETCH_EXT] = 0;
        cnt[CNT_FETCH_SH] = 0;
        cnt[CNT_SSS] = 0;
    }
    if (t < N_QUEUES) cnt[CNT_CLASS + t] = 0;
}

// ---- accumulate ------------------------------------------------------------------------
// Per pixel, in sample order: firefly clamp (mod.rs:90-93), f64 sum.
__global__ void k_accumulate(Paths P, PtConsts C, uint32_t samples_in_slab, double* accum, float* aux) {
    uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= C.npix) return;
    double r = 0, g = 0, b = 0, l1 = 0, l2 = 0;
    uint32_t taken = 0;
    for (uint32_t s = 0; s < samples_in_slab; s++) {
        uint32_t slot = s * C.npix + pix;
        if (C.adaptive_tol > 0.0f && (__float_as_uint(P.prev[slot].w) & FL_INACTIVE)) continue;
        taken++;
        float4 L = P.L[slot];
        float3 l = xyz(L);
        float lum = luminance(l);
        float k = 1.0f;
        if (lum > C.clamp) {
            k = C.clamp / lum;
            l = l * k;
        }
        r += (double)l.x;
        g += (double)l.y;
        b += (double)l.z;
        const double lc = (double)luminance(l);
        l1 += lc;
        l2 += lc * lc;
        if (C.aovs) {
            float4 a = P.aux_a[slot], nn = P.aux_n[slot], dd = P.aux_d[slot];
            float* A = aux + 12 * (size_t)pix;
            A[0] += a.x; A[1] += a.y; A[2] += a.z;
            A[3] += nn.x; A[4] += nn.y; A[5] += nn.z;
            A[6] += a.w;
            if (A[11] == 0.0f && dd.w > 0.0f) A[7] = (float)__float_as_uint(nn.w);
            A[8] += dd.x * k; A[9] += dd.y * k; A[10] += dd.z * k;
            A[11] += dd.w;
        }
    }
    double* acc = accum + 4 * (size_t)pix;
    acc[0] += r;
    acc[1] += g;
    acc[2] += b;
    acc[3] += (double)taken;
    double* st = C.lum_stats + 4 * (size_t)pix;
    st[0] += l1;
    st[1] += l2;
    st[2] += (double)taken;
}

// ---- image: radiance sums / sample weight, f64 division rounded to f32 -------------------
__global__ void k_resolve(const double* __restrict__ accum, float* __restrict__ rgb, uint32_t npix) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npix) return;
    const double4 a = reinterpret_cast<const double4*>(accum)[i];
    const double w = a.w > 0.0 ? a.w : 1.0;
    rgb[3 * (size_t)i] = (float)(a.x / w);
    rgb[3 * (size_t)i + 1] = (float)(a.y / w);
    rgb[3 * (size_t)i + 2] = (float)(a.z / w);
}

// ---- ray batch (rt_intersect_batch) ------------------------------------------------------
template <int BLOCK, bool ANY, bool QUAD = false>
__global__ void __launch_bounds__(BLOCK, RT_TRAV_MIN_BLOCKS) k_intersect(DevScene S, const float4* __restrict__ org,
                                                     const float4* __restrict__ dir, uint64_t n, uint32_t* prim,
                                                     uint32_t* inst, float* tout, uint32_t* fetch, uint32_t* err) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    __shared__ LeafShared leaf_sh[BLOCK / 32];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    uint32_t qk = 0xFFFFFFFFu;  // closest (or blocking) quadric of this lane's ray
    float qt = 0.0f;
    auto load = [&](uint32_t j, float3& o, float3& d, float& tmax, uint64_t& seed, float&) {
        float4 o4 = __ldg(org + j), d4 = __ldg(dir + j);
        o = xyz(o4);
        d = xyz(d4);
        tmax = d4.w;
        qk = 0xFFFFFFFFu;
        if (QUAD) {
            const float dl = fmaxf(length(d), 1e-30f);
            float tw;
            qk = quadrics_closest(S, o, d / dl, tmax * dl, tw);
            if (qk != 0xFFFFFFFFu) tmax = qt = ANY ? -1.0f : tw / dl;
        }
    };
    auto finish = [&](bool done, uint32_t i, const TravState& ts) {
        if (!done) return;
        if (ANY) {
            prim[i] = (ts.found || qk != 0xFFFFFFFFu) ? 1u : 0u;
        } else {
            uint32_t p = 0xFFFFFFFFu, ii = 0xFFFFFFFFu;
            float t = INFINITY;
            if (ts.found) {
                p = __float_as_uint(__ldg(&S.tris[3 * (size_t)ts.hit.tri].w));
                ii = __ldg(&S.inst[ts.hit.inst].y);
                t = ts.hit.t;
            } else if (qk != 0xFFFFFFFFu) {
                p = 0u;
                ii = RT_HIT_QUADRIC | qk;
                t = qt;
            }
            prim[i] = p;
            if (inst) inst[i] = ii;
            if (tout) tout[i] = t;
        }
    };
    ray_pump<ANY, false, false, QUAD>(S, (uint32_t)n, fetch, err, st, leaf_sh[threadIdx.x >> 5], load, finish);
}

// ---- diagnostics: the device functions the render kernels use, on caller inputs ----------
// Transmittance of caller rays through the shadow kernel's query
// (rt_transmittance_batch): the same pump and cooperative leaves as k_shadow
// in scenes with presence cutouts.
template <int BLOCK, bool QUAD = false>
__global__ void __launch_bounds__(BLOCK, RT_TRAV_MIN_BLOCKS) k_transmit_batch(DevScene S, const float4* __restrict__ org,
                                                          const float4* __restrict__ dir, uint64_t n, float* out,
                                                          uint32_t* fetch, uint32_t* err) {
    __shared__ uint2 stack_sh[RT_SH_STACK * BLOCK];
    __shared__ LeafShared leaf_sh[BLOCK / 32];
    TravStack st;
    st.init(stack_sh + threadIdx.x, BLOCK);
    float qvis = 1.0f;
    auto load = [&](uint32_t j, float3& o, float3& d, float& tmax, uint64_t& seed, float&) {
        float4 o4 = __ldg(org + j), d4 = __ldg(dir + j);
        o = xyz(o4);
        d = xyz(d4);
        tmax = d4.w;
        qvis = 1.0f;
        if (QUAD) {
            const float dl = fmaxf(length(d), 1e-30f);
            qvis = quadrics_transmittance(S, o, d / dl, tmax * dl);
            if (qvis == 0.0f) tmax = -1.0f;  // nothing left for the BVH to find
        }
    };
    auto finish = [&](bool done, uint32_t i, const TravState& ts) {
        if (done) out[i] = ts.trans * qvis;
    };
    ray_pump<true, true, false, QUAD>(S, (uint32_t)n, fetch, err, st, leaf_sh[threadIdx.x >> 5], load, finish);
}

// Hair BSDF value and pdf for n (wo, wi, h) queries, 7 floats each.
__global__ void k_hair_eval_batch(DevHair hp, const float* __restrict__ q, uint32_t n, float* __restrict__ f,
                                  float* __restrict__ pdf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = q + 7ull * i;
    HairEval g;
    hair_prepare(hp, f3(r[0], r[1], r[2]), r[6], g);
    float pd;
    const float3 v = hair_f_pdf(hp, g, f3(r[3], r[4], r[5]), pd);
    f[3ull * i] = v.x;
    f[3ull * i + 1] = v.y;
    f[3ull * i + 2] = v.z;
    pdf[i] = pd;
}

// n consecutive hair samples for one (wo, h) from the stream of (pixel,
// sample): wi, f, pdf (pdf 0 where sampling failed). One thread.
__global__ void k_hair_sample_batch(DevHair hp, float3 wo, float h, uint64_t pixel, uint64_t sample, uint32_t n,
                                    float* __restrict__ out) {
    if (blockIdx.x || threadIdx.x) return;
    Pcg rng = pcg_for_pixel_sample(pixel, sample);
    HairEval g;
    hair_prepare(hp, wo, h, g);
    for (uint32_t i = 0; i < n; i++) {
        float3 wi = f3(0.0f, 0.0f, 0.0f), f = f3(0.0f, 0.0f, 0.0f);
        float pdf = 0.0f;
        if (!hair_sample(hp, g, rng, wi, f, pdf)) pdf = 0.0f;
        float* o = out + 7ull * i;
        o[0] = wi.x, o[1] = wi.y, o[2] = wi.z, o[3] = f.x, o[4] = f.y, o[5] = f.z, o[6] = pdf;
    }
}

// The first n u32 draws of Pcg32::for_pixel_sample(pixel[i], sample[i]).
__global__ void k_pcg_streams(const uint64_t* __restrict__ pixel, const uint64_t* __restrict__ sample, uint32_t m,
                              uint32_t n, uint32_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    Pcg r = pcg_for_pixel_sample(pixel[i], sample[i]);
    for (uint32_t k = 0; k < n; k++) out[(size_t)i * n + k] = r.next_u32();
}

// Light-BVH pick (light_sample) at points p with uniforms u; light ~0 when
// the scene has no lights.
__global__ void k_light_sample_batch(DevScene S, const float* __restrict__ p, const float* __restrict__ u, uint32_t m,
                                     uint32_t* __restrict__ light, float* __restrict__ pmf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    uint32_t li = 0xFFFFFFFFu;
    float pm = 0.0f;
    if (!light_sample(S, f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), u[i], li, pm)) {
        li = 0xFFFFFFFFu;
        pm = 0.0f;
    }
    light[i] = li;
    pmf[i] = pm;
}

// Light-BVH pick probability (light_pmf) of light[i] at p[i].
__global__ void k_light_pmf_batch(DevScene S, const float* __restrict__ p, const uint32_t* __restrict__ light,
                                  uint32_t m, float* __restrict__ pmf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    pmf[i] = light_pmf(S, f3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), light[i]);
}

// White-furnace estimator of one material: per thread, `per` BSDF samples
// from its own PCG stream; sums of lum(f)|cos|/pdf and of the RGB weights.
__global__ void k_furnace(DevMaterial m, float3 wo, float eta, uint64_t per, uint64_t seed, double* out) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    Pcg rng = pcg_for_pixel_sample(t, seed);
    double a = 0, r = 0, g = 0, b = 0;
    for (uint64_t i = 0; i < per; i++) {
        BsdfSample s;
        if (bsdf_sample(m, wo, eta, rng, s)) {
            float k = fabsf(s.wi.z) / s.pdf;
            a += (double)(luminance(s.f) * k);
            r += (double)(s.f.x * k);
            g += (double)(s.f.y * k);
            b += (double)(s.f.z * k);
        }
    }
    out[4 * t] = a;
    out[4 * t + 1] = r;
    out[4 * t + 2] = g;
    out[4 * t + 3] = b;
}

}  // namespace rt
