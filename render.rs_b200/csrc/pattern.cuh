// pattern.cuh — procedural pattern graph on the device: the shading-time
// substitution of pattern outputs into a material's PbrParams.
//
// Reference: PatternNode::eval (src/texture/pattern.rs:126-226),
// BoundField::apply (:278-296), Material::resolved_pbr
// (src/scene/material.rs:95-101), the Perlin fBm behind PxrFractal
// (src/geometry/displace.rs:36-97) and shade_params (pt/mod.rs:389-439).
//
// A material's bindings reach at most RT_MAX_PATTERN_NODES consecutive
// nodes (node_lo + the bits of node_mask); inputs always point to lower
// nodes, so one pass in index order evaluates every reached node once into
// a small per-thread table, where the reference re-walks shared inputs
// recursively (same values: nodes are pure functions of the shading point).
// The resolved parameters are folded into a DevMaterial exactly as the host
// folds a plain material (flatten.cpp fold_material), in f32.
#pragma once

#include "rt_internal.h"
#include "rt_scene.h"

namespace rt {

// displace.rs:36-43: 64-bit mix of a lattice key (arithmetic right shifts
// of a signed 64-bit value, as on the reference's i64).
__device__ __forceinline__ uint32_t lattice_hash(int64_t x) {
    x = (int64_t)((uint64_t)x * 0x9e3779b97f4a7c15ull);
    x ^= x >> 29;
    x = (int64_t)((uint64_t)x * 0xbf58476d1ce4e5b9ull);
    x ^= x >> 32;
    return (uint32_t)(uint64_t)x;
}

// displace.rs:45-80: gradient noise over the integer lattice with the 12
// cube-edge gradients (+-1 in two axes), quintic fade, trilinear blend.
__device__ __forceinline__ float perlin(float px, float py, float pz) {
    const float cx = floorf(px), cy = floorf(py), cz = floorf(pz);
    const float fx = px - cx, fy = py - cy, fz = pz - cz;
    const int64_t ix = (int64_t)cx, iy = (int64_t)cy, iz = (int64_t)cz;
    float corner[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int64_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        const uint64_t key = (uint64_t)(ix + dx) * 73856093ull ^ (uint64_t)(iy + dy) * 19349663ull ^
                             (uint64_t)(iz + dz) * 83492791ull;
        const uint32_t h = lattice_hash((int64_t)key) % 12u;
        // h 0-3: (+-1, +-1, 0); 4-7: (+-1, 0, +-1); 8-11: (0, +-1, +-1).
        const float g0 = h < 8u ? ((h & 1u) ? -1.0f : 1.0f) : 0.0f;
        const float g1 = h < 4u ? ((h & 2u) ? -1.0f : 1.0f) : (h < 8u ? 0.0f : ((h & 1u) ? -1.0f : 1.0f));
        const float g2 = h < 4u ? 0.0f : ((h & 2u) ? -1.0f : 1.0f);
        corner[k] = g0 * (fx - (float)dx) + g1 * (fy - (float)dy) + g2 * (fz - (float)dz);
    }
    auto fade = [](float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); };
    auto lerp = [](float a, float b, float t) { return a + (b - a) * t; };
    const float u = fade(fx), v = fade(fy), w = fade(fz);
    const float y0 = lerp(lerp(corner[0], corner[1], u), lerp(corner[2], corner[3], u), v);
    const float y1 = lerp(lerp(corner[4], corner[5], u), lerp(corner[6], corner[7], u), v);
    return lerp(y0, y1, w);
}

__device__ __forceinline__ float lum3(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// One node at a shading point; `v` holds the outputs of nodes node_lo.. so
// far, `lo` is node_lo.
__device__ __forceinline__ float3 pattern_node(const DevScene& S, const DevPattern& g, const float3* v, uint32_t lo,
                                               float s, float t, float3 p, float footprint) {
    auto input = [&](int k) {
        return g.in[k] == 0xFFFFFFFFu ? f3(g.c[k][0], g.c[k][1], g.c[k][2]) : v[g.in[k] - lo];
    };
    switch (g.type) {
        case RT_PATTERN_CHECKER: {
            const float fs = s * g.s0, ft = t * g.s1;
            const int64_t cell = (int64_t)(floorf(fs) + floorf(ft));
            const float3 a = f3(g.c[0][0], g.c[0][1], g.c[0][2]), b = f3(g.c[1][0], g.c[1][1], g.c[1][2]);
            const float3 sharp = (cell & 1) ? b : a;
            const float w = fminf(footprint * fmaxf(fabsf(g.s0), fabsf(g.s1)), 1.0f);
            return sharp * (1.0f - w) + (a + b) * (0.5f * w);
        }
        case RT_PATTERN_FRACTAL: {
            float sum = 0.0f, amp = 1.0f, freq = g.s0;
            for (uint32_t o = 0; o < g.u0; o++) {
                sum += amp * perlin(p.x * freq, p.y * freq, p.z * freq);
                amp *= g.s1;
                freq *= g.s2;
            }
            const float x = fminf(fmaxf(sum * 0.5f + 0.5f, 0.0f), 1.0f);
            return f3(x, x, x);
        }
        case RT_PATTERN_MIX: {
            const float m = fminf(fmaxf(input(2).x, 0.0f), 1.0f);
            return input(0) * (1.0f - m) + input(1) * m;
        }
        case RT_PATTERN_COLOR_CORRECT: {
            const float3 in = input(0);
            const float e = 1.0f / fmaxf(g.s0, 1e-6f);
            float3 out = f3(powf(fmaxf(in.x * g.c[1][0] + g.c[2][0], 0.0f), e),
                            powf(fmaxf(in.y * g.c[1][1] + g.c[2][1], 0.0f), e),
                            powf(fmaxf(in.z * g.c[1][2] + g.c[2][2], 0.0f), e));
            if (fabsf(g.s1 - 1.0f) > 1e-9f) {
                const float l = lum3(out);
                out = f3(l, l, l) + (out - f3(l, l, l)) * g.s1;
            }
            return out;
        }
        case RT_PATTERN_RAMP: {
            if (g.u1 == 0u) return f3(1.0f, 0.0f, 1.0f);  // the reference's missing colour
            const float x = fminf(fmaxf(g.u2 ? t : s, 0.0f), 1.0f);
            const float4* r = S.ramp + g.u0;
            float4 prev = __ldg(r);
            if (x <= prev.x) return f3(prev.y, prev.z, prev.w);
            for (uint32_t i = 1; i < g.u1; i++) {
                const float4 cur = __ldg(r + i);
                if (x <= cur.x) {
                    const float a = (x - prev.x) / fmaxf(cur.x - prev.x, 1e-9f);
                    return f3(prev.y, prev.z, prev.w) * (1.0f - a) + f3(cur.y, cur.z, cur.w) * a;
                }
                prev = cur;
            }
            return f3(prev.y, prev.z, prev.w);
        }
        default: return f3(1.0f, 0.0f, 1.0f);
    }
}

// BoundField::apply: scalars take channel 0; roughnesses clamp to
// [0.005, 1] (presence bindings are refused when the scene is built).
__device__ __forceinline__ void apply_field(DevPbr& q, uint32_t field, float3 v) {
    auto set3 = [&](float* dst) {
        dst[0] = v.x;
        dst[1] = v.y;
        dst[2] = v.z;
    };
    switch (field) {
        case RT_FIELD_DIFFUSE_COLOR: set3(q.diffuse_color); break;
        case RT_FIELD_DIFFUSE_GAIN: q.diffuse_gain = v.x; break;
        case RT_FIELD_DIFFUSE_ROUGHNESS: q.diffuse_roughness = v.x; break;
        case RT_FIELD_SPECULAR_FACE_COLOR: set3(q.spec_face); break;
        case RT_FIELD_SPECULAR_EDGE_COLOR: set3(q.spec_edge); break;
        case RT_FIELD_SPECULAR_ROUGHNESS: q.spec_rough = fminf(fmaxf(v.x, 0.005f), 1.0f); break;
        case RT_FIELD_CLEARCOAT_GAIN: q.cc_gain = v.x; break;
        case RT_FIELD_FUZZ_GAIN: q.fuzz_gain = v.x; break;
        case RT_FIELD_FUZZ_COLOR: set3(q.fuzz_color); break;
        case RT_FIELD_GLASS_GAIN: q.glass_gain = v.x; break;
        case RT_FIELD_GLASS_ROUGHNESS: q.glass_rough = fminf(fmaxf(v.x, 0.005f), 1.0f); break;
        case RT_FIELD_REFRACTION_COLOR: set3(q.refraction); break;
        case RT_FIELD_GLOW: set3(q.glow); break;
        default: break;
    }
}

// The host's fold_material in f32: lobe weights (pbr.rs:188-201), F0
// (pbr.rs:86-96), under-layer scale (bxdf.rs:137-143), Oren-Nayar A/B, GGX
// alphas, the first-hit albedo. Keeps d's area light, id and class.
__device__ __forceinline__ void fold_pbr(const DevPbr& q, DevMaterial& d) {
    const float3 face = f3(q.spec_face[0], q.spec_face[1], q.spec_face[2]);
    float3 f0 = f3(0.0f, 0.0f, 0.0f);
    if (lum3(face) > 1e-6f) {
        f0 = face;
    } else if (q.spec_ior > 1.0f) {
        const float r = (q.spec_ior - 1.0f) / (q.spec_ior + 1.0f);
        f0 = f3(r * r, r * r, r * r);
    }
    const bool has_spec = lum3(f0) > 1e-6f;
    const float3 dc = f3(q.diffuse_color[0], q.diffuse_color[1], q.diffuse_color[2]);
    const float3 fc = f3(q.fuzz_color[0], q.fuzz_color[1], q.fuzz_color[2]);
    const float wd = q.diffuse_gain * lum3(dc), ws = sqrtf(lum3(f0)), wc = q.cc_gain * 0.2f,
                wf = q.fuzz_gain * lum3(fc) * 0.3f, wg = q.glass_gain;
    const float total = wd + ws + wc + wf + wg;
    const bool lobes = total > 1e-9f;
    const float inv = lobes ? 1.0f / total : 0.0f;
    d.w_diff = wd * inv;
    d.w_spec = ws * inv;
    d.w_coat = wc * inv;
    d.w_fuzz = wf * inv;
    d.w_glass = wg * inv;
    d.has_lobes = lobes ? 1.0f : 0.0f;
    const float uls = fminf(fmaxf((1.0f - lum3(f0)) * (1.0f - 0.04f * q.cc_gain), 0.0f), 1.0f);
    const float sigma2 = q.diffuse_roughness * q.diffuse_roughness;
    d.on_a = 1.0f - sigma2 / (2.0f * (sigma2 + 0.33f));
    d.on_b = 0.45f * sigma2 / (sigma2 + 0.09f);
    auto alpha_of = [](float r) { return fminf(fmaxf(r * r, 2.5e-5f), 1.0f); };
    d.alpha_spec = alpha_of(q.spec_rough);
    d.alpha_coat = alpha_of(q.cc_rough);
    d.alpha_glass = alpha_of(q.glass_rough);
    d.coat_gain = q.cc_gain;
    d.glass_scale = q.glass_gain * uls;
    d.ior = q.glass_ior;
    d.presence = fminf(fmaxf(q.presence, 0.0f), 1.0f);
    const float f0a[3] = {f0.x, f0.y, f0.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        d.kd[k] = q.diffuse_color[k] * q.diffuse_gain * uls * (1.0f / RT_PI);
        d.f0[k] = f0a[k];
        d.f90[k] = q.spec_edge[k];
        d.kfuzz[k] = q.fuzz_color[k] * q.fuzz_gain * (1.0f / RT_PI);
        d.refr[k] = q.refraction[k];
        d.emission[k] = q.emission[k] + q.glow[k];
        d.albedo[k] = fminf(q.diffuse_color[k] * q.diffuse_gain + (has_spec ? f0a[k] : 0.0f) +
                                q.refraction[k] * q.glass_gain,
                            1.0f);
    }
}

// Material `mat` at a shading point: base parameters with every bound
// pattern output substituted in binding order, folded into `d` (which
// must hold the material's plain record on entry). Kept out of line: only
// patterned hits call it, and inlined its node table and fold would raise
// the shade kernel's register count for every scene (128 -> 192).
__device__ __noinline__ void resolve_material(const DevScene& S, const DevMatPat& mp, float s, float t, float3 p,
                                                 float footprint, DevMaterial& d) {
    float3 v[RT_MAX_PATTERN_NODES];
    for (uint32_t k = 0; k < RT_MAX_PATTERN_NODES; k++) {
        if (!((mp.node_mask >> k) & 1u)) continue;
        const DevPattern g = S.patterns[mp.node_lo + k];
        v[k] = pattern_node(S, g, v, mp.node_lo, s, t, p, footprint);
    }
    DevPbr q = S.pbr[mp.pbr_index];
    for (uint32_t b = 0; b < mp.bind_n; b++) {
        const uint2 fb = __ldg(S.binds + mp.bind_off + b);
        apply_field(q, fb.x, v[fb.y - mp.node_lo]);
    }
    fold_pbr(q, d);
}

}  // namespace rt
