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

// st at a hit: coordinates, density (st units per world unit) and the
// world-space gradients of s and t.
struct HitSt {
    float s, t, dens;
    float3 gs, gt;
};

// ---- file textures (src/texture/cache.rs) -------------------------------------------
// One texel of a mip level with the wrap mode applied (cache.rs:186-203).
__device__ __forceinline__ float3 tex_texel(const DevScene& S, const DevMip& m, int64_t x, int64_t y, uint32_t wrap) {
    const int64_t w = m.w, h = m.h;
    if (wrap == RT_WRAP_PERIODIC) {
        x = ((x % w) + w) % w;
        y = ((y % h) + h) % h;
    } else if (wrap == RT_WRAP_CLAMP) {
        x = x < 0 ? 0 : (x >= w ? w - 1 : x);
        y = y < 0 ? 0 : (y >= h ? h - 1 : y);
    } else if (x < 0 || x >= w || y < 0 || y >= h) {
        return f3(0.0f, 0.0f, 0.0f);
    }
    const float4 v = __ldg(S.texels + m.offset + (size_t)y * m.w + (size_t)x);
    return f3(v.x, v.y, v.z);
}

// Bilinear lookup at (s, t), t = 0 at the top row (cache.rs:205-229).
__device__ __forceinline__ float3 tex_bilinear(const DevScene& S, const DevMip& m, float s, float t, uint32_t wrap) {
    const float fx = s * (float)m.w - 0.5f, fy = t * (float)m.h - 0.5f;
    const float x0 = floorf(fx), y0 = floorf(fy);
    const float ax = fx - x0, ay = fy - y0;
    const int64_t ix = (int64_t)x0, iy = (int64_t)y0;
    return tex_texel(S, m, ix, iy, wrap) * ((1.0f - ax) * (1.0f - ay)) +
           tex_texel(S, m, ix + 1, iy, wrap) * (ax * (1.0f - ay)) +
           tex_texel(S, m, ix, iy + 1, wrap) * ((1.0f - ax) * ay) + tex_texel(S, m, ix + 1, iy + 1, wrap) * (ax * ay);
}

// Trilinear lookup with the mip chosen by the footprint's diameter in st
// units (cache.rs:230-252).
__device__ __forceinline__ float3 tex_sample(const DevScene& S, const DevTexture& T, float s, float t, float footprint,
                                             uint32_t wrap) {
    const float texels = fmaxf(footprint * T.base, 1e-9f);
    const float mip_f = fminf(fmaxf(log2f(texels), 0.0f), (float)(T.n_mips - 1));
    const uint32_t m0 = (uint32_t)floorf(mip_f), m1 = min(m0 + 1, T.n_mips - 1);
    const float a = mip_f - (float)m0;
    const float3 lo = tex_bilinear(S, S.tex_mips[T.first_mip + m0], s, t, wrap);
    if (a < 1e-6f || m1 == m0) return lo;
    return lo * (1.0f - a) + tex_bilinear(S, S.tex_mips[T.first_mip + m1], s, t, wrap) * a;
}

// Elliptical weighted average along the footprint axes du (major) and dv
// (minor) in st units (cache.rs:283-377): the mip from the minor axis
// (anisotropy capped at 16), Gaussian weights exp(-2 r^2) over the
// ellipse's texels (at most 4096 of them, else trilinear).
__device__ __forceinline__ float3 tex_sample_ewa(const DevScene& S, const DevTexture& T, float s, float t, float2 du,
                                                 float2 dv, uint32_t wrap) {
    float major = sqrtf(du.x * du.x + du.y * du.y), minor = sqrtf(dv.x * dv.x + dv.y * dv.y);
    float2 am = du, an = dv;
    if (minor > major) {
        const float tmp = major;
        major = minor;
        minor = tmp;
        am = dv;
        an = du;
    }
    if (major <= 1e-9f) return tex_sample(S, T, s, t, 0.0f, wrap);
    if (minor < major / 16.0f) minor = major / 16.0f;
    const float level = fminf(fmaxf(log2f(fmaxf(minor * T.base, 1e-9f)), 0.0f), (float)(T.n_mips - 1));
    const DevMip m = S.tex_mips[T.first_mip + (uint32_t)floorf(level)];
    const float mw = (float)m.w, mh = (float)m.h;
    const float px = s * mw - 0.5f, py = t * mh - 0.5f;
    const float dux = am.x * mw, duy = am.y * mh, dvx = an.x * mw, dvy = an.y * mh;
    float a = duy * duy + dvy * dvy + 1.0f, b = -2.0f * (dux * duy + dvx * dvy), c = dux * dux + dvx * dvx + 1.0f;
    const float f = a * c - 0.25f * b * b;
    if (f <= 1e-12f) return tex_sample(S, T, s, t, minor, wrap);
    a /= f;
    b /= f;
    c /= f;
    const float det = -b * b + 4.0f * a * c;
    if (det <= 0.0f) return tex_sample(S, T, s, t, minor, wrap);
    const float ur = sqrtf(4.0f * c * det) / det, vr = sqrtf(4.0f * a * det) / det;
    const int64_t x0 = (int64_t)floorf(px - ur), x1 = (int64_t)ceilf(px + ur);
    const int64_t y0 = (int64_t)floorf(py - vr), y1 = (int64_t)ceilf(py + vr);
    if ((x1 - x0) * (y1 - y0) > 4096) return tex_sample(S, T, s, t, minor, wrap);
    float3 sum = f3(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    for (int64_t y = y0; y <= y1; y++) {
        const float ddy = (float)y - py;
        for (int64_t x = x0; x <= x1; x++) {
            const float ddx = (float)x - px;
            const float r2 = a * ddx * ddx + b * ddx * ddy + c * ddy * ddy;
            if (r2 < 1.0f) {
                const float w = expf(-2.0f * r2);
                sum = sum + tex_texel(S, m, x, y, wrap) * w;
                wsum += w;
            }
        }
    }
    if (wsum <= 1e-9f) return tex_sample(S, T, s, t, minor, wrap);
    return sum / wsum;
}

// TextureRef::resolve (pattern.rs:25-38): the texture of a node at (s, t),
// with (s, t) made cell-local for a UDIM set (tile 1001 + s cell + 10 t
// cell, s cells clamped to 0..9); ~0 when missing or not in the set.
__device__ __forceinline__ uint32_t tex_resolve(const DevScene& S, const DevPattern& g, float& s, float& t) {
    if (g.u2 == 0u) return g.u0;
    const float sc = fminf(fmaxf(floorf(s), 0.0f), 9.0f), tc = fmaxf(floorf(t), 0.0f);
    const uint32_t tile = 1001u + (uint32_t)sc + 10u * (uint32_t)tc;
    for (uint32_t k = 0; k < g.u2; k++) {
        const uint2 e = __ldg(S.udim + g.udim_off + k);
        if (e.x == tile) {
            s -= sc;
            t -= tc;
            return e.y;
        }
    }
    return 0xFFFFFFFFu;
}

// pattern.rs:93-124: lookups with t flipped into image rows; a missing
// texture reads magenta.
__device__ __forceinline__ float3 sample_tex(const DevScene& S, const DevPattern& g, float s, float t,
                                             float footprint) {
    const uint32_t tex = tex_resolve(S, g, s, t);
    if (tex == 0xFFFFFFFFu) return f3(1.0f, 0.0f, 1.0f);
    return tex_sample(S, S.textures[tex], s, 1.0f - t, footprint, g.u1);
}

// Everything a node reads at a shading point (pattern.rs:69-82).
struct PatCtx {
    float s, t;
    float3 p, n;
    float footprint;
    float2 dst_major, dst_minor;
};

// One node at a shading point; `v` holds the outputs of nodes node_lo.. so
// far, `lo` is node_lo.
__device__ __forceinline__ float3 pattern_node(const DevScene& S, const DevPattern& g, const float3* v, uint32_t lo,
                                               const PatCtx& cx) {
    const float s = cx.s, t = cx.t, footprint = cx.footprint;
    const float3 p = cx.p;
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
        case RT_PATTERN_TEXTURE: {  // pattern.rs:134-149
            const float ts = s * g.s0, tt = t * g.s1;
            const float aniso =
                fabsf(cx.dst_major.x) + fabsf(cx.dst_major.y) + fabsf(cx.dst_minor.x) + fabsf(cx.dst_minor.y);
            if (aniso > 1e-12f) {
                float ls = ts, lt = tt;
                const uint32_t tex = tex_resolve(S, g, ls, lt);
                if (tex == 0xFFFFFFFFu) return f3(1.0f, 0.0f, 1.0f);
                const float2 du = make_float2(cx.dst_major.x * g.s0, -(cx.dst_major.y * g.s1));
                const float2 dv = make_float2(cx.dst_minor.x * g.s0, -(cx.dst_minor.y * g.s1));
                return tex_sample_ewa(S, S.textures[tex], ls, 1.0f - lt, du, dv, g.u1);
            }
            return sample_tex(S, g, ts, tt, footprint * fmaxf(fabsf(g.s0), fabsf(g.s1)));
        }
        case RT_PATTERN_TRIPLANAR: {  // pattern.rs:200-214
            const float3 an = f3(fabsf(cx.n.x), fabsf(cx.n.y), fabsf(cx.n.z));
            const float total = fmaxf(an.x + an.y + an.z, 1e-9f);
            const float f = g.s0;
            return sample_tex(S, g, p.y * f, p.z * f, footprint) * (an.x / total) +
                   sample_tex(S, g, p.z * f, p.x * f, footprint) * (an.y / total) +
                   sample_tex(S, g, p.x * f, p.y * f, footprint) * (an.z / total);
        }
        default: return f3(1.0f, 0.0f, 1.0f);
    }
}

// BoundField::apply (texture/pattern.rs:270-290): scalars take channel 0;
// roughnesses clamp to [0.005, 1], presence to [0, 1].
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
        case RT_FIELD_PRESENCE: q.presence = fminf(fmaxf(v.x, 0.0f), 1.0f); break;
        default: break;
    }
}

// The host's fold_material in f32: lobe weights (pbr.rs:188-201), F0
// (pbr.rs:86-96), under-layer scale (bxdf.rs:137-143), Oren-Nayar A/B, GGX
// alphas, the first-hit albedo. Keeps d's area light, id, class, interior
// medium and subsurface walk.
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
        d.albedo[k] = fminf(q.diffuse_color[k] * q.diffuse_gain + (has_spec ? f0a[k] : 0.0f) + q.sss_albedo[k] +
                                q.refraction[k] * q.glass_gain,
                            1.0f);
    }
}

// A patterned material at a shading point (shade_params, pt/mod.rs:389-439):
// the footprint is the cone width times the st density, and the cone's
// ellipse on the surface (minor axis the cone width, major stretched by
// 1/|cos| along the projected ray) is carried into st by the gradients;
// base parameters with every bound pattern output substituted in binding
// order are folded into `d` (which holds the material's plain record on
// entry). Kept out of line: only patterned hits call it, and inlined its
// node table and fold would raise the shade kernel's register count.
__device__ __noinline__ void resolve_material(const DevScene& S, const DevMatPat& mp, const HitSt& hs, float3 p,
                                              float3 n, float3 dir, float cone_width, DevMaterial& d) {
    PatCtx cx{hs.s, hs.t, p, n, cone_width * hs.dens, make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
    if (dot(hs.gs, hs.gs) + dot(hs.gt, hs.gt) > 1e-18f && cone_width > 0.0f) {
        const float3 dn = normalize_ref(dir);
        const float cs = fmaxf(fabsf(dot(dn, n)), 1.0f / 16.0f);
        float3 t1 = dn - n * dot(dn, n);
        if (dot(t1, t1) < 1e-12f) t1 = fabsf(n.x) < 0.9f ? cross(f3(1.0f, 0.0f, 0.0f), n) : cross(f3(0.0f, 1.0f, 0.0f), n);
        t1 = normalize_ref(t1) * (cone_width / cs);
        const float3 t2 = normalize_ref(cross(n, t1)) * cone_width;
        cx.dst_major = make_float2(dot(hs.gs, t1), dot(hs.gt, t1));
        cx.dst_minor = make_float2(dot(hs.gs, t2), dot(hs.gt, t2));
    }
    float3 v[RT_MAX_PATTERN_NODES];
    for (uint32_t k = 0; k < RT_MAX_PATTERN_NODES; k++) {
        if (!((mp.node_mask >> k) & 1u)) continue;
        const DevPattern g = S.patterns[mp.node_lo + k];
        v[k] = pattern_node(S, g, v, mp.node_lo, cx);
    }
    DevPbr q = S.pbr[mp.pbr_index];
    for (uint32_t b = 0; b < mp.bind_n; b++) {
        const uint2 fb = __ldg(S.binds + mp.bind_off + b);
        apply_field(q, fb.x, v[fb.y - mp.node_lo]);
    }
    fold_pbr(q, d);
}

}  // namespace rt
