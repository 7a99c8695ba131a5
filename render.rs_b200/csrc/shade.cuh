// shade.cuh — f32 light transport pieces for the shade kernel.
//
// Restatements, in f32, of the reference's CPU path
// (anders94/render.rs, src/raytracer/pt/*) with the GPU-side float
// conventions of its Metal kernel (src/raytracer/metal/kernel_pt.metal):
//  * PCG32: u32 stream bit-identical to Pcg32 (sampler.rs:12-42);
//    uniforms are (u >> 8) * 2^-24 as pcg_f32 (kernel_pt.metal:192-194).
//  * BSDF: PbrParams lobe stack — Oren-Nayar, GGX with VNDF sampling and
//    height-correlated Smith, clearcoat, fuzz, rough dielectric
//    (bxdf.rs:16-374); one-sample lobe selection with the weighted pdf.
//  * light BVH sample / pmf (light_sampler.rs:150-238) over the same
//    48-B node array.
#pragma once

#include "traverse.cuh"

namespace rt {

#define RT_PI 3.14159265358979323846f

// ---- PCG32 -------------------------------------------------------------------
struct Pcg {
    uint64_t state, inc;
    __device__ __forceinline__ uint32_t next_u32() {
        uint64_t old = state;
        state = old * 6364136223846793005ull + inc;
        uint32_t xs = (uint32_t)(((old >> 18) ^ old) >> 27);
        uint32_t rot = (uint32_t)(old >> 59);
        return __funnelshift_r(xs, xs, rot);
    }
    __device__ __forceinline__ float next_f() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
};

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Pcg32::for_pixel_sample (sampler.rs:24-32) via Pcg32::new (:12-21).
__device__ __forceinline__ Pcg pcg_for_pixel_sample(uint64_t pixel, uint64_t sample) {
    uint64_t seed = splitmix((pixel * 0x9e3779b97f4a7c15ull) ^ sample);
    uint64_t stream = splitmix(sample) | 1ull;
    Pcg r;
    r.state = 0;
    r.inc = (stream << 1) | 1ull;
    r.next_u32();
    r.state += seed;
    r.next_u32();
    return r;
}

// ---- shading frame (bxdf.rs:16-39) ---------------------------------------------------
struct Frame {
    float3 t, b, n;
    __device__ __forceinline__ explicit Frame(float3 nn) : n(nn) {
        float3 t0 = fabsf(n.x) > 0.9f ? f3(0, 1, 0) : f3(1, 0, 0);
        t = normalize_ref(cross(n, t0));
        b = cross(n, t);
    }
    __device__ __forceinline__ float3 to_local(float3 w) const { return f3(dot(w, t), dot(w, b), dot(w, n)); }
    __device__ __forceinline__ float3 to_world(float3 w) const { return t * w.x + b * w.y + n * w.z; }
};

// ---- lobes (bxdf.rs:57-232) ---------------------------------------------------------
__device__ __forceinline__ float fresnel_dielectric(float cos_i, float eta) {
    cos_i = fminf(fmaxf(cos_i, 0.0f), 1.0f);
    float sin2_t = (1.0f - cos_i * cos_i) / (eta * eta);
    if (sin2_t >= 1.0f) return 1.0f;
    float cos_t = sqrtf(1.0f - sin2_t);
    float r_par = (eta * cos_i - cos_t) / (eta * cos_i + cos_t);
    float r_perp = (cos_i - eta * cos_t) / (cos_i + eta * cos_t);
    return 0.5f * (r_par * r_par + r_perp * r_perp);
}
__device__ __forceinline__ float ggx_d(float3 h, float a) {
    if (h.z <= 0.0f) return 0.0f;
    float a2 = a * a;
    float d = h.z * h.z * (a2 - 1.0f) + 1.0f;
    return a2 / (RT_PI * d * d);
}
__device__ __forceinline__ float ggx_lambda(float3 w, float a) {
    float c2 = w.z * w.z;
    if (c2 <= 0.0f) return 0.0f;
    float tan2 = fmaxf(1.0f - c2, 0.0f) / c2;
    return (sqrtf(1.0f + a * a * tan2) - 1.0f) * 0.5f;
}
__device__ __forceinline__ float ggx_g1(float3 w, float a) { return 1.0f / (1.0f + ggx_lambda(w, a)); }
__device__ __forceinline__ float ggx_g2(float3 wo, float3 wi, float a) {
    return 1.0f / (1.0f + ggx_lambda(wo, a) + ggx_lambda(wi, a));
}
// Heitz 2018 visible-normal sampling (bxdf.rs:104-123).
__device__ __forceinline__ float3 ggx_sample_vndf(float3 wo, float a, float u1, float u2) {
    float3 v = normalize_ref(f3(a * wo.x, a * wo.y, wo.z));
    float lensq = v.x * v.x + v.y * v.y;
    float3 t1 = lensq > 1e-12f ? f3(-v.y, v.x, 0.0f) * rsqrtf(lensq) : f3(1, 0, 0);
    float3 t2 = cross(v, t1);
    float r = sqrtf(u1), phi = 2.0f * RT_PI * u2;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float p1 = r * cp, p2 = r * sp;
    float s = 0.5f * (1.0f + v.z);
    p2 = (1.0f - s) * sqrtf(fmaxf(1.0f - p1 * p1, 0.0f)) + s * p2;
    float3 nh = t1 * p1 + t2 * p2 + v * sqrtf(fmaxf(1.0f - p1 * p1 - p2 * p2, 0.0f));
    return normalize_ref(f3(a * nh.x, a * nh.y, fmaxf(nh.z, 1e-9f)));
}
__device__ __forceinline__ float ggx_pdf_h(float3 wo, float3 h, float a) {
    float odh = dot(wo, h);
    if (odh <= 0.0f || wo.z <= 0.0f) return 0.0f;
    return ggx_g1(wo, a) * odh * ggx_d(h, a) / wo.z;
}
__device__ __forceinline__ float3 schlick(float3 f0, float3 f90, float c) {
    float m = fminf(fmaxf(1.0f - c, 0.0f), 1.0f);
    float m2 = m * m;
    return f0 + (f90 - f0) * (m2 * m2 * m);
}
__device__ __forceinline__ float3 eval_spec(float3 f0, float3 f90, float a, float3 wo, float3 wi) {
    float3 h = normalize_ref(wo + wi);
    float d = ggx_d(h, a), g = ggx_g2(wo, wi, a);
    return schlick(f0, f90, fmaxf(dot(wo, h), 0.0f)) * (d * g / fmaxf(4.0f * wo.z * wi.z, 1e-9f));
}
__device__ __forceinline__ float spec_pdf(float3 wo, float3 wi, float a) {
    float3 h = normalize_ref(wo + wi);
    float odh = fmaxf(dot(wo, h), 1e-9f);
    return ggx_pdf_h(wo, h, a) / (4.0f * odh);
}
__device__ __forceinline__ float3 eval_diffuse(const DevMaterial& m, float3 wo, float3 wi) {
    float sin_o = sqrtf(fmaxf(1.0f - wo.z * wo.z, 0.0f));
    float sin_i = sqrtf(fmaxf(1.0f - wi.z * wi.z, 0.0f));
    float cos_dphi = 0.0f;
    if (sin_o > 1e-6f && sin_i > 1e-6f) cos_dphi = fminf(fmaxf((wo.x * wi.x + wo.y * wi.y) / (sin_o * sin_i), -1.f), 1.f);
    float sin_a, tan_b;
    if (wo.z < wi.z) {
        sin_a = sin_o;
        tan_b = sin_i / fmaxf(wi.z, 1e-6f);
    } else {
        sin_a = sin_i;
        tan_b = sin_o / fmaxf(wo.z, 1e-6f);
    }
    return f3(m.kd[0], m.kd[1], m.kd[2]) * (m.on_a + m.on_b * fmaxf(cos_dphi, 0.0f) * sin_a * tan_b);
}

// bxdf.rs:193-232 glass transmission (f, pdf within the lobe).
__device__ __forceinline__ float3 glass_transmit(const DevMaterial& m, float3 wo, float3 wi, float eta, float& pdf) {
    float a = m.alpha_glass;
    float3 h = normalize_ref(wo + wi * eta);
    if (h.z < 0.0f) h = -h;
    float odh = dot(wo, h), idh = dot(wi, h);
    pdf = 0.0f;
    if (odh <= 0.0f || idh >= 0.0f) return f3(0, 0, 0);
    float fres = fresnel_dielectric(odh, eta);
    float d = ggx_d(h, a), g = ggx_g2(wo, f3(wi.x, wi.y, -wi.z), a);
    float sd = odh + eta * idh;
    if (fabsf(sd) < 1e-9f) return f3(0, 0, 0);
    // (1/eta^2) radiance factor times the eta^2 of the Jacobian cancel.
    float k = m.glass_scale * (1.0f - fres) * d * g * fabsf(idh * odh / (wi.z * wo.z)) / (sd * sd);
    pdf = ggx_pdf_h(wo, h, a) * fabsf(eta * eta * idh) / (sd * sd);
    return f3(m.refr[0], m.refr[1], m.refr[2]) * k;
}

// bxdf.rs:241-299 composite eval + pdf; wo.z > 0.
__device__ __forceinline__ float3 bsdf_eval(const DevMaterial& m, float3 wo, float3 wi, float eta, float& pdf) {
    pdf = 0.0f;
    if (m.has_lobes == 0.0f) return f3(0, 0, 0);
    if (wi.z > 0.0f) {
        float3 f = f3(0, 0, 0);
        float cos_pdf = wi.z * (1.0f / RT_PI);
        if (m.w_diff > 0.0f) {
            f = f + eval_diffuse(m, wo, wi);
            pdf += m.w_diff * cos_pdf;
        }
        if (m.w_fuzz > 0.0f) {
            float a = 1.0f - wi.z, b = 1.0f - wo.z;
            float rim = 0.5f * (a * a * a * a + b * b * b * b);
            f = f + f3(m.kfuzz[0], m.kfuzz[1], m.kfuzz[2]) * rim;
            pdf += m.w_fuzz * cos_pdf;
        }
        if (m.w_spec > 0.0f) {
            f = f + eval_spec(f3(m.f0[0], m.f0[1], m.f0[2]), f3(m.f90[0], m.f90[1], m.f90[2]), m.alpha_spec, wo, wi);
            pdf += m.w_spec * spec_pdf(wo, wi, m.alpha_spec);
        }
        if (m.w_coat > 0.0f) {
            float c = m.coat_gain;
            f = f + eval_spec(f3(0.04f * c, 0.04f * c, 0.04f * c), f3(c, c, c), m.alpha_coat, wo, wi);
            pdf += m.w_coat * spec_pdf(wo, wi, m.alpha_coat);
        }
        if (m.w_glass > 0.0f) {
            float a = m.alpha_glass;
            float3 h = normalize_ref(wo + wi);
            float fres = fresnel_dielectric(fmaxf(dot(wo, h), 0.0f), eta);
            float d = ggx_d(h, a), g = ggx_g2(wo, wi, a);
            float v = m.glass_scale * fres * d * g / fmaxf(4.0f * wo.z * wi.z, 1e-9f);
            f = f + f3(v, v, v);
            pdf += m.w_glass * fres * spec_pdf(wo, wi, a);
        }
        return f;
    }
    if (m.w_glass <= 0.0f) return f3(0, 0, 0);
    float pl;
    float3 f = glass_transmit(m, wo, wi, eta, pl);
    float3 h = normalize_ref(wo + wi * eta);
    if (h.z < 0.0f) h = -h;
    float fres = fresnel_dielectric(fmaxf(dot(wo, h), 0.0f), eta);
    pdf = m.w_glass * (1.0f - fres) * pl;
    return f;
}

struct BsdfSample {
    float3 wi, f;
    float pdf;
    bool transmitted, specular;
};

// bxdf.rs:309-374 — same draw order: lobe pick, then 2 (+1 for glass R/T).
__device__ __forceinline__ bool bsdf_sample(const DevMaterial& m, float3 wo, float eta, Pcg& rng, BsdfSample& s) {
    if (m.has_lobes == 0.0f) return false;
    float wd = m.w_diff, ws = m.w_spec, wc = m.w_coat, wf = m.w_fuzz, wg = m.w_glass;
    float pick = rng.next_f();
    s.transmitted = false;
    s.specular = pick >= wd + wf;
    float3 wi;
    if (pick < wd + wf) {
        float u = rng.next_f(), v = rng.next_f();
        float r = sqrtf(u), sp, cp;
        sincosf(2.0f * RT_PI * v, &sp, &cp);
        wi = f3(r * cp, r * sp, sqrtf(fmaxf(1.0f - u, 0.0f)));
    } else if (pick < wd + wf + ws || pick < wd + wf + ws + wc) {
        float a = pick < wd + wf + ws ? m.alpha_spec : m.alpha_coat;
        float u1 = rng.next_f(), u2 = rng.next_f();
        float3 h = ggx_sample_vndf(wo, a, u1, u2);
        wi = h * (2.0f * dot(wo, h)) - wo;  // reflect(-wo, h)
        if (wi.z <= 0.0f) return false;
    } else if (wg > 0.0f) {
        float u1 = rng.next_f(), u2 = rng.next_f();
        float3 h = ggx_sample_vndf(wo, m.alpha_glass, u1, u2);
        float fres = fresnel_dielectric(fmaxf(dot(wo, h), 0.0f), eta);
        if (rng.next_f() < fres) {
            wi = h * (2.0f * dot(wo, h)) - wo;
            if (wi.z <= 0.0f) return false;
        } else {
            float ci = dot(wo, h);
            float sin2_t = (1.0f - ci * ci) / (eta * eta);
            if (sin2_t >= 1.0f) return false;
            float ct = sqrtf(1.0f - sin2_t);
            wi = normalize_ref((-wo) / eta + h * (ci / eta - ct));
            if (wi.z >= 0.0f) return false;
            s.transmitted = true;
        }
    } else {
        return false;
    }
    float pdf;
    float3 f = bsdf_eval(m, wo, wi, eta, pdf);
    if (pdf <= 0.0f) return false;
    s.wi = wi;
    s.f = f;
    s.pdf = pdf;
    return true;
}

// ---- light BVH (light_sampler.rs:74-87, 150-238) -------------------------------------
__device__ __forceinline__ float node_importance(const LightNode& n, float3 p) {
    float cx = (n.mn[0] + n.mx[0]) * 0.5f, cy = (n.mn[1] + n.mx[1]) * 0.5f, cz = (n.mn[2] + n.mx[2]) * 0.5f;
    float dx = p.x - cx, dy = p.y - cy, dz = p.z - cz;
    float d2 = dx * dx + dy * dy + dz * dz;
    float rx = (n.mx[0] - n.mn[0]) * 0.5f, ry = (n.mx[1] - n.mn[1]) * 0.5f, rz = (n.mx[2] - n.mn[2]) * 0.5f;
    float r2 = rx * rx + ry * ry + rz * rz;
    return n.power / fmaxf(fmaxf(d2, r2), 1e-6f);
}

__device__ __forceinline__ bool light_sample(const DevScene& S, float3 p, float u, uint32_t& light, float& pmf) {
    bool has_f = S.n_lbvh > 0, has_i = S.n_inf > 0;
    if (!has_f && !has_i) return false;
    pmf = 1.0f;
    bool inf;
    if (has_f && has_i) {
        if (u < S.p_infinite) {
            u /= S.p_infinite;
            pmf *= S.p_infinite;
            inf = true;
        } else {
            u = (u - S.p_infinite) / (1.0f - S.p_infinite);
            pmf *= 1.0f - S.p_infinite;
            inf = false;
        }
    } else {
        inf = has_i;
    }
    if (inf) {
        float acc = 0.0f, target = u * S.inf_total;
        for (uint32_t k = 0; k < S.n_inf; k++) {
            float w = S.inf_power[k];
            acc += w;
            if (target <= acc || k == S.n_inf - 1) {
                light = S.inf_lights[k];
                pmf *= w / fmaxf(S.inf_total, 1e-12f);
                return true;
            }
        }
        return false;
    }
    uint32_t node = 0;
    for (uint32_t guard = 0; guard < 64; guard++) {
        const LightNode& nd = S.lbvh[node];
        if (nd.b == 0xFFFFFFFFu) {
            light = nd.a;
            return true;
        }
        float ia = node_importance(S.lbvh[nd.a], p), ib = node_importance(S.lbvh[nd.b], p);
        float tot = ia + ib;
        float pa = tot > 1e-30f ? ia / tot : 0.5f;
        if (u < pa) {
            u = fminf(u / pa, 1.0f - 1e-7f);
            pmf *= pa;
            node = nd.a;
        } else {
            u = fminf((u - pa) / (1.0f - pa), 1.0f - 1e-7f);
            pmf *= 1.0f - pa;
            node = nd.b;
        }
    }
    return false;
}

__device__ __forceinline__ float light_pmf(const DevScene& S, float3 p, uint32_t light) {
    bool has_f = S.n_lbvh > 0, has_i = S.n_inf > 0;
    for (uint32_t k = 0; k < S.n_inf; k++)
        if (S.inf_lights[k] == light) return (has_f ? S.p_infinite : 1.0f) * S.inf_power[k] / fmaxf(S.inf_total, 1e-12f);
    uint32_t leaf = light < S.n_lights ? S.light_leaf[light] : 0xFFFFFFFFu;
    if (leaf == 0xFFFFFFFFu) return 0.0f;
    float pmf = has_i ? 1.0f - S.p_infinite : 1.0f;
    uint32_t node = leaf;
    for (uint32_t guard = 0; guard < 64 && S.lbvh[node].parent != 0xFFFFFFFFu; guard++) {
        uint32_t parent = S.lbvh[node].parent;
        const LightNode& pn = S.lbvh[parent];
        float ia = node_importance(S.lbvh[pn.a], p), ib = node_importance(S.lbvh[pn.b], p);
        float tot = ia + ib;
        float mine = node == pn.a ? ia : ib;
        pmf *= tot > 1e-30f ? mine / tot : 0.5f;
        node = parent;
    }
    return pmf;
}

// ---- environment map of a dome light (src/scene/envmap.rs:83-160) -----------------
__device__ __forceinline__ void env_texel_of(const DevScene& S, float3 dir, uint32_t* x, uint32_t* y) {
    float3 d = normalize_ref(dir);
    float u = atan2f(d.x, -d.z) * (0.5f / RT_PI);
    u -= floorf(u);  // rem_euclid(1)
    float v = fminf(fmaxf(acosf(fminf(fmaxf(d.y, -1.0f), 1.0f)) / RT_PI, 0.0f), 1.0f);
    *x = min((uint32_t)(u * (float)S.env_w), S.env_w - 1);
    *y = min((uint32_t)(v * (float)S.env_h), S.env_h - 1);
}

__device__ __forceinline__ float3 env_eval(const DevScene& S, float3 dir) {
    uint32_t x, y;
    env_texel_of(S, dir, &x, &y);
    return xyz(__ldg(S.env + (size_t)y * S.env_w + x));
}

// Solid-angle pdf of env_sample: texel weight * w * h / (total * 2 pi^2 sin theta).
__device__ __forceinline__ float env_pdf(const DevScene& S, float3 dir) {
    uint32_t x, y;
    env_texel_of(S, dir, &x, &y);
    const float sin_t = sinf(RT_PI * ((float)y + 0.5f) / (float)S.env_h);
    if (sin_t < 1e-9f) return 0.0f;
    const float4 c = __ldg(S.env + (size_t)y * S.env_w + x);
    const float tw = (0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z) * sin_t;
    return tw * (float)S.env_w * (float)S.env_h / (S.env_total * 2.0f * RT_PI * RT_PI * sin_t);
}

// Index of the CDF interval holding `target` (the reference's binary_search:
// an exact match gives its own index, otherwise the entry before the
// insertion point), clamped to [0, n - 1]; cdf has n + 1 entries.
__device__ __forceinline__ uint32_t env_cdf_find(const float* cdf, uint32_t n, float target) {
    uint32_t lo = 0, hi = n + 1;  // first index with cdf >= target, in [lo, hi]
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(cdf + mid) < target) lo = mid + 1;
        else hi = mid;
    }
    uint32_t i = (lo <= n && __ldg(cdf + lo) == target) ? lo : (lo > 0 ? lo - 1 : 0);
    return min(i, n - 1);
}

__device__ __forceinline__ float3 env_sample(const DevScene& S, float u1, float u2, float3* rad, float* pdf) {
    const uint32_t y = env_cdf_find(S.env_marg, S.env_h, u1 * S.env_total);
    const float row = fmaxf(__ldg(S.env_marg + y + 1) - __ldg(S.env_marg + y), 1e-12f);
    const float* cond = S.env_cond + (size_t)y * (S.env_w + 1);
    const uint32_t x = env_cdf_find(cond, S.env_w, u2 * row);
    const float u = ((float)x + 0.5f) / (float)S.env_w, v = ((float)y + 0.5f) / (float)S.env_h;
    float sp, cp, st, ct;
    sincosf(u * 2.0f * RT_PI, &sp, &cp);
    sincosf(v * RT_PI, &st, &ct);
    const float3 dir = f3(st * sp, ct, -st * cp);
    *rad = xyz(__ldg(S.env + (size_t)y * S.env_w + x));
    *pdf = env_pdf(S, dir);
    return dir;
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
    float a2 = a * a, b2 = b * b;
    return a2 + b2 <= 0.0f ? 0.0f : a2 / (a2 + b2);
}

// ---- IES profiles (src/scene/ies.rs) -----------------------------------------------
// interp_axis (ies.rs:89-106): bracketing angles and the blend between them.
__device__ __forceinline__ void ies_axis(const float* a, uint32_t n, float x, uint32_t& i0, uint32_t& i1, float& t) {
    t = 0.0f;
    if (x <= a[0]) {
        i0 = i1 = 0;
        return;
    }
    if (x >= a[n - 1]) {
        i0 = i1 = n - 1;
        return;
    }
    for (uint32_t i = 0; i + 1 < n; i++) {
        if (x <= a[i + 1]) {
            i0 = i;
            i1 = i + 1;
            t = (x - a[i]) / fmaxf(a[i + 1] - a[i], 1e-9f);
            return;
        }
    }
    i0 = i1 = n - 1;
}

// IesProfile::factor (ies.rs:108-142): candela toward the light-local
// emission direction (vertical angle from local -y, horizontal angle from
// local +x toward +z, folded into the profile's symmetry range), bilinear
// over the grid, divided by the mean candela.
__device__ __forceinline__ float ies_factor(const DevScene& S, const DevIes& P, float3 emit_world) {
    const float3 l = f3(P.m[0] * emit_world.x + P.m[1] * emit_world.y + P.m[2] * emit_world.z,
                        P.m[3] * emit_world.x + P.m[4] * emit_world.y + P.m[5] * emit_world.z,
                        P.m[6] * emit_world.x + P.m[7] * emit_world.y + P.m[8] * emit_world.z);
    const float3 d = normalize_ref(l);
    const float theta = acosf(fminf(fmaxf(-d.y, -1.0f), 1.0f)) * (180.0f / RT_PI);
    float phi = atan2f(d.z, d.x) * (180.0f / RT_PI);
    if (phi < 0.0f) phi += 360.0f;
    const float* va = S.ies_data + P.off;
    const float* ha = va + P.n_v;
    const float* cd = ha + P.n_h;
    const float hmax = ha[P.n_h - 1];
    if (hmax <= 0.0f) {
        phi = 0.0f;
    } else if (hmax <= 90.0f) {
        const float q = fmodf(phi, 180.0f);
        phi = q > 90.0f ? 180.0f - q : q;
    } else if (hmax <= 180.0f) {
        const float q = fmodf(phi, 360.0f);
        phi = q > 180.0f ? 360.0f - q : q;
    }
    uint32_t v0, v1, h0, h1;
    float tv, th;
    ies_axis(va, P.n_v, theta, v0, v1, tv);
    ies_axis(ha, P.n_h, phi, h0, h1, th);
    const float c00 = cd[h0 * P.n_v + v0], c01 = cd[h0 * P.n_v + v1], c10 = cd[h1 * P.n_v + v0],
                c11 = cd[h1 * P.n_v + v1];
    return ((c00 * (1.0f - tv) + c01 * tv) * (1.0f - th) + (c10 * (1.0f - tv) + c11 * tv) * th) / P.average;
}

}  // namespace rt
