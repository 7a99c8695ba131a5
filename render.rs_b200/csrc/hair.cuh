// hair.cuh — Marschner hair on curve hits, f32 (src/raytracer/pt/hair.rs).
//
// R, TT and TRT lobes plus a residual (d'Eon 2011 longitudinal lobes,
// trimmed-logistic azimuthal lobes, Fresnel and absorption attenuation, as
// pbrt-v3 formulates them), in the fiber frame: x along the fiber, y and z
// spanning the normal plane; f is per solid angle with no cosine factor.
#pragma once

#include "shade.cuh"

namespace rt {

#define RT_HAIR_PMAX 3

// hair.rs:104-126: I0 by its series (10 terms) and log I0 with the
// asymptotic form above 12.
__device__ __forceinline__ float hair_i0(float x) {
    float val = 0.0f, x2i = 1.0f, ifact = 1.0f, i4 = 1.0f;
    for (int i = 0; i < 10; i++) {
        if (i > 1) ifact *= (float)i;
        val += x2i / (i4 * ifact * ifact);
        x2i *= x * x;
        i4 *= 4.0f;
    }
    return val;
}
__device__ __forceinline__ float hair_log_i0(float x) {
    if (x > 12.0f) return x + 0.5f * (-logf(2.0f * RT_PI * x) + 1.0f / (8.0f * x));
    return logf(hair_i0(x));
}
// hair.rs:129-137
__device__ __forceinline__ float hair_mp(float cos_ti, float cos_to, float sin_ti, float sin_to, float v) {
    const float a = cos_ti * cos_to / v, b = sin_ti * sin_to / v;
    if (v <= 0.1f) return expf(hair_log_i0(a) - b - 1.0f / v + 0.6931f + logf(1.0f / (2.0f * v)));
    return expf(-b) * hair_i0(a) / (sinhf(1.0f / v) * 2.0f * v);
}
// hair.rs:139-157
__device__ __forceinline__ float hair_fresnel(float cos_i, float eta_i, float eta_t) {
    cos_i = fminf(fmaxf(cos_i, -1.0f), 1.0f);
    if (cos_i <= 0.0f) {
        const float e = eta_i;
        eta_i = eta_t;
        eta_t = e;
        cos_i = -cos_i;
    }
    const float sin_i = sqrtf(fmaxf(1.0f - cos_i * cos_i, 0.0f));
    const float sin_t = eta_i / eta_t * sin_i;
    if (sin_t >= 1.0f) return 1.0f;
    const float cos_t = sqrtf(fmaxf(1.0f - sin_t * sin_t, 0.0f));
    const float rpa = (eta_t * cos_i - eta_i * cos_t) / (eta_t * cos_i + eta_i * cos_t);
    const float rpe = (eta_i * cos_i - eta_t * cos_t) / (eta_i * cos_i + eta_t * cos_t);
    return 0.5f * (rpa * rpa + rpe * rpe);
}
__device__ __forceinline__ float hair_logistic(float x, float s) {
    x = fabsf(x);
    const float e = expf(-x / s);
    return e / (s * (1.0f + e) * (1.0f + e));
}
__device__ __forceinline__ float hair_logistic_cdf(float x, float s) { return 1.0f / (1.0f + expf(-x / s)); }
__device__ __forceinline__ float hair_trimmed_logistic(float x, float s) {
    return hair_logistic(x, s) / (hair_logistic_cdf(RT_PI, s) - hair_logistic_cdf(-RT_PI, s));
}
__device__ __forceinline__ float hair_phi(int p, float gamma_o, float gamma_t) {
    return 2.0f * p * gamma_t - 2.0f * gamma_o + p * RT_PI;
}
__device__ __forceinline__ float hair_np(float phi, int p, float s, float gamma_o, float gamma_t) {
    float dphi = phi - hair_phi(p, gamma_o, gamma_t);
    // hair.rs:213-218 wraps by 2 pi steps; one remainder is the same angle.
    dphi = remainderf(dphi, 2.0f * RT_PI);
    return hair_trimmed_logistic(dphi, s);
}

// Per-(wo, h) geometry and the lobes' attenuation (hair.rs:160-183, 224-258).
struct HairEval {
    float sin_to, cos_to, phi_o, gamma_o, gamma_t;
    float3 ap[RT_HAIR_PMAX + 1];
    float w[RT_HAIR_PMAX + 1];  // lobe selection weights: luminance of ap, normalised
};
__device__ __forceinline__ void hair_prepare(const DevHair& hp, float3 wo, float h, HairEval& g) {
    g.sin_to = fminf(fmaxf(wo.x, -1.0f), 1.0f);
    g.cos_to = sqrtf(fmaxf(1.0f - g.sin_to * g.sin_to, 0.0f));
    g.phi_o = atan2f(wo.z, wo.y);
    g.gamma_o = asinf(fminf(fmaxf(h, -1.0f), 1.0f));
    const float sin_tt = g.sin_to / hp.eta;
    const float cos_tt = sqrtf(fmaxf(1.0f - sin_tt * sin_tt, 0.0f));
    const float etap = sqrtf(fmaxf(hp.eta * hp.eta - g.sin_to * g.sin_to, 0.0f)) / fmaxf(g.cos_to, 1e-9f);
    const float sin_gt = fminf(fmaxf(h / etap, -1.0f), 1.0f);
    const float cos_gt = sqrtf(fmaxf(1.0f - sin_gt * sin_gt, 0.0f));
    g.gamma_t = asinf(sin_gt);
    const float l = 2.0f * cos_gt / fmaxf(cos_tt, 1e-9f);
    const float3 t = f3(expf(-hp.sigma_a[0] * l), expf(-hp.sigma_a[1] * l), expf(-hp.sigma_a[2] * l));
    const float cos_gamma_o = sqrtf(fmaxf(1.0f - h * h, 0.0f));
    const float f = hair_fresnel(g.cos_to * cos_gamma_o, 1.0f, hp.eta);
    g.ap[0] = f3(f, f, f);
    g.ap[1] = t * ((1.0f - f) * (1.0f - f));
    for (int p = 2; p < RT_HAIR_PMAX; p++) g.ap[p] = g.ap[p - 1] * t * f;
    const float3 last = g.ap[RT_HAIR_PMAX - 1];
    g.ap[RT_HAIR_PMAX] = f3(last.x * f * t.x / fmaxf(1.0f - t.x * f, 1e-6f), last.y * f * t.y / fmaxf(1.0f - t.y * f, 1e-6f),
                            last.z * f * t.z / fmaxf(1.0f - t.z * f, 1e-6f));
    float total = 0.0f;
    for (int p = 0; p <= RT_HAIR_PMAX; p++) total += (g.w[p] = luminance(g.ap[p]));
    for (int p = 0; p <= RT_HAIR_PMAX; p++) g.w[p] = total > 1e-12f ? g.w[p] / total : (p == 0 ? 1.0f : 0.0f);
}

// hair::f and hair::pdf (hair.rs:262-324) for a prepared wo.
__device__ __forceinline__ float3 hair_f_pdf(const DevHair& hp, const HairEval& g, float3 wi, float& pdf) {
    const float sin_ti = fminf(fmaxf(wi.x, -1.0f), 1.0f);
    const float cos_ti = sqrtf(fmaxf(1.0f - sin_ti * sin_ti, 0.0f));
    const float phi = atan2f(wi.z, wi.y) - g.phi_o;
    float3 f = f3(0.0f, 0.0f, 0.0f);
    float pd = 0.0f;
    for (int p = 0; p <= RT_HAIR_PMAX; p++) {
        const float mp = hair_mp(cos_ti, g.cos_to, sin_ti, g.sin_to, hp.v[p]);
        const float np = p < RT_HAIR_PMAX ? hair_np(phi, p, hp.s, g.gamma_o, g.gamma_t) : 1.0f / (2.0f * RT_PI);
        f = f + g.ap[p] * (mp * np);
        pd += g.w[p] * mp * np;
    }
    pdf = fmaxf(pd, 0.0f);
    return f;
}

// hair::sample (hair.rs:327-374): a lobe by attenuation energy, d'Eon's
// longitudinal inverse, a trimmed-logistic azimuth; false when the pdf
// of the direction vanishes.
__device__ __forceinline__ bool hair_sample(const DevHair& hp, const HairEval& g, Pcg& rng, float3& wi, float3& f,
                                            float& pdf) {
    float u = rng.next_f();
    int p = RT_HAIR_PMAX;
    for (int i = 0; i <= RT_HAIR_PMAX; i++) {
        if (u < g.w[i]) {
            p = i;
            break;
        }
        u -= g.w[i];
    }
    const float v = hp.v[p];
    const float u1 = fmaxf(rng.next_f(), 1e-9f), u2 = rng.next_f();
    const float cos_theta = 1.0f + v * logf(u1 + (1.0f - u1) * expf(-2.0f / v));
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    const float sin_ti = -cos_theta * g.sin_to + sin_theta * cosf(2.0f * RT_PI * u2) * g.cos_to;
    const float cos_ti = sqrtf(fmaxf(1.0f - sin_ti * sin_ti, 0.0f));
    const float u3 = rng.next_f();
    float dphi;
    if (p < RT_HAIR_PMAX) {
        const float lo = hair_logistic_cdf(-RT_PI, hp.s), k = hair_logistic_cdf(RT_PI, hp.s) - lo;
        const float x = -hp.s * logf(1.0f / fminf(fmaxf(u3 * k + lo, 1e-9f), 1.0f - 1e-7f) - 1.0f);
        dphi = hair_phi(p, g.gamma_o, g.gamma_t) + fminf(fmaxf(x, -RT_PI), RT_PI);
    } else {
        dphi = 2.0f * RT_PI * u3;
    }
    float sp, cp;
    sincosf(g.phi_o + dphi, &sp, &cp);
    wi = f3(sin_ti, cos_ti * cp, cos_ti * sp);
    f = hair_f_pdf(hp, g, wi, pdf);
    return pdf > 1e-12f;
}

// hair.rs:378-411: the fiber frame at a curve hit and the impact parameter
// h from the (viewer-facing) normal.
struct FiberFrame {
    float3 x, y, z;
    float h;
    __device__ __forceinline__ FiberFrame(float3 tangent, float3 n, float3 wo) {
        x = normalize_ref(tangent);
        float3 zz = wo - x * dot(wo, x);
        if (dot(zz, zz) < 1e-12f) zz = n - x * dot(n, x);
        z = normalize_ref(zz);
        y = normalize_ref(cross(z, x));
        const float3 np = normalize_ref(n - x * dot(n, x));
        h = fminf(fmaxf(dot(np, y), -1.0f), 1.0f);
    }
    __device__ __forceinline__ float3 to_local(float3 w) const { return f3(dot(w, x), dot(w, y), dot(w, z)); }
    __device__ __forceinline__ float3 to_world(float3 w) const { return x * w.x + y * w.y + z * w.z; }
};

}  // namespace rt
