// media.cuh — participating media and subsurface walks on the device, f32.
//
// Restates src/scene/medium.rs (density field, Henyey-Greenstein phase)
// and src/raytracer/pt/volume.rs (spectral one-sample distance sampling in
// homogeneous media, weighted delta tracking and ratio tracking against the
// channel-max majorant in fBm media, equiangular sampling toward point
// lights) for the wavefront kernels, plus the per-path stack of nested
// media (src/raytracer/pt/mod.rs:34-67) packed into 64 bits.
#pragma once

#include "pattern.cuh"

namespace rt {

#define RT_MEDIUM_NONE 0xFFFFFFFFu
// Tracking loops stop after this many tentative collisions (volume.rs:123,
// 177 bound theirs the same way); a loop that reaches it keeps its weight.
#define RT_MEDIUM_STEPS 10000

__device__ __forceinline__ float3 med_sigma_t(const DevMedium& m) {
    return f3(m.sigma_a[0] + m.sigma_s[0], m.sigma_a[1] + m.sigma_s[1], m.sigma_a[2] + m.sigma_s[2]);
}
__device__ __forceinline__ float3 med_sigma_s(const DevMedium& m) { return f3(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]); }
__device__ __forceinline__ float comp3(float3 v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }
__device__ __forceinline__ float3 exp3f(float3 st, float t) { return f3(expf(-st.x * t), expf(-st.y * t), expf(-st.z * t)); }

// Medium::density_at (medium.rs:57-66): fBm of displace.rs:82-97 (amplitude
// 1, offset 0) remapped by coverage and sharpness.
__device__ __forceinline__ float med_density(const DevMedium& m, float3 p) {
    if (m.density != RT_DENSITY_FBM) return 1.0f;
    float sum = 0.0f, amp = 1.0f, freq = m.frequency;
    const uint32_t oct = m.octaves > 1u ? m.octaves : 1u;
    for (uint32_t o = 0; o < oct; o++) {
        sum += amp * perlin(p.x * freq, p.y * freq, p.z * freq);
        amp *= m.gain;
        freq *= m.lacunarity;
    }
    return fminf(fmaxf((sum * 0.5f + 0.5f - (1.0f - m.coverage)) * m.sharpness, 0.0f), 1.0f);
}

// medium.rs:73-76.
__device__ __forceinline__ float hg_phase(float g, float cos_theta) {
    const float denom = 1.0f + g * g + 2.0f * g * cos_theta;
    return (1.0f - g * g) / (4.0f * RT_PI * denom * sqrtf(fmaxf(denom, 1e-9f)));
}

// medium.rs:80-103: a direction around the propagation direction -wo; the
// pdf is the phase of the direction.
__device__ __forceinline__ float3 hg_sample(float g, float3 wo, float u1, float u2, float& pdf) {
    float cos_theta;
    if (fabsf(g) < 1e-3f) {
        cos_theta = 1.0f - 2.0f * u1;
    } else {
        const float sq = (1.0f - g * g) / (1.0f + g - 2.0f * g * u1);
        cos_theta = -(1.0f + g * g - sq * sq) / (2.0f * g);
    }
    const float sin_theta = sqrtf(fmaxf(1.0f - cos_theta * cos_theta, 0.0f));
    float sp, cp;
    sincosf(2.0f * RT_PI * u2, &sp, &cp);
    const float3 w = -wo;
    const float3 a = fabsf(w.x) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(1.0f, 0.0f, 0.0f);
    const float3 t = normalize_ref(cross(w, a));
    const float3 b = cross(w, t);
    const float3 wi = normalize_ref(t * (sin_theta * cp) + b * (sin_theta * sp) + w * cos_theta);
    pdf = hg_phase(g, -dot(wo, wi));
    return wi;
}

// Scatter at t (weight = transmittance x sigma_s / pdf) or pass the segment
// (weight = transmittance / pass probability): volume.rs:11-20.
struct MedEvent {
    bool scatter;
    float t;
    float3 w;
};

// volume.rs:51-105: homogeneous extinction st, scattering ss; the sampling
// channel is picked in proportion to the path throughput.
__device__ __forceinline__ MedEvent homog_sample(float3 st, float3 ss, float t_max, float3 beta, Pcg& rng) {
    MedEvent ev{false, 0.0f, f3(1.0f, 1.0f, 1.0f)};
    if ((st.x + st.y + st.z) * (1.0f / 3.0f) <= 1e-9f) return ev;
    const float3 b = f3(fmaxf(beta.x, 0.0f), fmaxf(beta.y, 0.0f), fmaxf(beta.z, 0.0f));
    const float total = b.x + b.y + b.z;
    const float3 w = total > 1e-12f ? b / total : f3(1.0f / 3.0f, 1.0f / 3.0f, 1.0f / 3.0f);
    const float u = rng.next_f();
    const int c = u < w.x ? 0 : (u < w.x + w.y ? 1 : 2);
    const float sigma_c = fmaxf(comp3(st, c), 1e-9f);
    const float t = -logf(fmaxf(1.0f - rng.next_f(), 1e-12f)) / sigma_c;
    if (t < t_max) {
        const float3 tr = exp3f(st, t);
        const float pdf = w.x * st.x * tr.x + w.y * st.y * tr.y + w.z * st.z * tr.z;
        if (pdf <= 1e-30f) {
            ev.w = f3(0.0f, 0.0f, 0.0f);
            return ev;
        }
        ev.scatter = true;
        ev.t = t;
        ev.w = ss * tr / pdf;
        return ev;
    }
    const float3 tr = exp3f(st, t_max);
    const float pdf = w.x * tr.x + w.y * tr.y + w.z * tr.z;
    ev.w = pdf > 1e-30f ? tr / pdf : f3(0.0f, 0.0f, 0.0f);
    return ev;
}

// volume.rs:35-49 and 109-156: distance sampling along the unit-direction
// ray (o, d) over [0, t_max] clamped to the medium's extent.
__device__ __forceinline__ MedEvent med_sample(const DevMedium& m, float3 o, float3 d, float t_max, float3 beta,
                                               Pcg& rng) {
    t_max = fminf(t_max, m.max_distance);
    const float3 st = med_sigma_t(m), ss = med_sigma_s(m);
    if (m.density != RT_DENSITY_FBM) return homog_sample(st, ss, t_max, beta, rng);
    MedEvent ev{false, 0.0f, f3(1.0f, 1.0f, 1.0f)};
    const float maj = m.majorant;
    if (maj <= 1e-9f) return ev;
    float t = 0.0f;
    float3 weight = f3(1.0f, 1.0f, 1.0f);
    for (int i = 0; i < RT_MEDIUM_STEPS; i++) {
        t -= logf(fmaxf(1.0f - rng.next_f(), 1e-12f)) / maj;
        if (t >= t_max) break;
        const float rho = med_density(m, o + d * t);
        const float3 sh = st * rho;
        const float p_real = fminf(fmaxf((sh.x + sh.y + sh.z) * (1.0f / 3.0f) / maj, 0.0f), 1.0f);
        if (rng.next_f() < p_real) {
            ev.scatter = true;
            ev.t = t;
            ev.w = weight * (ss * rho) / (maj * p_real);
            return ev;
        }
        const float p_null = fmaxf(1.0f - p_real, 1e-9f);
        weight = weight * f3((1.0f - sh.x / maj) / p_null, (1.0f - sh.y / maj) / p_null, (1.0f - sh.z / maj) / p_null);
        if (maxc(weight) < 1e-6f) {
            ev.w = f3(0.0f, 0.0f, 0.0f);
            return ev;
        }
    }
    ev.w = weight;
    return ev;
}

// volume.rs:160-193: transmittance of one segment, closed form or ratio
// tracking.
__device__ __forceinline__ float3 med_transmittance(const DevMedium& m, float3 o, float3 d, float dist, Pcg& rng) {
    dist = fminf(dist, m.max_distance);
    const float3 st = med_sigma_t(m);
    if (m.density != RT_DENSITY_FBM) return exp3f(st, dist);
    const float maj = m.majorant;
    if (maj <= 1e-9f) return f3(1.0f, 1.0f, 1.0f);
    float t = 0.0f;
    float3 tr = f3(1.0f, 1.0f, 1.0f);
    for (int i = 0; i < RT_MEDIUM_STEPS; i++) {
        t -= logf(fmaxf(1.0f - rng.next_f(), 1e-12f)) / maj;
        if (t >= dist) break;
        const float rho = med_density(m, o + d * t) / maj;
        tr = tr * f3(1.0f - st.x * rho, 1.0f - st.y * rho, 1.0f - st.z * rho);
        if (maxc(tr) < 1e-5f) return f3(0.0f, 0.0f, 0.0f);
    }
    return tr;
}

// volume.rs:199-235 (Kulla-Fajardo equiangular sampling) and 240-249.
__device__ __forceinline__ float equiangular_pdf(float3 o, float3 d, float t_max, float3 lp, float t) {
    const float delta = dot(lp - o, d);
    const float h = fmaxf(length(lp - (o + d * delta)), 1e-6f);
    const float span = fmaxf(atanf((t_max - delta) / h) - atanf(-delta / h), 1e-9f);
    return h / (span * (h * h + (t - delta) * (t - delta)));
}
__device__ __forceinline__ float equiangular_sample(float3 o, float3 d, float t_max, float3 lp, float u, float& pdf) {
    const float delta = dot(lp - o, d);
    const float h = fmaxf(length(lp - (o + d * delta)), 1e-6f);
    const float ta = atanf(-delta / h);
    const float span = fmaxf(atanf((t_max - delta) / h) - ta, 1e-9f);
    const float t = fminf(fmaxf(delta + h * tanf(ta + u * span), 0.0f), t_max);
    pdf = h / (span * (h * h + (t - delta) * (t - delta)));
    return t;
}
__device__ __forceinline__ float distance_pdf_approx(const DevMedium& m, float t, float t_max) {
    const float3 st = med_sigma_t(m);
    const float s = fmaxf((st.x + st.y + st.z) * (1.0f / 3.0f), 1e-9f);
    return t < t_max ? s * expf(-s * t) : expf(-s * t_max);
}

// ---- nested media (pt/mod.rs:34-67) --------------------------------------------
// A path's stack in a uint2: bits 0-3 of x the depth (0..8), then eight
// 7-bit medium indices, four in x (bits 4..31) and four in y (bits 0..27).
// The atmosphere is the implicit bottom; pushes beyond 8 are dropped and
// pops below 0 ignored, as the reference's fixed array does.
__device__ __forceinline__ uint32_t mstack_depth(uint2 s) { return s.x & 15u; }
__device__ __forceinline__ uint32_t mstack_entry(uint2 s, uint32_t i) {
    return i < 4u ? (s.x >> (4u + 7u * i)) & 127u : (s.y >> (7u * (i - 4u))) & 127u;
}
__device__ __forceinline__ uint32_t mstack_top(uint2 s, uint32_t atmosphere) {
    const uint32_t dp = mstack_depth(s);
    return dp ? mstack_entry(s, dp - 1u) : atmosphere;
}
__device__ __forceinline__ void mstack_push(uint2& s, uint32_t m) {
    const uint32_t dp = mstack_depth(s);
    if (dp >= 8u) return;
    if (dp < 4u) {
        const uint32_t sh = 4u + 7u * dp;
        s.x = (s.x & ~(127u << sh)) | ((m & 127u) << sh);
    } else {
        const uint32_t sh = 7u * (dp - 4u);
        s.y = (s.y & ~(127u << sh)) | ((m & 127u) << sh);
    }
    s.x = (s.x & ~15u) | (dp + 1u);
}
__device__ __forceinline__ void mstack_pop(uint2& s) {
    const uint32_t dp = mstack_depth(s);
    if (dp) s.x = (s.x & ~15u) | (dp - 1u);
}

// ---- per-thread closest hit -------------------------------------------------------
// One ray walked to its closest hit by a single thread (quadrics first, then
// the BVH below the closest quadric), for the sequential loops of subsurface
// walks and medium-aware shadow rays. d must be unit length: t is the
// distance; `time` is the path's shutter time (read with MOT, scenes with
// motion blur). Returns the hit record in the layout k_extend writes.
template <bool MOT = false>
__device__ __forceinline__ bool trace_closest(const DevScene& S, TravStack& st, float3 o, float3 d, float tmax,
                                              uint32_t* err, uint4& hr, float time = 0.0f) {
    float tq = tmax;
    const uint32_t qk = S.n_quadrics ? quadrics_closest(S, o, d, tmax, tq) : 0xFFFFFFFFu;
    if (qk != 0xFFFFFFFFu) tmax = tq;
    PhaseState ps;
    bool found = false;
    if (trav_begin(S, ps.ts, st, o, d, tmax, MOT ? time : 0.0f)) {
        phase_begin(ps);
        for (;;) {
            if (++ps.ts.steps > S.max_steps) {
                atomicOr(err, RT_DEVERR_ITER);
                break;
            }
            if (ps.pending) {
                if (op_leaf<false, MOT>(S, ps, st, err)) break;
            } else if (ps.need_pop) {
                if (!op_pop(ps, st)) break;
            } else if (op_node<false>(S, ps, st, err)) {
                break;
            }
        }
        found = ps.ts.found;
    }
    if (found) {
        const TraceHit& h = ps.ts.hit;
        const uint32_t uv = (uint32_t)__half_as_ushort(__float2half_rn(h.b1)) |
                            ((uint32_t)__half_as_ushort(__float2half_rn(h.b2)) << 16);
        hr = make_uint4(__float_as_uint(h.t), h.tri, h.inst, uv);
        return true;
    }
    if (qk != 0xFFFFFFFFu) {
        hr = make_uint4(__float_as_uint(tq), RT_TRI_QUADRIC | qk, 0xFFFFFFFFu, 0u);
        return true;
    }
    return false;
}

}  // namespace rt
