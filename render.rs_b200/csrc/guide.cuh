// guide.cuh — the learned directional proposal (device side).
//
// Network: multiresolution hash-grid encoding of the shading position
// (16 levels x 2 features, 2^19 entries per level, FP16 table; Müller et al.
// 2022, "Instant neural graphics primitives") plus the shading normal and the
// outgoing direction, into an MLP of three hidden layers of 64 (BF16 weights,
// FP32 accumulate, ReLU) whose 40 outputs parameterise a mixture of 8
// von Mises-Fisher lobes (mean direction, concentration, weight).
//
// The reference has no counterpart (path guiding is an unimplemented stretch
// goal in its ROADMAP.md:34); this proposal is MIS-combined with the
// reference's BSDF sampling (one-sample MIS) so the estimator stays
// unbiased whatever the network outputs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "shade.cuh"

namespace rt {

static const int G_LEVELS = 16;
static const int G_FEAT = 2;
static const int G_LOG2_T = 19;
static const uint32_t G_T = 1u << G_LOG2_T;
static const int G_IN = 48;     // 32 hash features + normal(3) + wo(3) + zero pad
static const int G_HID = 64;
static const int G_OUT = 48;    // 40 used: 8 lobes x (mean xyz, kappa, weight)
static const int G_LOBES = 8;
static const int G_NW0 = G_HID * G_IN, G_NW1 = G_HID * G_HID, G_NW2 = G_HID * G_HID, G_NW3 = G_OUT * G_HID;
static const int G_NWEIGHTS = G_NW0 + G_NW1 + G_NW2 + G_NW3;
static const int G_NBIAS = G_HID * 3 + G_OUT;
static const int G_NPARAMS = G_NWEIGHTS + G_NBIAS;  // MLP parameters (table separate)

// Which records of a buffer a training or inference launch processes. With
// `total` null: the launch's own count. Otherwise the count lives in device
// memory and the launch takes slice s of `steps` equal slices of
// min(*total, steps * cap), so a slab's training batches are chosen on the
// device without a host round trip.
struct BatchSel {
    const uint32_t* total;
    uint32_t s, steps;
};

__device__ __forceinline__ uint32_t batch_slice(const BatchSel& b, uint32_t cap, uint32_t& begin) {
    begin = 0;
    if (!b.total) return cap;
    uint64_t t = min((uint64_t)*b.total, (uint64_t)cap * b.steps);
    begin = (uint32_t)(t * b.s / b.steps);
    return (uint32_t)(t * (b.s + 1) / b.steps) - begin;
}

struct GuideDev {
    const __half2* table;     // [levels][T] feature pairs (FP16)
    const __nv_bfloat16* w;   // MLP weights, row-major [out][in], layers concatenated
    const float* b;           // biases
    float res[G_LEVELS];      // grid resolution per level
    float lo[3], inv_ext[3];  // scene bounds -> [0,1]^3
    uint32_t wait_polls;      // polls of a tensor-core pipeline wait before it reports an error
};

// Table slot of a grid vertex. Vertices are stored in 2x2x2 blocks of 8
// consecutive entries (32 bytes, one memory sector), so the 8 corners of a
// cell touch 1 to 8 sectors, 3.4 on average, instead of 8. Blocks are placed
// by the spatial hash of Teschner et al. 2003 (the primes instant-ngp uses),
// or densely on coarse levels whose blocks all fit in the table.
__host__ __device__ __forceinline__ uint32_t grid_blocks(uint32_t res1) { return (res1 + 1u) >> 1; }
__host__ __device__ __forceinline__ bool grid_dense(uint32_t res1) {
    const uint64_t nb = grid_blocks(res1);
    return nb * nb * nb * 8u <= G_T;
}
__device__ __forceinline__ uint32_t grid_index(uint32_t x, uint32_t y, uint32_t z, uint32_t res1, bool dense) {
    const uint32_t intra = (x & 1u) | ((y & 1u) << 1) | ((z & 1u) << 2);
    const uint32_t bx = x >> 1, by = y >> 1, bz = z >> 1, nb = grid_blocks(res1);
    const uint32_t block = dense ? bx + (by + bz * nb) * nb : (bx * 1u ^ by * 2654435761u ^ bz * 805459861u);
    return (block * 8u + intra) & (G_T - 1u);
}

// Encode one position: 32 features (16 levels x 2), trilinear in each level.
__device__ __forceinline__ void hash_encode(const GuideDev& G, float3 pn, float* feat) {
#pragma unroll
    for (int l = 0; l < G_LEVELS; l++) {
        float r = G.res[l];
        uint32_t res1 = (uint32_t)r + 2u;
        bool dense = grid_dense(res1);
        float fx = pn.x * r, fy = pn.y * r, fz = pn.z * r;
        float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
        float tx = fx - ix, ty = fy - iy, tz = fz - iz;
        uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
        float a0 = 0.f, a1 = 0.f;
        const __half2* T = G.table + (size_t)l * G_T;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            uint32_t dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
            float w = (dx ? tx : 1.f - tx) * (dy ? ty : 1.f - ty) * (dz ? tz : 1.f - tz);
            float2 v = __half22float2(T[grid_index(x0 + dx, y0 + dy, z0 + dz, res1, dense)]);
            a0 += w * v.x;
            a1 += w * v.y;
        }
        feat[2 * l] = a0;
        feat[2 * l + 1] = a1;
    }
}

__device__ __forceinline__ float3 guide_normalize_pos(const GuideDev& G, float3 p) {
    float3 q = f3((p.x - G.lo[0]) * G.inv_ext[0], (p.y - G.lo[1]) * G.inv_ext[1], (p.z - G.lo[2]) * G.inv_ext[2]);
    return f3(fminf(fmaxf(q.x, 0.f), 1.f), fminf(fmaxf(q.y, 0.f), 1.f), fminf(fmaxf(q.z, 0.f), 1.f));
}

// ---- von Mises-Fisher mixture ----------------------------------------------------
// Raw outputs per lobe j: o[5j..5j+2] mean (unnormalised), o[5j+3] log kappa,
// o[5j+4] weight logit. kappa = exp(clamp(., -4, 9)); weights = softmax.
// The renderer reads the mixture in decoded form (48 floats, written by the
// forward pass): lobe j's (mu.xyz, kappa) at [4j, 4j+4), its weight at
// [32 + j] and at [40 + j] the log of its weighted density at mu.w = 0,
// A_j = log w_j + log(kappa_j / (2 pi (1 - e^{-2 kappa_j}))) - kappa_j, so that
// q(w) = sum_j exp(A_j + kappa_j mu_j.w).
//
// Raw outputs -> the decoded record (48 floats, layout above), stored as
// it is computed so few values stay live. The logarithms are taken where
// they are cheap: log w_j = (o_j - max) - log(sum of e^(o_i - max)), one
// logarithm for the whole softmax, and log kappa_j is the clamped output
// itself. log(1 - e^{-2 kappa}) uses the fast intrinsics: 1 - e^{-2 kappa}
// >= 1 - e^{-2 e^-4} = 0.036, so its absolute error stays near 1e-6, a
// relative 1e-6 on the density. Means are normalised with rsqrt (relative
// error below 2^-22).
__device__ __forceinline__ void mixture_decode_store(const float* o, float* dst) {
    float4* d4 = reinterpret_cast<float4*>(dst);
    float mx = -1e30f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) mx = fmaxf(mx, o[5 * j + 4]);
    float e[G_LOBES], k[G_LOBES], sw = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        const float3 v = f3(o[5 * j], o[5 * j + 1], o[5 * j + 2]);
        const float len2 = dot(v, v);
        const float3 mu = len2 > 1e-16f ? v * rsqrtf(len2) : f3(0.f, 0.f, 1.f);
        k[j] = __expf(fminf(fmaxf(o[5 * j + 3], -4.f), 9.f));
        d4[j] = make_float4(mu.x, mu.y, mu.z, k[j]);
        e[j] = __expf(o[5 * j + 4] - mx);
        sw += e[j];
    }
    const float inv_sw = __frcp_rn(sw), log_sw = __logf(sw);
    const float log_2pi = 1.8378770664093453f;
    float A[G_LOBES];
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        e[j] *= inv_sw;
        const float log_k = fminf(fmaxf(o[5 * j + 3], -4.f), 9.f);
        A[j] = (o[5 * j + 4] - mx) - log_sw + log_k - log_2pi - __logf(1.f - __expf(-2.f * k[j])) - k[j];
    }
    d4[8] = make_float4(e[0], e[1], e[2], e[3]);
    d4[9] = make_float4(e[4], e[5], e[6], e[7]);
    d4[10] = make_float4(A[0], A[1], A[2], A[3]);
    d4[11] = make_float4(A[4], A[5], A[6], A[7]);
}

// log of the vMF density kappa / (2 pi (1 - e^{-2 kappa})) exp(kappa (mu.w - 1)).
__device__ __forceinline__ float vmf_log_pdf(float3 mu, float kappa, float3 w) {
    float norm = logf(kappa) - logf(2.f * RT_PI) - log1pf(-__expf(-2.f * kappa));
    return norm + kappa * (dot(mu, w) - 1.f);
}

// The renderer's view of a decoded mixture: read in place from its record
// (global memory, L1-resident after the first touch) instead of copying its
// 48 floats into per-thread storage, which spilled to local memory and held
// registers through the whole shade.
struct MixtureRef {
    const float4* p;  // 12 float4: 8 x (mu.xyz, kappa), weights (2), A (2)
};

__device__ __forceinline__ float mixture_pdf(const MixtureRef& m, float3 w) {
    const float4 a0 = m.p[10], a1 = m.p[11];
    const float A[G_LOBES] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    float p = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        const float4 l = m.p[j];
        p += __expf(A[j] + l.w * dot(f3(l.x, l.y, l.z), w));
    }
    return p;
}

// Sample: pick a lobe by weight, then a direction around its mean
// (W. Jakob, "Numerically stable sampling of the von Mises-Fisher
// distribution on S^2", 2012).
__device__ __forceinline__ float3 mixture_sample(const MixtureRef& m, float u0, float u1, float u2) {
    const float4 w0 = m.p[8], w1 = m.p[9];
    const float wt[G_LOBES] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    int j = G_LOBES - 1;
    float acc = 0.f;
#pragma unroll
    for (int k = 0; k < G_LOBES; k++) {
        acc += wt[k];
        if (u0 < acc) {
            j = k;
            break;
        }
    }
    const float4 l = m.p[j];
    const float kappa = l.w;
    const float3 mu = f3(l.x, l.y, l.z);
    float wz = 1.f + logf(u1 + (1.f - u1) * __expf(-2.f * kappa)) / kappa;
    wz = fminf(fmaxf(wz, -1.f), 1.f);
    float sr = sqrtf(fmaxf(1.f - wz * wz, 0.f)), s, c;
    sincosf(2.f * RT_PI * u2, &s, &c);
    float3 t = fabsf(mu.x) > 0.9f ? f3(0, 1, 0) : f3(1, 0, 0);
    float3 a = normalize_ref(cross(mu, t)), b = cross(mu, a);
    return normalize_ref(a * (sr * c) + b * (sr * s) + mu * wz);
}

// Loss -weight * log q(w) for raw outputs o; writes d loss / d o into g (40 used).
__device__ __forceinline__ float mixture_loss_grad(const float* o, float3 w, float weight, float* g) {
    float mx = -1e30f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) mx = fmaxf(mx, o[5 * j + 4]);
    float pi[G_LOBES], lv[G_LOBES], kap[G_LOBES], len[G_LOBES], dmw[G_LOBES];
    float3 mu[G_LOBES];
    float sw = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        float3 v = f3(o[5 * j], o[5 * j + 1], o[5 * j + 2]);
        len[j] = fmaxf(length(v), 1e-8f);
        mu[j] = v / len[j];
        float lk = fminf(fmaxf(o[5 * j + 3], -4.f), 9.f);
        kap[j] = __expf(lk);
        pi[j] = __expf(o[5 * j + 4] - mx);
        sw += pi[j];
        dmw[j] = dot(mu[j], w);
    }
    float lmax = -1e30f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        pi[j] /= sw;
        lv[j] = logf(fmaxf(pi[j], 1e-30f)) + vmf_log_pdf(mu[j], kap[j], w);
        lmax = fmaxf(lmax, lv[j]);
    }
    float s = 0.f;
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) s += __expf(lv[j] - lmax);
    float logq = lmax + logf(s);
#pragma unroll
    for (int j = 0; j < G_LOBES; j++) {
        float r = __expf(lv[j] - logq);   // responsibility
        float k = kap[j];
        // d log vmf / d kappa = 1/kappa + (mu.w - 1) - 2 / (e^{2 kappa} - 1)
        float dlk = 1.f / k + (dmw[j] - 1.f) - 2.f / fmaxf(__expf(2.f * k) - 1.f, 1e-30f);
        float lk = o[5 * j + 3];
        float dk = (lk > -4.f && lk < 9.f) ? -weight * r * dlk * k : 0.f;
        float3 gm = (w - mu[j] * dmw[j]) * (-weight * r * k / len[j]);
        g[5 * j] = gm.x;
        g[5 * j + 1] = gm.y;
        g[5 * j + 2] = gm.z;
        g[5 * j + 3] = dk;
        g[5 * j + 4] = -weight * (r - pi[j]);
    }
#pragma unroll
    for (int j = 5 * G_LOBES; j < G_OUT; j++) g[j] = 0.f;
    return -weight * logq;
}

}  // namespace rt
