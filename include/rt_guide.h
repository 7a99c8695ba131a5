/*
 * rt_guide.h — the learned directional proposal of librtcuda.so.
 *
 * A hash-grid + MLP network (16 levels x 2 features, 2^19 FP16 entries per
 * level; 3 hidden layers of 64, BF16 weights, FP32 accumulation on the
 * tcgen05 tensor cores) maps a shading point (position, normal, outgoing
 * direction) to a mixture of 8 von Mises-Fisher lobes over incident
 * directions. It is trained online with Adam on the path tracer's own
 * radiance samples and used by rt_render_samples when params.guided = 1,
 * one-sample-MIS'd against BSDF sampling.
 *
 * The reference has no counterpart: path guiding is listed as an
 * unimplemented stretch goal (ROADMAP.md:34). These entry points exist so
 * the network can be trained, inspected and gradient-checked on its own.
 *
 * Training record (16 floats): position xyz, normal xyz, outgoing
 * direction wo xyz, sampled incident direction wi xyz, weight
 * (lum(f cos Li) / pdf), 3 unused. Raw network output (48 floats): for
 * lobe j = 0..7, [5j..5j+2] mean (unnormalised), [5j+3] log concentration,
 * [5j+4] weight logit; [40..47] unused.
 * Status codes as rt_cuda.h.
 */
#ifndef RT_GUIDE_H
#define RT_GUIDE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rt_guide rt_guide;

#define RT_GUIDE_LEVELS 16
#define RT_GUIDE_TABLE_ENTRIES (1u << 19)
#define RT_GUIDE_MLP_PARAMS (64 * 48 + 64 * 64 + 64 * 64 + 48 * 64 + 64 * 3 + 48)
#define RT_GUIDE_RECORD_FLOATS 16
#define RT_GUIDE_OUTPUTS 48

/* New network for positions inside [lo, hi]; Adam learning rate `lr`. */
int rt_guide_create(const float* lo, const float* hi, uint64_t seed, float lr, rt_guide** out);
int rt_guide_destroy(rt_guide* g);
const char* rt_guide_last_error(void);

/* One training iteration (forward, backward, Adam) on n records.
 * `_device`: records in device memory, enqueued on `stream`; loss_out
 * (host, may be NULL) receives the summed loss and forces a sync. */
int rt_guide_train_step(rt_guide* g, const float* records, uint32_t n, float* loss_out);
int rt_guide_train_step_device(rt_guide* g, const float* records, uint32_t n, float* loss_out, void* stream);

/* Raw outputs for n records (only position, normal and wo are read). */
int rt_guide_infer(rt_guide* g, const float* records, uint32_t n, float* raw_out);
int rt_guide_infer_device(rt_guide* g, const float* records, uint32_t n, float* raw_out, void* stream);

/* The decoded mixture the renderer samples from, for n records (host
 * pointers), 48 floats per record: lobe j's (mu.xyz, kappa) at [4j, 4j+4),
 * its weight at [32 + j] and at [40 + j] the log of its weighted density at
 * mu.w = 0, A_j = log w_j + log(kappa_j / (2 pi (1 - e^{-2 kappa_j}))) -
 * kappa_j, so that q(w) = sum_j exp(A_j + kappa_j mu_j.w). */
int rt_guide_infer_mixture(rt_guide* g, const float* records, uint32_t n, float* mixture_out);

/* Gradients of the summed loss without updating (host pointers):
 * g_mlp: RT_GUIDE_MLP_PARAMS floats (weights row-major [out][in] per layer,
 * then biases); g_table: RT_GUIDE_LEVELS * RT_GUIDE_TABLE_ENTRIES * 2 floats
 * or NULL; raw_out: n * 48 floats or NULL. */
int rt_guide_grads(rt_guide* g, const float* records, uint32_t n, float* g_mlp, float* g_table, float* raw_out,
                   float* loss);

/* Parameter access (MLP as f32, table as IEEE fp16 bit patterns). */
int rt_guide_get_params(rt_guide* g, float* mlp, uint16_t* table_fp16);
int rt_guide_set_params(rt_guide* g, const float* mlp, const uint16_t* table_fp16);
/* Grid resolution per level and the position normalisation. */
int rt_guide_info(rt_guide* g, float* res16, float* lo3, float* inv_extent3);

/* Diagnostic: D[128][N] = A[128][K] * B[N][K]^T on one CTA's tcgen05 path
 * (bf16 bit patterns in, f32 out). N, K multiples of 16. */
int rt_tc_gemm_selftest(const uint16_t* A, const uint16_t* B, int N, int K, float* D);

#ifdef __cplusplus
}
#endif

#endif /* RT_GUIDE_H */
