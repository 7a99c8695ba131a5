// guide.cu — training and inference of the learned directional proposal.
//
// Kernels (one training iteration = encode -> forward -> backward -> hash
// backward -> Adam; inference = encode -> forward):
//   k_guide_encode    hash-grid features (+ normal, wo) -> X0 rows, bf16
//   k_guide_fwd       tcgen05 MLP forward, 128-row tiles in six independent
//                     pipelines of one persistent CTA per SM, weights resident
//                     in shared memory,
//                     accumulators in TMEM; stores activations (training) and
//                     the 48 raw outputs, or the decoded mixture when rendering
//   k_guide_bwd       vMF-mixture loss gradient in registers, then per layer
//                     two tcgen05 GEMMs: dW = dZ^T H (batch is the K dimension)
//                     and dH = dZ W; each CTA sums dW/db of its tiles into its
//                     own f32 row, k_guide_grad_reduce adds the rows in order
//   k_guide_hash_bwd  scatter-add of d loss / d features into the table
//                     gradient, in 2^-24 fixed point (integer sums do not
//                     depend on the order the atomics land in)
//   k_guide_adam      Adam on the f32 masters, refreshing the bf16 / fp16 copies
//                     (lazy on the hash table: entries without gradient skip)
// Loss: -w * log q(wi | x) with w = lum(f cos Li) / p_sample, the
// importance-weighted KL objective of neural importance sampling
// (Müller et al. 2019), estimated from the path tracer's own vertices.
// Training is deterministic: no gradient is summed by float atomics, so a
// render with the same seed trains the same network bit for bit.

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "guide.cuh"
#include "rt_guide.h"
#include "tc_mma.cuh"

using namespace rt;

namespace {

thread_local std::string g_gerr;

int gfail(int code, const std::string& m) {
    g_gerr = m;
    return code;
}

#define G_TRY(expr)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess) return gfail(-2, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int TILE = 128;
constexpr uint32_t GERR_WAIT = 1u;

// Weight offsets (row-major [out][in]) and bias offsets per layer.
__host__ __device__ constexpr int w_off(int l) {
    return l == 0 ? 0 : l == 1 ? G_NW0 : l == 2 ? G_NW0 + G_NW1 : G_NW0 + G_NW1 + G_NW2;
}
__host__ __device__ constexpr int b_off(int l) { return l * G_HID; }
__host__ __device__ constexpr int l_in(int l) { return l == 0 ? G_IN : G_HID; }
__host__ __device__ constexpr int l_out(int l) { return l == 3 ? G_OUT : G_HID; }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&v);
}
// The same with ReLU folded into the conversion (a in the low half, as
// above): rounding keeps the sign, so this equals pack_bf16(max(a, 0), max(b, 0)).
__device__ __forceinline__ uint32_t pack_bf16_relu(float a, float b) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(b), "f"(a));
    return r;
}

// Copy a row-major [R][K] bf16 matrix into the core-matrix layout.
__device__ void stage_matrix(uint8_t* dst, const __nv_bfloat16* src, int R, int K) {
    int chunks = R * (K / 8);
    for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
        int r = c / (K / 8), kc = c % (K / 8);
        uint4 v = *reinterpret_cast<const uint4*>(src + (size_t)r * K + kc * 8);
        *reinterpret_cast<uint4*>(dst + core_offset(r, kc * 8, K)) = v;
    }
}
// Copy the transpose of a row-major [R][K] bf16 matrix (i.e. a [K][R] operand).
__device__ void stage_transpose(uint8_t* dst, const __nv_bfloat16* src, int R, int K) {
    for (int i = threadIdx.x; i < R * K; i += blockDim.x) {
        int r = i / K, k = i % K;
        *reinterpret_cast<__nv_bfloat16*>(dst + core_offset(k, r, R)) = src[i];
    }
}

}  // namespace

// ---- encode -------------------------------------------------------------------
// rec: 16 floats per record (pos xyz, normal xyz, wo xyz, wi xyz, weight, -).
// One record -> 48 network inputs (32 hash-grid features, normal, wo, zeros).
__device__ __forceinline__ void encode_record(const GuideDev& G, const float* r, float* feat) {
    hash_encode(G, guide_normalize_pos(G, f3(r[0], r[1], r[2])), feat);
#pragma unroll
    for (int k = 0; k < 6; k++) feat[32 + k] = r[3 + k];
#pragma unroll
    for (int k = 38; k < G_IN; k++) feat[k] = 0.f;
}

// Encoding runs as its own kernel at full occupancy: its cost is the 128
// scattered table reads per record, which need many threads in flight (inside
// the 128-thread forward CTAs they ran 1.7x slower than here). The grid is
// sized for the record capacity but at most ENCODE_CTAS_PER_SM per SM, and
// strides over the records: a launch whose count (read on the device) is
// small then ends in a few microseconds instead of retiring one CTA per 256
// records of capacity.
constexpr uint32_t ENCODE_CTAS_PER_SM = 8;
__global__ void __launch_bounds__(256) k_guide_encode(GuideDev G, const float* __restrict__ rec, uint32_t n,
                                                      BatchSel B, __nv_bfloat16* X0) {
    uint32_t begin;
    n = batch_slice(B, n, begin);
    rec += 16 * (size_t)begin;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float feat[G_IN];
        encode_record(G, rec + 16 * (size_t)i, feat);
        uint4* out = reinterpret_cast<uint4*>(X0 + (size_t)i * G_IN);
#pragma unroll
        for (int c = 0; c < G_IN / 8; c++)
            out[c] = make_uint4(pack_bf16(feat[8 * c], feat[8 * c + 1]), pack_bf16(feat[8 * c + 2], feat[8 * c + 3]),
                                pack_bf16(feat[8 * c + 4], feat[8 * c + 5]),
                                pack_bf16(feat[8 * c + 6], feat[8 * c + 7]));
    }
}

// ---- forward ------------------------------------------------------------------
// One persistent CTA per SM runs FWD_GROUPS independent 128-row tile
// pipelines (one per 128 threads, one warpgroup) that share the weights in
// shared memory; a pipeline's layers are latency-bound (MMA -> commit -> TMEM
// load -> epilogue), so six tiles in flight per SM hide each other's waits.
// (Three CTAs of two pipelines each held the same work, but the weights three
// times, and in some launches ran one CTA per SM at a time.) A tile keeps
// one activation buffer: X (K = 48), then H1, H2, H3 (K = 64) overwrite it in
// turn, which is safe because a layer's MMA has finished reading its input
// when the epilogue runs.
// Shared memory: W0 6144 | W1 8192 | W2 8192 | W3 6144 | ACT 16384 per group.
// TMEM: 64 columns per group, allocated as the next power of two.
constexpr int FWD_GROUPS = 6, FWD_THREADS = FWD_GROUPS * TILE;
constexpr uint32_t FWD_TMEM_COLS = 512;
static_assert(64 * FWD_GROUPS <= FWD_TMEM_COLS && FWD_GROUPS <= 7, "forward: TMEM columns and named barriers");
constexpr int F_W0 = 0, F_W1 = 6144, F_W2 = F_W1 + 8192, F_W3 = F_W2 + 8192, F_ACT = F_W3 + 6144,
              F_BYTES = F_ACT + FWD_GROUPS * 16384;

// Modes: raw outputs (inference API), training (raw outputs + the hidden
// activations the backward pass reads), rendering (the decoded mixture of
// guide.cuh, 48 floats).
enum { FWD_RAW = 0, FWD_TRAIN = 1, FWD_RENDER = 2 };

template <int MODE>
__global__ void __launch_bounds__(FWD_THREADS, 1) k_guide_fwd(GuideDev G, const __nv_bfloat16* __restrict__ X0,
                                                              uint32_t n, BatchSel B, __nv_bfloat16* acts,
                                                              float* out, uint32_t* err) {
    constexpr bool TRAIN = MODE == FWD_TRAIN;
    uint32_t begin;
    n = batch_slice(B, n, begin);
    if ((uint64_t)blockIdx.x * TILE >= n) return;  // no tile for this CTA: skip the weight staging
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t mbar[FWD_GROUPS];
    __shared__ uint32_t tmem_base;
    __shared__ uint32_t group_failed[FWD_GROUPS];
    __shared__ __align__(16) float bias[G_NBIAS];
    const int tid = threadIdx.x, warp = tid >> 5, grp = tid / TILE, gt = tid % TILE;
    stage_matrix(sm + F_W0, G.w + w_off(0), G_HID, G_IN);
    stage_matrix(sm + F_W1, G.w + w_off(1), G_HID, G_HID);
    stage_matrix(sm + F_W2, G.w + w_off(2), G_HID, G_HID);
    stage_matrix(sm + F_W3, G.w + w_off(3), G_OUT, G_HID);
    for (int i = tid; i < G_NBIAS; i += FWD_THREADS) bias[i] = G.b[i];
    if (warp == 0) tmem_alloc(&tmem_base, FWD_TMEM_COLS);
    if (tid < FWD_GROUPS) {
        mbar_init(&mbar[tid], 1);
        group_failed[tid] = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // Group grp owns TMEM columns [64 grp, 64 grp + 64); warp w reads lanes 32 (w % 4) ...
    const uint32_t acc = tmem_base + 64u * grp;
    const uint32_t lane_addr = acc + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t s0 = smem_u32(sm);
    const uint32_t act = F_ACT + 16384u * grp;
    uint32_t phase = 0;
    // Tiles go to the CTAs first, then to their pipelines (tile = grp x grid +
    // CTA), so a launch of fewer tiles than pipelines still spreads over
    // every SM.
    for (uint32_t tile = grp * gridDim.x + blockIdx.x; tile * TILE < n; tile += gridDim.x * FWD_GROUPS) {
        uint32_t row = tile * TILE + gt;
        bool valid = row < n;
        const uint4* xr = reinterpret_cast<const uint4*>(X0 + (size_t)row * G_IN);
#pragma unroll
        for (int c = 0; c < G_IN / 8; c++)
            *reinterpret_cast<uint4*>(sm + act + core_offset(gt, 8 * c, G_IN)) = valid ? xr[c] : make_uint4(0, 0, 0, 0);
        bool failed = false;
        for (int l = 0; l < 4; l++) {
            const int K = l_in(l), N = l_out(l);
            const uint32_t w_sm = l == 0 ? F_W0 : l == 1 ? F_W1 : l == 2 ? F_W2 : F_W3;
            fence_proxy_async_smem();
            group_sync(grp);
            if (gt == 0) {
                tc_fence_after();
                tc_gemm_issue(acc, s0 + act, s0 + w_sm, N, K, false);
                tc_commit(&mbar[grp]);
            }
            if (!mbar_wait_or_drain(&mbar[grp], phase, G.wait_polls)) group_failed[grp] = 1;
            phase ^= 1u;
            group_sync(grp);
            if (group_failed[grp]) {
                failed = true;
                break;
            }
            tc_fence_after();
            if (l < 3) {
                // Hidden layer: bias, ReLU, bf16 into the activation buffer,
                // 32 columns at a time (fewer live registers).
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    uint32_t r[32];
                    tmem_ld16_nowait(lane_addr + 32 * h, r);
                    tmem_ld16_nowait(lane_addr + 32 * h + 16, r + 16);
                    tmem_ld_wait();
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int k = 32 * h + 8 * c;
                        const float4 ba = *reinterpret_cast<const float4*>(&bias[b_off(l) + k]);
                        const float4 bb = *reinterpret_cast<const float4*>(&bias[b_off(l) + k + 4]);
                        const float* f = reinterpret_cast<const float*>(r + 8 * c);
                        const uint4 q = make_uint4(pack_bf16_relu(f[0] + ba.x, f[1] + ba.y),
                                                   pack_bf16_relu(f[2] + ba.z, f[3] + ba.w),
                                                   pack_bf16_relu(f[4] + bb.x, f[5] + bb.y),
                                                   pack_bf16_relu(f[6] + bb.z, f[7] + bb.w));
                        *reinterpret_cast<uint4*>(sm + act + core_offset(gt, k, G_HID)) = q;
                        if (TRAIN && valid)
                            reinterpret_cast<uint4*>(acts + ((size_t)row * 3 + l) * G_HID)[k / 8] = q;
                    }
                }
            } else {
                uint32_t r[G_OUT];
#pragma unroll
                for (int c = 0; c < G_OUT / 16; c++) tmem_ld16_nowait(lane_addr + c * 16, r + 16 * c);
                tmem_ld_wait();
                if (valid) {
                    float v[G_OUT];
#pragma unroll
                    for (int k = 0; k < G_OUT; k += 4) {
                        const float4 b4 = *reinterpret_cast<const float4*>(&bias[b_off(3) + k]);
                        v[k] = __uint_as_float(r[k]) + b4.x;
                        v[k + 1] = __uint_as_float(r[k + 1]) + b4.y;
                        v[k + 2] = __uint_as_float(r[k + 2]) + b4.z;
                        v[k + 3] = __uint_as_float(r[k + 3]) + b4.w;
                    }
                    if (MODE == FWD_RENDER) {
                        mixture_decode_store(v, out + (size_t)row * G_OUT);
                    } else {
                        float4* o = reinterpret_cast<float4*>(out + (size_t)row * G_OUT);
#pragma unroll
                        for (int c = 0; c < G_OUT / 4; c++)
                            o[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                    }
                }
            }
            tc_fence_before();
        }
        if (failed) {
            if (gt == 0) atomicOr(err, GERR_WAIT);
            break;
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem_base, FWD_TMEM_COLS);
        tmem_relinquish();
    }
}

// ---- backward -----------------------------------------------------------------
// Shared memory: WT0 [48][64] 6144 | WT1 8192 | WT2 8192 | WT3 [64][48] 6144 |
//                DZ [128][64] 16384 | DZT [128][128] 32768 | HT [80][128] 20480
// HT holds the layer input transposed plus one row of ones and zero rows up
// to K_in + 16: the dW GEMM then also yields column K_in = sum over the batch
// of dZ, the bias gradient (no per-neuron warp reductions).
// TMEM: dW (and the bias column) in columns [0, 80), dH in [128, 192).
constexpr int B_WT0 = 0, B_WT1 = 6144, B_WT2 = B_WT1 + 8192, B_WT3 = B_WT2 + 8192, B_DZ = B_WT3 + 6144,
              B_DZT = B_DZ + 16384, B_HT = B_DZT + 32768, B_BYTES = B_HT + 20480;
constexpr uint32_t B_TMEM_DH = 128;

__global__ void __launch_bounds__(TILE) k_guide_bwd(GuideDev G, const __nv_bfloat16* __restrict__ X0,
                                                    const __nv_bfloat16* __restrict__ acts,
                                                    const float* __restrict__ out, const float* __restrict__ rec,
                                                    uint32_t n, BatchSel B, float* part,
                                                    float* dX0, float* loss_sum, uint32_t* err) {
    uint32_t begin;
    n = batch_slice(B, n, begin);
    rec += 16 * (size_t)begin;
    // This CTA's row of dW / db partial sums (weights, then biases): its
    // tiles add into it in tile order; k_guide_grad_reduce adds the rows.
    float* gW = part + (size_t)blockIdx.x * G_NPARAMS;
    float* gb = gW + G_NWEIGHTS;
    for (int i = threadIdx.x; i < G_NPARAMS; i += blockDim.x) gW[i] = 0.f;
    __syncthreads();
    if ((uint64_t)blockIdx.x * TILE >= n) return;
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ float red[TILE / 32];
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int l = 0; l < 4; l++) {
        const uint32_t dst = l == 0 ? B_WT0 : l == 1 ? B_WT1 : l == 2 ? B_WT2 : B_WT3;
        stage_transpose(sm + dst, G.w + w_off(l), l_out(l), l_in(l));
    }
    for (int i = tid; i < 32768 / 16; i += TILE) reinterpret_cast<uint4*>(sm + B_DZT)[i] = make_uint4(0, 0, 0, 0);
    // HT rows 64..79 (layers with K_in = 64): a row of ones, then zeros.
    for (int k = 64; k < 80; k++)
        *reinterpret_cast<__nv_bfloat16*>(sm + B_HT + core_offset(k, tid, TILE)) = __float2bfloat16_rn(k == 64 ? 1.f : 0.f);
    if (warp == 0) tmem_alloc(&tmem_base, 256);
    if (tid == 0) mbar_init(&mbar, 1);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tb = tmem_base;
    const uint32_t lane_addr = tb + ((uint32_t)(warp * 32) << 16);
    const uint32_t s0 = smem_u32(sm);
    uint32_t phase = 0;
    bool failed = false;
    float loss = 0.f;
    for (uint32_t tile = blockIdx.x; tile * TILE < n && !failed; tile += gridDim.x) {
        uint32_t row = tile * TILE + tid;
        bool valid = row < n;
        float dz[64];
        if (valid) {
            float o[G_OUT];
            const float4* op = reinterpret_cast<const float4*>(out + (size_t)row * G_OUT);
#pragma unroll
            for (int c = 0; c < G_OUT / 4; c++) {
                float4 q = op[c];
                o[4 * c] = q.x;
                o[4 * c + 1] = q.y;
                o[4 * c + 2] = q.z;
                o[4 * c + 3] = q.w;
            }
            const float* r = rec + 16 * (size_t)row;
            loss += mixture_loss_grad(o, f3(r[9], r[10], r[11]), r[12], dz);
        } else {
#pragma unroll
            for (int k = 0; k < 64; k++) dz[k] = 0.f;
        }
        for (int l = 3; l >= 0 && !failed; l--) {
            const int K_in = l_in(l), N_out = l_out(l);
            // dZ (K-major over N_out) and dZ^T (rows = neurons, K = batch).
#pragma unroll
            for (int c = 0; c < 8; c++)
                if (8 * c < N_out) {
                    uint4 q = make_uint4(pack_bf16(dz[8 * c], dz[8 * c + 1]), pack_bf16(dz[8 * c + 2], dz[8 * c + 3]),
                                         pack_bf16(dz[8 * c + 4], dz[8 * c + 5]), pack_bf16(dz[8 * c + 6], dz[8 * c + 7]));
                    *reinterpret_cast<uint4*>(sm + B_DZ + core_offset(tid, 8 * c, N_out)) = q;
                }
#pragma unroll
            for (int k = 0; k < 64; k++)
                if (k < N_out) *reinterpret_cast<__nv_bfloat16*>(sm + B_DZT + core_offset(k, tid, TILE)) = __float2bfloat16_rn(dz[k]);
            // Layer input H (rows of this tile) -> registers and H^T operand.
            float h[64];
            if (l > 0) {
                const uint4* hp = reinterpret_cast<const uint4*>(acts + ((size_t)row * 3 + (l - 1)) * G_HID);
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    uint4 q = valid ? hp[c] : make_uint4(0, 0, 0, 0);
                    __nv_bfloat162 p2[4];
                    memcpy(p2, &q, 16);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        float2 f = __bfloat1622float2(p2[e]);
                        h[8 * c + 2 * e] = f.x;
                        h[8 * c + 2 * e + 1] = f.y;
                    }
                }
            } else {
                const uint4* hp = reinterpret_cast<const uint4*>(X0 + (size_t)row * G_IN);
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    uint4 q = (valid && c < G_IN / 8) ? hp[c] : make_uint4(0, 0, 0, 0);
                    __nv_bfloat162 p2[4];
                    memcpy(p2, &q, 16);
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        float2 f = __bfloat1622float2(p2[e]);
                        h[8 * c + 2 * e] = f.x;
                        h[8 * c + 2 * e + 1] = f.y;
                    }
                }
            }
            // H^T rows 0..K_in-1, then (layer 0) a row of ones and zeros up to
            // row 63; for K_in = 64 the ones row 64 and zeros were set up front.
#pragma unroll
            for (int k = 0; k < 64; k++) {
                const float hv = k < K_in ? h[k] : (k == K_in ? 1.f : 0.f);
                *reinterpret_cast<__nv_bfloat16*>(sm + B_HT + core_offset(k, tid, TILE)) = __float2bfloat16_rn(hv);
            }
            fence_proxy_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc_fence_after();
                // dW[n][k] = sum_m dZ[m][n] H[m][k]  (M = 128 padded neurons, N = K_in + 16, K = batch);
                // column K_in is the bias gradient.
                tc_gemm_issue(tb, s0 + B_DZT, s0 + B_HT, K_in + 16, TILE, false);
                // dH[m][k] = sum_n dZ[m][n] W[n][k]  (N = K_in, K = N_out)
                const uint32_t wt = l == 0 ? B_WT0 : l == 1 ? B_WT1 : l == 2 ? B_WT2 : B_WT3;
                tc_gemm_issue(tb + B_TMEM_DH, s0 + B_DZ, s0 + wt, K_in, N_out, false);
                tc_commit(&mbar);
            }
            bool ok = mbar_wait_or_drain(&mbar, phase, G.wait_polls);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            tc_fence_after();
            float v[64], vb[16];
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c * 16 < K_in) tmem_ld16(lane_addr + c * 16, v + 16 * c);
            tmem_ld16(lane_addr + K_in, vb);
            if (tid < N_out) {
                float* g = gW + w_off(l) + (size_t)tid * K_in;
#pragma unroll
                for (int k = 0; k < 64; k++)
                    if (k < K_in) g[k] += v[k];
                gb[b_off(l) + tid] += vb[0];
            }
#pragma unroll
            for (int c = 0; c < 4; c++)
                if (c * 16 < K_in) tmem_ld16(lane_addr + B_TMEM_DH + c * 16, v + 16 * c);
            if (l > 0) {
#pragma unroll
                for (int k = 0; k < 64; k++) dz[k] = h[k] > 0.f ? v[k] : 0.f;
            } else if (valid) {
                float4* d = reinterpret_cast<float4*>(dX0 + (size_t)row * 32);
#pragma unroll
                for (int c = 0; c < 8; c++) d[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
            }
            tc_fence_before();
            __syncthreads();
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, off);
    if ((tid & 31) == 0) red[warp] = loss;
    __syncthreads();
    if (tid == 0) atomicAdd(loss_sum, red[0] + red[1] + red[2] + red[3]);
    if (failed && tid == 0) atomicOr(err, GERR_WAIT);
    if (warp == 0) {
        tmem_dealloc(tb, 256);
        tmem_relinquish();
    }
}

// Adds the backward CTAs' partial rows to the MLP gradient, in CTA order.
__global__ void k_guide_grad_reduce(const float* __restrict__ part, int rows, float* gw) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G_NPARAMS) return;
    float s = 0.f;
    for (int b = 0; b < rows; b++) s += part[(size_t)b * G_NPARAMS + i];
    gw[i] += s;
}

// Table gradients are summed as integers in units of 2^-24 (each
// contribution rounded, clamped to +-2^30): the sum is the same whatever
// order the scattered atomics arrive in.
#define G_FIX_SCALE 16777216.0f
__device__ __forceinline__ unsigned long long to_fix(float v) {
    return (unsigned long long)__float2ll_rn(fminf(fmaxf(v, -1073741824.0f), 1073741824.0f) * G_FIX_SCALE);
}
__device__ __forceinline__ float from_fix(unsigned long long q) { return (float)(long long)q * (1.0f / G_FIX_SCALE); }

// ---- hash-grid backward ---------------------------------------------------------
__global__ void k_guide_hash_bwd(GuideDev G, const float* __restrict__ rec, const float* __restrict__ dX0, uint32_t n,
                                 BatchSel B, unsigned long long* gtable) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, begin;
    n = batch_slice(B, n, begin);
    rec += 16 * (size_t)begin;
    if (i >= n) return;
    const float* r = rec + 16 * (size_t)i;
    float3 pn = guide_normalize_pos(G, f3(r[0], r[1], r[2]));
    const float* dx = dX0 + 32 * (size_t)i;
    for (int l = 0; l < G_LEVELS; l++) {
        float rs = G.res[l];
        uint32_t res1 = (uint32_t)rs + 2u;
        bool dense = grid_dense(res1);
        float fx = pn.x * rs, fy = pn.y * rs, fz = pn.z * rs;
        float ix = floorf(fx), iy = floorf(fy), iz = floorf(fz);
        float tx = fx - ix, ty = fy - iy, tz = fz - iz;
        uint32_t x0 = (uint32_t)ix, y0 = (uint32_t)iy, z0 = (uint32_t)iz;
        float g0 = dx[2 * l], g1 = dx[2 * l + 1];
        unsigned long long* T = gtable + (size_t)l * G_T * 2;
        for (int c = 0; c < 8; c++) {
            uint32_t ddx = c & 1, ddy = (c >> 1) & 1, ddz = (c >> 2) & 1;
            float w = (ddx ? tx : 1.f - tx) * (ddy ? ty : 1.f - ty) * (ddz ? tz : 1.f - tz);
            uint32_t idx = grid_index(x0 + ddx, y0 + ddy, z0 + ddz, res1, dense);
            const float a = w * g0, b = w * g1;
            if (a != 0.f) atomicAdd(T + 2 * (size_t)idx, to_fix(a));
            if (b != 0.f) atomicAdd(T + 2 * (size_t)idx + 1, to_fix(b));
        }
    }
}

// ---- Adam -----------------------------------------------------------------------------
struct AdamArgs {
    float lr, b1, b2, eps;
    const float* c;  // device: c[0] = 1/(1-b1^t), c[1] = 1/(1-b2^t), c[2] = 1 when the step runs
};

// Step counter and bias corrections on the device: a step whose batch slice is
// empty is skipped (no update, no count).
__global__ void k_guide_adam_tick(BatchSel B, uint32_t cap, AdamArgs A, uint32_t* step, float* c) {
    uint32_t begin;
    uint32_t n = batch_slice(B, cap, begin);
    if (n == 0) {
        c[2] = 0.f;
        return;
    }
    uint32_t t = ++*step;
    c[0] = 1.f / (1.f - powf(A.b1, (float)t));
    c[1] = 1.f / (1.f - powf(A.b2, (float)t));
    c[2] = 1.f;
}

__global__ void k_guide_adam_mlp(AdamArgs A, float* p, float* g, float* m, float* v, __nv_bfloat16* w16, int n_weights,
                                 int n_total) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_total || A.c[2] == 0.f) return;
    const float c1 = A.c[0], c2 = A.c[1];
    float gi = g[i];
    float mi = A.b1 * m[i] + (1.f - A.b1) * gi;
    float vi = A.b2 * v[i] + (1.f - A.b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - A.lr * (mi * c1) / (sqrtf(vi * c2) + A.eps);
    p[i] = pi;
    g[i] = 0.f;
    if (i < n_weights) w16[i] = __float2bfloat16_rn(pi);
}

__global__ void k_guide_adam_table(AdamArgs A, float* p, unsigned long long* g, float* m, float* v, __half* t16,
                                   uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || A.c[2] == 0.f) return;
    const float c1 = A.c[0], c2 = A.c[1];
    // Lazy (sparse) Adam: a table entry no record touched this step keeps its
    // parameter and moments. A batch touches a few percent of the 16M
    // entries, so the step reads the gradient table and updates only those.
    const unsigned long long q = g[i];
    if (q == 0ull) return;
    float gi = from_fix(q);
    float mi = A.b1 * m[i] + (1.f - A.b1) * gi;
    float vi = A.b2 * v[i] + (1.f - A.b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i] - A.lr * (mi * c1) / (sqrtf(vi * c2) + A.eps);
    p[i] = pi;
    g[i] = 0ull;
    t16[i] = __float2half_rn(pi);
}

// ---- tcgen05 GEMM self-test: D[128][N] = A[128][K] B[N][K]^T -------------------------------
__global__ void __launch_bounds__(TILE) k_tc_selftest(const __nv_bfloat16* A, const __nv_bfloat16* B, int N, int K,
                                                      float* D, uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t sm[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5;
    stage_matrix(sm, A, TILE, K);
    stage_matrix(sm + TILE * K * 2, B, N, K);
    if (warp == 0) tmem_alloc(&tmem_base, 256);
    if (tid == 0) mbar_init(&mbar, 1);
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    uint32_t tb = tmem_base;
    uint32_t s0 = smem_u32(sm);
    if (tid == 0) {
        tc_gemm_issue(tb, s0, s0 + TILE * K * 2, N, K, false);
        tc_commit(&mbar);
    }
    bool ok = mbar_wait_bounded(&mbar, 0);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicOr(err, GERR_WAIT);
    } else {
        tc_fence_after();
        for (int c = 0; c < N / 16; c++) {
            float v[16];
            tmem_ld16(tb + ((uint32_t)(warp * 32) << 16) + c * 16, v);
            for (int i = 0; i < 16; i++) D[(size_t)tid * N + c * 16 + i] = v[i];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tmem_dealloc(tb, 256);
        tmem_relinquish();
    }
}

// ---- host side ------------------------------------------------------------------------------
struct rt_guide {
    GuideDev G{};
    float* w32 = nullptr;      // f32 masters: weights then biases (G_NPARAMS)
    float* gw = nullptr;       // gradients (same layout)
    float* mw = nullptr;
    float* vw = nullptr;
    __nv_bfloat16* w16 = nullptr;
    float* t32 = nullptr;      // table master (levels * T * 2)
    unsigned long long* gt = nullptr;  // table gradient, 2^-24 fixed point
    float* part = nullptr;     // backward CTAs' dW / db partial rows (bwd_rows x G_NPARAMS)
    int bwd_rows = 0;
    float* mt = nullptr;
    float* vt = nullptr;
    __half* t16 = nullptr;
    // scratch for a batch: inputs and outputs for `cap` records, activations
    // and input gradients for `train_cap` (training batches only)
    uint32_t cap = 0, train_cap = 0;
    __nv_bfloat16* X0 = nullptr;
    __nv_bfloat16* acts = nullptr;
    float* out = nullptr;
    float* dX0 = nullptr;
    float* loss = nullptr;
    uint32_t* err = nullptr;
    float* rec_dev = nullptr;  // staging for host-pointer calls
    uint32_t rec_cap = 0;
    int sms = 148;
    uint32_t* step = nullptr;  // device: Adam steps taken
    float* adam_c = nullptr;   // device: bias corrections of the current step
    float lr = 1e-2f;
    std::vector<void*> allocs;

    template <class T>
    int alloc(T** p, size_t n) {
        void* v = nullptr;
        cudaError_t e = cudaMalloc(&v, std::max<size_t>(n, 1) * sizeof(T));
        if (e != cudaSuccess) return gfail(-3, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        allocs.push_back(v);
        *p = (T*)v;
        return 0;
    }
    void release(void* q) {
        if (!q) return;
        cudaFree(q);
        allocs.erase(std::remove(allocs.begin(), allocs.end(), q), allocs.end());
    }
    int ensure(uint32_t n, bool train) {
        int rc = 0;
        if (n > cap) {
            release(X0);
            release(out);
            cap = std::max(n, 1u << 16);
            rc = rc ? rc : alloc(&X0, (size_t)cap * G_IN);
            rc = rc ? rc : alloc(&out, (size_t)cap * G_OUT);
            // Zeroed, so rows a failed forward pass did not write hold an
            // empty mixture rather than stale bits.
            if (!rc && cudaMemset(out, 0, (size_t)cap * G_OUT * 4) != cudaSuccess) rc = gfail(-2, "cudaMemset");
        }
        if (train && n > train_cap) {
            release(acts);
            release(dX0);
            train_cap = std::max(n, 1u << 16);
            rc = rc ? rc : alloc(&acts, (size_t)train_cap * 3 * G_HID);
            rc = rc ? rc : alloc(&dX0, (size_t)train_cap * 32);
        }
        return rc;
    }
    ~rt_guide() {
        cudaDeviceSynchronize();
        for (void* p : allocs) cudaFree(p);
    }
};

static int launch_forward(rt_guide* g, const float* rec, uint32_t n, int mode, cudaStream_t st,
                          BatchSel B = BatchSel{nullptr, 0, 1}) {
    if (n == 0) return 0;
    int rc = g->ensure(n, mode == FWD_TRAIN);
    if (rc) return rc;
    const uint32_t enc_grid = std::min<uint32_t>((n + 255) / 256, (uint32_t)g->sms * ENCODE_CTAS_PER_SM);
    k_guide_encode<<<enc_grid, 256, 0, st>>>(g->G, rec, n, B, g->X0);
    uint32_t tiles = (n + TILE - 1) / TILE;
    int grid = (int)std::min<uint32_t>(tiles, (uint32_t)g->sms);
    if (mode == FWD_TRAIN)
        k_guide_fwd<FWD_TRAIN><<<grid, FWD_THREADS, F_BYTES, st>>>(g->G, g->X0, n, B, g->acts, g->out, g->err);
    else if (mode == FWD_RENDER)
        k_guide_fwd<FWD_RENDER><<<grid, FWD_THREADS, F_BYTES, st>>>(g->G, g->X0, n, B, g->acts, g->out, g->err);
    else
        k_guide_fwd<FWD_RAW><<<grid, FWD_THREADS, F_BYTES, st>>>(g->G, g->X0, n, B, g->acts, g->out, g->err);
    G_TRY(cudaGetLastError());
    return 0;
}

static int launch_backward(rt_guide* g, const float* rec, uint32_t n, cudaStream_t st,
                           BatchSel B = BatchSel{nullptr, 0, 1}) {
    uint32_t tiles = (n + TILE - 1) / TILE;
    int grid = (int)std::min<uint32_t>(tiles, (uint32_t)g->bwd_rows);
    G_TRY(cudaMemsetAsync(g->loss, 0, 4, st));
    k_guide_bwd<<<grid, TILE, B_BYTES, st>>>(g->G, g->X0, g->acts, g->out, rec, n, B, g->part, g->dX0, g->loss,
                                             g->err);
    k_guide_grad_reduce<<<(G_NPARAMS + 255) / 256, 256, 0, st>>>(g->part, grid, g->gw);
    k_guide_hash_bwd<<<(n + 127) / 128, 128, 0, st>>>(g->G, rec, g->dX0, n, B, g->gt);
    G_TRY(cudaGetLastError());
    return 0;
}

static void launch_adam(rt_guide* g, uint32_t n, cudaStream_t st, BatchSel B = BatchSel{nullptr, 0, 1}) {
    AdamArgs A{g->lr, 0.9f, 0.99f, 1e-8f, g->adam_c};
    k_guide_adam_tick<<<1, 1, 0, st>>>(B, n, A, g->step, g->adam_c);
    k_guide_adam_mlp<<<(G_NPARAMS + 255) / 256, 256, 0, st>>>(A, g->w32, g->gw, g->mw, g->vw, g->w16, G_NWEIGHTS,
                                                             G_NPARAMS);
    uint32_t tn = (uint32_t)(G_LEVELS * G_T * 2);
    k_guide_adam_table<<<(tn + 255) / 256, 256, 0, st>>>(A, g->t32, g->gt, g->mt, g->vt, g->t16, tn);
}

// ---- entry points for the renderer (guide_internal.h) ------------------------------
namespace rt {

int guide_infer_counted(rt_guide* g, const float* rec, const uint32_t* n_dev, uint32_t cap, float** raw_out,
                        cudaStream_t st) {
    int rc = launch_forward(g, rec, cap, FWD_RENDER, st, BatchSel{n_dev, 0, 1});
    *raw_out = g->out;
    return rc;
}

int guide_train_slices(rt_guide* g, const float* rec, const uint32_t* total_dev, uint32_t cap, uint32_t steps,
                       cudaStream_t st) {
    for (uint32_t s = 0; s < steps; s++) {
        const BatchSel B{total_dev, s, steps};
        int rc = launch_forward(g, rec, cap, FWD_TRAIN, st, B);
        rc = rc ? rc : launch_backward(g, rec, cap, st, B);
        if (rc) return rc;
        launch_adam(g, cap, st, B);
    }
    G_TRY(cudaGetLastError());
    return 0;
}

int guide_reserve(rt_guide* g, uint32_t n) { return g->ensure(n, false); }

const float* guide_loss_ptr(rt_guide* g) { return g->loss; }
const uint32_t* guide_err_ptr(rt_guide* g) { return g->err; }
GuideDev guide_dev(rt_guide* g) { return g->G; }
void guide_set_wait_polls(rt_guide* g, uint32_t polls) { g->G.wait_polls = polls ? polls : (1u << 24); }

}  // namespace rt

static int check_err(rt_guide* g, cudaStream_t st) {
    uint32_t e = 0;
    G_TRY(cudaMemcpyAsync(&e, g->err, 4, cudaMemcpyDeviceToHost, st));
    G_TRY(cudaStreamSynchronize(st));
    if (e) {
        cudaMemsetAsync(g->err, 0, 4, st);
        return gfail(-4, "tensor-core pipeline wait timed out");
    }
    return 0;
}

extern "C" {

const char* rt_guide_last_error(void) { return g_gerr.c_str(); }

int rt_guide_create(const float* lo, const float* hi, uint64_t seed, float lr, rt_guide** out) {
    if (!lo || !hi || !out) return gfail(-1, "NULL argument");
    *out = nullptr;
    auto* g = new rt_guide();
    g->lr = lr;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        delete g;
        return gfail(-2, "no CUDA device");
    }
    cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, dev);
    size_t tn = (size_t)G_LEVELS * G_T * 2;
    int rc = 0;
    rc = rc ? rc : g->alloc(&g->w32, G_NPARAMS);
    rc = rc ? rc : g->alloc(&g->gw, G_NPARAMS);
    rc = rc ? rc : g->alloc(&g->mw, G_NPARAMS);
    rc = rc ? rc : g->alloc(&g->vw, G_NPARAMS);
    rc = rc ? rc : g->alloc(&g->w16, G_NWEIGHTS);
    rc = rc ? rc : g->alloc(&g->t32, tn);
    rc = rc ? rc : g->alloc(&g->gt, tn);
    g->bwd_rows = g->sms * 2;
    rc = rc ? rc : g->alloc(&g->part, (size_t)g->bwd_rows * G_NPARAMS);
    rc = rc ? rc : g->alloc(&g->mt, tn);
    rc = rc ? rc : g->alloc(&g->vt, tn);
    rc = rc ? rc : g->alloc(&g->t16, tn);
    rc = rc ? rc : g->alloc(&g->loss, 1);
    rc = rc ? rc : g->alloc(&g->err, 1);
    rc = rc ? rc : g->alloc(&g->step, 1);
    rc = rc ? rc : g->alloc(&g->adam_c, 4);
    rc = rc ? rc : g->ensure(1u << 16, true);
    if (rc) {
        delete g;
        return rc;
    }
    cudaFuncSetAttribute(k_guide_fwd<FWD_RAW>, cudaFuncAttributeMaxDynamicSharedMemorySize, F_BYTES);
    cudaFuncSetAttribute(k_guide_fwd<FWD_TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, F_BYTES);
    cudaFuncSetAttribute(k_guide_fwd<FWD_RENDER>, cudaFuncAttributeMaxDynamicSharedMemorySize, F_BYTES);
    cudaFuncSetAttribute(k_guide_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, B_BYTES);
    cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024);
    // Init: He-uniform weights, zero biases; table U(-1e-4, 1e-4) (instant-ngp).
    std::mt19937_64 rng(seed);
    std::vector<float> p(G_NPARAMS, 0.f);
    for (int l = 0; l < 4; l++) {
        float lim = std::sqrt(6.0f / (float)l_in(l));
        std::uniform_real_distribution<float> U(-lim, lim);
        for (int i = 0; i < l_out(l) * l_in(l); i++) p[w_off(l) + i] = U(rng);
    }
    // Padded inputs (x >= 38) and padded outputs (rows >= 40) stay zero.
    for (int o = 0; o < G_HID; o++)
        for (int k = 38; k < G_IN; k++) p[w_off(0) + o * G_IN + k] = 0.f;
    for (int o = 40; o < G_OUT; o++)
        for (int k = 0; k < G_HID; k++) p[w_off(3) + o * G_HID + k] = 0.f;
    std::vector<float> t(tn);
    std::uniform_real_distribution<float> Ut(-1e-4f, 1e-4f);
    for (auto& x : t) x = Ut(rng);
    int r2 = rt_guide_set_params(g, p.data(), nullptr);
    if (!r2) {
        std::vector<__half> th(tn);
        for (size_t i = 0; i < tn; i++) th[i] = __float2half_rn(t[i]);
        cudaMemcpy(g->t32, t.data(), tn * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(g->t16, th.data(), tn * 2, cudaMemcpyHostToDevice);
    }
    cudaMemset(g->gw, 0, G_NPARAMS * 4);
    cudaMemset(g->mw, 0, G_NPARAMS * 4);
    cudaMemset(g->vw, 0, G_NPARAMS * 4);
    cudaMemset(g->gt, 0, tn * 8);
    cudaMemset(g->mt, 0, tn * 4);
    cudaMemset(g->vt, 0, tn * 4);
    cudaMemset(g->err, 0, 4);
    cudaMemset(g->step, 0, 4);
    g->G.table = reinterpret_cast<const __half2*>(g->t16);
    g->G.wait_polls = 1u << 24;
    g->G.w = g->w16;
    g->G.b = g->w32 + G_NWEIGHTS;
    // Level resolutions: geometric from 16 to 2048.
    double b = std::exp((std::log(2048.0) - std::log(16.0)) / (G_LEVELS - 1));
    for (int l = 0; l < G_LEVELS; l++) g->G.res[l] = (float)std::floor(16.0 * std::pow(b, l));
    for (int a = 0; a < 3; a++) {
        float ext = std::max(hi[a] - lo[a], 1e-6f);
        g->G.lo[a] = lo[a];
        g->G.inv_ext[a] = 1.0f / ext;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (r2 || e != cudaSuccess) {
        delete g;
        return r2 ? r2 : gfail(-2, cudaGetErrorString(e));
    }
    *out = g;
    return 0;
}

int rt_guide_destroy(rt_guide* g) {
    delete g;
    return 0;
}

int rt_guide_set_params(rt_guide* g, const float* mlp, const uint16_t* table_fp16) {
    if (!g) return gfail(-1, "NULL guide");
    if (mlp) {
        std::vector<__nv_bfloat16> w(G_NWEIGHTS);
        for (int i = 0; i < G_NWEIGHTS; i++) w[i] = __float2bfloat16_rn(mlp[i]);
        // The f32 master holds the bf16-rounded weights so both copies agree.
        std::vector<float> m(mlp, mlp + G_NPARAMS);
        for (int i = 0; i < G_NWEIGHTS; i++) m[i] = __bfloat162float(w[i]);
        G_TRY(cudaMemcpy(g->w32, m.data(), G_NPARAMS * 4, cudaMemcpyHostToDevice));
        G_TRY(cudaMemcpy(g->w16, w.data(), G_NWEIGHTS * 2, cudaMemcpyHostToDevice));
    }
    if (table_fp16) {
        size_t tn = (size_t)G_LEVELS * G_T * 2;
        std::vector<float> t(tn);
        for (size_t i = 0; i < tn; i++) {
            __half_raw hr;
            hr.x = table_fp16[i];
            t[i] = __half2float(__half(hr));
        }
        G_TRY(cudaMemcpy(g->t16, table_fp16, tn * 2, cudaMemcpyHostToDevice));
        G_TRY(cudaMemcpy(g->t32, t.data(), tn * 4, cudaMemcpyHostToDevice));
    }
    return 0;
}

int rt_guide_get_params(rt_guide* g, float* mlp, uint16_t* table_fp16) {
    if (!g) return gfail(-1, "NULL guide");
    G_TRY(cudaDeviceSynchronize());
    if (mlp) G_TRY(cudaMemcpy(mlp, g->w32, G_NPARAMS * 4, cudaMemcpyDeviceToHost));
    if (table_fp16) G_TRY(cudaMemcpy(table_fp16, g->t16, (size_t)G_LEVELS * G_T * 4, cudaMemcpyDeviceToHost));
    return 0;
}

int rt_guide_info(rt_guide* g, float* res_out, float* lo_out, float* inv_ext_out) {
    if (!g) return gfail(-1, "NULL guide");
    for (int l = 0; l < G_LEVELS; l++) res_out[l] = g->G.res[l];
    for (int a = 0; a < 3; a++) {
        lo_out[a] = g->G.lo[a];
        inv_ext_out[a] = g->G.inv_ext[a];
    }
    return 0;
}

int rt_guide_infer_device(rt_guide* g, const float* rec, uint32_t n, float* raw_out, void* stream) {
    if (!g || (n && (!rec || !raw_out))) return gfail(-1, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    int rc = launch_forward(g, rec, n, FWD_RAW, st);
    if (rc) return rc;
    if (n) G_TRY(cudaMemcpyAsync(raw_out, g->out, (size_t)n * G_OUT * 4, cudaMemcpyDeviceToDevice, st));
    return 0;
}

int rt_guide_train_step_device(rt_guide* g, const float* rec, uint32_t n, float* loss_out, void* stream) {
    if (!g || (n && !rec)) return gfail(-1, "NULL argument");
    cudaStream_t st = (cudaStream_t)stream;
    if (n == 0) return 0;
    int rc = launch_forward(g, rec, n, FWD_TRAIN, st);
    rc = rc ? rc : launch_backward(g, rec, n, st);
    if (rc) return rc;
    launch_adam(g, n, st);
    G_TRY(cudaGetLastError());
    if (loss_out) {
        G_TRY(cudaMemcpyAsync(loss_out, g->loss, 4, cudaMemcpyDeviceToHost, st));
        return check_err(g, st);
    }
    return 0;
}

// Gradients without an update (host pointers), for checks against the f64 network oracle.
int rt_guide_grads(rt_guide* g, const float* rec_host, uint32_t n, float* g_mlp, float* g_table, float* raw_out,
                   float* loss) {
    if (!g || !rec_host || n == 0) return gfail(-1, "bad argument");
    float* rec = nullptr;
    G_TRY(cudaMalloc(&rec, (size_t)n * 64));
    G_TRY(cudaMemcpy(rec, rec_host, (size_t)n * 64, cudaMemcpyHostToDevice));
    size_t tn = (size_t)G_LEVELS * G_T * 2;
    cudaMemset(g->gw, 0, G_NPARAMS * 4);
    cudaMemset(g->gt, 0, tn * 8);
    int rc = launch_forward(g, rec, n, FWD_TRAIN, 0);
    rc = rc ? rc : launch_backward(g, rec, n, 0);
    if (!rc) rc = check_err(g, 0);
    if (!rc && g_mlp) G_TRY(cudaMemcpy(g_mlp, g->gw, G_NPARAMS * 4, cudaMemcpyDeviceToHost));
    if (!rc && g_table) {
        std::vector<long long> q(tn);
        G_TRY(cudaMemcpy(q.data(), g->gt, tn * 8, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < tn; i++) g_table[i] = (float)q[i] * (1.0f / G_FIX_SCALE);
    }
    if (!rc && raw_out) G_TRY(cudaMemcpy(raw_out, g->out, (size_t)n * G_OUT * 4, cudaMemcpyDeviceToHost));
    if (!rc && loss) G_TRY(cudaMemcpy(loss, g->loss, 4, cudaMemcpyDeviceToHost));
    cudaMemset(g->gw, 0, G_NPARAMS * 4);
    cudaMemset(g->gt, 0, tn * 8);
    cudaFree(rec);
    return rc;
}

int rt_guide_train_step(rt_guide* g, const float* rec_host, uint32_t n, float* loss) {
    if (!g || !rec_host || n == 0) return gfail(-1, "bad argument");
    if (n > g->rec_cap) {
        if (g->rec_dev) cudaFree(g->rec_dev);
        g->rec_dev = nullptr;
        G_TRY(cudaMalloc(&g->rec_dev, (size_t)n * 64));
        g->rec_cap = n;
    }
    G_TRY(cudaMemcpy(g->rec_dev, rec_host, (size_t)n * 64, cudaMemcpyHostToDevice));
    int rc = rt_guide_train_step_device(g, g->rec_dev, n, loss, 0);
    if (!rc) G_TRY(cudaDeviceSynchronize());
    return rc;
}

int rt_guide_infer(rt_guide* g, const float* rec_host, uint32_t n, float* raw_host) {
    if (!g || !rec_host || !raw_host || n == 0) return gfail(-1, "bad argument");
    float* rec = nullptr;
    G_TRY(cudaMalloc(&rec, (size_t)n * 64));
    G_TRY(cudaMemcpy(rec, rec_host, (size_t)n * 64, cudaMemcpyHostToDevice));
    int rc = launch_forward(g, rec, n, FWD_RAW, 0);
    if (!rc) rc = check_err(g, 0);
    if (!rc) G_TRY(cudaMemcpy(raw_host, g->out, (size_t)n * G_OUT * 4, cudaMemcpyDeviceToHost));
    cudaFree(rec);
    return rc;
}

int rt_guide_infer_mixture(rt_guide* g, const float* rec_host, uint32_t n, float* mix_host) {
    if (!g || !rec_host || !mix_host || n == 0) return gfail(-1, "bad argument");
    float* rec = nullptr;
    G_TRY(cudaMalloc(&rec, (size_t)n * 64));
    G_TRY(cudaMemcpy(rec, rec_host, (size_t)n * 64, cudaMemcpyHostToDevice));
    int rc = launch_forward(g, rec, n, FWD_RENDER, 0);
    if (!rc) rc = check_err(g, 0);
    if (!rc) G_TRY(cudaMemcpy(mix_host, g->out, (size_t)n * G_OUT * 4, cudaMemcpyDeviceToHost));
    cudaFree(rec);
    return rc;
}

int rt_tc_gemm_selftest(const uint16_t* A, const uint16_t* B, int N, int K, float* D) {
    if (!A || !B || !D || N % 16 || N < 16 || N > 256 || K % 16 || K < 16 || (128 * K + N * K) * 2 > 128 * 1024)
        return gfail(-1, "bad shape");
    void *dA, *dB, *dD, *dE;
    G_TRY(cudaMalloc(&dA, 128 * K * 2));
    G_TRY(cudaMalloc(&dB, N * K * 2));
    G_TRY(cudaMalloc(&dD, 128 * N * 4));
    G_TRY(cudaMalloc(&dE, 4));
    cudaMemcpy(dA, A, 128 * K * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(dB, B, N * K * 2, cudaMemcpyHostToDevice);
    cudaMemset(dE, 0, 4);
    cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, 128 * 1024);
    k_tc_selftest<<<1, TILE, (128 * K + N * K) * 2>>>((const __nv_bfloat16*)dA, (const __nv_bfloat16*)dB, N, K,
                                                      (float*)dD, (uint32_t*)dE);
    cudaError_t e = cudaDeviceSynchronize();
    uint32_t err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(D, dD, 128 * N * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&err, dE, 4, cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dE);
    if (e != cudaSuccess) return gfail(-2, cudaGetErrorString(e));
    if (err) return gfail(-4, "tensor-core wait timed out");
    return 0;
}

}  // extern "C"
