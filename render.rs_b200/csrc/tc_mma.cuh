// tc_mma.cuh — 5th-generation tensor core (tcgen05) building blocks, sm_100a.
//
// One CTA computes D[128 x N] (f32, in tensor memory) = A[128 x K] * B[N x K]^T
// with A and B in shared memory as bf16, both K-major, laid out as the
// canonical no-swizzle ("interleaved") UMMA layout: 8-row x 16-byte core
// matrices; core (row group g, k chunk c) of an R x K operand sits at
//     g * (K/8 * 128) + c * 128 bytes,
// i.e. leading-byte offset (between the two K halves of one MMA) = 128 B and
// stride-byte offset (between 8-row groups) = K * 16 B. One thread issues the
// MMAs (K/16 of them), a tcgen05.commit arrives on an mbarrier, every thread
// waits on it (bounded), and the epilogue reads D with tcgen05.ld
// (32x32b shape: warp w owns TMEM lanes 32w..32w+31 = rows of D).
//
// Descriptor bit layouts follow the PTX ISA's tcgen05 "shared memory
// descriptor" and "instruction descriptor" tables (also mirrored by
// CUTLASS's UMMA::SmemDescriptor / UMMA::InstrDescriptor).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace rt {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) of an R x K bf16 operand in the core-matrix layout.
__host__ __device__ __forceinline__ uint32_t core_offset(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor, kind::f16: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
                 "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void tc_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Non-blocking test of a barrier phase.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* mbar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait: returns false (and the caller records an error) if the
// barrier phase has not completed after `limit` polls. Polls block for a
// while (try_wait) unless the limit is tiny (at most 64), where they return
// at once (test_wait) so that such a limit really runs out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* mbar, uint32_t phase, uint32_t limit = (1u << 24)) {
    if (limit <= 64) {
        for (uint32_t i = 0; i < limit; i++)
            if (mbar_test_wait(mbar, phase)) return true;
        return false;
    }
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_try_wait(mbar, phase)) return true;
    return false;
}
// A pipeline wait with a settable limit. When it runs out the caller
// reports an error, but the MMAs it already issued are still drained first
// (a second wait with the default limit), so no tensor-core work writes the
// TMEM the caller then frees. Returns false when the first wait ran out.
__device__ __forceinline__ bool mbar_wait_or_drain(uint64_t* mbar, uint32_t phase, uint32_t limit) {
    if (mbar_wait_bounded(mbar, phase, limit)) return true;
    mbar_wait_bounded(mbar, phase);
    return false;
}

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// The same without the wait, so several loads share one tcgen05.wait::ld.
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Barrier over the 128 threads of tile group `grp` (named barrier 1 + grp;
// immediate ids, so the kernel reserves only the barriers it uses).
__device__ __forceinline__ void group_sync(uint32_t grp) {
    switch (grp) {
        case 0: asm volatile("bar.sync 1, 128;" ::: "memory"); break;
        case 1: asm volatile("bar.sync 2, 128;" ::: "memory"); break;
        case 2: asm volatile("bar.sync 3, 128;" ::: "memory"); break;
        case 3: asm volatile("bar.sync 4, 128;" ::: "memory"); break;
        case 4: asm volatile("bar.sync 5, 128;" ::: "memory"); break;
        case 5: asm volatile("bar.sync 6, 128;" ::: "memory"); break;
        default: asm volatile("bar.sync 7, 128;" ::: "memory"); break;
    }
}

// Issue D = A * B^T for a 128-row tile (thread 0 of the CTA issues).
// a_saddr / b_saddr: shared addresses of the operands in the core layout.
__device__ __forceinline__ void tc_gemm_issue(uint32_t d_tmem, uint32_t a_saddr, uint32_t b_saddr, int N, int K,
                                              bool accumulate_first) {
    const uint32_t idesc = umma_idesc_bf16_f32(128, N);
    for (int ks = 0; ks < K / 16; ks++) {
        uint64_t ad = umma_smem_desc(a_saddr + ks * 256u, 128u, (uint32_t)K * 16u);
        uint64_t bd = umma_smem_desc(b_saddr + ks * 256u, 128u, (uint32_t)K * 16u);
        tc_mma_bf16(d_tmem, ad, bd, idesc, (ks > 0 || accumulate_first) ? 1u : 0u);
    }
}

}  // namespace rt
