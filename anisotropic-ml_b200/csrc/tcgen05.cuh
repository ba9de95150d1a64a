// Thin inline-PTX wrappers for the sm_100a tensor-core path (tcgen05 MMA with
// TMEM accumulators, operands in shared memory) and the mbarrier it signals.
//
// Shared-memory operand layout used throughout: K-major, no swizzle. Element
// (row, k) of a rows x K bf16 tile sits at byte
//   (row % 8) * 16 + (row / 8) * (K * 16) + (k % 8) * 2 + (k / 8) * 128,
// i.e. 8x8 core matrices of 128 contiguous bytes, K-adjacent core matrices 128
// bytes apart (leading byte offset) and 8-row groups K*16 bytes apart (stride
// byte offset). The same bytes read as an MN-major operand describe the
// transpose, with the two offsets exchanged.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace amlp {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int K) {
    return (row & 7) * 16 + (row >> 3) * (K * 16) + (k & 7) * 2 + (k >> 3) * 128;
}

// UMMA shared-memory descriptor: start address, leading / stride byte offsets
// (all in 16-byte units), version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D f32, A and B bf16, M = 128, N, B major.
__host__ __device__ constexpr uint32_t idesc_bf16(int N, int b_mn_major) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)b_mn_major << 16) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Allocation by one whole warp; the TMEM address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void tmem_ld8_issue(uint32_t taddr, uint32_t *r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}

// After tcgen05.wait::ld: the empty statements redefine the loaded registers,
// so that no use of them can be scheduled above the wait.
template <int N>
__device__ __forceinline__ void tmem_wait_ld(uint32_t *r, float *v) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < N; ++k) {
        asm volatile("" : "+r"(r[k]));
        v[k] = __uint_as_float(r[k]);
    }
}

// 8 consecutive 32-bit columns of this thread's TMEM lane written from v;
// complete once tmem_wait_st() returns.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float *v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
                 "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
                 "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
                 : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// 8 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v) {
    uint32_t r[8];
    tmem_ld8_issue(taddr, r);
    tmem_wait_ld<8>(r, v);
}

// n (<= NMAX, warp-uniform) chunks of 8 columns at taddr, taddr + 8, ... with
// one wait for all of them; v[8 c + k] is column 8 c + k.
template <int NMAX>
__device__ __forceinline__ void tmem_ld8_many(uint32_t taddr, int n, float *v) {
    uint32_t r[8 * NMAX];
#pragma unroll
    for (int c = 0; c < NMAX; ++c)
        if (c < n) tmem_ld8_issue(taddr + 8 * c, r + 8 * c);
    tmem_wait_ld<8 * NMAX>(r, v);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}

constexpr int kWaitLimit = 1 << 22;  // polls of a bounded mbarrier wait

// Bounded wait for the completion of `phase`; false after `limit` polls (at once for 0).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int limit = kWaitLimit) {
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

// One arrival on the mbarrier that also expects `bytes` of asynchronous copies.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bulk copy of `bytes` from global memory into this CTA's shared memory (no
// tensor map, no multicast), completing on the mbarrier. Both addresses
// 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Prefetch of `bytes` of global memory into L2 (no shared-memory destination,
// no completion to wait for). Address 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void *src, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// bf16 pair (hi, lo) with hi + lo == v to about 2^-16 relative.
__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16 &hi, __nv_bfloat16 &lo) {
    hi = __float2bfloat16_rn(v);
    lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

}  // namespace tc
}  // namespace amlp
