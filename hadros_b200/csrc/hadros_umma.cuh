// hadros_umma.cuh — PTX wrappers for the 5th-generation tensor cores
// (tcgen05: MMA into tensor memory, loads from it, commits), mbarriers and
// bulk copies, and the shared-memory matrix and instruction descriptors, as
// the surrogate's inference kernel and its training GEMMs use them.
#pragma once

#include <cstdint>

namespace hadros {
namespace umma {

constexpr long kWaitLimit = 1L << 22;        // try_wait rounds before giving up

__device__ __forceinline__ uint32_t saddr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait; false (and the abort flag set) when the limit ran out or
// another thread already aborted.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag)
{
    for (long it = 0; it < kWaitLimit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}
// mbar_wait by every lane of a warp, which leaves it converged and agreeing
// (the tcgen05.ld that follows is warp-collective).
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag)
{
    const bool ok = mbar_wait(bar, parity, abort_flag);
    return __all_sync(0xffffffffu, ok) != 0;
}
// Bounded wait that ignores the abort flag (draining on the abort path).
__device__ __forceinline__ bool mbar_wait_plain(uint32_t bar, uint32_t parity)
{
    for (long it = 0; it < kWaitLimit; ++it)
        if (mbar_try(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
                 : "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, both K-major.
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tc_ld2(uint32_t taddr, uint32_t& r0, uint32_t& r1)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];\n" : "=r"(r0), "=r"(r1) : "r"(taddr));
}
// The wait, with the loaded registers as operands so that no use of them is
// scheduled before it.
__device__ __forceinline__ void tc_wait_ld(uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.wait::ld.sync.aligned;\n"
        : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
          "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
          "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
          "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
          "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
        :
        : "memory");
}
__device__ __forceinline__ void tc_wait_ld(uint32_t& r0, uint32_t& r1)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" : "+r"(r0), "+r"(r1) : : "memory");
}

// (a0, a1) + (b0, b1) with one packed FP32x2 addition.
__device__ __forceinline__ void add_f32x2(uint32_t& a0, uint32_t& a1, float2 b)
{
    asm("{\n.reg .b64 x, y;\nmov.b64 x, {%0, %1};\nmov.b64 y, {%2, %3};\n"
        "add.rn.f32x2 x, x, y;\nmov.b64 {%0, %1}, x;\n}\n"
        : "+r"(a0), "+r"(a1)
        : "f"(b.x), "f"(b.y));
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), descriptor version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t addr)
{
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t(1) << 16) | (uint64_t(1024 >> 4) << 32) |
           (uint64_t(1) << 46) | (uint64_t(2) << 61);
}
// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

// Shared-memory matrix descriptor of an MN-major operand, 128-byte swizzle:
// atoms of 64 MN-contiguous BF16 (one 128-byte row per k) by 8 k, atoms
// along K `sbo` bytes apart, atoms along MN `lbo` bytes apart.
__device__ __forceinline__ uint64_t sdesc_mn(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((addr & 0x3FFFFu) >> 4) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46) | (uint64_t(2) << 61);
}
// Instruction descriptor of kind::f16 with the operands' majors: bit 15 A,
// bit 16 B (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_bf16_major(int M, int N, bool a_mn, bool b_mn)
{
    return idesc_bf16(M, N) | (a_mn ? (1u << 15) : 0u) | (b_mn ? (1u << 16) : 0u);
}

}  // namespace umma
}  // namespace hadros
