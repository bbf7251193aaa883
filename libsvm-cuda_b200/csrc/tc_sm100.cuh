// tc_sm100.cuh -- sm_100a tensor-core primitives (tcgen05 MMA with TMEM
// accumulators, shared-memory operand descriptors, mbarriers) used by the
// tensor forms of the kernel-row and kernel-block products.
//
// Operand tiles are K-major with the 128-byte swizzle: a tile of R rows x 64
// bf16 (128 B per row) is stored as R/8 atoms of 8 rows x 128 B (1024 B,
// 1024-byte aligned); inside an atom the 16-byte piece q of row r sits at
// piece position q ^ (r % 8).  One MMA consumes K = 16 bf16 (32 B of each
// row); the four MMAs of a 64-wide chunk advance the descriptor's start
// address by 32 B.  Layout and descriptor fields follow the PTX ISA's
// "shared memory descriptor" and "instruction descriptor" tables for
// tcgen05.mma (kind::f16).
//
// Every wait on an mbarrier is bounded: after `kSpinLimit` polls it gives up
// and returns false, and the caller records an error instead of hanging.
#pragma once
#include <cstdint>

namespace svmb {
namespace tc {

constexpr unsigned kSpinLimit = 1u << 26;        // polls of an mbarrier before giving up
constexpr uint64_t kWaitNs = 5000000000ull;     // or 5 s of wall time, whichever comes first

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// ---- mbarriers --------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// true once the barrier's phase with the given parity has completed
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// bounded wait (at most kSpinLimit polls and kWaitNs of wall time); false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 1023u) == 1023u && global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// the same, but also gives up as soon as *abort is non-zero (another role of
// the block ran out of time and stopped feeding this barrier)
__device__ __forceinline__ bool mbar_wait_or(uint64_t *bar, unsigned parity, const volatile int *abort)
{
    if (mbar_try(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 255u) == 255u && (*abort != 0 || global_ns() - t0 > kWaitNs)) return false;
    }
    return false;
}

// one arrival (release at CTA scope)
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// ---- proxy / tcgen05 ordering -----------------------------------------------
// generic-proxy writes to shared memory (st.shared, cp.async) -> visible to the
// tensor core's async proxy
__device__ __forceinline__ void fence_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- tensor memory ----------------------------------------------------------
// issued by one full warp; writes the TMEM base address to *dst (shared)
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish()
{
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp receives lane
// (taddr.lane + t), columns taddr.col .. +15
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 8 consecutive 32-bit columns
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float *v)
{
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- descriptors ------------------------------------------------------------
// K-major operand tile with the 128-byte swizzle; atoms of 8 rows are 1024 B apart
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);          // start address
    d |= (uint64_t)1u << 16;                          // leading byte offset (unused with swizzle)
    d |= (uint64_t)(1024u >> 4) << 32;                // stride byte offset: next 8-row atom
    d |= (uint64_t)1u << 46;                          // descriptor version (sm_100)
    d |= (uint64_t)2u << 61;                          // layout: 128-byte swizzle
    return d;
}

// kind::f16 instruction descriptor: A and B both bf16 (or both fp16), f32
// accumulator, both K-major
__host__ __device__ constexpr uint32_t idesc_f16_f32(int M, int N, bool bf16)
{
    return (1u << 4)                           // D format f32
           | ((bf16 ? 1u : 0u) << 7)           // A format: 0 fp16, 1 bf16
           | ((bf16 ? 1u : 0u) << 10)          // B format (same as A)
           | ((uint32_t)(N >> 3) << 17)        // N / 8
           | ((uint32_t)(M >> 4) << 24);       // M / 16
}
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) { return idesc_f16_f32(M, N, true); }
// kind::tf32 instruction descriptor: A and B tf32 (format 2), f32 accumulator, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32_f32(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// the same with tf32 operands (K = 8 per instruction: 32 bytes of a 128-byte row, as for 16-bit types)
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// the mbarrier receives one arrival when every MMA issued so far by this thread has completed
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// ---- cp.async (16-byte pieces, zero fill when src_bytes == 0) ----------------
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void *gptr, uint32_t src_bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(gptr), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
// the same with a run-time count (0..3): at most n of this thread's groups still pending
__device__ __forceinline__ void cp_async_wait_n(int n)
{
    if (n <= 0) cp_async_wait<0>();
    else if (n == 1) cp_async_wait<1>();
    else if (n == 2) cp_async_wait<2>();
    else cp_async_wait<3>();
}

// byte offset of 16-byte piece q (0..7) of row r inside a 128B-swizzled K-major tile
__host__ __device__ __forceinline__ uint32_t sw128_offset(int r, int q)
{
    return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((q ^ (r & 7)) << 4));
}

}  // namespace tc
}  // namespace svmb
