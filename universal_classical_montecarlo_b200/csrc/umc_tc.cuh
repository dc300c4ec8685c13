// umc_tc.cuh -- fifth-generation tensor-core primitives (tcgen05, TMEM, mbarrier)
// for the learned proposal's small matrix products on sm_100a.
//
// Operand staging: BF16 operands live in shared memory in the canonical
// K-major, no-swizzle layout the UMMA shared-memory descriptor describes:
// 8 rows x 16 bytes "core matrices" (8 consecutive K elements of 8 rows), with
// the descriptor's leading byte offset (LBO) the distance between core
// matrices adjacent in K and its stride byte offset (SBO) the distance between
// 8-row groups.  Here every operand of R rows stores its core matrices
// K-block-major:
//     byte(r, k) = ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// so LBO = 16 R, SBO = 128, and the operand of the K = 16 step s starts at
// byte 32 R s (rows r0.. of it at + 16 r0).
//
// Accumulators: D = A B^T with A (M x K) and B (N x K) both K-major, FP32 in
// tensor memory: row i of an M = 128 tile is TMEM lane i, column j is column
// base + j.  Warp w of the CTA may read lanes 32 (w % 4) .. 32 (w % 4) + 31, so
// with 128 threads thread t reads row t (tcgen05.ld 32x32b).
//
// Synchronisation (one elected thread issues the MMAs):
//   writers: st.shared; fence.proxy.async.shared::cta; tcgen05.fence::before;
//            barrier
//   issuer : tcgen05.fence::after; tcgen05.mma ...; tcgen05.commit -> mbarrier
//   readers: mbarrier wait (bounded); tcgen05.fence::after; tcgen05.ld;
//            tcgen05.wait::ld
// Every wait has an iteration limit: on expiry it returns false and the
// caller records a status bit and finishes without touching the result.
#pragma once

#include <cstdint>

namespace umc {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) of an operand with R rows (see header).
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t R, uint32_t r, uint32_t k)
{
    return ((k >> 3) * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// UMMA shared-memory descriptor: start >> 4 in [0,14), LBO >> 4 in [16,30),
// SBO >> 4 in [32,46), version 1 in [46,48), base offset 0, layout SWIZZLE_NONE.
__host__ __device__ constexpr uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo)
{
    return uint64_t((start >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Descriptor of K step s of an R-row operand whose first byte is `base`,
// restricted to rows r0 .. (r0 multiple of 8).
__host__ __device__ constexpr uint64_t operand_desc(uint32_t base, uint32_t R, uint32_t s, uint32_t r0 = 0)
{
    return smem_desc(base + 32u * R * s + 16u * r0, 16u * R, 128u);
}

// Instruction descriptor, kind::f16: FP32 accumulate (bits 4-5 = 1), A and B
// BF16 (bits 7-9 = 1, 10-12 = 1), both K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// ---- tensor memory ------------------------------------------------------
// Whole warp; writes the allocated base address to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A B^T, one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate)
{
    const uint32_t acc = accumulate ? 1u : 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrive on the mbarrier once all previously issued MMAs of this thread finish.
__device__ __forceinline__ void mma_commit(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(mbar))
                 : "memory");
}

// ---- mbarrier -------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

constexpr uint32_t kWaitSpins = 1u << 22;

// Waits for the phase with the given parity to complete; false after the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity)
{
    const uint32_t a = smem_addr(mbar);
    for (uint32_t it = 0; it < kWaitSpins; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

// ---- named barriers -----------------------------------------------------------
// Barrier over `count` threads on named barrier `id` (1..15; 0 is
// __syncthreads) that also ORs a predicate over them (bar.red.or).
__device__ __forceinline__ bool bar_or(uint32_t id, uint32_t count, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, %2, %3, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(r)
        : "r"(v ? 1u : 0u), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

// ---- TMEM -> registers ------------------------------------------------------
// 16 consecutive FP32 columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Lane address of this warp's quadrant: lanes 32 (warp % 4) .., column col.
__device__ __forceinline__ uint32_t tmem_lane_addr(uint32_t base, uint32_t col)
{
    const uint32_t quad = (threadIdx.x >> 5) & 3u;
    return base + ((quad * 32u) << 16) + col;
}

}  // namespace tc
}  // namespace umc
