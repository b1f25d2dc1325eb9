// Minimal sm_100a tensor-core helpers (tcgen05 + TMEM) for single-CTA bf16
// GEMM tiles whose operands live in shared memory in the canonical
// no-swizzle layout:
//
//   K-major operand (rows x K): 8-row x 16-byte core matrices; element
//   (r, k) at (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
//   bytes. Our buffers use LBO = 128 (the 8-column chunks of one 8-row
//   group are contiguous) and SBO = 1024 for 64-column matrices.
//
//   The same bytes read as an MN-major operand (MN = the column index,
//   K = the row index) have 8-element MN groups 128 bytes apart and 8-row K
//   groups 1024 bytes apart: descriptor SBO = 128, LBO = 1024. This is how
//   the backward GEMMs read transposed operands without a transposed copy.
//
// One elected thread issues tcgen05.mma; completion is signalled by
// tcgen05.commit on an mbarrier that every thread waits on (with an
// iteration bound), after which accumulators are read with tcgen05.ld.
#pragma once

#include <cstdint>

namespace yrc {
namespace umma {

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1 (sm_100), no swizzle.
__device__ __forceinline__ uint64_t Desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Instruction descriptor of kind::f16: bf16 A and B, fp32 accumulator,
// M x N tile, K-major (false) or MN-major (true) operands.
__host__ __device__ constexpr uint32_t IDesc(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void Mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

__device__ __forceinline__ void Commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(SmemAddr(mbar))
                 : "memory");
}

// Initialises an mbarrier and makes the initialisation visible to the
// tensor core's arrive (tcgen05.commit).
__device__ __forceinline__ void MbarInit(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the mbarrier phase with the given parity; gives up after
// `max_tries` polls and returns false.
__device__ __forceinline__ bool MbarWait(uint64_t* mbar, uint32_t parity, uint32_t max_tries) {
    const uint32_t addr = SmemAddr(mbar);
    for (uint32_t i = 0; i < max_tries; ++i) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void FenceBeforeSync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void FenceAfterSync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes this thread's st.shared visible to the tensor core (async proxy).
__device__ __forceinline__ void FenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Warp-wide TMEM allocation of `ncols` columns (power of two >= 32); the
// base address is written to shared memory.
__device__ __forceinline__ void TmemAlloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(SmemAddr(smem_dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void TmemFree(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this warp's 32 TMEM lanes (one per thread).
__device__ __forceinline__ void Ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void WaitLd() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of element (row, col) of a 64-column bf16 matrix in the
// canonical K-major layout (LBO 128, SBO 1024).
__host__ __device__ constexpr uint32_t Canon64(int row, int col) {
    return static_cast<uint32_t>((row >> 3) * 1024 + (col >> 3) * 128 + (row & 7) * 16 + (col & 7) * 2);
}

}  // namespace umma
}  // namespace yrc
