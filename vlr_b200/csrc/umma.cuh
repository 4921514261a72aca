// Thin device helpers for the sm_100a tensor-core path (tcgen05.* PTX):
// shared-memory matrix descriptors, the kind::f16 instruction descriptor,
// TMEM allocation, MMA issue/commit, and TMEM loads.
//
// Operand tiles live in shared memory in the no-swizzle ("interleave")
// canonical layout, built from 8-row x 16-byte core matrices.  The tiles this
// project writes are "chunk-major": for a tile of R rows and C bf16 columns,
// element (r, c) sits at
//     (c / 8) * (R * 16) + r * 16 + (c % 8) * 2        bytes,
// i.e. every 8-column chunk is a contiguous R x 16 B block.  The same bytes
// can be read by the MMA in two ways:
//   K-major  (rows = M or N, columns = K):  SBO = 128 (next 8 rows),
//            LBO = R * 16 (next 8 columns of K);
//   MN-major (rows = K, columns = M or N):  LBO = 128 (next 8 rows of K),
//            SBO = R * 16 (next 8 columns of M/N).
// That lets an activation tile written once for the forward product serve as
// the transposed operand of the weight-gradient product.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace vlrb {
namespace umma {

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all >> 4), descriptor version 1 at bits 46-47.
__device__ __forceinline__ uint64_t smemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;   // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor for kind::f16 with BF16 A/B and FP32 accumulation.
// aMN / bMN select the MN-major reading of the operand.
__host__ __device__ constexpr uint32_t instrDescBf16(uint32_t M, uint32_t N, bool aMN, bool bMN) {
    return (1u << 4)                       // D format: F32
         | (1u << 7)                       // A format: BF16
         | (1u << 10)                      // B format: BF16
         | ((aMN ? 1u : 0u) << 15)
         | ((bMN ? 1u : 0u) << 16)
         | ((N >> 3) << 17)
         | ((M >> 4) << 24);
}

// D[tmem] (+)= A * B for one K = 16 step, issued by a single thread.
__device__ __forceinline__ void mmaBf16(uint32_t tmemD, uint64_t aDesc, uint64_t bDesc, uint32_t idesc,
                                        bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :: "r"(tmemD), "l"(aDesc), "l"(bDesc), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

// Arrive on an mbarrier once every MMA this thread issued so far completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smemAddr(mbar)) : "memory");
}

__device__ __forceinline__ void mbarInit(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smemAddr(mbar)), "r"(count) : "memory");
}

__device__ __forceinline__ uint64_t globalTimerNs() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for phase `parity` of the mbarrier to complete: gives up after
// `limitNs` nanoseconds and returns false (the caller records the error and
// skips the dependent work).
__device__ __forceinline__ bool mbarWait(uint64_t* mbar, uint32_t parity, uint64_t limitNs = 1000000000ull) {
    const uint32_t a = smemAddr(mbar);
    const uint64_t t0 = globalTimerNs();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
        if (globalTimerNs() - t0 > limitNs) return false;
    }
}

// Generic-proxy shared-memory writes -> visible to the tensor core.
__device__ __forceinline__ void fenceProxyAsync() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fenceBeforeSync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fenceAfterSync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM allocation by one full warp; the base address lands in *dst (shared).
__device__ __forceinline__ void tmemAlloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smemAddr(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemFree(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: the
// warp reads its own 32-lane sub-partition, thread t gets lane base + t).
__device__ __forceinline__ void tmemLoad16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// TMEM address of (lane, column).
__device__ __forceinline__ uint32_t tmemAt(uint32_t base, uint32_t lane, uint32_t col) {
    return base + (lane << 16) + col;
}

// Byte offset of element (r, c) in a chunk-major bf16 tile of R rows.
__host__ __device__ constexpr uint32_t chunkOffset(uint32_t R, uint32_t r, uint32_t c) {
    return (c >> 3) * (R * 16u) + r * 16u + (c & 7u) * 2u;
}

// Descriptors of a chunk-major tile with R rows, advanced to K step `ks`
// (16 columns per step for the K-major reading, 16 rows for the MN-major one).
__device__ __forceinline__ uint64_t descKMajor(uint32_t tileAddr, uint32_t R, uint32_t ks) {
    return smemDesc(tileAddr + ks * 2u * R * 16u, R * 16u, 128u);
}
__device__ __forceinline__ uint64_t descMNMajor(uint32_t tileAddr, uint32_t R, uint32_t ks) {
    return smemDesc(tileAddr + ks * 256u, 128u, R * 16u);
}

} // namespace umma
} // namespace vlrb
