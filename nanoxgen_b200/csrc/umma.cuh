// umma.cuh -- the sm_100a tensor-core primitives the surrogate kernels use:
// TMEM allocation, tcgen05.mma (kind::f16, BF16 x BF16 -> FP32) with both
// operands in shared memory, tcgen05.commit to an mbarrier, tcgen05.ld of
// the FP32 accumulator, and the proxy / thread-sync fences between them.
//
// Shared-memory operands use the SWIZZLE_NONE canonical layout: "core
// matrices" of 8 rows x 16 bytes stored as 128 contiguous bytes.  One tile
// of R rows and K columns (bf16) is stored K-chunk-outer:
//   offset(r, k) = ((k / 8) * (R / 8) + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2
// Read along k it is a K-major operand (8-row groups 128 B apart, the two
// 8-column chunks of one K=16 step R*16 B apart); read along r it is an
// MN-major operand of the transposed matrix (8-element groups of the
// columns R*16 B apart, 8-row K groups 128 B apart).  The same buffer thus
// serves the forward product and the weight-gradient product.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace nxg {
namespace umma {

__device__ __forceinline__ uint32_t tile_offset(uint32_t r, uint32_t k, uint32_t rows) {
    return ((k >> 3) * (rows >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_address(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm_100 format: start >> 4 in bits 0-13,
// leading byte offset >> 4 in 16-29, stride byte offset >> 4 in 32-45,
// version 1 in bits 46-47, base offset 0, no swizzle).
__device__ __forceinline__ uint64_t descriptor(uint32_t address, uint32_t leading_bytes, uint32_t stride_bytes) {
    return static_cast<uint64_t>((address >> 4) & 0x3fffu) |
           (static_cast<uint64_t>((leading_bytes >> 4) & 0x3fffu) << 16) |
           (static_cast<uint64_t>((stride_bytes >> 4) & 0x3fffu) << 32) | (uint64_t{1} << 46);
}

// K-major operand of a tile with `rows` rows, K-step `step` (16 columns).
__device__ __forceinline__ uint64_t kmajor(uint32_t base, uint32_t rows, uint32_t step) {
    const uint32_t chunk = rows * 16u;  // bytes between 8-column chunks
    return descriptor(base + step * 2u * chunk, chunk, 128u);
}

// MN-major operand read from a tile of `rows` rows: the operand's K runs
// along the tile's rows, its M/N along the tile's columns.  K-step `step`
// covers tile rows 16*step .. 16*step+15.
__device__ __forceinline__ uint64_t mnmajor(uint32_t base, uint32_t rows, uint32_t step) {
    return descriptor(base + step * 256u, 128u, rows * 16u);
}

// Instruction descriptor: D F32, A and B BF16, operand majorness, N, M.
__host__ __device__ constexpr uint32_t instr_bf16(uint32_t m, uint32_t n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn) << 15) |
           (static_cast<uint32_t>(b_mn) << 16) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t instr, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(instr), "r"(accumulate)
        : "memory");
}

// Arrives once on `bar` when every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_address(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes become visible to the tensor cores.
__device__ __forceinline__ void fence_shared_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Whole warp: allocates `columns` TMEM columns (power of two >= 32) and
// writes the base address to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t columns) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_address(slot)), "r"(columns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t address, uint32_t columns) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(address), "r"(columns) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w .. 32w+31); the wait is tied to the registers so no use can move above it.
__device__ __forceinline__ void load16(uint32_t address, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(address)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) { v[i] = __uint_as_float(r[i]); }
}

__device__ __forceinline__ void load2(uint32_t address, float &a, float &b) {
    uint32_t r0, r1;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : "=r"(r0), "=r"(r1) : "r"(address) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" : "+r"(r0), "+r"(r1) : : "memory");
    a = __uint_as_float(r0);
    b = __uint_as_float(r1);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_address(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(smem_address(bar)), "r"(parity)
        : "memory");
    return done != 0u;
}

// Bounded wait for the phase with the given parity; false when the limit
// runs out (the caller records an error and stops issuing work).
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (uint32_t i = 0; i < kWaitLimit; ++i) {
        if (mbar_try_wait(bar, parity)) { return true; }
    }
    return false;
}

} // namespace umma
} // namespace nxg
