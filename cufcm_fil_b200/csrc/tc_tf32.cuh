// tc_tf32.cuh -- 5th-generation tensor-core building blocks for FP32-accurate tile
// products on sm_100a: D (FP32, in tensor memory) = A^T B with A, B given as
// FP32 tiles [K][M] and [K][N] (the operands of the line patches' blocked
// Gauss-Jordan update), evaluated as three TF32 products
//   A^T B ~ Ahi^T Bhi + Ahi^T Blo + Alo^T Bhi,   a = ahi + alo, ahi = tf32(a),
// which keeps ~22 bits of each product (FP32 has 24), accumulated in FP32.
//
// Operands sit in shared memory in the canonical K-major layout without
// swizzling: 8 rows x 16 bytes (4 TF32 along K) per core matrix, the K chunks
// of one group of 8 rows next to each other (leading byte offset 128 B), the
// groups of 8 rows 2048 B apart (stride byte offset) for K = 64.  One thread
// issues tcgen05.mma (kind::tf32, cta_group::1, M = 64, N = 64, K = 8 per
// instruction) and commits to an mbarrier; the accumulator rows are read back
// with tcgen05.ld (row m of an M = 64 tile lives in TMEM lane (m % 16) + 32 (m / 16)).
#pragma once

#include <cstdint>

#include "tma.cuh"

namespace cufil {
namespace tc {

constexpr int kTileK = 64;                   // K of one tile product
constexpr int kTileMN = 64;                  // M = N = 64
constexpr int kOperandFloats = kTileMN * kTileK;  // 4096 floats = 16 KB per operand part
constexpr uint32_t kTmemCols = 64;           // FP32 accumulator columns

// Index (in floats) of element (mn, k) of a 64 x 64 operand in the canonical K-major layout.
__host__ __device__ constexpr int canon(int mn, int k) { return (mn & 7) * 4 + (k & 3) + (k >> 2) * 32 + (mn >> 3) * 512; }

// The inverse map: row (m or n) and k of the element at canonical index q.
__host__ __device__ constexpr int canon_mn(int q) { return (q >> 9) * 8 + ((q & 31) >> 2); }
__host__ __device__ constexpr int canon_k(int q) { return ((q & 511) >> 5) * 4 + (q & 3); }

// FP32 -> (TF32 high part rounded to nearest, FP32 remainder).
__device__ __forceinline__ void split_tf32(float a, float &hi, float &lo) {
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(a));
    hi = __uint_as_float(h);
    lo = a - hi;
}

// Shared-memory matrix descriptor: start address, leading byte offset 128, stride byte offset 2048,
// descriptor version 1, no swizzle (all offsets in 16-byte units).
__device__ __forceinline__ uint64_t smem_desc(const float *p) {
    const uint64_t addr = (static_cast<uint64_t>(smem_u32(p)) >> 4) & 0x3FFFull;
    return addr | (static_cast<uint64_t>(128 >> 4) << 16) | (static_cast<uint64_t>(2048 >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, TF32 A and B, both K-major, N = 64, M = 64.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((64u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdescTf32), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// The three TF32 products of one 64 x 64 x 64 tile (8 K steps of 8, 32 bytes of K per step, i.e. two
// 128-byte K chunks: the start addresses advance by 256 bytes).  Issued by one thread.
__device__ __forceinline__ void issue_tile_products(uint32_t tmem_d, const float *ahi, const float *alo,
                                                    const float *bhi, const float *blo) {
    const uint64_t dah = smem_desc(ahi), dal = smem_desc(alo), dbh = smem_desc(bhi), dbl = smem_desc(blo);
#pragma unroll
    for (int s = 0; s < kTileK / 8; ++s) {
        const uint64_t o = static_cast<uint64_t>(s) * (256 >> 4);
        mma_tf32(tmem_d, dal + o, dbh + o, s > 0 ? 1u : 0u);
        mma_tf32(tmem_d, dah + o, dbl + o, 1u);
        mma_tf32(tmem_d, dah + o, dbh + o, 1u);
    }
}

// BF16 operands (kind::f16): 8 rows x 16 bytes (8 BF16 along K) per core matrix, the K chunks of a group of
// 8 rows 128 B apart, the groups 1024 B apart (K chunk of 64); element (mn, k) at canon16(mn, k).
__host__ __device__ constexpr int canon16(int mn, int k) { return (mn & 7) * 8 + (k & 7) + (k >> 3) * 64 + (mn >> 3) * 512; }

__device__ __forceinline__ uint64_t smem_desc16(const void *p) {
    const uint64_t addr = (static_cast<uint64_t>(smem_u32(p)) >> 4) & 0x3FFFull;
    return addr | (static_cast<uint64_t>(128 >> 4) << 16) | (static_cast<uint64_t>(1024 >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 32, M = 128.
constexpr uint32_t kIdescBf16 = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(kIdescBf16), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// Arrives on `bar` once every tcgen05.mma this thread issued has completed.
__device__ __forceinline__ void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy writes to shared memory become visible to the tensor core.
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Allocation by one whole warp; the base address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

// 32 consecutive accumulator columns of this thread's TMEM lane (warp-wide).
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// TMEM address of the accumulator columns [col0, col0 + 32) for the lanes of warp w's sub-partition.
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int warp, int col0) {
    return base + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + static_cast<uint32_t>(col0);
}

}  // namespace tc
}  // namespace cufil
