// tcgen05 (5th-generation tensor core) building blocks for sm_100a, written in inline PTX.
//
// One CTA of 128 threads owns a 128-row tile.  Operands live in shared memory in the
// K-major, no-swizzle canonical UMMA layout: the tile is cut into 8-element (16-byte) K
// chunks; chunk c of all R rows forms a block of R x 16 bytes made of 8-row x 16-byte core
// matrices (128 contiguous bytes each), consecutive 8-row groups 128 bytes apart.  Chunk
// blocks are consecutive, so
//     byte offset(row, k) = (k / 8) * (R * 16) + (row / 8) * 128 + (row % 8) * 16 + (k % 8) * 2
// and the shared-memory descriptor of one K=16 MMA step s uses start = base + 2 s (R * 16),
// leading-byte offset (between the two K chunks) = R * 16 and stride-byte offset (between
// 8-row groups) = 128.  The accumulator D (128 x N FP32) lives in tensor memory: row r is TMEM
// lane r, column j is TMEM column base + j, so thread r of the CTA (warp r / 32) reads its own
// row with tcgen05.ld.32x32b.
//
// Descriptor bit layouts follow the sm100 UMMA definitions (shared-memory descriptor: start
// address >> 4 in bits 0-13, leading byte offset >> 4 in 16-29, stride byte offset >> 4 in
// 32-45, version 1 in 46-47, layout type in 61-63 with 0 = no swizzle; instruction
// descriptor for kind::f16: D format bits 4-5 (1 = F32), A/B format bits 7-9 / 10-12
// (1 = BF16), K-major A and B (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in 24-28).
#ifndef CLOTHSTEP_TC_CUH
#define CLOTHSTEP_TC_CUH

#include <cuda_bf16.h>
#include <stdint.h>

namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, k) in a K-major no-swizzle tile with R rows.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int R, int row, int k) {
    return (uint32_t)((k >> 3) * (R * 16) + (row >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((start >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // version 1 (sm100)
    // base offset 0, lbo mode 0, layout type 0 (no swizzle)
    return d;
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128.
__host__ __device__ __forceinline__ uint32_t idesc_bf16_f32(int M, int N) {
    uint32_t d = 0;
    d |= 1u << 4;                        // D format F32
    d |= 1u << 7;                        // A format BF16
    d |= 1u << 10;                       // B format BF16
    d |= ((uint32_t)(N >> 3) & 0x3Fu) << 17;
    d |= ((uint32_t)(M >> 4) & 0x1Fu) << 24;
    return d;
}

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by warp 0; the address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait on an mbarrier phase; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t max_tries = 1u << 20) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t i = 0; i < max_tries; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// D (+)= A x B^T for one K = 16 step; issued by a single thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives on `bar` once all previously issued MMAs of this thread have completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// Issues the K/16 MMAs of D[128 x N] (+)= A[128 x K] B[N x K]^T for K-major tiles at a_base
// (128 rows) and b_base (N rows).  Single thread.
__device__ __forceinline__ void gemm_tile(uint32_t tmem_d, uint32_t a_base, uint32_t b_base, int K, int N,
                                          bool accumulate) {
    const uint32_t idesc = idesc_bf16_f32(128, N);
    const uint32_t a_lbo = 128 * 16, b_lbo = (uint32_t)N * 16;
    for (int s = 0; s < K / 16; s++) {
        uint64_t ad = smem_desc(a_base + 2u * s * a_lbo, a_lbo, 128);
        uint64_t bd = smem_desc(b_base + 2u * s * b_lbo, b_lbo, 128);
        mma_bf16(tmem_d, ad, bd, idesc, (accumulate || s > 0) ? 1u : 0u);
    }
}

// Loads 16 consecutive FP32 columns of this thread's TMEM lane (row).
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

// TMEM address of (lane = 32 * warp, column col) relative to the allocation base.
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int warp, int col) {
    return base + ((uint32_t)(32 * warp) << 16) + (uint32_t)col;
}

__device__ __forceinline__ void st_bf16(unsigned char* tile, int R, int row, int k, float v) {
    *reinterpret_cast<__nv_bfloat16*>(tile + kmajor_offset(R, row, k)) = __float2bfloat16_rn(v);
}

}  // namespace tc

#endif
