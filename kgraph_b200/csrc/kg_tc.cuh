// Fifth-generation tensor core (tcgen05) building blocks for sm_100a: TMEM
// allocation, shared-memory operand descriptors, the BF16 MMA with an FP32
// accumulator in TMEM, its completion barrier, the TMEM read-back, and the
// tensor-memory-accelerator (TMA) tile loads that feed it.
//
// Two operand layouts are described.
//
// (1) No swizzle, K-major "core matrices", staged by the threads themselves:
// 8 rows x 16 bytes per core matrix; row r, element k of a tile with K columns
// sits at byte (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2 with LBO = 128 (the
// next 8 elements along K) and SBO = K*16 (the next 8 rows).  One MMA consumes
// K = 16 (two core matrices along K); the next K step starts 256 bytes further.
//
// (2) 128-byte swizzle, written by TMA (cp.async.bulk.tensor, tensor map with
// CU_TENSOR_MAP_SWIZZLE_128B, box inner extent 64 BF16 = 128 bytes).  A
// K-major tile is rows x 128 bytes (64 elements of K per row), 8-row groups
// 1024 bytes apart (SBO = 1024; LBO unused); a K = 16 step advances the start
// address by 32 bytes inside the swizzle atom.  An MN-major tile (the operand
// stored K x MN, MN contiguous) is one 64 (MN) x 64 (K) box per 64 columns of
// MN: 64 rows of K x 128 bytes, 8-row groups 1024 bytes apart (SBO), the
// next 64 columns of MN one box (8192 bytes) further (LBO); a K = 16 step
// advances the start address by 2048 bytes.  Tiles start on 1024-byte
// boundaries so the swizzle phase is that of the address.
//
// Descriptor bit layouts follow the sm_100 UMMA descriptors (SmemDescriptor:
// start>>4 @0, LBO>>4 @16, SBO>>4 @32, version 1 @46, layout type @61 (0 no
// swizzle, 2 128-byte swizzle); InstrDescriptor: D format @4, A/B format
// @7/@10, A/B major @15/@16 (1 = MN-major), N>>3 @17, M>>4 @24).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace kgb {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of (row r, element k) in a K-major core-matrix tile of K columns (bf16).
__device__ __forceinline__ uint32_t kmajor_off(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;   // descriptor version for sm_100; base offset 0, no swizzle
    return d;
}

// The same with the 128-byte swizzle layout type.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return smem_desc(saddr, lbo, sbo) | ((uint64_t)2 << 61);
}

// kind::f16 instruction descriptor: BF16 x BF16 -> FP32, both operands K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
// The same with A and / or B MN-major (stored K x M / K x N, MN contiguous).
__host__ __device__ constexpr uint32_t idesc_bf16_f32_major(uint32_t M, uint32_t N, uint32_t a_mn, uint32_t b_mn) {
    return idesc_bf16_f32(M, N) | (a_mn << 15) | (b_mn << 16);
}

// kind::f8f6f4 instruction descriptor: E4M3 x E4M3 (format code 0 for both)
// -> FP32, both operands K-major.  Same bit layout as kind::f16.
__host__ __device__ constexpr uint32_t idesc_e4m3_f32(uint32_t M, uint32_t N) {
    return (1u << 4) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Byte offset of (row r, byte k) in a K-major core-matrix tile whose rows are
// Kb bytes (8-bit elements: byte k is element k).  Same layout as kmajor_off in
// bytes: 8 rows x 16 bytes per core matrix, LBO = 128, SBO = Kb * 8.
__device__ __forceinline__ uint32_t kmajor_off8(uint32_t r, uint32_t k, uint32_t Kb) {
    return (r >> 3) * (Kb * 8) + (k >> 4) * 128 + (r & 7) * 16 + (k & 15);
}

__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Whole warp: allocate `cols` TMEM columns (power of two >= 32); the base
// address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *dst, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One thread: arm *bar for `bytes` of TMA transactions (and arrive once).
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// One thread: a plain arrive on *bar.
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// One thread: TMA load of the box at (x, y) of a 2-D tensor map (a kernel
// parameter declared __grid_constant__) into shared memory at dst; completion
// is counted in bytes on *bar.  This GPU's memory only, no multicast; x times
// the element size is a multiple of 16 bytes at every call site.
__device__ __forceinline__ void tma_load_2d(void *dst, const void *tmap, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// One thread: D[tmem] (+)= A[smem] * B[smem]^T for one K=16 step.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// One thread: D[tmem] (+)= A[smem] * B[smem]^T for one K=32 step of E4M3
// operands (32 bytes of each row: the same 256 bytes of the K-major tile as one
// BF16 step).
__device__ __forceinline__ void mma_e4m3(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// One thread: arrive on *bar when every MMA this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// Bounded wait for phase `parity` of *bar; false when the bound ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit_cycles) {
    const long long t0 = clock64();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (clock64() - t0 > limit_cycles) return false;
    }
}

// Warp: 32 consecutive FP32 columns of this warp's 32 TMEM lanes (lane = row).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace kgb
