// tc_umma.cuh -- fifth-generation tensor-core (tcgen05) building blocks for
// sm_100a, written as inline PTX: tensor-memory allocation, shared-memory
// matrix descriptors, kind::f16 MMAs with FP32 accumulators in tensor
// memory, commit/mbarrier completion and tensor-memory loads.
//
// Operand layout: K-major, no swizzle ("interleaved" canonical layout).  The
// unit is a core matrix of 8 rows x 16 bytes (8 fp16 along K) stored as 128
// contiguous bytes.  For a tile of R rows and K columns (R % 8 == 0,
// K % 16 == 0) the byte offset of element (r, k) is
//     (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2,
// SBO = (K / 8) * 128: the K-adjacent core matrices of one 8-row group are
// contiguous (leading byte offset 128), the row groups follow each other.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace negf {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Byte offset of element (r, k) of a K-major operand tile with K columns.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor (64 bits): start address >> 4 in [0,14),
// leading byte offset >> 4 in [16,30), stride byte offset >> 4 in [32,46),
// descriptor version 1 in [46,48), base offset 0, layout type 0 (no swizzle)
// in [61,64).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::f16 with fp16 A and B, FP32 accumulator,
// both operands K-major: D format F32 (1) in [4,6), A/B format F16 (0) in
// [7,10) / [10,13), negate A in bit 13, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ __forceinline__ uint32_t idesc_f16(int M, int N, bool neg_a) {
    return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24) | (neg_a ? (1u << 13) : 0u);
}

// ------------------------------------------------------------ tensor memory
// Allocation and release are warp-wide (.sync.aligned): call from one whole
// warp.  The allocated base address is written to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}
// Generic-proxy shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, one thread issues.  accumulate = 0
// overwrites D.
__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// The mbarrier at `bar` receives one arrival when every MMA issued so far by
// this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// ------------------------------------------------------------------ mbarrier
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_u32(bar)));
}
// Waits for the phase with the given parity to complete, at most `limit`
// polls.  Returns false if it gave up (the caller records an error).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ------------------------------------------------------------ tensor loads
// 32 lanes x 16 consecutive 32-bit columns: thread t of the warp receives
// row (lane base + t), columns [col, col+16).  The warp may only address the
// 32 lanes of its sub-partition: lanes 32 * (warp % 4) ...
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
        "[%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// ------------------------------------------------------- split fp16 operands
// x = 2^e (hi + lo) with hi = fp16(x 2^-e), lo = fp16(x 2^-e - hi): 22
// significant bits.  The exponent e is chosen per row of A and per column of
// B so that the largest magnitude maps into [2^14, 2^15) (fp16 overflows at
// 65520).  e is clamped to [-60, 60], so that a row exponent plus a column
// exponent is a normal float's exponent and an epilogue rescales with one
// multiply (rows above 2^74 or below 2^-46 lie far outside the range of these
// Green's functions; for them the clamp only costs fp16 range).
__device__ __forceinline__ int scale_exponent(float maxabs) {
    if (!(maxabs > 0.0f)) return 0;
    const int ex = (int)((__float_as_uint(maxabs) >> 23) & 0xFF) - 127;  // floor(log2) for normals
    const int e = ex - 14;
    return e < -60 ? -60 : (e > 60 ? 60 : e);
}
__device__ __forceinline__ float exp2i(int e) { return __uint_as_float((uint32_t)(e + 127) << 23); }

struct Split2 {
    __half hi, lo;
};
__device__ __forceinline__ Split2 split_fp16(float xs) {
    Split2 s;
    s.hi = __float2half_rn(xs);
    s.lo = __float2half_rn(xs - __half2float(s.hi));
    return s;
}

}  // namespace tc
}  // namespace negf
