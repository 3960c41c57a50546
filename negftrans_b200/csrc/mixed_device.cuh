// mixed_device.cuh -- device building blocks of the mixed-precision RGF path:
// complex products on the tcgen05 tensor cores in split fp16 with FP32
// accumulation, and the FP32 blocked Gauss-Jordan inverse whose trailing
// updates use them.
//
// Complex product C = W * B (W: rows x K, B: K x cols).  Every operand value
// x is stored as 2^e (hi + lo), hi = fp16(x 2^-e), lo = fp16(x 2^-e - hi),
// with one exponent e per row of W and one per column of B (chosen so the
// largest magnitude of the row / column maps into [2^14, 2^15)).  Three
// split products hi*hi + hi*lo + lo*hi keep ~2^-21 of the normwise accuracy
// (lo*lo is below that); fp16 products are exact and accumulate in FP32 in
// tensor memory.  The complex product is four real MMAs into separate real
// and imaginary accumulators: re += Wr Br, re += (-Wi) Bi (negated A
// operand, no negated copy in shared memory), im += Wr Bi, im += Wi Br.
// Unit of work: one 128-row tile of C x TN columns, K in chunks of KB = 32.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tc_umma.cuh"

namespace negf {
namespace mx {

constexpr int NT = 256;       // threads per CTA
constexpr int NWARP = NT / 32;
constexpr int TM = 128;       // rows of an MMA tile (tensor-memory lanes)
constexpr int KB = 32;        // K of one staged chunk = panel width of the inverse
constexpr int TN = 64;        // columns of C per tile
constexpr uint32_t WAIT_LIMIT = 1u << 26;  // mbarrier polls before a wait gives up

// ------------------------------------------------------------ complex FP32
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {  // c + a b
    c.x = fmaf(a.x, b.x, c.x);
    c.x = fmaf(-a.y, b.y, c.x);
    c.y = fmaf(a.x, b.y, c.y);
    c.y = fmaf(a.y, b.x, c.y);
    return c;
}
__device__ __forceinline__ float2 cfms(float2 a, float2 b, float2 c) {  // c - a b
    c.x = fmaf(-a.x, b.x, c.x);
    c.x = fmaf(a.y, b.y, c.x);
    c.y = fmaf(-a.x, b.y, c.y);
    c.y = fmaf(-a.y, b.x, c.y);
    return c;
}
// 1/a in FP64 arithmetic, rounded once (pivots can be small and |a|^2 may
// underflow in FP32)
__device__ __forceinline__ float2 crcp(float2 a) {
    const double x = a.x, y = a.y, s = 1.0 / (x * x + y * y);
    return make_float2((float)(x * s), (float)(-y * s));
}
// 1/a in FP32 with a power-of-two prescale, so |a|^2 neither overflows nor
// underflows: a = 2^e (u + i v) with max(|u|, |v|) in [1, 2), 1/a =
// 2^-e (u - i v) / (u^2 + v^2); a few ulp.  Zero or non-finite a gives a
// non-finite result.
__device__ __forceinline__ float2 crcp_f32(float2 a) {
    const int eb = (__float_as_int(fmaxf(fabsf(a.x), fabsf(a.y))) >> 23) & 0xff;
    const float sc = __int_as_float((254 - min(max(eb, 1), 253)) << 23);  // 2^(127 - eb)
    const float u = a.x * sc, v = a.y * sc;
    const float r = __frcp_rn(fmaf(u, u, v * v)) * sc;
    return make_float2(u * r, -v * r);
}
__device__ __forceinline__ float cabs1f(float2 a) { return fabsf(a.x) + fabsf(a.y); }

// ------------------------------------------------------- tile shared memory
// sa[0..3]: W tile (TM x KB) re_hi, re_lo, im_hi, im_lo; sb[0..3]: B tile
// (TN x KB, K-major: one row per output column).  rexp / cexp: exponents.
struct TileSmem {
    __half *sa[4];
    __half *sb[4];
    int *rexp;   // [TM]
    int *cexp;   // [TN]
    uint64_t *bar;
    uint32_t *tslot;
};
__host__ __device__ constexpr size_t tile_smem_bytes() {
    return 4 * (size_t)TM * KB * 2 + 4 * (size_t)TN * KB * 2 + TM * 4 + TN * 4 + 16 + 16;
}
// base must be 128-byte aligned
__device__ inline TileSmem carve_tile(unsigned char *base) {
    TileSmem t;
    unsigned char *p = base;
    for (int q = 0; q < 4; ++q) { t.sa[q] = (__half *)p; p += (size_t)TM * KB * 2; }
    for (int q = 0; q < 4; ++q) { t.sb[q] = (__half *)p; p += (size_t)TN * KB * 2; }
    t.rexp = (int *)p; p += TM * 4;
    t.cexp = (int *)p; p += TN * 4;
    t.bar = (uint64_t *)p; p += 16;
    t.tslot = (uint32_t *)p;
    return t;
}

// Store 8 consecutive K values (already scaled) of row r of a tile as the
// four split planes.  k8 = index of the 8-wide K group.
__device__ __forceinline__ void store_split8(__half *const (&dst)[4], int r, int k8, const float2 (&v)[8]) {
    __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const tc::Split2 a = tc::split_fp16(v[q].x), b = tc::split_fp16(v[q].y);
        rh[q] = a.hi; rl[q] = a.lo; ih[q] = b.hi; il[q] = b.lo;
    }
    const uint32_t off = tc::kmajor_offset(r, 8 * k8, KB);
    *(uint4 *)((unsigned char *)dst[0] + off) = *(const uint4 *)rh;
    *(uint4 *)((unsigned char *)dst[1] + off) = *(const uint4 *)rl;
    *(uint4 *)((unsigned char *)dst[2] + off) = *(const uint4 *)ih;
    *(uint4 *)((unsigned char *)dst[3] + off) = *(const uint4 *)il;
}

// Issue the MMAs of one staged K chunk (thread 0 only).  D: re at column
// tcol, im at tcol + TN.  first = overwrite the accumulators.
__device__ inline void issue_chunk(const TileSmem &t, uint32_t tbase, bool first) {
    constexpr uint32_t SBO = (KB / 8) * 128, LBO = 128;
    const uint32_t id = tc::idesc_f16(TM, TN, false), idn = tc::idesc_f16(TM, TN, true);
    const uint32_t dre = tbase, dim = tbase + TN;
    uint32_t a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) { a[q] = tc::smem_u32(t.sa[q]); b[q] = tc::smem_u32(t.sb[q]); }
    // split pairs (A part, B part): hi*hi, hi*lo, lo*hi
    const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
#pragma unroll
    for (int ks = 0; ks < KB / 16; ++ks) {
        const uint32_t koff = ks * 256;  // two core matrices along K per K16 step
#pragma unroll
        for (int s = 0; s < 3; ++s) {
            const uint64_t are = tc::sdesc(a[0 + pa[s]] + koff, LBO, SBO);
            const uint64_t aim = tc::sdesc(a[2 + pa[s]] + koff, LBO, SBO);
            const uint64_t bre = tc::sdesc(b[0 + pb[s]] + koff, LBO, SBO);
            const uint64_t bim = tc::sdesc(b[2 + pb[s]] + koff, LBO, SBO);
            const uint32_t acc = (first && ks == 0 && s == 0) ? 0u : 1u;
            tc::mma_f16(dre, are, bre, id, acc);
            tc::mma_f16(dre, aim, bim, idn, 1u);
            tc::mma_f16(dim, are, bim, id, acc);
            tc::mma_f16(dim, aim, bre, id, 1u);
        }
    }
}

// Waits for the MMAs committed to t.bar (parity ph) in every thread; on
// timeout sets *err (the caller stops and releases tensor memory).
__device__ __forceinline__ void wait_mma(const TileSmem &t, uint32_t &ph, int *err) {
    if (!tc::mbar_wait(t.bar, ph, WAIT_LIMIT)) *err = 1;
    ph ^= 1u;
    tc::fence_after_sync();
}

// Tensor-memory setup / teardown (warp 0 allocates; 2*TN columns).
__device__ inline uint32_t tile_setup(const TileSmem &t) {
    if (threadIdx.x < 32) tc::tmem_alloc(t.tslot, 2 * TN);
    if (threadIdx.x == 0) tc::mbar_init(t.bar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    return *t.tslot;
}
__device__ inline void tile_teardown(const TileSmem &t, uint32_t tbase) {
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(tbase, 2 * TN);
    if (threadIdx.x == 0) tc::mbar_inval(t.bar);
}

// Reads the accumulators of this thread's tile row into re[16], im[16] for
// the 16 columns [c16*16, c16*16+16).  Warps w and w+4 share lanes
// 32*(w%4)..; the caller splits the column groups between them.
__device__ __forceinline__ void load_acc16(uint32_t tbase, int c16, float (&re)[16], float (&im)[16]) {
    const int warp = threadIdx.x >> 5;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    tc::tmem_ld16(tbase + lane_base + c16 * 16, re);
    tc::tmem_ld16(tbase + lane_base + TN + c16 * 16, im);
    tc::tmem_wait_ld();
}

}  // namespace mx
}  // namespace negf
