// negf_mixed.cu -- mixed-precision RGF transmission on sm_100a.
//
// The FP64 path (negf_engine.cu) inverts every Schur complement in complex
// FP64 on the FP64 tensor cores.  Here the same sweep (math_kernel.f90:81-128
// restated as a right-connected factorization) runs with
//   * the Schur complement S = D_k - gR(k) formed in FP64 and rounded to
//     complex FP32 (D_k generated on chip from the V table, grid.f90:236-333);
//   * its inverse by blocked Gauss-Jordan with partial pivoting: 32-column
//     panels eliminated in FP32 registers, rank-32 trailing updates on the
//     tcgen05 tensor cores in split fp16 with FP32 accumulation
//     (mixed_device.cuh);
//   * every generator gR(k) kept in HBM (complex FP32),
// followed by one step of iterative refinement of the columns the
// transmission trace reads: with x0 the first block column G(:,1) restricted
// to the open channels of the right lead computed from the stored factors,
// the residual r = E_1 - A x0 of the whole block-tridiagonal system is formed
// in FP64 (A generated in FP64), the correction d = A_lo^-1 r is applied with
// the stored factors, and tau (grid.f90:362-383) is evaluated from
// x0 + d in FP64.  Jobs whose correction is not small enough, and jobs the
// policy sends there (near a subband threshold, small eta), are re-run by the
// FP64 path.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "engine_internal.h"
#include "mixed_device.cuh"
#include "negf_gpu.h"
#include "rgf_device.cuh"

using namespace negf::mx;
namespace tc = negf::tc;

namespace {

// ------------------------------------------------------------ shared memory
// Per-CTA state of the FP32 Gauss-Jordan inverse.
struct GjSmem {
    int *prow;       // [N] row permutation of the stored factors (the identity here)
    int *iprow;      // [N] its inverse
    float2 *sP;      // [32][32] inverse of the current diagonal block, P(r, c) at r * 32 + c
    int *spr;        // [32] pivot lane of each step of the diagonal-block inverse
    float2 *srow;    // [2][32] the pivot row of a step, double-buffered by step parity
    float *rmax;     // [2][TM]  per-thread-half row maxima while staging W (self test)
};
__host__ __device__ inline int rup(int a, int b) { return (a + b - 1) / b * b; }
__host__ __device__ inline size_t gj_smem_bytes(int N) {
    const int n4 = rup(N, 4);
    size_t b = 32 * 32 * 8 + 32 * 4 + 2 * 32 * 8 + 2 * TM * 4;
    b += 2 * (size_t)n4 * 4;
    return (b + 127) / 128 * 128;
}
__device__ inline GjSmem carve_gj(unsigned char *base, int N) {
    GjSmem s;
    const int n4 = rup(N, 4);
    s.sP = (float2 *)base;
    s.srow = s.sP + 32 * 32;
    s.spr = (int *)(s.srow + 2 * 32);
    s.rmax = (float *)(s.spr + 32);
    s.prow = (int *)(s.rmax + 2 * TM);
    s.iprow = s.prow + n4;
    return s;
}
__device__ inline void gj_identity(const GjSmem &s, int N) {
    for (int i = threadIdx.x; i < N; i += NT) { s.prow[i] = i; s.iprow[i] = i; }
}

// ------------------------------------------------------------ job teams
// The CTAs that share one job: a thread-block cluster of n = 1 or 2 CTAs.
// With n = 2 the rows of every per-row phase and the output tiles of every
// trailing update are split between the two, and the phases are separated
// by cluster barriers (release / acquire at cluster scope, so the global
// writes of one CTA are visible to the other after it).  Loads of the shared
// working matrix go through L2 (ld.global.cg): its lines may have been
// rewritten by the other SM since this SM's L1 last held them.
struct Team {
    int rank, n;
    int *gx;        // per-job global exponents (n > 1): rexpW [ntr * TM], then cexpB [ntc * PTN]
    int *slot;      // shared [2]: this CTA's contribution to team_or, by call parity
    uint32_t par;
};
__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void team_sync(const Team &t) {
    if (t.n > 1) cluster_sync();
    else __syncthreads();
}
// OR of a CTA-uniform flag over the team; every thread of both CTAs calls it
// at the same point and gets the same result.  The slot of a parity is
// rewritten two calls later, after the peer has passed the barrier between.
__device__ inline int team_or(Team &t, int v) {
    if (t.n == 1) return v;
    int *sl = t.slot + (t.par & 1u);
    if (threadIdx.x == 0) *sl = v;
    cluster_sync();
    int r = 0;
    for (int q = 0; q < t.n; ++q) {
        uint32_t ra;
        int x;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(ra) : "r"(tc::smem_u32(sl)), "r"(q));
        asm volatile("ld.shared::cluster.s32 %0, [%1];\n" : "=r"(x) : "r"(ra) : "memory");
        r |= x;
    }
    t.par++;
    return r;
}
// [lo, hi) of this CTA's share of `count` items in units of `gran`
__device__ __forceinline__ int2 team_range(const Team &t, int count, int gran) {
    const int units = (count + gran - 1) / gran;
    const int u0 = units * t.rank / t.n, u1 = units * (t.rank + 1) / t.n;
    return make_int2(min(count, u0 * gran), min(count, u1 * gran));
}
__device__ __forceinline__ float2 ldcg2(const float2 *p) { return __ldcg(p); }

// ------------------------------------------------ diagonal-block inverse
// Sortable 32-bit key: |re|+|im| bits (non-negative floats order as
// unsigned integers) with the low 10 bits replaced by 1023 - row, so the
// warp maximum is one redux and ties go to the lower row.  Magnitudes that
// differ only in those bits (relative 2^-13) count as a tie.
__device__ __forceinline__ uint32_t pivot_key32(float v, int row) {
    return (__float_as_uint(v) & ~0x3FFu) | (uint32_t)(0x3FF - row);
}

// P = inv(A(k0:k0+m, k0:k0+m)) (m <= 32) by one warp: lane r holds row r of
// the block in registers, padded to 32 x 32 with identity rows; Gauss-Jordan
// with implicit partial pivoting inside the block (largest |re|+|im| among
// the unused rows, as zgetf2 chooses).  The row shifts left by one column per
// step, so step k always pivots on R[0] and appends the inverse column at
// R[31] (after 32 steps R[j] is the in-place result's column j); the rolled
// loop keeps every register index static.  Each step is uniform across the
// warp: one redux for the pivot lane p, the pivot row by shuffles from p, its
// reciprocal in FP32 on every lane.  P is written to s.sP in natural order,
// P(r, c) = R(pr[r], ipr[c]) (pr[k] the pivot lane of step k), with the
// identity on the padding.  Returns the 1-based step of the first zero pivot
// (0 if none).
__device__ __noinline__ int invert_diag_warp(const float2 *__restrict__ A, int ld, int k0, int m, const GjSmem &s) {
    const int lane = threadIdx.x & 31;
    const bool valid = lane < m;
    float2 R[32];
#pragma unroll
    for (int j = 0; j < 32; ++j)
        R[j] = (valid && j < m) ? ldcg2(A + (k0 + lane) + (size_t)ld * (k0 + j))
                                : make_float2((!valid && j == lane) ? 1.0f : 0.0f, 0.0f);
    int *spr = s.spr;
    bool used = false;
    int myk = 0, info = 0;
#pragma unroll 1
    for (int k = 0; k < 32; ++k) {
        float v = cabs1f(R[0]);
        if (!(v == v)) v = 0.0f;  // NaN rows rank as zero pivots
        const uint32_t wk = __reduce_max_sync(0xffffffffu, used ? 0u : pivot_key32(v, lane));
        // 32 - k unused lanes remain, so p is one of them
        const int p = 0x3FF - (int)(wk & 0x3FFu);
        if ((wk >> 10) == 0 && info == 0) info = k + 1;
        const bool piv = lane == p;
        const float2 d = crcp_f32(make_float2(__shfl_sync(0xffffffffu, R[0].x, p),
                                              __shfl_sync(0xffffffffu, R[0].y, p)));
        // the pivot row becomes its scaled copy: base 0, multiplier -1
        const float2 f = piv ? make_float2(-1.0f, 0.0f) : R[0];
#pragma unroll
        for (int j = 1; j < 32; ++j) {
            const float2 rp = cmul(make_float2(__shfl_sync(0xffffffffu, R[j].x, p),
                                               __shfl_sync(0xffffffffu, R[j].y, p)), d);
            R[j - 1] = cfms(f, rp, piv ? make_float2(0.f, 0.f) : R[j]);
        }
        R[31] = make_float2(-(f.x * d.x - f.y * d.y), -(f.x * d.y + f.y * d.x));
        if (piv) {
            used = true;
            myk = k;
        }
        if (lane == 0) spr[k] = p;
    }
    __syncwarp();
    float2 *sP = s.sP;
#pragma unroll
    for (int j = 0; j < 32; ++j) sP[myk * 32 + spr[j]] = R[j];
    __syncwarp();
    return info > m ? 0 : info;
}

// ------------------------------------------------- trailing-update staging
// W tile: rows I0..I0+TM-1 of the panel columns [k0, k0+nbt) of A, one
// exponent per row over its nbt values.  Thread (row r = tid % TM, half h =
// tid / TM) loads the K groups 2h and 2h+1 (8 values each).
__device__ inline void stage_w(const TileSmem &t, const GjSmem &s, const float2 *__restrict__ A, int ld, int N,
                               int I0, int k0, int nbt) {
    const int tid = threadIdx.x, r = tid % TM, h = tid / TM, i = I0 + r;
    float2 v[2][8];
    float m = 0.0f;
#pragma unroll
    for (int g = 0; g < 2; ++g)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int kk = 8 * (2 * h + g) + q;
            v[g][q] = (i < N && kk < nbt) ? A[i + (size_t)ld * (k0 + kk)] : make_float2(0.f, 0.f);
            m = fmaxf(m, fmaxf(fabsf(v[g][q].x), fabsf(v[g][q].y)));
        }
    s.rmax[h * TM + r] = m;
    __syncthreads();
    const int e = tc::scale_exponent(fmaxf(s.rmax[r], s.rmax[TM + r]));
    const float sc = tc::exp2i(-e);
    if (h == 0) t.rexp[r] = e;
#pragma unroll
    for (int g = 0; g < 2; ++g) {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[g][q] = make_float2(v[g][q].x * sc, v[g][q].y * sc);
        store_split8(t.sa, r, 2 * h + g, v[g]);
    }
}

// ---------------------------------------------- pipelined trailing update
// The panel's W (N x nbt) and its rows of the other columns (nbt x (N - nbt))
// are converted once per panel into split-fp16 tiles in the CTA's global
// scratch (W: TM-row tiles of 32 KB with one exponent per row; B: PTN-column
// tiles of 8 KB with one exponent per column).  The TM x PTN output tiles then
// run through a warp-specialised pipeline whose roles synchronise only
// through mbarriers:
//   warp 0, lane 0      bulk copies of the W tile of each row tile (one
//                       buffer) and of the B tile (three buffers), one TMA
//                       tile load of the old C values (three buffers) of tile
//                       t+3 as soon as tile t's C has been stored, and the
//                       TMA tile stores of finished C tiles;
//   warp 1, lane 0      the tcgen05 MMAs of each tile into one of two
//                       tensor-memory accumulators;
//   warps 4-7           the epilogue: accumulator (tcgen05.ld, one lane
//                       quadrant per warp) times 2^(row + column exponent)
//                       added to the old C in shared memory.
// The leading dimension must be a multiple of 8 (16-byte TMA strides; rows
// N..ld-1 are never touched).
constexpr int PTN = 32;                         // columns of an output tile
constexpr int NCB = 3;                          // C buffers
constexpr int NBB = 2;                          // B buffers
constexpr int NKB = 2;                          // K chunks of KB in one update at most (rank 64)
constexpr uint32_t WTILE = 4u * TM * KB * 2;     // 32 KB
constexpr uint32_t BTILE = 4u * PTN * KB * 2;    // 8 KB
constexpr uint32_t CTILE = (uint32_t)TM * PTN * 8;  // 32 KB: PTN columns of TM float2
static_assert(NCB * CTILE >= 32u * NT * 8, "panel_w stages 32 values per thread in the C buffers");
struct Pipe {
    unsigned char *sW;               // NKB chunks of WTILE bytes: the W tile of one row tile
    unsigned char *sB;               // NBB buffers of NKB * BTILE bytes (no arrays of pointers, so the
    unsigned char *sC;               // struct stays in registers): NCB buffers of CTILE bytes
    uint64_t *fullW, *emptyW;        // [1], [1]
    uint64_t *fullB, *emptyB;        // [NBB]
    uint64_t *fullC, *doneC;         // [NCB]: C loaded / C updated by the epilogue
    uint64_t *accFull, *accEmpty;    // [2]
    uint64_t *drain;                 // [1] completion of every MMA before tensor memory is freed
    uint64_t *laReady;               // [1] the look-ahead tile is stored (next diagonal block final)
    int *rexpW;                      // [ntr * TM] row exponents of W
    int *cexpB;                      // [ntc * PTN] column exponents of the pivot rows
    uint32_t *tslot;
    unsigned char *wt, *bt;          // global: W tiles (NKB * WTILE per row tile), B tiles (NKB * BTILE
                                     // per column tile; an update of one K chunk uses the first)
    uint32_t tbase;
    uint32_t nW, nB, nT, nLA;        // W tiles, B tiles, output tiles, look-aheads so far (phase counters)
};
constexpr int PIPE_BARS = 2 + 2 * NBB + 2 * NCB + 4 + 1 + 1;
__host__ __device__ inline size_t pipe_smem_bytes(int N) {
    const int ntr = (N + TM - 1) / TM, ntc = (N + PTN - 1) / PTN;
    return (size_t)NKB * WTILE + NBB * (size_t)NKB * BTILE + NCB * (size_t)CTILE + PIPE_BARS * 8 + 8 + 4 * (size_t)ntr * TM +
           4 * (size_t)ntc * PTN + 16;
}
// global scratch of one CTA for the panel tiles
__host__ __device__ inline size_t pipe_scratch_bytes(int N) {
    const int ntr = (N + TM - 1) / TM, ntc = (N + PTN - 1) / PTN;
    return (size_t)ntr * NKB * WTILE + (size_t)ntc * NKB * BTILE;
}
__device__ inline Pipe carve_pipe(unsigned char *base, int N, unsigned char *gscratch) {
    Pipe P;
    const int ntr = (N + TM - 1) / TM, ntc = (N + PTN - 1) / PTN;
    unsigned char *q = base;
    P.sW = q; q += NKB * WTILE;
    P.sC = q; q += NCB * CTILE;
    P.sB = q; q += NBB * NKB * BTILE;
    uint64_t *bar = (uint64_t *)q;
    P.fullW = bar; P.emptyW = bar + 1;
    P.fullB = bar + 2; P.emptyB = P.fullB + NBB;
    P.fullC = P.emptyB + NBB; P.doneC = P.fullC + NCB;
    P.accFull = P.doneC + NCB; P.accEmpty = P.accFull + 2;
    P.drain = P.accEmpty + 2;
    P.laReady = P.drain + 1;
    q += PIPE_BARS * 8 + 8;
    P.rexpW = (int *)q; q += 4 * (size_t)ntr * TM;
    P.cexpB = (int *)q; q += 4 * (size_t)ntc * PTN;
    P.tslot = (uint32_t *)q;
    P.wt = gscratch;
    P.bt = gscratch + (size_t)ntr * NKB * WTILE;
    P.nW = P.nB = P.nT = P.nLA = 0;
    return P;
}
// 128 tensor-memory columns: two accumulators of PTN complex columns (re, im)
__device__ inline void pipe_setup(Pipe &P) {
    if (threadIdx.x < 32) tc::tmem_alloc(P.tslot, 4 * PTN);
    if (threadIdx.x == 0) {
        tc::mbar_init(P.fullW, 1);
        tc::mbar_init(P.emptyW, 1);
        for (int i = 0; i < NBB; ++i) { tc::mbar_init(&P.fullB[i], 1); tc::mbar_init(&P.emptyB[i], 1); }
        for (int i = 0; i < NCB; ++i) { tc::mbar_init(&P.fullC[i], 1); tc::mbar_init(&P.doneC[i], 4); }
        for (int i = 0; i < 2; ++i) { tc::mbar_init(&P.accFull[i], 1); tc::mbar_init(&P.accEmpty[i], 4); }
        tc::mbar_init(P.drain, 1);
        tc::mbar_init(P.laReady, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    P.tbase = *P.tslot;
}
__device__ inline void pipe_teardown(const Pipe &P) {
    // the MMA issuer's last commit: every MMA it issued has completed (bounded;
    // on the normal path they have long finished)
    if (threadIdx.x == 32) {
        tc::mma_commit(P.drain);
        tc::mbar_wait(P.drain, 0, WAIT_LIMIT);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(P.tbase, 4 * PTN);
}

__device__ __forceinline__ void expect_bytes(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc::smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tc::smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     tc::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// this thread's committed bulk stores have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
// ... and have completed
__device__ __forceinline__ void bulk_wait0() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

// The working matrices of the C tiles: a 4-D tensor map (row, column, matrix,
// CTA) of complex FP32 elements moved as 8-byte words, N x N valid elements
// per matrix, and the (matrix, CTA) coordinates of the one being inverted.
struct CMat {
    const CUtensorMap *tm;
    int z, w;
};
__device__ __forceinline__ void tma_load4(void *dst, const CUtensorMap *tm, int x, int y, int z, int w,
                                          uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(tc::smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(tc::smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store4(const CUtensorMap *tm, int x, int y, int z, int w, const void *src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(
                     reinterpret_cast<uint64_t>(tm)),
                 "r"(x), "r"(y), "r"(z), "r"(w), "r"(tc::smem_u32(src))
                 : "memory");
}

// MMAs of one K chunk: A (TM x KB, plane stride TM*KB*2), B (n x KB, plane
// stride n*KB*2), D re at d0, im at d0 + n.  first = overwrite.
__device__ inline void issue_split_mma(uint32_t a0, uint32_t b0, int n, uint32_t d0, bool first) {
    constexpr uint32_t SBO = (KB / 8) * 128, LBO = 128;
    const uint32_t id = tc::idesc_f16(TM, n, false), idn = tc::idesc_f16(TM, n, true);
    const uint32_t aplane = TM * KB * 2, bplane = n * KB * 2;
    const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
#pragma unroll
    for (int ks = 0; ks < KB / 16; ++ks) {
        const uint32_t koff = ks * 256;
#pragma unroll
        for (int sp = 0; sp < 3; ++sp) {
            const uint64_t are = tc::sdesc(a0 + (0 + pa[sp]) * aplane + koff, LBO, SBO);
            const uint64_t aim = tc::sdesc(a0 + (2 + pa[sp]) * aplane + koff, LBO, SBO);
            const uint64_t bre = tc::sdesc(b0 + (0 + pb[sp]) * bplane + koff, LBO, SBO);
            const uint64_t bim = tc::sdesc(b0 + (2 + pb[sp]) * bplane + koff, LBO, SBO);
            const uint32_t acc = (first && ks == 0 && sp == 0) ? 0u : 1u;
            tc::mma_f16(d0, are, bre, id, acc);
            tc::mma_f16(d0, aim, bim, idn, 1u);
            tc::mma_f16(d0 + n, are, bim, id, acc);
            tc::mma_f16(d0 + n, aim, bre, id, 1u);
        }
    }
}

// The panel's column block once its diagonal block is inverted (P in s.sP):
// W = -A(:, K) P on the rows outside K and P - I on the rows of K, so that
// the rank-m update A(:, J) += W A_old(K, J) of every other column J completes
// the elimination.  A(:, K) receives its final values (W outside K, P on K);
// W goes to the split-fp16 W tiles with one exponent per row.  One thread per
// row; the row's panel values are staged in the pipe's C buffers (idle
// between trailing updates) so that the k loop stays rolled.  Tile rows
// N .. ntr*TM-1 are zero.
// Rows [rlo, rhi) of the ntr * TM tile rows; with gexp the row exponents
// also go to global memory for the other CTA of the team.
__device__ inline void panel_w(const Pipe &P, const GjSmem &s, float2 *__restrict__ A, int ld, int N, int k0,
                               int m, int rlo, int rhi, int *gexp) {
    const int tid = threadIdx.x;
    float2 *xs = (float2 *)P.sC;  // [32][NT]: 64 KB of the three contiguous C buffers
    for (int row = rlo + tid; row < rhi; row += NT) {
        float2 w[32];
        const int rk = row - k0;
        if (row >= N) {
#pragma unroll
            for (int c = 0; c < 32; ++c) w[c] = make_float2(0.f, 0.f);
        } else if (rk >= 0 && rk < m) {
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const float2 p = s.sP[rk * 32 + c];
                if (c < m) A[row + (size_t)ld * (k0 + c)] = p;
                w[c] = (c == rk) ? make_float2(p.x - 1.0f, p.y) : p;
            }
        } else {
            // all 32 loads in flight before the first staging store
#pragma unroll
            for (int k = 0; k < 32; ++k) w[k] = (k < m) ? ldcg2(A + row + (size_t)ld * (k0 + k)) : make_float2(0.f, 0.f);
#pragma unroll
            for (int k = 0; k < 32; ++k) xs[k * NT + tid] = w[k];
#pragma unroll
            for (int c = 0; c < 32; ++c) w[c] = make_float2(0.f, 0.f);
#pragma unroll 1
            for (int k = 0; k < m; ++k) {
                const float2 x = xs[k * NT + tid];
                const float4 *pk = (const float4 *)(s.sP + k * 32);
#pragma unroll
                for (int c2 = 0; c2 < 16; ++c2) {
                    const float4 p = pk[c2];
                    w[2 * c2] = cfma(x, make_float2(p.x, p.y), w[2 * c2]);
                    w[2 * c2 + 1] = cfma(x, make_float2(p.z, p.w), w[2 * c2 + 1]);
                }
            }
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                w[c] = make_float2(-w[c].x, -w[c].y);
                if (c < m) A[row + (size_t)ld * (k0 + c)] = w[c];
            }
        }
        float mx = 0.0f;
#pragma unroll
        for (int c = 0; c < 32; ++c) mx = fmaxf(mx, fmaxf(fabsf(w[c].x), fabsf(w[c].y)));
        const int e = tc::scale_exponent(mx);
        const float sc = tc::exp2i(-e);
        P.rexpW[row] = e;
        if (gexp) gexp[row] = e;
        unsigned char *tile = P.wt + (size_t)(row / TM) * NKB * WTILE;
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const tc::Split2 u = tc::split_fp16(w[8 * g + q].x * sc), v = tc::split_fp16(w[8 * g + q].y * sc);
                rh[q] = u.hi; rl[q] = u.lo; ih[q] = v.hi; il[q] = v.lo;
            }
            const uint32_t off = tc::kmajor_offset(row % TM, 8 * g, KB);
            *(uint4 *)(tile + 0 * (TM * KB * 2) + off) = *(const uint4 *)rh;
            *(uint4 *)(tile + 1 * (TM * KB * 2) + off) = *(const uint4 *)rl;
            *(uint4 *)(tile + 2 * (TM * KB * 2) + off) = *(const uint4 *)ih;
            *(uint4 *)(tile + 3 * (TM * KB * 2) + off) = *(const uint4 *)il;
        }
    }
}
// W of a 64-column panel [k0, k0+64) whose columns already hold their final
// Gauss-Jordan values: W = A(:, K) - E_K (the identity on the panel's rows),
// so that A(:, J) += W A_old(K, J) eliminates the whole panel from every other
// column J.  Two K chunks per row tile, one exponent per row over all 64
// values.  Rows [rlo, rhi) of the ntr * TM tile rows (rows N.. are zero);
// with gexp the row exponents also go to global memory.
__device__ __noinline__ void panel_w64(const Pipe &P, const float2 *__restrict__ A, int ld, int N, int k0, int rlo,
                                 int rhi, int *gexp) {
    for (int row = rlo + threadIdx.x; row < rhi; row += NT) {
        const int rk = row - k0;
        auto ld8 = [&](int c0, float2 (&v)[8]) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                float2 x = row < N ? ldcg2(A + row + (size_t)ld * (k0 + c0 + q)) : make_float2(0.f, 0.f);
                if (c0 + q == rk) x.x -= 1.0f;
                v[q] = x;
            }
        };
        // the row maximum first (16 loads in flight), then the values again, eight at a time
        float mx = 0.0f;
#pragma unroll 1
        for (int c0 = 0; c0 < 64; c0 += 16) {
            float2 a[8], b[8];
            ld8(c0, a);
            ld8(c0 + 8, b);
#pragma unroll
            for (int q = 0; q < 8; ++q)
                mx = fmaxf(mx, fmaxf(fmaxf(fabsf(a[q].x), fabsf(a[q].y)), fmaxf(fabsf(b[q].x), fabsf(b[q].y))));
        }
        const int e = tc::scale_exponent(mx);
        const float sc = tc::exp2i(-e);
        P.rexpW[row] = e;
        if (gexp) gexp[row] = e;
        unsigned char *tile = P.wt + (size_t)(row / TM) * NKB * WTILE;
#pragma unroll 1
        for (int g = 0; g < 8; ++g) {
            float2 w[8];
            ld8(8 * g, w);
            __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const tc::Split2 u = tc::split_fp16(w[q].x * sc), v = tc::split_fp16(w[q].y * sc);
                rh[q] = u.hi; rl[q] = u.lo; ih[q] = v.hi; il[q] = v.lo;
            }
            unsigned char *t = tile + (size_t)(g / 4) * WTILE;
            const uint32_t off = tc::kmajor_offset(row % TM, 8 * (g % 4), KB);
            *(uint4 *)(t + 0 * (TM * KB * 2) + off) = *(const uint4 *)rh;
            *(uint4 *)(t + 1 * (TM * KB * 2) + off) = *(const uint4 *)rl;
            *(uint4 *)(t + 2 * (TM * KB * 2) + off) = *(const uint4 *)ih;
            *(uint4 *)(t + 3 * (TM * KB * 2) + off) = *(const uint4 *)il;
        }
    }
}

// Which matrix columns the B tiles and output tiles of an update cover:
// either the rest columns of a panel (column tile jt holds rest columns jr =
// jt*PTN.., matrix column jr < skip0 ? jr : jr + nskip) or one column tile at
// cfix (cfix >= 0).  nrest = valid rest columns.
struct ColMap {
    int skip0, nskip, cfix, nrest;
    __device__ __forceinline__ int col(int jr) const { return cfix >= 0 ? cfix + jr : (jr < skip0 ? jr : jr + nskip); }
    __device__ __forceinline__ int ntc() const { return (nrest + PTN - 1) / PTN; }
};

// B tiles: rest column jr with the K values A(krow0 + kk, col(jr)), kk <
// nkr <= 32 * NKBT (the rows of the panel, old values), one exponent per
// column over all of them; four threads per column.  Rest columns [clo, chi)
// (multiples of 8); with gexp the column exponents also go to global memory
// for the other CTA of the team.  A single K chunk takes two groups of eight
// columns per warp and round (sixteen loads in flight).
// (not inlined: a separate register allocation keeps the sweep kernel's spills low)
template <int NKBT>
__device__ __noinline__ void convert_b(const Pipe &P, const float2 *__restrict__ A, int ld, int krow0, int nkr,
                                 const ColMap &cmap, int clo, int chi, int *gexp) {
    constexpr int GR = NKBT == 1 ? 2 : 1;  // column groups per warp and round
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane & 3;
    for (int c00 = clo + warp * 8; c00 < chi; c00 += GR * NWARP * 8) {
        float2 v[GR][8 * NKBT];
#pragma unroll
        for (int h = 0; h < GR; ++h) {
            const int jr = c00 + h * NWARP * 8 + (lane >> 2);
            const bool cv = jr < cmap.nrest && jr < chi;
            const int col = cmap.col(jr);
#pragma unroll
            for (int c = 0; c < NKBT; ++c)
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int kk = 32 * c + 8 * g + q;
                    v[h][8 * c + q] = (cv && kk < nkr) ? ldcg2(A + krow0 + kk + (size_t)ld * col) : make_float2(0.f, 0.f);
                }
        }
#pragma unroll
        for (int h = 0; h < GR; ++h) {
            const int c0 = c00 + h * NWARP * 8;
            if (c0 >= chi) break;  // uniform over the warp
            const int jr = c0 + (lane >> 2);
            float m = 0.0f;
#pragma unroll
            for (int q = 0; q < 8 * NKBT; ++q) m = fmaxf(m, fmaxf(fabsf(v[h][q].x), fabsf(v[h][q].y)));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
            const int e = tc::scale_exponent(m);
            const float sc = tc::exp2i(-e);
            if (g == 0) {
                P.cexpB[jr] = e;
                if (gexp) gexp[jr] = e;
            }
#pragma unroll
            for (int c = 0; c < NKBT; ++c) {
                __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const tc::Split2 a = tc::split_fp16(v[h][8 * c + q].x * sc), b = tc::split_fp16(v[h][8 * c + q].y * sc);
                    rh[q] = a.hi; rl[q] = a.lo; ih[q] = b.hi; il[q] = b.lo;
                }
                unsigned char *tile = P.bt + (size_t)(jr / PTN) * NKB * BTILE + (size_t)c * BTILE;
                const uint32_t off = tc::kmajor_offset(jr % PTN, 8 * g, KB);
                *(uint4 *)(tile + 0 * (PTN * KB * 2) + off) = *(const uint4 *)rh;
                *(uint4 *)(tile + 1 * (PTN * KB * 2) + off) = *(const uint4 *)rl;
                *(uint4 *)(tile + 2 * (PTN * KB * 2) + off) = *(const uint4 *)ih;
                *(uint4 *)(tile + 3 * (PTN * KB * 2) + off) = *(const uint4 *)il;
            }
        }
    }
}

// Look-ahead of a trailing update: the output tile that holds the next
// panel's diagonal block goes first; once it is stored, warp 2 (idle during
// the update) inverts that block into s.sP while the other tiles run.
struct LookAhead {
    int tile;                  // output tile index, -1: none
    const float2 *A;
    int ld, k0, m;             // the block A(k0:k0+m, k0:k0+m)
    int *info;                 // shared: its zero-pivot step (1-based), 0 if none
    int peer;                  // team of two: the other CTA's rank (it receives the result), else -1
};

// Copies P, the pivot lanes and the status of a diagonal-block inverse into
// the same shared-memory places of CTA `peer` of the cluster (one warp).
__device__ inline void send_diag(const GjSmem &s, int *info, int peer) {
    const int lane = threadIdx.x & 31;
    auto remote = [&](const void *p) -> uint32_t {
        uint32_t r;
        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(tc::smem_u32(p)), "r"(peer));
        return r;
    };
    for (int e = lane; e < 32 * 32; e += 32) {
        const float2 v = s.sP[e];
        asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};\n" ::"r"(remote(s.sP + e)), "f"(v.x), "f"(v.y) : "memory");
    }
    asm volatile("st.shared::cluster.s32 [%0], %1;\n" ::"r"(remote(s.spr + lane)), "r"(s.spr[lane]) : "memory");
    if (lane == 0) asm volatile("st.shared::cluster.s32 [%0], %1;\n" ::"r"(remote(info)), "r"(*info) : "memory");
}

// A(:, cols) += W * B (N rows) with nkb K chunks (W and B tiles already in the CTA's
// global scratch), pipelined (see above); the C tiles of matrix cm move by
// TMA, the columns as cmap says.  Output tiles [t0, t1) of the ntr x ntc
// tiles (row tile major; the look-ahead tile first), so that the CTAs of a
// team share the update.  Returns false if a wait timed out (uniform over
// the CTA).
__device__ inline bool trailing_pipe(Pipe &P, int N, const CMat &cm, const ColMap &cmap, int nkb, int t0, int t1,
                                     const GjSmem &s, const LookAhead &la) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nrest = cmap.nrest, ntc = cmap.ntc(), T = t1 - t0;
    const uint32_t wbytes = (uint32_t)nkb * WTILE, bbytes = (uint32_t)nkb * BTILE;
    const bool lad = la.tile >= t0 && la.tile < t1;
    // generic stores (W/B tiles in global, the staging in the C buffers) before
    // the bulk copies and TMA tiles that read or overwrite them
    asm volatile("fence.proxy.async;\n" ::: "memory");
    __syncthreads();
    const uint32_t bW = P.nW, bB = P.nB, bT = P.nT;
    int err = 0;
    // tile of local step v: the look-ahead tile, then the others in order
    auto tile_of = [&](int v) -> int {
        if (!lad) return t0 + v;
        if (v == 0) return la.tile;
        return t0 + v - 1 < la.tile ? t0 + v - 1 : t0 + v;
    };
    // first matrix column of tile t: the rest columns of a tile are contiguous
    // (the panel start and width are multiples of 32)
    auto tile_col0 = [&](int t) -> int { return cmap.col((t % ntc) * PTN); };
    // the W tile changes at the first step and wherever the row tile changes
    auto w_first = [&](int v) -> bool { return v == 0 || tile_of(v) / ntc != tile_of(v - 1) / ntc; };
    auto w_last = [&](int v) -> bool { return v == T - 1 || tile_of(v) / ntc != tile_of(v + 1) / ntc; };
    int nwl = 0;  // W loads of this update
    for (int v = 0; v < T; ++v) nwl += w_first(v);
    if (warp == 0) {
        // ------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t iw = bW;  // next W load
            auto load = [&](int u) -> bool {
                const int t = tile_of(u);
                if (w_first(u)) {
                    if (iw >= 1 && !tc::mbar_wait(P.emptyW, (iw - 1) & 1u, WAIT_LIMIT)) return false;
                    expect_bytes(P.fullW, wbytes);
                    bulk_copy(P.sW, P.wt + (size_t)(t / ntc) * NKB * WTILE, wbytes, P.fullW);
                    ++iw;
                }
                const uint32_t ib = bB + u, ic = bT + u;
                if (ib >= NBB && !tc::mbar_wait(&P.emptyB[ib % NBB], ((ib - NBB) / NBB) & 1u, WAIT_LIMIT))
                    return false;
                expect_bytes(&P.fullB[ib % NBB], bbytes);
                bulk_copy(P.sB + (ib % NBB) * NKB * BTILE, P.bt + (size_t)(t % ntc) * NKB * BTILE, bbytes,
                          &P.fullB[ib % NBB]);
                // the C buffer last held tile u - NCB, whose store this thread issued
                bulk_wait_read0();
                expect_bytes(&P.fullC[ic % NCB], CTILE);  // the whole box, out-of-range elements zero-filled
                tma_load4(P.sC + (ic % NCB) * CTILE, cm.tm, (t / ntc) * TM, tile_col0(t), cm.z, cm.w, &P.fullC[ic % NCB]);
                return true;
            };
            for (int u = 0; u < NCB && u < T && !err; ++u)
                if (!load(u)) err = 1;
            for (int v = 0; v < T && !err; ++v) {
                const uint32_t ic = bT + v;
                const int t = tile_of(v);
                if (!tc::mbar_wait(&P.doneC[ic % NCB], (ic / NCB) & 1u, WAIT_LIMIT)) { err = 1; break; }
                tma_store4(cm.tm, (t / ntc) * TM, tile_col0(t), cm.z, cm.w, P.sC + (ic % NCB) * CTILE);  // clipped
                bulk_commit();
                if (lad && v == 0) {
                    // the next diagonal block is final in global memory
                    bulk_wait0();
                    asm volatile("fence.proxy.async.global;\n" ::: "memory");
                    mbar_arrive(P.laReady);
                }
                if (v + NCB < T && !load(v + NCB)) err = 1;
            }
            if (lad && err && T > 0) mbar_arrive(P.laReady);  // release the look-ahead warp (its result is discarded)
            bulk_wait0();
            asm volatile("fence.proxy.async.global;\n" ::: "memory");
        }
        __syncwarp();
    } else if (warp == 1) {
        // --------------------------------------------------- MMA issuer
        if (lane == 0) {
            uint32_t iw = bW;  // next W use
            for (int t = 0; t < T; ++t) {
                const uint32_t ic = bT + t, ib = bB + t, a = ic & 1u;
                if (ic >= 2 && !tc::mbar_wait(&P.accEmpty[a], ((ic >> 1) & 1u) ^ 1u, WAIT_LIMIT)) { err = 1; break; }
                if (w_first(t)) {
                    if (!tc::mbar_wait(P.fullW, iw & 1u, WAIT_LIMIT)) { err = 1; break; }
                    ++iw;
                }
                if (!tc::mbar_wait(&P.fullB[ib % NBB], (ib / NBB) & 1u, WAIT_LIMIT)) { err = 1; break; }
                tc::fence_after_sync();
                for (int c = 0; c < nkb; ++c)
                    issue_split_mma(tc::smem_u32(P.sW + c * WTILE), tc::smem_u32(P.sB + (ib % NBB) * NKB * BTILE + c * BTILE),
                                    PTN, P.tbase + a * (2 * PTN), c == 0);
                tc::mma_commit(&P.accFull[a]);
                tc::mma_commit(&P.emptyB[ib % NBB]);
                if (w_last(t)) tc::mma_commit(P.emptyW);
            }
        }
        __syncwarp();
    } else if (warp == 2) {
        // ---------------------------------------------- look-ahead inverse
        if (lad) {
            int ok = 1;
            if (lane == 0) ok = tc::mbar_wait(P.laReady, P.nLA & 1u, WAIT_LIMIT) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) err = 1;
            else {
                const int r = invert_diag_warp(la.A, la.ld, la.k0, la.m, s);
                if (lane == 0) *la.info = r;
                __syncwarp();
                // the team's other CTA gets the same inverse (visible after the
                // cluster barrier that ends the update)
                if (la.peer >= 0) send_diag(s, la.info, la.peer);
            }
        }
    } else if (warp >= 4) {
        // ------------------------------------------------------ epilogue
        const int q4 = warp & 3, r = 32 * q4 + lane;
        const uint32_t lb = (uint32_t)(32 * q4) << 16;
        for (int t = 0; t < T && !err; ++t) {
            const uint32_t ic = bT + t, a = ic & 1u, cb = ic % NCB;
            if (!tc::mbar_wait(&P.accFull[a], (ic >> 1) & 1u, WAIT_LIMIT)) err = 1;
            if (!tc::mbar_wait(&P.fullC[cb], (ic / NCB) & 1u, WAIT_LIMIT)) err = 1;
            if (__any_sync(0xffffffffu, err)) { err = 1; break; }
            tc::fence_after_sync();
            const int tt = tile_of(t);
            const int it = tt / ntc, jt = tt % ntc, i = it * TM + r;
            const bool rv = i < N;
            const int er = rv ? P.rexpW[i] : 0;
            float2 *cs = (float2 *)(P.sC + cb * CTILE);
            const uint32_t dacc = P.tbase + lb + a * (2 * PTN);
#pragma unroll
            for (int g = 0; g < PTN / 16; ++g) {
                float re[16], im[16];
                tc::tmem_ld16(dacc + g * 16, re);
                tc::tmem_ld16(dacc + PTN + g * 16, im);
                float2 old[16];
#pragma unroll
                for (int q = 0; q < 16; ++q) old[q] = cs[(g * 16 + q) * TM + r];
                tc::tmem_wait_ld();
                if (rv) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const int jr = jt * PTN + g * 16 + q;
                        if (jr < nrest) {
                            const float f = tc::exp2i(er + P.cexpB[jr]);
                            cs[(g * 16 + q) * TM + r] = make_float2(fmaf(re[q], f, old[q].x), fmaf(im[q], f, old[q].y));
                        }
                    }
                }
            }
            // tensor memory read: the accumulator may take the next tile's MMAs
            tc::fence_before_sync();
            tc::fence_async_smem();  // the TMA store (async proxy) reads these values
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&P.accEmpty[a]);
                mbar_arrive(&P.doneC[cb]);
            }
        }
    }
    if (__syncthreads_or(err)) return false;
    P.nW += nwl;
    P.nB += T;
    P.nT += T;
    if (lad) P.nLA++;
    return true;
}

// In-place blocked Gauss-Jordan inverse of the N x N block A (leading
// dimension ld, complex FP32; the same matrix as cm) in panels of 32
// columns, pivoting only inside each panel's diagonal block: the Schur
// complements of the sweep keep their diagonal blocks well conditioned, and
// the FP64 refinement and the acceptance test of every job absorb the
// difference to full partial pivoting.  Per panel K: P = inv(A_KK) by one
// warp, the column block W (CUDA cores, FP32), one rank-32 update of all other
// columns on the tensor cores.  On return A = inv(A) in natural order.
// Returns (on warp 0) the 1-based column of the first zero pivot, 0 if none;
// *err = 1 if a tensor-core wait timed out.
__device__ int gj_invert(float2 *__restrict__ A, int N, int ld, const GjSmem &s, Pipe &P, const CMat &cm,
                         int *err, Team &tm) {
    int info = 0;
    const int ntr = (N + TM - 1) / TM;
    const int2 rr = team_range(tm, ntr * TM, 8);  // this CTA's rows of the panel products
    int *gr = tm.n > 1 ? tm.gx : nullptr, *gc = tm.n > 1 ? tm.gx + ntr * TM : nullptr;
    // every CTA of the team inverts the diagonal block (the same values)
    auto diag = [&](int k0, int m) {
        if (threadIdx.x < 32) {
            const int r = invert_diag_warp(A, ld, k0, m, s);
            if (r && !info) info = k0 + r;
        }
        __syncthreads();
    };
    // B tiles of the K rows [krow0, krow0 + nkr) for the columns of cmap, then
    // A(:, cols) += W B; every C tile of both CTAs is stored before it returns
    auto update = [&](const ColMap &cmap, int krow0, int nkr, const LookAhead &la) -> bool {
        const int ntc = cmap.ntc();
        const int2 cr = team_range(tm, ntc * PTN, 8);
        if (nkr > KB) convert_b<2>(P, A, ld, krow0, nkr, cmap, cr.x, cr.y, gc);
        else convert_b<1>(P, A, ld, krow0, nkr, cmap, cr.x, cr.y, gc);
        if (tm.n > 1) {
            // the W and B tiles of both CTAs (read by bulk copies) and their exponents
            asm volatile("fence.proxy.async;\n" ::: "memory");
            cluster_sync();
            for (int i = threadIdx.x; i < ntr * TM; i += NT) P.rexpW[i] = __ldcg(gr + i);
            for (int j = threadIdx.x; j < ntc * PTN; j += NT) P.cexpB[j] = __ldcg(gc + j);
        }
        const int2 tr = team_range(tm, ntr * ntc, 1);
        const bool ok = trailing_pipe(P, N, cm, cmap, nkr > KB ? 2 : 1, tr.x, tr.y, s, la);
        return !team_or(tm, !ok);
    };
    // 64-column panels once the working matrices of a wave no longer stay in
    // L2 (their rank-32 updates then stream from HBM); 32-column panels below
    const bool pairs = N > 256;
    const LookAhead none{-1, nullptr, 0, 0, 0, nullptr, -1};
    const int peer = tm.n > 1 ? 1 - tm.rank : -1;
    int *la_info = tm.slot + 2;  // shared int after the team's two exchange slots
    bool have_next = false;      // the next diagonal block was inverted during the last update
    int k0 = 0;
    while (k0 < N) {
        if (pairs && N - k0 >= 2 * KB) {
            // A 64-column panel K1 | K2: two 32-column steps on the panel's own
            // columns (K1 eliminated from K2, K2 from K1, each a one-column-tile
            // update), then W = A(:, K) - E_K and one rank-64 update of every
            // other column: half the passes over the working matrix of two
            // rank-32 updates, the same elimination.
            const int k1 = k0 + KB;
            if (have_next) {
                const int r = *la_info;
                if (r && !info) info = k0 + r;
                have_next = false;
            } else {
                diag(k0, KB);
            }
            panel_w(P, s, A, ld, N, k0, KB, rr.x, rr.y, gr);
            // the update of K2's columns first finishes K2's diagonal block (row
            // tile k1 / TM of its one column tile), inverted while the rest runs
            const LookAhead la1{k1 / TM, A, ld, k1, KB, la_info, peer};
            if (!update(ColMap{0, 0, k1, KB}, k0, KB, la1)) { *err = 1; return info; }
            {
                const int r = *la_info;
                if (r && !info) info = k1 + r;
            }
            panel_w(P, s, A, ld, N, k1, KB, rr.x, rr.y, gr);
            if (!update(ColMap{0, 0, k0, KB}, k1, KB, none)) { *err = 1; return info; }
            if (N > k0 + 2 * KB) {
                panel_w64(P, A, ld, N, k0, rr.x, rr.y, gr);
                // the next panel's diagonal block: row tile kn / TM, rest-column tile k0 / PTN
                const int kn = k0 + 2 * KB, ntc = (N - 2 * KB + PTN - 1) / PTN;
                const LookAhead la2{(kn / TM) * ntc + k0 / PTN, A, ld, kn, min(KB, N - kn), la_info, peer};
                if (!update(ColMap{k0, 2 * KB, -1, N - 2 * KB}, k0, 2 * KB, la2)) { *err = 1; return info; }
                have_next = true;
            }
            k0 += 2 * KB;
        } else {
            const int nbt = min(KB, N - k0);
            if (have_next) {
                // inverted during the previous update (s.sP, s.spr), its status in la_info
                const int r = *la_info;
                if (r && !info) info = k0 + r;
                have_next = false;
            } else {
                diag(k0, nbt);
            }
            panel_w(P, s, A, ld, N, k0, nbt, rr.x, rr.y, gr);
            if (nbt < N) {
                // the next panel's diagonal block (rows and columns kn.., in row tile
                // kn / TM and rest-column tile k0 / PTN) is inverted by warp 2 of the
                // CTA that updates that tile while this update runs
                const int kn = k0 + nbt;
                LookAhead la = none;
                if (kn < N) {
                    const int ntc = (N - nbt + PTN - 1) / PTN;
                    la = LookAhead{(kn / TM) * ntc + k0 / PTN, A, ld, kn, min(KB, N - kn), la_info, peer};
                }
                if (!update(ColMap{k0, nbt, -1, N - nbt}, k0, nbt, la)) { *err = 1; return info; }
                have_next = la.tile >= 0;
            } else {
                team_sync(tm);
            }
            k0 += nbt;
        }
    }
    return info;
}

// ----------------------------------------------------------- self tests
// C = W(:, 0:K) * B(rowmap[0:K], :) for one 128 x 64 tile per CTA with the
// staging, MMAs and epilogue of the trailing update (K <= 32; K values of B
// gathered through rowmap like the pivot rows).
__global__ void __launch_bounds__(NT, 1)
    k_tc_product_check(const float2 *__restrict__ W, int ldw, const float2 *__restrict__ B, int ldb,
                       const int *__restrict__ rowmap, float2 *__restrict__ C, int ldc, int M, int ncol, int K,
                       int *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    GjSmem s = carve_gj(smem, 32);
    TileSmem t = carve_tile(smem + gj_smem_bytes(32));
    const int tid = threadIdx.x, warp = tid >> 5;
    const int I0 = blockIdx.x * TM, J0 = blockIdx.y * TN;
    for (int k = tid; k < K; k += NT) s.prow[k] = rowmap[k];
    const uint32_t tbase = tile_setup(t);
    uint32_t ph = 0;
    int err = 0;
    {
        // B: column j of the tile is B column J0 + j, K values B(rowmap[kk], .)
        const int j = tid >> 2, g = tid & 3, jc = J0 + j;
        float2 v[8];
        float m = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int kk = 8 * g + q;
            v[q] = (jc < ncol && kk < K) ? B[s.prow[kk] + (size_t)ldb * jc] : make_float2(0.f, 0.f);
            m = fmaxf(m, fmaxf(fabsf(v[q].x), fabsf(v[q].y)));
        }
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
        const int e = tc::scale_exponent(m);
        const float sc = tc::exp2i(-e);
        if (g == 0) t.cexp[j] = e;
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = make_float2(v[q].x * sc, v[q].y * sc);
        store_split8(t.sb, j, g, v);
    }
    stage_w(t, s, W, ldw, M, I0, 0, K);
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
        tc::fence_after_sync();
        issue_chunk(t, tbase, true);
        tc::mma_commit(t.bar);
    }
    wait_mma(t, ph, &err);
    if (!err) {
        const int r = 32 * (warp & 3) + (tid & 31), i = I0 + r;
        for (int c16 = 2 * (warp >> 2); c16 < 2 * (warp >> 2) + 2; ++c16) {
            float re[16], im[16];
            load_acc16(tbase, c16, re, im);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int jc = J0 + c16 * 16 + q;
                if (i < M && jc < ncol) {
                    const float f = tc::exp2i(t.rexp[r] + t.cexp[c16 * 16 + q]);
                    C[i + (size_t)ldc * jc] = make_float2(re[q] * f, im[q] * f);
                }
            }
        }
    }
    if (err && tid == 0) atomicExch(status, 1);
    tile_teardown(t, tbase);
}

// Inverse of each of nmat N x N complex FP32 matrices (one CTA each):
// work holds the matrices (leading dimension ld, matrix b at b * ld * N; tm
// maps them as (row, column, 0, b)), out receives the inverses.
__global__ void __launch_bounds__(NT, 1)
    k_tc_inverse_check(float2 *__restrict__ work, int N, int ld, float2 *__restrict__ out, int *__restrict__ info,
                       int *status, unsigned char *pscratch, const __grid_constant__ CUtensorMap tm) {
    extern __shared__ __align__(128) unsigned char smem[];
    GjSmem s = carve_gj(smem, N);
    Pipe P = carve_pipe(smem + gj_smem_bytes(N), N, pscratch + (size_t)blockIdx.x * pipe_scratch_bytes(N));
    pipe_setup(P);
    int err = 0;
    float2 *A = work + (size_t)blockIdx.x * ld * N;
    const CMat cm{&tm, 0, (int)blockIdx.x};
    __shared__ int team_slots[4];
    Team team{0, 1, nullptr, team_slots, 0};
    const int inf = gj_invert(A, N, ld, s, P, cm, &err, team);
    if (!err) {
        float2 *o = out + (size_t)blockIdx.x * N * N;
        for (int j = 0; j < N; ++j)
            for (int r = threadIdx.x; r < N; r += NT) o[r + (size_t)N * j] = A[r + (size_t)ld * j];
    }
    if (threadIdx.x == 0) {
        info[blockIdx.x] = inf;
        if (err) atomicExch(status, 1);
    }
    pipe_teardown(P);
}

// =================================================== mixed-precision sweep
// Storage of one job of a wave (offsets from MixedLayout, the same for every
// job):
//   tiles  Nz matrices in split-fp16 tile form: slot b = gR(b) of the sweep
//          (b = 1 .. Nz-1, 0-based slices), slot 0 = G_11.  Each matrix is
//          the raw Gauss-Jordan result R (inv(S)(r, c) = R(prow[r], iprow[c]))
//          cut into tiles of TM rows x KB columns; tile (rt, kc) is 32 KB at
//          (rt * nkc + kc) * 32 KB: four planes (re hi, re lo, im hi, im lo)
//          of fp16 in the K-major core-matrix layout, R(t, k) scaled by
//          2^-rexp[t] (one exponent per row over all columns)
//   prow   [Nz][N] the pivot rows of each slot, rexp [Nz][N] the row exponents
//   x      [Nz][ncap][N] x0: column j = G(:, 1) times the open channel oc[j]
//   rc     [Nz][ncap][N] the FP64 residual r, then the correction stage c
//   d      [2][ncap][N] the correction, two slices at a time
//   oc     [ncap] open channels of the right lead, then n_open
// complex FP32 everywhere (column j of a slice at j * N).
// The sweep's job vectors in shared memory, and the lead self-energies in
// global memory (see carve_job_slim).
__host__ __device__ inline size_t job_smem_bytes_slim(int N) {
    const int n4 = rup(N, 4);
    const size_t b = 3 * (size_t)n4 * 4 + 16;
    return (b + 127) / 128 * 128;
}
__host__ __device__ inline size_t job_sig_bytes(int N) { return 2 * (size_t)rup(N, 2) * 16; }

struct MixedLayout {
    int N, Nz, ld, ntr, nkc, ncap;
    size_t mat_bytes;  // one matrix in split tiles
    int last_rows;     // rows stored of the last row tile (the valid ones, rounded up to 8)
    uint32_t last_plane;  // bytes of one plane of a last-row-tile tile (last_rows / 8 core-matrix rows)
    size_t off_tiles, off_prow, off_rexp, off_x, off_rc, off_d, off_oc, job_bytes;
    size_t off_gx;         // in a wave slot's scratch: the team's exponent exchange
    size_t off_sig;        // ... then the lead self-energies of each CTA of the team
    size_t scratch_bytes;  // per wave slot (the CTAs of one job)
};
constexpr size_t TILE_BYTES = 4 * (size_t)TM * KB * 2;  // 32 KB
inline size_t align256(size_t x) { return (x + 255) / 256 * 256; }
MixedLayout make_layout(int N, int Nz, int ld, int ncap) {
    MixedLayout L;
    L.N = N; L.Nz = Nz; L.ld = ld; L.ncap = ncap;
    L.ntr = (N + TM - 1) / TM;
    L.nkc = (N + KB - 1) / KB;
    // the last row tile keeps only its valid rows: a plane of it is the first
    // last_rows / 8 core-matrix rows of a full plane (up to 11 % of the factor
    // storage at N = 797, so more jobs fit a wave)
    L.last_rows = ((N - (L.ntr - 1) * TM) + 7) / 8 * 8;
    L.last_plane = (uint32_t)(L.last_rows / 8) * (KB / 8) * 128;
    L.mat_bytes = (size_t)(L.ntr - 1) * L.nkc * TILE_BYTES + (size_t)L.nkc * 4 * L.last_plane;
    size_t o = 0;
    L.off_tiles = o; o = align256(o + (size_t)Nz * L.mat_bytes);
    L.off_prow = o; o = align256(o + (size_t)Nz * N * 4);
    L.off_rexp = o; o = align256(o + (size_t)Nz * N * 4);
    L.off_x = o; o = align256(o + (size_t)Nz * ncap * N * 8);
    L.off_rc = o; o = align256(o + (size_t)Nz * ncap * N * 8);
    L.off_d = o; o = align256(o + (size_t)2 * ncap * N * 8);
    L.off_oc = o; o = align256(o + (size_t)(ncap + 4) * 4);
    L.job_bytes = o;
    // sweep: two working matrices, the panel tiles and the exponents exchanged
    // by a team; passes: the B operand of one product in split tiles
    L.off_gx = align256((size_t)2 * N * ld * 8 + pipe_scratch_bytes(N));
    const size_t gx_bytes = 4 * ((size_t)L.ntr * TM + (size_t)((N + PTN - 1) / PTN) * PTN);
    L.off_sig = align256(L.off_gx + gx_bytes);
    L.scratch_bytes = align256(std::max(L.off_sig + 2 * job_sig_bytes(N), (size_t)L.nkc * ncap * 256));
    return L;
}

// shared memory of k_mixed_sweep: Gauss-Jordan state, the update pipeline,
// the job's index vectors and the team's exchange slots
inline size_t sweep_smem_bytes(int N) {
    return gj_smem_bytes(N) + (pipe_smem_bytes(N) + 127) / 128 * 128 + job_smem_bytes_slim(N) + 16;
}

// Byte offset of factor tile (rt, kc) in a stored matrix, and its plane stride.
__host__ __device__ inline size_t factor_tile_off(const MixedLayout &L, int rt, int kc) {
    return rt < L.ntr - 1 ? ((size_t)rt * L.nkc + kc) * TILE_BYTES
                          : (size_t)(L.ntr - 1) * L.nkc * TILE_BYTES + (size_t)kc * 4 * L.last_plane;
}
__host__ __device__ inline uint32_t factor_plane(const MixedLayout &L, int rt) {
    return rt < L.ntr - 1 ? (uint32_t)(TM * KB * 2) : L.last_plane;
}

struct MixedArgs {
    negf::Geo g;
    MixedLayout L;
    const double2 *voff;   // [Nz][N][ld] -c2 V(G_i - G_j) (the context's table)
    const double *E;       // energies
    const int2 *jobs;      // per wave slot: (energy index, k-point)
    int njobs;
    int cpj;               // CTAs (one cluster) per job in the sweep: 1 or 2
    int pa;                // factor ring stages of the passes
    unsigned char *jobmem; // njobs job regions
    unsigned char *scratch;
    double *tau, *dnorm, *xnorm, *dprev;
    int *status;           // 0 in progress; > 0 zero pivot (info); MIX_DONE converged;
                           // -1 too many open channels; -2 tensor wait timed out
    double tol;            // acceptance bound on the estimated remaining |dtau|
};
constexpr int MIX_DONE = 0x40000000;

// The job's N-sized vectors used by negf::job_vectors / d_element / open_cols.
__host__ __device__ inline size_t job_smem_bytes(int N) {
    const int n4 = rup(N, 4), n2 = rup(N, 2);
    size_t b = 3 * (size_t)n4 * 4 + 16;
    b = (b + 15) / 16 * 16;
    b += 2 * (size_t)n2 * 16 + 2 * (size_t)n2 * 8;
    return (b + 127) / 128 * 128;
}
// The sweep's variant: only nx, ny and the open-channel list in its own
// space; gamma_L / gamma_R (needed only while the open channels are listed at
// the start of a job) at gscr, the lead self-energies (read only by the
// diagonal of the end slices) in global memory at gsig.
__device__ inline negf::Smem carve_job_slim(unsigned char *base, int N, unsigned char *gscr, unsigned char *gsig) {
    negf::Smem s{};
    const int n4 = rup(N, 4), n2 = rup(N, 2);
    s.nx = (int *)base;
    s.ny = s.nx + n4;
    s.rows = s.ny + n4;
    s.nrows = s.rows + n4;
    s.sigL = (double2 *)gsig;
    s.sigR = s.sigL + n2;
    s.gL = (double *)gscr;
    s.gR = s.gL + n2;
    return s;
}
__device__ inline negf::Smem carve_job(unsigned char *base, int N) {
    negf::Smem s{};
    const int n4 = rup(N, 4), n2 = rup(N, 2);
    s.nx = (int *)base;
    s.ny = s.nx + n4;
    s.rows = s.ny + n4;
    s.nrows = s.rows + n4;
    size_t off = ((size_t)3 * n4 * 4 + 16 + 15) / 16 * 16;
    s.sigL = (double2 *)(base + off);
    s.sigR = s.sigL + n2;
    s.gL = (double *)(s.sigR + n2);
    s.gR = s.gL + n2;
    return s;
}

// M = round32(D_k - inv(prev)) in FP64: the off-diagonal part of D_k
// (-c2 V(G_i - G_j), the same for every energy and k-point) streams from the
// precomputed table, the diagonal is generated (negf::d_element,
// grid.f90:236-333), rows [rlo, rhi).
__device__ inline void form_mixed(float2 *__restrict__ M, const negf::Geo &g, const negf::Smem &js,
                                  const double2 *__restrict__ voff, int k, double2 E, int ik,
                                  const float2 *__restrict__ R, int rlo, int rhi) {
    const int N = g.N, ld = g.ld;
    const double2 *vs = g.vhat + (size_t)g.W * g.H * k;
    const double2 *vk = voff + (size_t)N * ld * k;
    // work items (row, 8-column chunk), rows fastest: every thread busy, loads
    // coalesced along the rows, sixteen loads in flight per item
    constexpr int CH = 8;
    const int nrows = rhi - rlo, nch = (N + CH - 1) / CH, nitem = nrows * nch;
    for (int it = threadIdx.x; it < nitem; it += NT) {
        const int t = rlo + it % nrows, j0 = (it / nrows) * CH;
        double2 d[CH];
        float2 r[CH];
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int j = j0 + q;
            d[q] = make_double2(0.0, 0.0);
            r[q] = make_float2(0.f, 0.f);
            if (j < N) {
                d[q] = __ldg(vk + t + (size_t)ld * j);
                if (R) r[q] = ldcg2(R + t + (size_t)ld * j);
            }
        }
#pragma unroll
        for (int q = 0; q < CH; ++q) {
            const int j = j0 + q;
            if (j == t) d[q] = negf::d_element(g, js, vs, k, E, ik, t, t, js.nx[t], js.ny[t]);
            if (j < N) M[t + (size_t)ld * j] = make_float2((float)(d[q].x - (double)r[q].x),
                                                           (float)(d[q].y - (double)r[q].y));
        }
    }
}

// -c2 V(G_i - G_j) for every slice: out[k][j][i] (leading dimension ld), the
// off-diagonal elements of negf::d_element.  Grid (Nz), one slice per CTA.
__global__ void __launch_bounds__(NT) k_voff(negf::Geo g, double2 *__restrict__ out) {
    const int N = g.N, ld = g.ld, k = blockIdx.x;
    const double2 *vs = g.vhat + (size_t)g.W * g.H * k;
    double2 *o = out + (size_t)N * ld * k;
    for (int j = 0; j < N; ++j) {
        const int nxj = g.nx[j], nyj = g.ny[j];
        for (int i = threadIdx.x; i < ld; i += NT) {
            double2 v = make_double2(0.0, 0.0);
            if (i < N) {
                const double2 t = vs[(g.nx[i] - nxj + g.ngx) + g.W * (g.ny[i] - nyj + g.ngy)];
                v = make_double2(-t.x * g.c2, -t.y * g.c2);
            }
            o[i + (size_t)ld * j] = v;
        }
    }
}

// Stores the raw inverse R (working layout) as the split tiles of slot b,
// with its pivot rows and row exponents.
__device__ inline void store_factor(const float2 *__restrict__ R, const MixedLayout &L, const GjSmem &s,
                                    int *rexpN, unsigned char *jm, int b, const Team &tm) {
    const int N = L.N, ld = L.ld, tid = threadIdx.x;
    int *prow_g = (int *)(jm + L.off_prow) + (size_t)b * N;
    int *rexp_g = (int *)(jm + L.off_rexp) + (size_t)b * N;
    unsigned char *tiles = jm + L.off_tiles + (size_t)b * L.mat_bytes;
    const int2 rr = team_range(tm, N, 8);
    for (int t = rr.x + tid; t < rr.y; t += NT) {
        float m = 0.0f;
#pragma unroll 8
        for (int j = 0; j < N; ++j) {
            const float2 v = ldcg2(R + t + (size_t)ld * j);
            m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
        }
        const int e = tc::scale_exponent(m);
        rexpN[t] = e;
        rexp_g[t] = e;
        prow_g[t] = s.prow[t];
    }
    team_sync(tm);
    if (tm.n > 1) {
        for (int t = tid; t < N; t += NT) rexpN[t] = __ldcg(rexp_g + t);
        __syncthreads();
    }
    // this CTA's tiles (row tile major)
    const int2 ur = team_range(tm, L.ntr * L.nkc, 1);
    const int r = tid % TM, h = tid / TM;
    for (int u = ur.x; u < ur.y; ++u) {
        const int rt = u / L.nkc, kc = u % L.nkc;
        const int row = rt * TM + r;
        if (rt == L.ntr - 1 && r >= L.last_rows) continue;  // not stored
        const float sc = tc::exp2i(row < N ? -rexpN[row] : 0);
        unsigned char *tile = tiles + factor_tile_off(L, rt, kc);
        const uint32_t pl = factor_plane(L, rt);
#pragma unroll
        for (int g2 = 0; g2 < 2; ++g2) {
            const int kg = 2 * h + g2;
            float2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int col = kc * KB + 8 * kg + q;
                float2 x = (row < N && col < N) ? ldcg2(R + row + (size_t)ld * col) : make_float2(0.f, 0.f);
                v[q] = make_float2(x.x * sc, x.y * sc);
            }
            __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const tc::Split2 a = tc::split_fp16(v[q].x), bb = tc::split_fp16(v[q].y);
                rh[q] = a.hi; rl[q] = a.lo; ih[q] = bb.hi; il[q] = bb.lo;
            }
            const uint32_t off = tc::kmajor_offset(r, 8 * kg, KB);
            *(uint4 *)(tile + 0 * pl + off) = *(const uint4 *)rh;
            *(uint4 *)(tile + 1 * pl + off) = *(const uint4 *)rl;
            *(uint4 *)(tile + 2 * pl + off) = *(const uint4 *)ih;
            *(uint4 *)(tile + 3 * pl + off) = *(const uint4 *)il;
        }
    }
    __syncthreads();
}

// One CTA per job (persistent over the wave): the right-connected sweep
// gR(b) = inv(D_b - gR(b+1)), b = Nz-1 .. 1, then G_11 = inv(D_0 - gR(1))
// (math_kernel.f90:81-118), every inverse stored as a split-tile factor, and
// x0(:, j) = G_11(:, oc[j]) for the open channels oc of the right lead.
// tmC maps the CTA's two working matrices as (row, column, 0|1, CTA).
__global__ void __launch_bounds__(NT, 1) k_mixed_sweep(MixedArgs a, const __grid_constant__ CUtensorMap tmC) {
    extern __shared__ __align__(128) unsigned char smem[];
    const MixedLayout &L = a.L;
    const negf::Geo &g = a.g;
    const int N = L.N, Nz = L.Nz, ld = L.ld, tid = threadIdx.x;
    // a.cpj CTAs (one cluster) per job; slot = the job's wave slot in the scratch
    const int slot = blockIdx.x / a.cpj, nslot = gridDim.x / a.cpj;
    GjSmem s = carve_gj(smem, N);
    size_t off = gj_smem_bytes(N);
    unsigned char *pipe_smem = smem + off;
    off += (pipe_smem_bytes(N) + 127) / 128 * 128;
    unsigned char *jscr = a.scratch + (size_t)slot * L.scratch_bytes;
    float2 *W0 = (float2 *)jscr;
    float2 *W1 = W0 + (size_t)N * ld;
    Pipe P = carve_pipe(pipe_smem, N, (unsigned char *)(W1 + (size_t)N * ld));
    const int rank = (int)(blockIdx.x % a.cpj);
    negf::Smem js = carve_job_slim(smem + off, N, P.sC, jscr + L.off_sig + (size_t)rank * job_sig_bytes(N));
    off += job_smem_bytes_slim(N);
    int *rexpN = P.rexpW;  // free while a factor is stored
    Team tm{rank, a.cpj, (int *)(jscr + L.off_gx), (int *)(smem + off), 0u};
    for (int i = tid; i < N; i += NT) { js.nx[i] = g.nx[i]; js.ny[i] = g.ny[i]; }
    gj_identity(s, N);
    pipe_setup(P);
    const int2 fr = team_range(tm, N, 8);  // this CTA's rows of the formation and of x0
    for (int w = slot; w < a.njobs; w += nslot) {
        const int2 jb = a.jobs[w];
        const double e = a.E[jb.x];
        const double2 E = make_double2(e, g.eta);
        unsigned char *jm = a.jobmem + (size_t)w * L.job_bytes;
        negf::job_vectors(g, js, E, e, jb.y);
        __syncthreads();
        negf::open_cols(N, js, js.gR);
        __syncthreads();
        const int nopen = *js.nrows;  // the same in every CTA of the team
        int *oc = (int *)(jm + L.off_oc);
        if (nopen > L.ncap) {
            if (tid == 0 && tm.rank == 0) a.status[w] = -1;
            __syncthreads();
            continue;
        }
        if (tm.rank == 0) {
            for (int j = tid; j < nopen; j += NT) oc[j] = js.rows[j];
            if (tid == 0) oc[L.ncap] = nopen;
        }
        float2 *cur = W0, *oth = W1;
        int zc = 0, info = 0, err = 0;
        for (int b = Nz - 1; b >= 0; --b) {
            form_mixed(oth, g, js, a.voff, b, E, jb.y, b < Nz - 1 ? cur : nullptr, fr.x, fr.y);
            team_sync(tm);
            float2 *tt = cur; cur = oth; oth = tt;
            zc ^= 1;
            const CMat cm{&tmC, zc, slot};
            const int r = gj_invert(cur, N, ld, s, P, cm, &err, tm);
            if (r && !info) info = r;
            if (err) break;  // uniform over the team (team_or)
            store_factor(cur, L, s, rexpN, jm, b, tm);
        }
        if (!err) {
            float2 *x0 = (float2 *)(jm + L.off_x);  // slice 0
            for (int j = 0; j < L.ncap; ++j) {
                const int jc = j < nopen ? s.iprow[js.rows[j]] : -1;
                for (int r = fr.x + tid; r < fr.y; r += NT)
                    x0[r + (size_t)N * j] = jc >= 0 ? ldcg2(cur + s.prow[r] + (size_t)ld * jc) : make_float2(0.f, 0.f);
            }
        }
        if (tid == 0 && tm.rank == 0) a.status[w] = err ? -2 : info;
        // the next job's formation overwrites the working matrices that x0 read
        team_sync(tm);
        if (err) break;
    }
    pipe_teardown(P);
    // no CTA leaves while the other may still read its shared memory (team_or)
    if (tm.n > 1) cluster_sync();
}

// ======================================================= refinement passes
// y = alpha * (gR(slot) v) + wadd with gR(slot) applied from its split-tile
// factor: gR(r, c) = R(prow[r], iprow[c]), so with v_p(k) = v(prow[k]) and
// z = R v_p, y(iprow[t]) = alpha z(t) + wadd(iprow[t]).  v = v1 - v2 (v2 may be
// null).  The B operand v_p is converted once per product into split tiles
// (one exponent per column over all N rows) in the CTA's scratch; then for
// each 128-row tile of R the K chunks stream through a pipeline of bulk
// copies (A: a ring of pa 32 KB factor tiles, as deep as shared memory allows
// for the vector block's width; B: one chunk) into tcgen05 MMAs.
enum PassMode { PASS_X0 = 0, PASS_BACK = 1, PASS_CORR = 2 };
constexpr int PA_MIN = 3, PA_MAX = 6;  // A ring stages (one 32 KB factor tile each)
constexpr int PB = 3;                  // B ring stages (one K chunk of the vector block each)

struct PassSmem {
    int pa;               // A ring stages
    unsigned char *stA;   // pa x TILE_BYTES
    unsigned char *stB;   // PB x (ncap * 256)
    int *cexp;            // [ncap] column exponents of the current product's v
    unsigned *cmax;       // [ncap] column maxima (float bits) of the next product's v
    unsigned *cmaxPeer;   // [2][ncap] the team's other CTA's maxima, by exchange parity
    uint64_t *fullA, *emptyA, *fullB, *emptyB, *accFull, *accEmpty, *bReady;
    uint64_t *maxReady;   // the other CTA's maxima have arrived
    uint64_t *convReady;  // the other CTA has converted its chunks of the next v
    uint32_t *tslot;
    double *red;          // [2 * NWARP]
};
constexpr int PASS_BARS = 2 * PA_MAX + 2 * PB + 2 + 2 + 1 + 2;
__host__ __device__ inline size_t pass_smem_bytes(int N, int ncap, int pa) {
    size_t b = pa * TILE_BYTES + PB * (size_t)ncap * 256;
    b += 4 * (size_t)ncap * 4 + PASS_BARS * 8 + 16 + 2 * NWARP * 8;
    (void)N;
    return (b + 127) / 128 * 128;
}
__device__ inline PassSmem carve_pass(unsigned char *base, int ncap, int pa) {
    PassSmem p;
    unsigned char *q = base;
    p.pa = pa;
    p.stA = q; q += pa * TILE_BYTES;
    p.stB = q; q += PB * (size_t)ncap * 256;
    p.cexp = (int *)q; q += (size_t)ncap * 4;
    p.cmax = (unsigned *)q; q += (size_t)ncap * 4;
    p.cmaxPeer = (unsigned *)q; q += 2 * (size_t)ncap * 4;
    q = (unsigned char *)(((uintptr_t)q + 15) & ~(uintptr_t)15);
    uint64_t *bar = (uint64_t *)q;
    p.fullA = bar; p.emptyA = bar + PA_MAX;
    p.fullB = bar + 2 * PA_MAX; p.emptyB = p.fullB + PB;
    p.accFull = p.emptyB + PB; p.accEmpty = p.accFull + 2;
    p.bReady = p.accEmpty + 2;
    p.maxReady = p.bReady + 1;
    p.convReady = p.maxReady + 1;
    q += PASS_BARS * 8;
    p.tslot = (uint32_t *)q; q += 16;
    p.red = (double *)q;
    return p;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc::smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     tc::smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
                 : "memory");
}
// barrier 1 of the four epilogue warps; and its OR-reduction (a uniform
// decision for all four)
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, 128;\n" ::: "memory"); }
__device__ __forceinline__ int epi_any(int v) {
    int r;
    asm volatile(
        "{\n .reg .pred q;\n setp.ne.s32 q, %1, 0;\n bar.red.or.pred q, 1, 128, q;\n selp.s32 %0, 1, 0, q;\n}\n"
        : "=r"(r)
        : "r"(v)
        : "memory");
    return r;
}

// MMAs of one staged K chunk with N = npad output columns (one thread).
__device__ inline void issue_pass_chunk(const unsigned char *sA, const unsigned char *sB, int npad,
                                        uint32_t tbase, bool first) {
    constexpr uint32_t SBO = (KB / 8) * 128, LBO = 128;
    const uint32_t id = tc::idesc_f16(TM, npad, false), idn = tc::idesc_f16(TM, npad, true);
    const uint32_t dre = tbase, dim = tbase + npad;
    const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
    const uint32_t aplane = TM * KB * 2, bplane = npad * KB * 2;
    const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
#pragma unroll
    for (int ks = 0; ks < KB / 16; ++ks) {
        const uint32_t koff = ks * 256;
#pragma unroll
        for (int sp = 0; sp < 3; ++sp) {
            const uint64_t are = tc::sdesc(a0 + (0 + pa[sp]) * aplane + koff, LBO, SBO);
            const uint64_t aim = tc::sdesc(a0 + (2 + pa[sp]) * aplane + koff, LBO, SBO);
            const uint64_t bre = tc::sdesc(b0 + (0 + pb[sp]) * bplane + koff, LBO, SBO);
            const uint64_t bim = tc::sdesc(b0 + (2 + pb[sp]) * bplane + koff, LBO, SBO);
            const uint32_t acc = (first && ks == 0 && sp == 0) ? 0u : 1u;
            tc::mma_f16(dre, are, bre, id, acc);
            tc::mma_f16(dre, aim, bim, idn, 1u);
            tc::mma_f16(dim, are, bim, id, acc);
            tc::mma_f16(dim, aim, bre, id, 1u);
        }
    }
}

// Product s of a pass: y = alpha gR(slot) (v1 - v2) + wadd, written to out
// (and xacc += y); the next product's v is vn1 - y (vn1 null: y itself).
struct Prod {
    int slot;
    const float2 *v1, *v2;
    float2 *out;
    float alpha;
    const float2 *wadd;
    float2 *xacc;
    const float2 *vn1;
};
__device__ inline int pass_nprod(int mode, int Nz) { return mode == PASS_CORR ? Nz : Nz - 1; }
// x = x0 slices, rc = residual / correction stage, d = two correction slices,
// xa = the solution that d accumulates into (CORR, null on the last iteration)
__device__ inline Prod pass_prod(int mode, int s, int Nz, size_t sl, float2 *x, float2 *rc, float2 *d, float2 *xa) {
    Prod q;
    q.wadd = nullptr;
    q.xacc = nullptr;
    q.vn1 = nullptr;
    q.v2 = nullptr;
    if (mode == PASS_X0) {          // x0(b) = -gR(b) x0(b-1), b = s + 1
        const int b = s + 1;
        q.slot = b; q.v1 = x + (b - 1) * sl; q.out = x + b * sl; q.alpha = -1.f;
    } else if (mode == PASS_BACK) { // c(b) = r(b) - gR(b+1) c(b+1), b = Nz-2-s, in place of r
        const int b = Nz - 2 - s;
        q.slot = b + 1; q.v1 = rc + (b + 1) * sl; q.out = rc + b * sl; q.alpha = -1.f; q.wadd = rc + b * sl;
    } else {                        // d(b) = gR(b) (c(b) - d(b-1)), b = s
        const int b = s;
        q.slot = b; q.v1 = rc + b * sl; q.v2 = b ? d + ((b - 1) & 1) * sl : nullptr;
        q.out = d + (b & 1) * sl; q.alpha = 1.f;
        q.xacc = (b < Nz - 1 && xa) ? xa + b * sl : nullptr;
        q.vn1 = b + 1 < Nz ? rc + (b + 1) * sl : nullptr;  // the next product reads c(b+1) - d(b)
    }
    return q;
}

// Arrival on the barrier at the same shared-memory place of CTA `peer` of the
// cluster, releasing this thread's (and, through the barrier before it, its
// warps') earlier writes at cluster scope.
__device__ __forceinline__ void mbar_arrive_peer(uint64_t *bar, int peer) {
    uint32_t ra;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(ra) : "r"(tc::smem_u32(bar)), "r"(peer));
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(ra) : "memory");
}
// mbar_wait with acquire at cluster scope (the arrival came from the other CTA)
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t *bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = tc::smem_u32(bar);
    for (uint32_t it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// The epilogue warps' conversion of v = v1 - v2 into the split-fp16 B chunks
// (chunk kc at kc * npad * 256 B of bscr, planes of npad * KB fp16), one
// exponent per column.  First, if cmax is null, the column maxima by a pass
// over v; else the maxima the previous epilogue accumulated in cmax.
__device__ inline void pass_convert(const MixedLayout &L, const PassSmem &p, const float2 *__restrict__ v1,
                                    const float2 *__restrict__ v2, int nopen, int npad, unsigned char *bscr,
                                    bool from_cmax, int kc0, int kc1) {
    const int N = L.N, et = threadIdx.x - 128, ew = et >> 5, lane = et & 31;
    if (!from_cmax) {
        for (int j = ew; j < npad; j += 4) {
            float m = 0.0f;
            if (j < nopen)
                for (int k = lane; k < N; k += 32) {
                    float2 x = v1[k + (size_t)N * j];
                    if (v2) { const float2 y = v2[k + (size_t)N * j]; x.x -= y.x; x.y -= y.y; }
                    m = fmaxf(m, fmaxf(fabsf(x.x), fabsf(x.y)));
                }
            m = __uint_as_float(__reduce_max_sync(0xffffffffu, __float_as_uint(m)));
            if (lane == 0) p.cexp[j] = tc::scale_exponent(m);
        }
    } else {
        for (int j = et; j < npad; j += 128) p.cexp[j] = tc::scale_exponent(__uint_as_float(p.cmax[j]));
    }
    epi_bar();
    for (int j = et; j < npad; j += 128) p.cmax[j] = 0u;
    const uint32_t bplane = npad * KB * 2;
    const int nitem = (kc1 - kc0) * npad * 4;  // this CTA's chunks [kc0, kc1)
    // two items per thread per round: all 32 loads in flight before the first use
    for (int i0 = et; i0 < nitem; i0 += 256) {
        float2 x1[2][8], x2[2][8];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int item = i0 + 128 * h;
            const int g4 = item & 3, j = (item >> 2) % npad, kc = kc0 + (item >> 2) / npad;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = kc * KB + 8 * g4 + q;
                const bool ok = item < nitem && k < N && j < nopen;
                x1[h][q] = ok ? v1[k + (size_t)N * j] : make_float2(0.f, 0.f);
                x2[h][q] = (ok && v2) ? v2[k + (size_t)N * j] : make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int item = i0 + 128 * h;
            if (item >= nitem) break;
            const int g4 = item & 3, j = (item >> 2) % npad, kc = kc0 + (item >> 2) / npad;
            const float sc = tc::exp2i(-p.cexp[j]);
            __align__(16) __half rh[8], rl[8], ih[8], il[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const tc::Split2 a = tc::split_fp16((x1[h][q].x - x2[h][q].x) * sc),
                                 b = tc::split_fp16((x1[h][q].y - x2[h][q].y) * sc);
                rh[q] = a.hi; rl[q] = a.lo; ih[q] = b.hi; il[q] = b.lo;
            }
            unsigned char *dst = bscr + (size_t)kc * npad * 256 + tc::kmajor_offset(j, 8 * g4, KB);
            *(uint4 *)(dst + 0 * bplane) = *(const uint4 *)rh;
            *(uint4 *)(dst + 1 * bplane) = *(const uint4 *)rl;
            *(uint4 *)(dst + 2 * bplane) = *(const uint4 *)ih;
            *(uint4 *)(dst + 3 * bplane) = *(const uint4 *)il;
        }
    }
    // the bulk copies (async proxy) read what these generic stores wrote
    asm volatile("fence.proxy.async.global;\n" ::: "memory");
    epi_bar();
}

// Pipeline counters of the roles, carried across the jobs of a CTA.
struct PassCnt {
    uint32_t a, b, u, r, x;  // A stages, B stages, accumulators, products, maxima exchanges
};
// The row tiles [rt0, rt1) a CTA computes; with a team of two (peer >= 0)
// the other CTA computes the rest, and per product the two exchange their
// column maxima (DSMEM) and convert the K chunks of their own rows of the
// next vector into the job's shared B scratch.
struct PassPart {
    int rt0, rt1, kc0, kc1, peer;
};

// All products of one pass of one job through the warp-specialised pipeline:
//   warp 0, lane 0   streams the factor tiles of every product (row tile by
//                    row tile, K chunk by K chunk) through the A ring; they do
//                    not depend on the data, so it runs as far ahead as the
//                    ring allows, across products;
//   warp 2, lane 0   streams the B chunks of product s (the split vector
//                    block in the CTA's global scratch) through the B ring,
//                    once per row tile, as soon as the epilogue warps have
//                    converted v_s;
//   warp 1, lane 0   the MMAs of each row tile into one of two tensor-memory
//                    accumulators (2 ncap columns each);
//   warps 4-7        the epilogue of each row tile: y from the accumulator
//                    (tcgen05.ld, one lane quadrant per warp) times
//                    2^(row + column exponent), the stores, the column maxima
//                    of the next product's v (one redux per column); after the
//                    last row tile, the conversion of v_{s+1}.
// Returns false if a wait timed out (uniform over the CTA).
__device__ bool pass_run(const MixedLayout &L, const PassSmem &p, unsigned char *jm, unsigned char *bscr, int mode,
                         float2 *x, float2 *rc, float2 *d, float2 *xa, int nopen, int npad, uint32_t tbase,
                         PassCnt &cnt, const PassPart &pt) {
    const int N = L.N, Nz = L.Nz, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nprod = pass_nprod(mode, Nz), ntr = L.ntr, nkc = L.nkc;
    const int nrt = pt.rt1 - pt.rt0;  // this CTA's row tiles
    const size_t sl = (size_t)L.ncap * N;
    const uint32_t bbytes = (uint32_t)npad * 256, bst = (uint32_t)L.ncap * 256;
    int err = 0;
    if (warp == 0) {
        // -------------------------------------------------------- A producer
        if (lane == 0) {
            uint32_t ia = cnt.a;
            for (int s = 0; s < nprod && !err; ++s) {
                const Prod q = pass_prod(mode, s, Nz, sl, x, rc, d, xa);
                const unsigned char *tiles = jm + L.off_tiles + (size_t)q.slot * L.mat_bytes;
                for (int t = 0; t < nrt * nkc && !err; ++t, ++ia) {
                    const uint32_t st = ia % (uint32_t)p.pa;
                    if (ia >= (uint32_t)p.pa && !tc::mbar_wait(&p.emptyA[st], ((ia / p.pa) - 1) & 1u, WAIT_LIMIT)) { err = 1; break; }
                    const int rt = pt.rt0 + t / nkc, kc = t % nkc;
                    const unsigned char *src = tiles + factor_tile_off(L, rt, kc);
                    if (rt < ntr - 1) {
                        mbar_expect_tx(&p.fullA[st], (uint32_t)TILE_BYTES);
                        bulk_g2s(p.stA + st * TILE_BYTES, src, (uint32_t)TILE_BYTES, &p.fullA[st]);
                    } else {
                        // a last-row-tile tile: each plane to the start of its full-size
                        // plane in the stage (the rows past it are never read back)
                        mbar_expect_tx(&p.fullA[st], 4 * L.last_plane);
                        for (int pl = 0; pl < 4; ++pl)
                            bulk_g2s(p.stA + st * TILE_BYTES + (size_t)pl * (TM * KB * 2), src + (size_t)pl * L.last_plane,
                                     L.last_plane, &p.fullA[st]);
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 2) {
        // -------------------------------------------------------- B producer
        if (lane == 0) {
            uint32_t ib = cnt.b;
            for (int s = 0; s < nprod && !err; ++s) {
                if (!tc::mbar_wait(p.bReady, (cnt.r + s) & 1u, WAIT_LIMIT)) { err = 1; break; }
                // ... and the other CTA's chunks of the same vector
                if (pt.peer >= 0 && !mbar_wait_cluster(p.convReady, (cnt.r + s) & 1u, WAIT_LIMIT)) { err = 1; break; }
                for (int t = 0; t < nrt * nkc && !err; ++t, ++ib) {
                    const uint32_t st = ib % PB;
                    if (ib >= PB && !tc::mbar_wait(&p.emptyB[st], ((ib / PB) - 1) & 1u, WAIT_LIMIT)) { err = 1; break; }
                    mbar_expect_tx(&p.fullB[st], bbytes);
                    bulk_g2s(p.stB + st * bst, bscr + (size_t)(t % nkc) * bbytes, bbytes, &p.fullB[st]);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------ MMA issuer
        if (lane == 0) {
            uint32_t ia = cnt.a, ib = cnt.b, iu = cnt.u;
            for (int s = 0; s < nprod && !err; ++s) {
                for (int rt = pt.rt0; rt < pt.rt1 && !err; ++rt, ++iu) {
                    const uint32_t buf = iu & 1u, dacc = tbase + buf * (2 * L.ncap);
                    if (iu >= 2 && !tc::mbar_wait(&p.accEmpty[buf], ((iu >> 1) - 1) & 1u, WAIT_LIMIT)) { err = 1; break; }
                    for (int kc = 0; kc < nkc; ++kc, ++ia, ++ib) {
                        const uint32_t sa = ia % (uint32_t)p.pa, sb = ib % PB;
                        if (!tc::mbar_wait(&p.fullA[sa], (ia / p.pa) & 1u, WAIT_LIMIT) ||
                            !tc::mbar_wait(&p.fullB[sb], (ib / PB) & 1u, WAIT_LIMIT)) { err = 1; break; }
                        tc::fence_after_sync();
                        issue_pass_chunk(p.stA + sa * TILE_BYTES, p.stB + sb * bst, npad, dacc, kc == 0);
                        tc::mma_commit(&p.emptyA[sa]);
                        tc::mma_commit(&p.emptyB[sb]);
                    }
                    if (!err) tc::mma_commit(&p.accFull[buf]);
                }
            }
        }
        __syncwarp();
    } else if (warp >= 4) {
        // -------------------------------------------------------- epilogue
        const int q4 = warp & 3;
        const uint32_t lb = (uint32_t)(32 * q4) << 16;
        uint32_t iu = cnt.u;
        {
            const Prod q0 = pass_prod(mode, 0, Nz, sl, x, rc, d, xa);
            pass_convert(L, p, q0.v1, q0.v2, nopen, npad, bscr, false, pt.kc0, pt.kc1);
            if (tid == 128) {
                mbar_arrive(p.bReady);
                if (pt.peer >= 0) mbar_arrive_peer(p.convReady, pt.peer);
            }
        }
        for (int s = 0; s < nprod && !err; ++s) {
            const Prod q = pass_prod(mode, s, Nz, sl, x, rc, d, xa);
            const int *rexp_g = (const int *)(jm + L.off_rexp) + (size_t)q.slot * N;
            for (int rt = pt.rt0; rt < pt.rt1; ++rt, ++iu) {
                const uint32_t buf = iu & 1u, dacc = tbase + lb + buf * (2 * L.ncap);
                const int r = 32 * q4 + lane, i = rt * TM + r;
                const bool rv = i < N;
                const int er = rv ? rexp_g[i] : 0;
                if (epi_any(!tc::mbar_wait(&p.accFull[buf], (iu >> 1) & 1u, WAIT_LIMIT))) { err = 1; break; }
                tc::fence_after_sync();
                for (int c16 = 0; c16 < npad / 16; ++c16) {
                    float re[16], im[16];
                    tc::tmem_ld16(dacc + c16 * 16, re);
                    tc::tmem_ld16(dacc + npad + c16 * 16, im);
                    float2 wv[16], xv[16], nv[16];
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int j = c16 * 16 + u;
                        const bool ok = rv && j < nopen;
                        wv[u] = (ok && q.wadd) ? q.wadd[i + (size_t)N * j] : make_float2(0.f, 0.f);
                        xv[u] = (ok && q.xacc) ? q.xacc[i + (size_t)N * j] : make_float2(0.f, 0.f);
                        nv[u] = (ok && q.vn1) ? q.vn1[i + (size_t)N * j] : make_float2(0.f, 0.f);
                    }
                    tc::tmem_wait_ld();
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const int j = c16 * 16 + u;
                        float2 y = make_float2(0.f, 0.f);
                        if (rv && j < nopen) {
                            const float f = q.alpha * tc::exp2i(er + p.cexp[j]);
                            y = make_float2(fmaf(re[u], f, wv[u].x), fmaf(im[u], f, wv[u].y));
                        }
                        if (rv && j < L.ncap) {
                            q.out[i + (size_t)N * j] = y;
                            if (q.xacc && j < nopen) q.xacc[i + (size_t)N * j] = make_float2(xv[u].x + y.x, xv[u].y + y.y);
                        }
                        // |entry| of the next product's v in this column
                        const float2 vn = q.vn1 ? make_float2(nv[u].x - y.x, nv[u].y - y.y) : y;
                        const float m = (rv && j < nopen) ? fmaxf(fabsf(vn.x), fabsf(vn.y)) : 0.0f;
                        const unsigned wm = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
                        if (lane == 0 && wm) atomicMax(&p.cmax[j], wm);
                    }
                }
                // accumulator read: it may take the row tile after next
                tc::fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(&p.accEmpty[buf]);
            }
            if (err) break;
            if (s + 1 < nprod) {
                epi_bar();  // every store of y and every column maximum of this product
                if (pt.peer >= 0) {
                    // column maxima of the next v over both CTAs' rows
                    const int et = tid - 128;
                    const uint32_t px = cnt.x + (uint32_t)s;
                    unsigned *dst = p.cmaxPeer + (px & 1u) * L.ncap;
                    for (int j = et; j < npad; j += 128) {
                        uint32_t ra;
                        asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(ra) : "r"(tc::smem_u32(dst + j)), "r"(pt.peer));
                        asm volatile("st.shared::cluster.u32 [%0], %1;\n" ::"r"(ra), "r"(p.cmax[j]) : "memory");
                    }
                    epi_bar();
                    if (tid == 128) mbar_arrive_peer(p.maxReady, pt.peer);
                    if (epi_any(!mbar_wait_cluster(p.maxReady, px & 1u, WAIT_LIMIT))) { err = 1; break; }
                    for (int j = et; j < npad; j += 128) p.cmax[j] = max(p.cmax[j], dst[j]);
                    epi_bar();
                }
                const Prod qn = pass_prod(mode, s + 1, Nz, sl, x, rc, d, xa);
                pass_convert(L, p, qn.v1, qn.v2, nopen, npad, bscr, true, pt.kc0, pt.kc1);
                if (tid == 128) {
                    mbar_arrive(p.bReady);
                    if (pt.peer >= 0) mbar_arrive_peer(p.convReady, pt.peer);
                }
            }
        }
    }
    if (__syncthreads_or(err)) return false;
    cnt.a += (uint32_t)(nprod * nrt * nkc);
    cnt.b += (uint32_t)(nprod * nrt * nkc);
    cnt.u += (uint32_t)(nprod * nrt);
    cnt.r += (uint32_t)nprod;
    cnt.x += (uint32_t)(nprod - 1);
    return true;
}

// One CTA per job: PASS_X0 x0(b) = -gR(b) x0(b-1), b = 1..Nz-1 (x0(0) from the
// sweep); PASS_BACK c(Nz-1) = r(Nz-1), c(b) = r(b) - gR(b+1) c(b+1) in place
// of r; PASS_CORR d(0) = G_11 c(0), d(b) = gR(b) (c(b) - d(b-1)), then
// tau = sum_ij gamma_L,i gamma_R,oc_j |2 dz^2 (x0 + d)(Nz-1)(i, j)|^2 in FP64
// (grid.f90:362-383) and the norms of d and x0 + d on the rows that enter it.
__global__ void __launch_bounds__(NT, 1) k_mixed_pass(MixedArgs a, int mode, int iter, int last) {
    extern __shared__ __align__(128) unsigned char smem[];
    const MixedLayout &L = a.L;
    const int N = L.N, Nz = L.Nz, tid = threadIdx.x;
    PassSmem p = carve_pass(smem, L.ncap, a.pa);
    // the job vectors of the tau step live in the A ring, idle by then
    negf::Smem js = carve_job(p.stA, N);
    uint32_t ncols = 32;
    while (ncols < 4u * L.ncap) ncols <<= 1;  // two accumulators of 2 ncap columns
    if (tid < 32) tc::tmem_alloc(p.tslot, ncols);
    if (tid == 0) {
        for (int s = 0; s < p.pa; ++s) { tc::mbar_init(&p.fullA[s], 1); tc::mbar_init(&p.emptyA[s], 1); }
        for (int s = 0; s < PB; ++s) { tc::mbar_init(&p.fullB[s], 1); tc::mbar_init(&p.emptyB[s], 1); }
        for (int s = 0; s < 2; ++s) { tc::mbar_init(&p.accFull[s], 1); tc::mbar_init(&p.accEmpty[s], 4); }
        tc::mbar_init(p.bReady, 1);
        tc::mbar_init(p.maxReady, 1);
        tc::mbar_init(p.convReady, 1);
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    // a.cpj CTAs (one cluster) per job, as in the sweep: each computes its share
    // of the row tiles of every product
    const int cpj = a.cpj, rank = (int)(blockIdx.x % cpj), slot = (int)(blockIdx.x / cpj);
    const int nslot = (int)(gridDim.x / cpj);
    if (cpj > 1) cluster_sync();  // both CTAs' barriers exist before either arrives on the other's
    __shared__ int ok_slots[2];
    Team team{rank, cpj, nullptr, ok_slots, 0u};
    const int rt0 = L.ntr * rank / cpj, rt1 = L.ntr * (rank + 1) / cpj;
    const PassPart pt{rt0, rt1, min(L.nkc, rt0 * (TM / KB)), min(L.nkc, rt1 * (TM / KB)), cpj > 1 ? 1 - rank : -1};
    const uint32_t tbase = *p.tslot;
    PassCnt cnt{0, 0, 0, 0, 0};
    unsigned char *bscr = a.scratch + (size_t)slot * L.scratch_bytes;
    const size_t sl = (size_t)L.ncap * N;  // float2 per slice of a vector array
    bool ok = true;
    for (int w = slot; w < a.njobs && ok; w += nslot) {
        if (a.status[w] != 0) continue;
        unsigned char *jm = a.jobmem + (size_t)w * L.job_bytes;
        const int nopen = ((const int *)(jm + L.off_oc))[L.ncap];
        const int npad = max(16, rup(nopen, 16));
        float2 *x = (float2 *)(jm + L.off_x), *rc = (float2 *)(jm + L.off_rc), *d = (float2 *)(jm + L.off_d);
        // unless this is the last iteration, CORR folds d into x(b) for b < Nz-1
        // on the way (the last slice is kept so that tau is formed from x + d in FP64)
        ok = pass_run(L, p, jm, bscr, mode, x, rc, d, (mode == PASS_CORR && !last) ? x : nullptr, nopen, npad,
                      tbase, cnt, pt);
        // the same outcome in both CTAs of a team; the barrier also makes each
        // CTA's rows of the vectors visible to the other
        if (cpj > 1) ok = !team_or(team, !ok);
        if (mode == PASS_CORR && rank == 0) {
            if (ok) {
                // tau of x0 + d at the last slice, FP64
                const negf::Geo &g = a.g;
                const int2 jb = a.jobs[w];
                const double e = a.E[jb.x];
                for (int i = tid; i < N; i += NT) { js.nx[i] = g.nx[i]; js.ny[i] = g.ny[i]; }
                __syncthreads();
                negf::job_vectors(g, js, make_double2(e, g.eta), e, jb.y);
                __syncthreads();
                const int *oc = (const int *)(jm + L.off_oc);
                const float2 *xl = x + (size_t)(Nz - 1) * sl, *dl = d + ((Nz - 1) & 1) * sl;
                const double c2 = g.c2;
                double tau = 0.0, dn = 0.0, xn = 0.0;
                for (int e2 = tid; e2 < N * nopen; e2 += NT) {
                    const int i = e2 % N, j = e2 / N;
                    const double gl = js.gL[i];
                    if (gl == 0.0) continue;
                    const float2 a0 = xl[i + (size_t)N * j], a1 = dl[i + (size_t)N * j];
                    const double gx = ((double)a0.x + (double)a1.x) * c2, gy = ((double)a0.y + (double)a1.y) * c2;
                    tau += gl * js.gR[oc[j]] * (gx * gx + gy * gy);
                    dn += (double)a1.x * a1.x + (double)a1.y * a1.y;
                    xn += ((double)a0.x + a1.x) * ((double)a0.x + a1.x) + ((double)a0.y + a1.y) * ((double)a0.y + a1.y);
                }
                // fixed-order block reduction (bitwise repeatable)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    tau += __shfl_xor_sync(0xffffffffu, tau, o);
                    dn += __shfl_xor_sync(0xffffffffu, dn, o);
                    xn += __shfl_xor_sync(0xffffffffu, xn, o);
                }
                if ((tid & 31) == 0) {
                    p.red[(tid >> 5)] = tau;
                    p.red[NWARP + (tid >> 5)] = dn;
                }
                __syncthreads();
                if (tid == 0) {
                    double T = 0, D = 0;
                    for (int q = 0; q < NWARP; ++q) { T += p.red[q]; D += p.red[NWARP + q]; }
                    a.tau[w] = T;
                    a.dnorm[w] = sqrt(D);
                }
                __syncthreads();
                if ((tid & 31) == 0) p.red[tid >> 5] = xn;
                __syncthreads();
                if (tid == 0) {
                    double X = 0;
                    for (int q = 0; q < NWARP; ++q) X += p.red[q];
                    a.xnorm[w] = sqrt(X);
                    // remaining error after this correction: |d_k| times the contraction,
                    // estimated as |d_1| / |x| after the first step and |d_k| / |d_k-1| later
                    const double dn = a.dnorm[w], xnv = sqrt(X);
                    // no trace term (no open channel of the left lead, e.g. E at the
                    // band bottom): tau = 0 exactly, whatever the solution; an exactly
                    // zero solution with a zero correction has converged as well
                    const double corr = xnv > 0 ? dn / xnv : (dn > 0 ? INFINITY : 0.0);
                    const double rho = iter == 1 ? corr : (a.dprev[w] > 0 ? dn / a.dprev[w] : INFINITY);
                    const double est = 2.0 * fmax(a.tau[w], 1.0) * corr * rho;
                    a.dprev[w] = dn;
                    if (est < a.tol && isfinite(a.tau[w])) a.status[w] = MIX_DONE;
                }
                __syncthreads();
                // not converged and another iteration follows: fold d into the last slice
                if (!last && a.status[w] == 0)
                    for (int e2 = tid; e2 < N * nopen; e2 += NT) {
                        float2 *xv = (float2 *)xl + e2;
                        const float2 dv = dl[e2];
                        *xv = make_float2(xv->x + dv.x, xv->y + dv.y);
                    }
                __syncthreads();
            }
        }
        if (!ok && tid == 0 && rank == 0) a.status[w] = -2;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid < 32) tc::tmem_dealloc(tbase, ncols);
    // no CTA leaves while the other may still write its shared memory
    if (cpj > 1) cluster_sync();
}

// FP64 residual of the block-tridiagonal system for x0, one CTA per (job,
// slice b): r(b) = E_1 delta_b0 - x0(b-1) - D_b x0(b) - x0(b+1), D_b in FP64
// and the product on the FP64 tensor cores (DMMA warp tiles of
// negf::WarpAcc), 64 x 64 output tiles, K in chunks of 16, two stages: the
// table chunk of the next stage streams in by cp.async and the next x0 chunk
// (FP32) is loaded into registers while the current chunk is multiplied,
// then widened to FP64 into the other stage.  The product uses the
// -c2 V(G_i - G_j) table as it is, diagonal included; the epilogue replaces
// its diagonal term by the generated one (negf::d_element):
// D_b x = T_b x + (d_ii - T_b(i,i)) x_i.
__global__ void __launch_bounds__(NT, 2) k_mixed_residual(MixedArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const MixedLayout &L = a.L;
    const negf::Geo &g = a.g;
    const int N = L.N, Nz = L.Nz, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // jobs fastest: the CTAs in flight share slice b's D table in L2
    const int w = blockIdx.x, b = blockIdx.y;
    if (a.status[w] != 0) return;
    constexpr int KC = negf::KC, AP = negf::AP, BP = negf::BP, CM = negf::CM, CN = negf::CN;
    double2 *sA = (double2 *)smem;           // [2][KC][AP]
    double2 *sB = sA + 2 * KC * AP;          // [2][KC][BP]
    negf::Smem js = carve_job(smem + (size_t)2 * KC * (AP + BP) * 16, N);
    unsigned char *jm = a.jobmem + (size_t)w * L.job_bytes;
    const int *oc = (const int *)(jm + L.off_oc);
    const int nopen = oc[L.ncap];
    const int npad = max(16, rup(nopen, 16));
    const int2 jb = a.jobs[w];
    const double e = a.E[jb.x];
    const double2 E = make_double2(e, g.eta);
    for (int i = tid; i < N; i += NT) { js.nx[i] = g.nx[i]; js.ny[i] = g.ny[i]; }
    __syncthreads();
    negf::job_vectors(g, js, E, e, jb.y);
    __syncthreads();
    const size_t sl = (size_t)L.ncap * N;
    const float2 *x = (const float2 *)(jm + L.off_x);
    const float2 *xb = x + b * sl;
    float2 *out = (float2 *)(jm + L.off_rc) + b * sl;
    const double2 *vs = g.vhat + (size_t)g.W * g.H * b;
    const double2 *vt = a.voff + (size_t)N * L.ld * b;
    const int wm0 = (warp >> 2) * negf::WM, wn0 = (warp & 3) * negf::WN;
    const int nkc = (N + KC - 1) / KC;
    constexpr int BQ = (KC * CN) / NT;  // x0 values per thread per chunk
    for (int J0 = 0; J0 < npad; J0 += CN) {
        for (int I0 = 0; I0 < N; I0 += CM) {
            const bool active = (I0 + wm0 < N) && (J0 + wn0 < npad);
            negf::WarpAcc acc;
            acc.zero();
            float2 xr[BQ];
            auto load_a = [&](int st, int k0) {
                double2 *dA = sA + st * KC * AP;
#pragma unroll
                for (int q = 0; q < (KC * CM) / NT; ++q) {
                    const int e2 = tid + NT * q, kk = e2 / CM, ii = e2 % CM, k = k0 + kk, i = I0 + ii;
                    const bool v = k < N && i < N;
                    negf::cp_async16(dA + kk * AP + ii, vt + (v ? (i + (size_t)L.ld * k) : 0), v);
                }
                negf::cp_async_commit();
            };
            auto load_x = [&](int k0) {
#pragma unroll
                for (int q = 0; q < BQ; ++q) {
                    const int e2 = tid + NT * q, jj = e2 / KC, kk = e2 % KC, j = J0 + jj, k = k0 + kk;
                    xr[q] = (j < nopen && k < N) ? xb[k + (size_t)N * j] : make_float2(0.f, 0.f);
                }
            };
            auto store_x = [&](int st) {
                double2 *dB = sB + st * KC * BP;
#pragma unroll
                for (int q = 0; q < BQ; ++q) {
                    const int e2 = tid + NT * q, jj = e2 / KC, kk = e2 % KC;
                    dB[kk * BP + jj] = make_double2(xr[q].x, xr[q].y);
                }
            };
            load_a(0, 0);
            load_x(0);
            store_x(0);
            for (int c = 0; c < nkc; ++c) {
                negf::cp_async_wait<0>();
                // chunk c is in stage c & 1, and every warp has finished chunk c - 1,
                // so stage (c + 1) & 1 may be refilled
                __syncthreads();
                if (c + 1 < nkc) {
                    load_a((c + 1) & 1, (c + 1) * KC);
                    load_x((c + 1) * KC);
                }
                if (active) {
                    const double2 *cA = sA + (c & 1) * KC * AP;
                    const double2 *cB = sB + (c & 1) * KC * BP;
#pragma unroll
                    for (int kb = 0; kb < KC; kb += 4) acc.step(cA, AP, wm0, cB, BP, wn0, kb, lane);
                }
                if (c + 1 < nkc) store_x((c + 1) & 1);
            }
            // every warp is done with both stages before the next tile refills them
            __syncthreads();
            if (active) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int i = I0 + wm0 + 8 * m + (lane >> 2);
                    double2 dfix = make_double2(0.0, 0.0);
                    if (i < N) {
                        const double2 dii = negf::d_element(g, js, vs, b, E, jb.y, i, i, js.nx[i], js.ny[i]);
                        const double2 tii = vt[i + (size_t)L.ld * i];
                        dfix = make_double2(dii.x - tii.x, dii.y - tii.y);
                    }
#pragma unroll
                    for (int n = 0; n < 2; ++n)
#pragma unroll
                        for (int e3 = 0; e3 < 2; ++e3) {
                            const int j = J0 + wn0 + 8 * n + 2 * (lane & 3) + e3;
                            if (i < N && j < L.ncap) {
                                double rx = 0.0, ry = 0.0;
                                if (j < nopen) {
                                    const float2 xi = xb[i + (size_t)N * j];
                                    const double ax = acc.re[m][n][e3] + (dfix.x * xi.x - dfix.y * xi.y);
                                    const double ay = acc.im[m][n][e3] + (dfix.x * xi.y + dfix.y * xi.x);
                                    rx = -ax;
                                    ry = -ay;
                                    if (b > 0) { const float2 v = x[(b - 1) * sl + i + (size_t)N * j]; rx -= v.x; ry -= v.y; }
                                    if (b + 1 < Nz) { const float2 v = x[(b + 1) * sl + i + (size_t)N * j]; rx -= v.x; ry -= v.y; }
                                    if (b == 0 && i == oc[j]) rx += 1.0;
                                }
                                out[i + (size_t)N * j] = make_float2((float)rx, (float)ry);
                            }
                        }
                }
            }
        }
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
        else
            cudaGetLastError();
    }
    return fn;
}
// The C-tile map of the trailing update: nmat matrices per CTA (stride
// mat_stride bytes) for ncta CTAs (stride cta_stride), each N x N complex FP32
// with leading dimension ld; boxes of TM rows x PTN columns.
bool c_tile_map(CUtensorMap *m, void *base, int N, int ld, int nmat, size_t mat_stride, int ncta, size_t cta_stride) {
    EncodeTiledFn f = encode_tiled();
    if (!f || ld % 2 || mat_stride % 16 || cta_stride % 16 || ((uintptr_t)base & 15)) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)N, (cuuint64_t)N, (cuuint64_t)nmat, (cuuint64_t)ncta};
    const cuuint64_t strides[3] = {(cuuint64_t)ld * 8, (cuuint64_t)mat_stride, (cuuint64_t)cta_stride};
    const cuuint32_t box[4] = {(cuuint32_t)TM, (cuuint32_t)PTN, 1, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return f(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

#define CKM(x)                                                                             \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "negf_gpu: %s failed: %s\n", #x, cudaGetErrorString(e_));      \
            return NEGF_ERR_CUDA;                                                          \
        }                                                                                  \
    } while (0)

}  // namespace

extern "C" int negf_tc_product_check(const float *d_W, int32_t ldw, const float *d_B, int32_t ldb,
                                     const int32_t *d_rowmap, float *d_C, int32_t ldc, int32_t M, int32_t ncol,
                                     int32_t K, void *stream) {
    if (!d_W || !d_B || !d_rowmap || !d_C || M < 1 || ncol < 1 || K < 1 || K > KB || ldw < M || ldc < M)
        return NEGF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t smem = gj_smem_bytes(32) + tile_smem_bytes();
    CKM(cudaFuncSetAttribute(k_tc_product_check, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int *d_status = nullptr;
    CKM(cudaMalloc(&d_status, sizeof(int)));
    CKM(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    dim3 grid((M + TM - 1) / TM, (ncol + TN - 1) / TN);
    k_tc_product_check<<<grid, NT, smem, st>>>((const float2 *)d_W, ldw, (const float2 *)d_B, ldb, d_rowmap,
                                                (float2 *)d_C, ldc, M, ncol, K, d_status);
    CKM(cudaGetLastError());
    int h = 0;
    CKM(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));
    cudaFree(d_status);
    return h ? NEGF_ERR_CUDA : NEGF_OK;
}

extern "C" int negf_tc_inverse_check(const float *d_A, int32_t N, int32_t nmat, float *d_out, int32_t *d_info,
                                     void *stream) {
    if (!d_A || !d_out || !d_info || N < 1 || N > 1023 || nmat < 1) return NEGF_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t smem = gj_smem_bytes(N) + pipe_smem_bytes(N);
    float2 *work = nullptr;
    int *d_status = nullptr;
    unsigned char *pscr = nullptr;
    const int ld = rup(N, 8);  // the TMA strides of the trailing update need ld % 8 == 0
    CKM(cudaMalloc(&pscr, pipe_scratch_bytes(N) * nmat));
    CKM(cudaMalloc(&work, sizeof(float2) * (size_t)ld * N * nmat));
    CKM(cudaMalloc(&d_status, sizeof(int)));
    CKM(cudaMemcpy2DAsync(work, sizeof(float2) * ld, d_A, sizeof(float2) * N, sizeof(float2) * N, (size_t)N * nmat,
                          cudaMemcpyDeviceToDevice, st));
    CKM(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    CUtensorMap tm;
    if (!c_tile_map(&tm, work, N, ld, 1, (size_t)ld * N * 8, nmat, (size_t)ld * N * 8)) {
        cudaFree(work);
        cudaFree(d_status);
        cudaFree(pscr);
        return NEGF_ERR_CUDA;
    }
    CKM(cudaFuncSetAttribute(k_tc_inverse_check, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_tc_inverse_check<<<nmat, NT, smem, st>>>(work, N, ld, (float2 *)d_out, d_info, d_status, pscr, tm);
    CKM(cudaGetLastError());
    int h = 0;
    CKM(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));
    cudaFree(work);
    cudaFree(d_status);
    cudaFree(pscr);
    return h ? NEGF_ERR_CUDA : NEGF_OK;
}

// ======================================================================= host
namespace {

negf::Geo mixed_geo(const negf_ctx *c) {
    negf::Geo g;
    g.N = c->N; g.Nz = c->Nz; g.ld = c->ld;
    g.ngx = c->ngx; g.ngy = c->ngy; g.W = 2 * c->ngx + 1; g.H = 2 * c->ngy + 1;
    g.nk = c->nk;
    g.vhat = c->d_vhat; g.nx = c->d_nx; g.ny = c->d_ny;
    g.ax = c->d_ax; g.ay = c->d_ay; g.kw = c->d_kw;
    g.delta = c->Lz / c->Nz;
    g.c2 = 2 * (g.delta * g.delta);
    g.V_L = c->V_L; g.V_R = c->V_R; g.eta = c->eta;
    g.lead_model = c->lead_model;
    return g;
}

constexpr double PI_M = 3.141592653589793;  // global.f90:28
constexpr int FP64_KEEP = 32;                // FP64 re-runs whose workspace fits beside the mixed buffers

// |k+G_i|^2 / 2 for mode i at k-point ik (grid.f90:258)
double kinetic(const negf_ctx *c, int ik, int i) {
    const double ax = (double)(2 * c->nx[i]) * PI_M / c->Lx + c->kpt[3 * ik];
    const double ay = (double)(2 * c->ny[i]) * PI_M / c->Ly + c->kpt[3 * ik + 1];
    return (ax * ax + ay * ay) / 2;
}

// k_mixed_pass on nw jobs of cpj CTAs each (a cluster per job)
cudaError_t launch_pass(const MixedArgs &a, int nw, int cpj, size_t smem, cudaStream_t st, int mode, int it, int last) {
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute la[1];
    la[0].id = cudaLaunchAttributeClusterDimension;
    la[0].val.clusterDim.x = cpj;
    la[0].val.clusterDim.y = 1;
    la[0].val.clusterDim.z = 1;
    lc.gridDim = dim3(nw * cpj);
    lc.blockDim = dim3(NT);
    lc.dynamicSmemBytes = smem;
    lc.stream = st;
    lc.attrs = la;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, k_mixed_pass, a, mode, it, last);
}

template <typename K>
int set_smem(K kern, size_t bytes) {
    CKM(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    return 0;
}

}  // namespace

int negf_internal_mixed(negf_ctx *c, const double *h_E, const double *d_E, int nE, double *h_tau_jobs,
                        int *h_info, double *device_ms) {
    const int nk = c->nk, njobs = nE * nk, N = c->N, Nz = c->Nz;
    negf_mixed_stats stats{};
    stats.n_jobs = njobs;
    *device_ms = 0;
    if (N > 1023) return NEGF_ERR_UNSUPPORTED;
    const negf_mixed_policy pol = c->mixed_policy;
    cudaStream_t st = c->stream;

    // ---- policy: which jobs run in FP64 from the start
    std::vector<int> f_ie, f_ik, m_jobs;
    std::vector<int> nopen_est(njobs, 0);
    int nmax = 0;
    for (int ik = 0; ik < nk; ++ik) {
        std::vector<double> kin(N);
        for (int i = 0; i < N; ++i) kin[i] = kinetic(c, ik, i);
        for (int ie = 0; ie < nE; ++ie) {
            const int q = ik * nE + ie;
            const double E = h_E[ie];
            bool fp64 = c->eta < pol.eta_fp64_below;
            int n = 0;
            for (int i = 0; i < N; ++i) {
                if (pol.threshold_window > 0 &&
                    (std::fabs(E - (c->V_L + kin[i])) < pol.threshold_window ||
                     std::fabs(E - (c->V_R + kin[i])) < pol.threshold_window))
                    fp64 = true;
                // open channel of the right lead (gamma_R != 0, grid.f90:355-360), with a
                // margin for rounding at the threshold
                if (2 * (E - c->V_R) - 2 * kin[i] > -1e-12 * (std::fabs(E) + 2 * kin[i])) ++n;
            }
            if (n > 127) fp64 = true;
            nopen_est[q] = n;
            if (fp64) {
                f_ie.push_back(ie);
                f_ik.push_back(ik);
                stats.n_fp64_policy++;
            } else {
                m_jobs.push_back(q);
                nmax = std::max(nmax, n);
            }
        }
    }
    int rc = 0;
    double mixed_ms = 0;
    if (!m_jobs.empty()) {
        const int ncap = std::max(16, rup(nmax, 16));
        const MixedLayout L = make_layout(N, Nz, c->ld, ncap);
        const size_t per_job = L.job_bytes + L.scratch_bytes;
        const size_t small_per_job = sizeof(int2) + 4 * sizeof(double) + sizeof(int);
        if (!c->d_voff) {
            // the energy-independent part of every D_k, once per context
            if (cudaMalloc(&c->d_voff, sizeof(double2) * (size_t)N * c->ld * Nz) != cudaSuccess) {
                cudaGetLastError();
                c->d_voff = nullptr;
                return NEGF_ERR_NOMEM;
            }
            k_voff<<<Nz, NT, 0, st>>>(mixed_geo(c), c->d_voff);
            CKM(cudaGetLastError());
        }
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        // the FP64 re-runs keep their own workspace (4 blocks per CTA): room is
        // kept for FP64_KEEP of them beside the mixed buffers (beyond that the
        // mixed buffers are released before the re-runs), less what the
        // context already holds
        const size_t fp64_ws = (size_t)std::min(c->num_sms, FP64_KEEP) * 4 * c->ld * N * 16;
        const size_t fp64_more = fp64_ws > c->ws_bytes ? fp64_ws - c->ws_bytes : 0;
        const size_t avail = free_b + c->mixed_bytes;
        const size_t budget = avail > fp64_more + ((size_t)2 << 30) ? (size_t)(0.95 * (avail - fp64_more)) - ((size_t)1 << 30) : 0;
        const size_t mem_jobs = budget / (per_job + small_per_job);
        int W = (int)std::min<size_t>({(size_t)m_jobs.size(), (size_t)c->num_sms, mem_jobs});
        // Two CTAs (one cluster) per job when a wave of single-CTA jobs would
        // leave at least half of the SMs idle (few jobs, or factor storage
        // bounding the wave): the job then sweeps on two SMs.
        int cpj = pol.ctas_per_job;
        if (cpj == 0) cpj = (2 * (size_t)W <= (size_t)c->num_sms) ? 2 : 1;
        const size_t sm_sweep = sweep_smem_bytes(N);
        int smem_optin = 0;
        CKM(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
        // a basis whose sweep state does not fit one SM's shared memory (about
        // N > 900) runs in FP64 like a job that does not fit device memory
        // the deepest factor ring of the passes that shared memory allows
        // (1 KB kept for the pass kernel's static shared memory)
        int pa = PA_MAX;
        while (pa > PA_MIN && pass_smem_bytes(N, ncap, pa) + 1024 > (size_t)smem_optin) --pa;
        if (sm_sweep > (size_t)smem_optin || pass_smem_bytes(N, ncap, pa) + 1024 > (size_t)smem_optin) W = 0;
        if (cpj == 2 && W >= 1) {
            CKM(cudaFuncSetAttribute(k_mixed_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_sweep));
            cudaLaunchConfig_t qc = {};
            cudaLaunchAttribute qa[1];
            qa[0].id = cudaLaunchAttributeClusterDimension;
            qa[0].val.clusterDim.x = 2;
            qa[0].val.clusterDim.y = 1;
            qa[0].val.clusterDim.z = 1;
            qc.gridDim = dim3(2 * W);
            qc.blockDim = dim3(NT);
            qc.dynamicSmemBytes = sm_sweep;
            qc.attrs = qa;
            qc.numAttrs = 1;
            int nclu = 0;
            CKM(cudaOccupancyMaxActiveClusters(&nclu, k_mixed_sweep, &qc));
            if (nclu < 1) cpj = 1;
            else W = std::min(W, nclu);
        }
        if (W < 1) {
            // not enough device memory (or shared memory) for one job: everything in FP64
            for (int q : m_jobs) { f_ie.push_back(q % nE); f_ik.push_back(q / nE); }
            stats.n_fp64_policy += (int)m_jobs.size();
            m_jobs.clear();
        } else {
            const size_t need = (size_t)W * (per_job + small_per_job) + 4096;
            if (need > c->mixed_bytes) {
                if (c->d_mixed) cudaFree(c->d_mixed);
                c->d_mixed = nullptr;
                c->mixed_bytes = 0;
                if (cudaMalloc(&c->d_mixed, need) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
                c->mixed_bytes = need;
            }
            stats.jobs_per_wave = W;
            stats.ctas_per_job = cpj;
            unsigned char *base = (unsigned char *)c->d_mixed;
            MixedArgs a;
            a.g = mixed_geo(c);
            a.voff = c->d_voff;
            a.L = L;
            a.E = d_E;
            a.jobmem = base;
            a.scratch = base + (size_t)W * L.job_bytes;
            unsigned char *smallp = a.scratch + (size_t)W * L.scratch_bytes;
            int2 *d_jobs = (int2 *)smallp;
            a.jobs = d_jobs;
            a.tau = (double *)align256((size_t)(d_jobs + W));
            a.dnorm = a.tau + W;
            a.xnorm = a.dnorm + W;
            a.dprev = a.xnorm + W;
            a.status = (int *)(a.dprev + W);
            a.tol = pol.tau_tolerance;
            a.cpj = cpj;
            const size_t sm_pass = pass_smem_bytes(N, ncap, pa);
            a.pa = pa;
            const size_t sm_res = (size_t)2 * negf::KC * (negf::AP + negf::BP) * 16 + job_smem_bytes(N);
            rc = set_smem(k_mixed_sweep, sm_sweep);
            if (!rc) rc = set_smem(k_mixed_pass, sm_pass);
            if (!rc) rc = set_smem(k_mixed_residual, sm_res);
            if (rc) return rc;
            CUtensorMap tmC;
            if (!c_tile_map(&tmC, a.scratch, N, c->ld, 2, (size_t)N * c->ld * 8, W, L.scratch_bytes))
                return NEGF_ERR_CUDA;
            std::vector<int2> wj(W);
            std::vector<double> tau(W), dn(W), xn(W);
            std::vector<int> status(W);
            for (size_t w0 = 0; w0 < m_jobs.size(); w0 += W) {
                const int nw = (int)std::min<size_t>(W, m_jobs.size() - w0);
                for (int w = 0; w < nw; ++w) wj[w] = make_int2(m_jobs[w0 + w] % nE, m_jobs[w0 + w] / nE);
                a.njobs = nw;
                CKM(cudaMemcpyAsync(d_jobs, wj.data(), sizeof(int2) * nw, cudaMemcpyHostToDevice, st));
                CKM(cudaEventRecord(c->ev0, st));
                {
                    cudaLaunchConfig_t lc = {};
                    cudaLaunchAttribute la[1];
                    la[0].id = cudaLaunchAttributeClusterDimension;
                    la[0].val.clusterDim.x = cpj;
                    la[0].val.clusterDim.y = 1;
                    la[0].val.clusterDim.z = 1;
                    lc.gridDim = dim3(nw * cpj);
                    lc.blockDim = dim3(NT);
                    lc.dynamicSmemBytes = sm_sweep;
                    lc.stream = st;
                    lc.attrs = la;
                    lc.numAttrs = 1;
                    CKM(cudaLaunchKernelEx(&lc, k_mixed_sweep, a, tmC));
                }
                CKM(launch_pass(a, nw, cpj, sm_pass, st, PASS_X0, 0, 0));
                // refinement steps; converged jobs (MIX_DONE) are skipped by the next ones
                for (int it = 1; it <= pol.max_refinements; ++it) {
                    const int last = it == pol.max_refinements;
                    k_mixed_residual<<<dim3(nw, Nz), NT, sm_res, st>>>(a);
                    CKM(cudaGetLastError());
                    CKM(launch_pass(a, nw, cpj, sm_pass, st, PASS_BACK, it, last));
                    CKM(launch_pass(a, nw, cpj, sm_pass, st, PASS_CORR, it, last));
                }
                CKM(cudaEventRecord(c->ev1, st));
                CKM(cudaMemcpyAsync(tau.data(), a.tau, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
                CKM(cudaMemcpyAsync(dn.data(), a.dnorm, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
                CKM(cudaMemcpyAsync(xn.data(), a.xnorm, sizeof(double) * nw, cudaMemcpyDeviceToHost, st));
                CKM(cudaMemcpyAsync(status.data(), a.status, sizeof(int) * nw, cudaMemcpyDeviceToHost, st));
                CKM(cudaStreamSynchronize(st));
                float ms = 0.f;
                CKM(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
                mixed_ms += ms;
                for (int w = 0; w < nw; ++w) {
                    const int q = m_jobs[w0 + w];
                    const double corr = xn[w] > 0 ? dn[w] / xn[w] : (dn[w] > 0 ? INFINITY : 0.0);
                    if (status[w] == MIX_DONE) {
                        h_tau_jobs[q] = tau[w];
                        h_info[q] = 0;
                        stats.n_mixed++;
                        stats.max_correction = std::max(stats.max_correction, corr);
                    } else {
                        if (status[w] == -2) return NEGF_ERR_CUDA;  // a tensor-core wait timed out
                        f_ie.push_back(q % nE);
                        f_ik.push_back(q / nE);
                        stats.n_fp64_rejected++;
                    }
                }
            }
        }
    }
    // ---- FP64 re-runs
    float ms64 = 0.f;
    if ((int)f_ie.size() > FP64_KEEP && c->d_mixed) {
        // more re-runs than the room kept for them: the mixed buffers go first
        cudaFree(c->d_mixed);
        c->d_mixed = nullptr;
        c->mixed_bytes = 0;
    }
    if (!f_ie.empty()) {
        std::vector<double> t64(f_ie.size());
        std::vector<int> i64(f_ie.size());
        rc = negf_internal_fp64_jobs(c, d_E, f_ie.data(), f_ik.data(), (int)f_ie.size(), t64.data(), i64.data(),
                                     &ms64);
        if (rc) return rc;
        for (size_t q = 0; q < f_ie.size(); ++q) {
            const int job = f_ik[q] * nE + f_ie[q];
            h_tau_jobs[job] = t64[q];
            h_info[job] = i64[q];
        }
    }
    stats.mixed_ms = mixed_ms;
    stats.fp64_ms = ms64;
    c->mixed_stats = stats;
    *device_ms = mixed_ms + ms64;
    return NEGF_OK;
}
