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
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "mixed_device.cuh"
#include "negf_gpu.h"

using namespace negf;
using namespace negf::mx;

namespace {

// ------------------------------------------------------------ shared memory
// Per-CTA state of the FP32 Gauss-Jordan inverse.
struct GjSmem {
    int *prow;       // [N] pivot row of column k
    int *iprow;      // [N] inverse permutation
    int *inP;        // [N] sub-panel tag (1..4) of the current panel's pivot rows, else 0
    uint32_t *rkey;  // [2][NWARP] warp candidate keys, double-buffered by step parity
    float2 *rrec;    // [2][NWARP] reciprocal of each warp's candidate
    float2 *cand;    // [2][NWARP][8] each warp's candidate row (sub-panel columns)
    float2 *sX;      // [32][8]  rows P_<p of sub-panel p before its update
    float2 *sY;      // [8][32]  rows P_p of the earlier sub-panels
    float *rmax;     // [2][TM]  per-thread-half row maxima while staging W
};
__host__ __device__ inline int rup(int a, int b) { return (a + b - 1) / b * b; }
__host__ __device__ inline size_t gj_smem_bytes(int N) {
    const int n4 = rup(N, 4);
    size_t b = 3 * (size_t)n4 * 4;
    b += 2 * NWARP * 4 + 2 * NWARP * 8 + 2 * NWARP * 8 * 8;
    b += 32 * 8 * 8 + 8 * 32 * 8 + 2 * TM * 4;
    return (b + 127) / 128 * 128;
}
__device__ inline GjSmem carve_gj(unsigned char *base, int N) {
    GjSmem s;
    const int n4 = rup(N, 4);
    s.prow = (int *)base;
    s.iprow = s.prow + n4;
    s.inP = s.iprow + n4;
    s.rkey = (uint32_t *)(s.inP + n4);
    s.rrec = (float2 *)(s.rkey + 2 * NWARP);
    s.cand = s.rrec + 2 * NWARP;
    s.sX = s.cand + 2 * NWARP * 8;
    s.sY = s.sX + 32 * 8;
    s.rmax = (float *)(s.sY + 8 * 32);
    return s;
}

// ------------------------------------------------------------- pivot steps
// Sortable 32-bit key: |re|+|im| bits (non-negative floats order as
// unsigned integers) with the low 10 bits replaced by 1023 - row, so the
// warp maximum is one redux and ties go to the lower row.  Magnitudes that
// differ only in those bits (relative 2^-13) count as a tie.  N <= 1023.
__device__ __forceinline__ uint32_t pivot_key32(float v, int row) {
    return (__float_as_uint(v) & ~0x3FFu) | (uint32_t)(0x3FF - row);
}

template <int RPT>
__device__ inline int warp_pivot_f(const float2 (&f)[RPT], unsigned used, int buf, const GjSmem &s) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t key = 0;
    int rbest = -1;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        if (!((used >> r) & 1u)) {
            float v = cabs1f(f[r]);
            if (!(v == v)) v = 0.0f;  // NaN rows rank as zero pivots
            const uint32_t k = pivot_key32(v, tid + NT * r);
            if (k > key) { key = k; rbest = r; }
        }
    }
    const uint32_t wk = __reduce_max_sync(0xffffffffu, key);
    if (lane == 0) s.rkey[buf * NWARP + warp] = wk;
    if (wk != 0 && key == wk) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
            if (r == rbest) s.rrec[buf * NWARP + warp] = crcp(f[r]);
        return rbest;
    }
    return -1;
}

// Gauss-Jordan steps on the 8 columns [kb, kb+nbe) held in registers (row
// tid + NT*r in w[r][.]), implicit partial pivoting (largest |re|+|im| among
// unused rows, as zgetf2 chooses).  One CTA barrier per step: each warp
// publishes its candidate key, reciprocal and updated row; the next column
// is updated first so its search overlaps the rest of the row update.
template <int RPT>
__device__ inline void factor_sub8(float2 (&w)[RPT][8], int kb, int nbe, unsigned &used, int &info, int tag,
                                   const GjSmem &s) {
    const int tid = threadIdx.x, warp = tid >> 5;
    float2 f[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) f[r] = w[r][0];
    int mine = warp_pivot_f<RPT>(f, used, 0, s);
    if (mine >= 0) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
            if (r == mine) {
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) s.cand[warp * 8 + jj] = w[r][jj];
            }
    }
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) {
        if (kk < nbe) {
            const int buf = kk & 1;
            __syncthreads();
            const uint32_t *rk = s.rkey + buf * NWARP;
            uint32_t key = rk[0];
            int q = 0;
#pragma unroll
            for (int j = 1; j < NWARP; ++j) {
                const uint32_t k = rk[j];
                if (k > key) { key = k; q = j; }
            }
            const float2 d = s.rrec[buf * NWARP + q];
            const float2 *srow = s.cand + (buf * NWARP + q) * 8;
            const int p = 0x3FF - (int)(key & 0x3FFu);
            if ((key >> 10) == 0 && info == 0) info = kb + kk + 1;
#pragma unroll
            for (int r = 0; r < RPT; ++r)
                if (tid + NT * r == p) used |= 1u << r;
            if (tid == 0) { s.prow[kb + kk] = p; s.inP[p] = tag; }
            const bool more = (kk + 1 < 8) && (kk + 1 < nbe);
            float2 gm[RPT];
#pragma unroll
            for (int r = 0; r < RPT; ++r) gm[r] = (tid + NT * r == p) ? make_float2(0.f, 0.f) : cmul(w[r][kk], d);
            if (kk + 1 < 8) {
                float2 fn[RPT];
                const float2 rn = srow[(kk + 1) & 7];
#pragma unroll
                for (int r = 0; r < RPT; ++r)
                    fn[r] = (tid + NT * r == p) ? cmul(rn, d) : cfms(gm[r], rn, w[r][(kk + 1) & 7]);
                mine = more ? warp_pivot_f<RPT>(fn, used, buf ^ 1, s) : -1;
            } else {
                mine = -1;
            }
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (tid + NT * r == p) {
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj) w[r][jj] = (jj == kk) ? d : cmul(srow[jj], d);
                } else {
#pragma unroll
                    for (int jj = 0; jj < 8; ++jj)
                        w[r][jj] = (jj == kk) ? make_float2(-gm[r].x, -gm[r].y) : cfms(gm[r], srow[jj], w[r][jj]);
                }
            }
            if (mine >= 0) {
                float2 *dst = s.cand + ((buf ^ 1) * NWARP + warp) * 8;
#pragma unroll
                for (int r = 0; r < RPT; ++r)
                    if (r == mine) {
#pragma unroll
                        for (int jj = 0; jj < 8; ++jj) dst[jj] = w[r][jj];
                    }
            }
        }
    }
    __syncthreads();
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

// B tile of the trailing update: column j < TN of the tile is matrix column
// col(J0 + j) (the columns outside the panel), its K values the pivot rows
// prow[k0 .. k0+nbt) of that column; one exponent per column.  Thread
// (column j = tid / 4, K group g = tid % 4).
__device__ inline void stage_b_pivot_rows(const TileSmem &t, const GjSmem &s, const float2 *__restrict__ A,
                                          int ld, int N, int k0, int nbt, int J0) {
    const int tid = threadIdx.x, j = tid >> 2, g = tid & 3;
    const int nrest = N - nbt, jr = J0 + j;
    const bool cv = jr < nrest;
    const int col = jr < k0 ? jr : jr + nbt;
    float2 v[8];
    float m = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int kk = 8 * g + q;
        v[q] = (cv && kk < nbt) ? A[s.prow[k0 + kk] + (size_t)ld * col] : make_float2(0.f, 0.f);
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

// A(:, rest) = mask(A(:, rest)) + W * A_old(prow[k0:k0+nbt], rest) with
// W = A(:, k0:k0+nbt): the combined effect of the panel's Gauss-Jordan steps
// on every other column (mask zeroes the panel's pivot rows), on the tensor
// cores.  Returns false if an MMA wait timed out.
__device__ inline bool trailing_update_tc(float2 *__restrict__ A, int N, int ld, int k0, int nbt, const GjSmem &s,
                                          const TileSmem &t, uint32_t tbase, uint32_t &ph) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const int nrest = N - nbt;
    int err = 0;
    for (int J0 = 0; J0 < nrest; J0 += TN) {
        stage_b_pivot_rows(t, s, A, ld, N, k0, nbt, J0);
        for (int I0 = 0; I0 < N; I0 += TM) {
            stage_w(t, s, A, ld, N, I0, k0, nbt);  // contains a barrier
            tc::fence_async_smem();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                issue_chunk(t, tbase, true);
                tc::mma_commit(t.bar);
            }
            wait_mma(t, ph, &err);
            // epilogue: warps 0-3 columns 0-31, warps 4-7 columns 32-63
            const int r = 32 * (warp & 3) + (tid & 31), i = I0 + r;
            const bool rv = i < N;
            const bool keep = rv && !s.inP[i];
            const int er = t.rexp[r];
#pragma unroll 1
            for (int c16 = 2 * (warp >> 2); c16 < 2 * (warp >> 2) + 2; ++c16) {
                float re[16], im[16];
                load_acc16(tbase, c16, re, im);
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const int j = c16 * 16 + q, jr = J0 + j;
                    if (rv && jr < nrest) {
                        const int col = jr < k0 ? jr : jr + nbt;
                        float2 *cp = A + i + (size_t)ld * col;
                        const float2 c = keep ? *cp : make_float2(0.f, 0.f);
                        const int ex = er + t.cexp[j];
                        *cp = make_float2(c.x + ldexpf(re[q], ex), c.y + ldexpf(im[q], ex));
                    }
                }
            }
            tc::fence_before_sync();
            __syncthreads();
            if (err) return false;
        }
    }
    return true;
}

// In-place blocked Gauss-Jordan inverse of the N x N block A (leading
// dimension ld, complex FP32) with implicit partial pivoting.  Panels of 32
// columns, four 8-column register sub-panels each: per sub-panel p,
// (i) bring it up to date with sub-panels < p, (ii) eliminate it,
// (iii) apply its steps to the earlier columns; then one rank-32 trailing
// update of all other columns on the tensor cores.  On return s.prow/s.iprow
// hold the permutations: inv(A)(r, c) = A(prow[r], iprow[c]).  Returns the
// LAPACK-style info (1-based column of the first zero pivot, 0 if none);
// *err = 1 if a tensor-core wait timed out.
template <int RPT>
__device__ int gj_invert_mixed(float2 *__restrict__ A, int N, int ld, const GjSmem &s, const TileSmem &t,
                               uint32_t tbase, uint32_t &ph, int *err) {
    const int tid = threadIdx.x;
    const float2 zero = make_float2(0.f, 0.f);
    int info = 0;
    unsigned used = 0;
#pragma unroll
    for (int r = 0; r < RPT; ++r)
        if (tid + NT * r >= N) used |= 1u << r;
    for (int i = tid; i < N; i += NT) s.inP[i] = 0;
    __syncthreads();
    for (int k0 = 0; k0 < N; k0 += KB) {
        const int nbt = min(KB, N - k0);
        for (int p = 0; p * 8 < nbt; ++p) {
            const int cp = k0 + p * 8, kprev = p * 8;
            const int nbp = min(8, nbt - kprev);
            if (p > 0) {
                for (int e = tid; e < kprev * 8; e += NT) {
                    const int kk = e / 8, c = e % 8;
                    s.sX[e] = (c < nbp) ? A[s.prow[k0 + kk] + (size_t)ld * (cp + c)] : zero;
                }
                __syncthreads();
            }
            float2 w[RPT][8];
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = tid + NT * r;
                const bool keep = (i < N) && !(s.inP[i] >= 1 && s.inP[i] <= p);
#pragma unroll
                for (int c = 0; c < 8; ++c) w[r][c] = (keep && c < nbp) ? A[i + (size_t)ld * (cp + c)] : zero;
                if (i < N) {
#pragma unroll 1
                    for (int kk0 = 0; kk0 < kprev; kk0 += 8) {
                        float2 wa[8];
#pragma unroll
                        for (int u = 0; u < 8; ++u) wa[u] = A[i + (size_t)ld * (k0 + kk0 + u)];
#pragma unroll
                        for (int u = 0; u < 8; ++u)
#pragma unroll
                            for (int c = 0; c < 8; ++c) w[r][c] = cfma(wa[u], s.sX[(kk0 + u) * 8 + c], w[r][c]);
                    }
                }
            }
            factor_sub8<RPT>(w, cp, nbp, used, info, p + 1, s);
            if (p > 0) {
                for (int e = tid; e < 8 * kprev; e += NT) {
                    const int c = e / kprev, q = e % kprev;
                    s.sY[c * 32 + q] = (c < nbp) ? A[s.prow[cp + c] + (size_t)ld * (k0 + q)] : zero;
                }
                __syncthreads();
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = tid + NT * r;
                    if (i < N) {
                        const bool keep = s.inP[i] != p + 1;
#pragma unroll 1
                        for (int q0 = 0; q0 < kprev; q0 += 8) {
                            float2 v[8];
#pragma unroll
                            for (int u = 0; u < 8; ++u) v[u] = keep ? A[i + (size_t)ld * (k0 + q0 + u)] : zero;
#pragma unroll
                            for (int u = 0; u < 8; ++u) {
#pragma unroll
                                for (int c = 0; c < 8; ++c) v[u] = cfma(w[r][c], s.sY[c * 32 + q0 + u], v[u]);
                                A[i + (size_t)ld * (k0 + q0 + u)] = v[u];
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = tid + NT * r;
                if (i < N) {
#pragma unroll
                    for (int c = 0; c < 8; ++c)
                        if (c < nbp) A[i + (size_t)ld * (cp + c)] = w[r][c];
                }
            }
            __syncthreads();
        }
        if (nbt < N && !trailing_update_tc(A, N, ld, k0, nbt, s, t, tbase, ph)) {
            *err = 1;
            return info;
        }
        __syncthreads();
        if (tid < nbt) s.inP[s.prow[k0 + tid]] = 0;
        __syncthreads();
    }
    for (int k = tid; k < N; k += NT) s.iprow[s.prow[k]] = k;
    __syncthreads();
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
                    const int ex = t.rexp[r] + t.cexp[c16 * 16 + q];
                    C[i + (size_t)ldc * jc] = make_float2(ldexpf(re[q], ex), ldexpf(im[q], ex));
                }
            }
        }
    }
    if (err && tid == 0) atomicExch(status, 1);
    tile_teardown(t, tbase);
}

// Inverse of each of nmat N x N complex FP32 matrices (one CTA each):
// work holds the matrices (overwritten), out receives the inverses.
template <int RPT>
__global__ void __launch_bounds__(NT, 1)
    k_tc_inverse_check(float2 *__restrict__ work, int N, float2 *__restrict__ out, int *__restrict__ info,
                       int *status) {
    extern __shared__ __align__(128) unsigned char smem[];
    GjSmem s = carve_gj(smem, N);
    TileSmem t = carve_tile(smem + gj_smem_bytes(N));
    const uint32_t tbase = tile_setup(t);
    uint32_t ph = 0;
    int err = 0;
    float2 *A = work + (size_t)blockIdx.x * N * N;
    const int inf = gj_invert_mixed<RPT>(A, N, N, s, t, tbase, ph, &err);
    if (!err) {
        float2 *o = out + (size_t)blockIdx.x * N * N;
        for (int j = 0; j < N; ++j) {
            const int jc = s.iprow[j];
            for (int r = threadIdx.x; r < N; r += NT) o[s.iprow[r] + (size_t)N * j] = A[r + (size_t)N * jc];
        }
    }
    if (threadIdx.x == 0) {
        info[blockIdx.x] = inf;
        if (err) atomicExch(status, 1);
    }
    tile_teardown(t, tbase);
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
    const size_t smem = gj_smem_bytes(N) + tile_smem_bytes();
    float2 *work = nullptr;
    int *d_status = nullptr;
    CKM(cudaMalloc(&work, sizeof(float2) * (size_t)N * N * nmat));
    CKM(cudaMalloc(&d_status, sizeof(int)));
    CKM(cudaMemcpyAsync(work, d_A, sizeof(float2) * (size_t)N * N * nmat, cudaMemcpyDeviceToDevice, st));
    CKM(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    if (N <= NT) {
        CKM(cudaFuncSetAttribute(k_tc_inverse_check<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tc_inverse_check<1><<<nmat, NT, smem, st>>>(work, N, (float2 *)d_out, d_info, d_status);
    } else if (N <= 2 * NT) {
        CKM(cudaFuncSetAttribute(k_tc_inverse_check<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tc_inverse_check<2><<<nmat, NT, smem, st>>>(work, N, (float2 *)d_out, d_info, d_status);
    } else {
        CKM(cudaFuncSetAttribute(k_tc_inverse_check<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_tc_inverse_check<4><<<nmat, NT, smem, st>>>(work, N, (float2 *)d_out, d_info, d_status);
    }
    CKM(cudaGetLastError());
    int h = 0;
    CKM(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKM(cudaStreamSynchronize(st));
    cudaFree(work);
    cudaFree(d_status);
    return h ? NEGF_ERR_CUDA : NEGF_OK;
}
