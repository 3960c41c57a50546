// rgf_device.cuh -- CTA-level building blocks of the FP64 recursive Green's
// function (RGF) engine for sm_100a.
//
// One CTA owns one (E,k) job at a time and runs its whole z sweep
// (math_kernel.f90:44-165) without leaving the kernel.  Blocks are never read
// from HBM: D_k = 2*dz^2*((E+i*eta)I - H_k) - 2I (grid.f90:236-333) is
// generated from the V(G-G') table while the previous inverse is subtracted.
// Inverses use a blocked Gauss-Jordan elimination with implicit partial
// pivoting (the pivot choice of LAPACK zgetf2: largest |re|+|im| among the
// rows not yet used), whose panel lives in registers; the rank-NB trailing
// update and the chain products are complex FP64 GEMMs tiled through shared
// memory.  The raw Gauss-Jordan result R satisfies
//     inv(M)(r, c) = R(prow[r], iprow[c])
// so consumers read it through two index gathers instead of permuting it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace negf {

constexpr int NT = 256;          // threads per CTA
constexpr int NWARP = NT / 32;
// Complex FP64 GEMMs run on the FP64 tensor cores (DMMA, mma.m8n8k4.f64):
// a CTA tile of CM x CN outputs is split into 2 x 4 warp tiles of WM x WN
// (4 x 2 m8n8 tiles each); warps whose tile lies outside the matrix skip
// their MMAs, so the padding waste is at 8-row granularity only.  Warps 0-3
// take rows 0-31 and warps 4-7 rows 32-63: warp w runs on SM sub-partition
// w % 4, so a tile of at most 32 rows (the open-channel rows of the chain
// product, the last row tile of a block) still keeps all four DMMA units busy.
constexpr int CM = 64, CN = 64;  // CTA tile
constexpr int WM = 32, WN = 16;  // warp tile
constexpr int KC = 16;           // k chunk staged per pipeline step
// k-major tiles use a 66-element row pitch: successive k rows shift by 8
// banks, so the four k rows of an m8n8k4 fragment load hit distinct banks.
constexpr int AP = CM + 2;       // padded row of a k-major A tile
constexpr int BP = CN + 2;       // padded row of a k-major B tile

// ------------------------------------------------------------ complex FP64
__device__ __forceinline__ double2 zmake(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// c + a*b
__device__ __forceinline__ double2 zfma(double2 a, double2 b, double2 c) {
    c.x = fma(a.x, b.x, c.x);
    c.x = fma(-a.y, b.y, c.x);
    c.y = fma(a.x, b.y, c.y);
    c.y = fma(a.y, b.x, c.y);
    return c;
}
// c - a*b
__device__ __forceinline__ double2 zfms(double2 a, double2 b, double2 c) {
    c.x = fma(-a.x, b.x, c.x);
    c.x = fma(a.y, b.y, c.x);
    c.y = fma(-a.x, b.y, c.y);
    c.y = fma(-a.y, b.x, c.y);
    return c;
}
// 1/a = conj(a) / |a|^2 with one division (block entries here are O(1..1e3),
// far from the overflow range of |a|^2).
__device__ __forceinline__ double2 zrcp(double2 a) {
    const double s = 1.0 / (a.x * a.x + a.y * a.y);
    return make_double2(a.x * s, -a.y * s);
}
__device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }

// Principal square root, Re >= 0, branch cut on the negative real axis
// (the Fortran intrinsic sqrt of complex*16 used at grid.f90:285-288).
__device__ __forceinline__ double2 zsqrt(double2 z) {
    if (z.x == 0.0 && z.y == 0.0) return make_double2(0.0, z.y);
    double t = sqrt(0.5 * (fabs(z.x) + hypot(z.x, z.y)));
    if (z.x >= 0.0) return make_double2(t, z.y / (2.0 * t));
    return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}
// exp(i*q*delta), grid.f90:325,330
__device__ __forceinline__ double2 self_energy(double2 q, double delta) {
    double s, c;
    sincos(q.x * delta, &s, &c);
    double m = exp(-q.y * delta);
    return make_double2(m * c, m * s);
}

// Exact lead of the discretised model: the semi-infinite chain of diagonal
// blocks d = 2 dz^2 (E - V - kin) - 2 with +1 couplings has the surface
// Green's function g = 1/(d - g) (the fixed point of Sancho-Rubio
// decimation), the root of g^2 - d g + 1 = 0 with |g| < 1; block 1 then
// gets d_1 - g.  Returns -g, the term added to the end blocks.
__device__ __forceinline__ double2 lattice_self_energy(double2 E, double V, double kin, double c2) {
    const double2 d = make_double2(c2 * (E.x - V - kin) - 2.0, c2 * E.y);
    const double2 disc = zsqrt(make_double2(d.x * d.x - d.y * d.y - 4.0, 2.0 * d.x * d.y));
    const double2 g1 = make_double2(0.5 * (d.x + disc.x), 0.5 * (d.y + disc.y));
    const double2 g2 = make_double2(0.5 * (d.x - disc.x), 0.5 * (d.y - disc.y));
    const double2 gs = (g1.x * g1.x + g1.y * g1.y <= g2.x * g2.x + g2.y * g2.y) ? g1 : g2;
    return make_double2(-gs.x, -gs.y);
}
// Im of that term at the real energy over dz^2: sin(theta)/dz^2 for an open
// lattice channel (d = -2 cos(theta), |d| < 2), 0 for a closed one.
__device__ __forceinline__ double lattice_gamma(double e, double V, double kin, double c2, double dz) {
    const double d = c2 * (e - V - kin) - 2.0;
    return fabs(d) < 2.0 ? sqrt(1.0 - 0.25 * d * d) / (dz * dz) : 0.0;
}

// ------------------------------------------------------------ cp.async
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// ------------------------------------------------------------ geometry
// Everything a CTA needs to generate D_k for any (E, k-point) job.
struct Geo {
    int N, Nz, ld;          // basis size, slices, leading dimension of workspace blocks
    int ngx, ngy, W, H;     // V table bounds, W = 2ngx+1, H = 2ngy+1
    int nk;
    const double2 *vhat;    // [Nz][H][W]  V_reciprocal_all, zero outside |i|<=ngx/2,|j|<=ngy/2
    const int *nx, *ny;     // [N]
    const double *ax, *ay;  // [nk][N]  2*pi*n/L + k  (grid.f90:258,285)
    const double *kw;       // [nk]     k-point weights
    double delta;           // Lz / Nz
    double c2;              // 2*delta**2 (grid.f90:311)
    double V_L, V_R, eta;
    int lead_model;         // 0 reference continuum lead term, 1 exact lattice surface GF
};

// One warp's pivot candidate: a sortable key and the reciprocal of its value.
struct Red {
    unsigned long long key;
    unsigned long long pad;
    double2 d;
};

// Key that orders candidates by |re|+|im| (v >= 0, so its bit pattern sorts
// as an unsigned integer), then by lower row index.  The low 11 bits of v
// carry the index; two magnitudes that agree in all but those bits (a
// relative difference below 2^-41) count as a tie.  Key 0 = no candidate.
__device__ __forceinline__ unsigned long long pivot_key(double v, int row) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b & ~0x7FFull) | (unsigned long long)(0x7FF - row);
}

// Shared memory carve-up (dynamic).
struct Smem {
    int *prow;      // [N] pivot row of column k
    int *iprow;     // [N] inverse permutation
    int *nx, *ny;   // [N]
    int *inP;       // [N] 1 if row is a pivot row of the current panel
    int *rows;      // [N] open-channel rows of the left lead (gamma_L != 0), ascending
    int *nrows;     // [1] their count
    double2 *sigL;  // [N] exp(i q_L dz)
    double2 *sigR;  // [N] exp(i q_R dz)
    double *gL;     // [N] gamma_L  sin(q dz)/dz^2 (grid.f90:365)
    double *gR;     // [N] gamma_R
    double2 *cand;  // [2][NWARP][32] each warp's pivot candidate row (double-buffered by step)
    Red *red;       // [2][NWARP] each warp's candidate key and reciprocal
    double *fred;   // [NWARP] float reductions
    double2 *big;   // union: sub-panel + block | trailing rows + W tile | GEMM stages
    int ldw;
};

__host__ __device__ inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

template <int NB>
__host__ __device__ inline size_t smem_bytes(int N) {
    int ldw = round_up(N, CM);
    size_t big = (size_t)NB * ldw + (size_t)NB * NB;         // sub-panel a + 16x16 block
    size_t trail = 32 * (size_t)(BP + AP);                    // rank-32 update: gathered rows + W tile
    size_t gemm = 2 * (size_t)KC * (AP + BP);
    if (trail > big) big = trail;
    if (gemm > big) big = gemm;
    size_t b = 0;
    b += 6 * (size_t)round_up(N, 4) * sizeof(int) + 4 * sizeof(int);
    b += 2 * (size_t)round_up(N, 2) * sizeof(double2);
    b += 2 * (size_t)round_up(N, 2) * sizeof(double);
    b += 2 * NWARP * 32 * sizeof(double2);
    b += 2 * NWARP * sizeof(Red) + NWARP * sizeof(double);
    b = (b + 255) / 256 * 256;
    return b + big * sizeof(double2);
}

template <int NB>
__device__ inline Smem carve(unsigned char *base, int N) {
    Smem s;
    const int n4 = round_up(N, 4), n2 = round_up(N, 2);
    s.prow = (int *)base;
    s.iprow = s.prow + n4;
    s.nx = s.iprow + n4;
    s.ny = s.nx + n4;
    s.inP = s.ny + n4;
    s.rows = s.inP + n4;
    s.nrows = s.rows + n4;
    s.sigL = (double2 *)(s.nrows + 4);
    s.sigR = s.sigL + n2;
    s.gL = (double *)(s.sigR + n2);
    s.gR = s.gL + n2;
    s.cand = (double2 *)(s.gR + n2);
    s.red = (Red *)(s.cand + 2 * NWARP * 32);
    s.fred = (double *)(s.red + 2 * NWARP);
    size_t off = (size_t)((unsigned char *)(s.fred + NWARP) - base);
    off = (off + 255) / 256 * 256;
    s.big = (double2 *)(base + off);
    s.ldw = round_up(N, CM);
    return s;
}

// ------------------------------------------------------- block generation
// Self energies of the two leads for one job (grid.f90:284-289, 323-331) and
// the transmission weights (grid.f90:354-360) at the real energy e_t.
__device__ inline void job_vectors(const Geo &g, const Smem &s, double2 E, double e_t, int ik) {
    for (int i = threadIdx.x; i < g.N; i += NT) {
        const double ax = g.ax[ik * g.N + i], ay = g.ay[ik * g.N + i];
        if (g.lead_model == 0) {
            double2 zl = make_double2(2.0 * (E.x - g.V_L) - ax * ax - ay * ay, 2.0 * E.y);
            double2 zr = make_double2(2.0 * (E.x - g.V_R) - ax * ax - ay * ay, 2.0 * E.y);
            s.sigL[i] = self_energy(zsqrt(zl), g.delta);
            s.sigR[i] = self_energy(zsqrt(zr), g.delta);
            double ql = sqrt(fmax(2.0 * (e_t - g.V_L) - ax * ax - ay * ay, 0.0));
            double qr = sqrt(fmax(2.0 * (e_t - g.V_R) - ax * ax - ay * ay, 0.0));
            s.gL[i] = sin(ql * g.delta) / (g.delta * g.delta);
            s.gR[i] = sin(qr * g.delta) / (g.delta * g.delta);
        } else {
            const double kin = (ax * ax + ay * ay) / 2;
            s.sigL[i] = lattice_self_energy(E, g.V_L, kin, g.c2);
            s.sigR[i] = lattice_self_energy(E, g.V_R, kin, g.c2);
            s.gL[i] = lattice_gamma(e_t, g.V_L, kin, g.c2, g.delta);
            s.gR[i] = lattice_gamma(e_t, g.V_R, kin, g.c2, g.delta);
        }
    }
}

// M = D_k - inv(prev), where inv(prev)(i,j) = R(prow[i], iprow[j]).
// D_k is generated from V_reciprocal_all (Dexp == nullptr) or read from an
// explicit (N,N,Nz) array with leading dimension N.  Four columns per pass
// keep four independent gathers in flight per thread.
__device__ inline double2 d_element(const Geo &g, const Smem &s, const double2 *vs, int k, double2 E,
                                    int ik, int i, int j, int nxj, int nyj) {
    const int dx = s.nx[i] - nxj + g.ngx, dy = s.ny[i] - nyj + g.ngy;
    const double2 v = __ldg(vs + dx + g.W * dy);
    if (i != j) return make_double2(-v.x * g.c2, -v.y * g.c2);
    const double ax = g.ax[ik * g.N + i], ay = g.ay[ik * g.N + i];
    const double hx = v.x + (ax * ax + ay * ay) / 2;
    double2 d = make_double2((-hx + E.x) * g.c2 - 2.0, (-v.y + E.y) * g.c2);
    if (k == 0) d = zadd(d, s.sigL[i]);
    if (k == g.Nz - 1) d = zadd(d, s.sigR[i]);
    return d;
}

__device__ inline void form_block(double2 *__restrict__ M, const Geo &g, const Smem &s, int k,
                                  double2 E, int ik, const double2 *__restrict__ R,
                                  const double2 *__restrict__ Dexp) {
    const int N = g.N, ld = g.ld;
    const double2 *vs = g.vhat ? g.vhat + (size_t)g.W * g.H * k : nullptr;
    const double2 *Dk = Dexp ? Dexp + (size_t)N * N * k : nullptr;
    for (int j0 = 0; j0 < N; j0 += 4) {
        // thread t reads row t of R (coalesced) and writes the row i of M it
        // belongs to, i = iprow[t] (prow[i] = t): scattered stores instead of
        // scattered loads
        for (int t = threadIdx.x; t < N; t += NT) {
            double2 d[4], r[4];
            const int i = R ? s.iprow[t] : t;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = j0 + q;
                d[q] = make_double2(0.0, 0.0);
                r[q] = make_double2(0.0, 0.0);
                if (j < N) {
                    if (Dk) d[q] = Dk[i + (size_t)N * j];
                    else d[q] = d_element(g, s, vs, k, E, ik, i, j, s.nx[j], s.ny[j]);
                    if (R) r[q] = R[t + (size_t)ld * s.iprow[j]];
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (j0 + q < N) M[i + (size_t)ld * (j0 + q)] = zsub(d[q], r[q]);
        }
    }
}

// out(i,j) = inv(R)(i,j) = R(prow[i], iprow[j]) (+ identity when add_eye).
__device__ inline void unpermute(double2 *__restrict__ out, int ldo, const double2 *__restrict__ R,
                                 int ld, int N, const Smem &s, double scale) {
    for (int j = 0; j < N; ++j) {
        const int jc = s.iprow[j];
        for (int t = threadIdx.x; t < N; t += NT) {  // coalesced loads, scattered stores
            double2 v = R[t + (size_t)ld * jc];
            out[s.iprow[t] + (size_t)ldo * j] = make_double2(v.x * scale, v.y * scale);
        }
    }
}

// Rows of G_{Nz,1} that the transmission trace reads: gamma_L,i != 0, the
// channels open in the left lead (grid.f90:355-365).  Row i of the chain
// product P * gR depends on row i of P only, so the chain can carry just
// these rows and produce the same values for them.
__device__ inline void open_rows(int N, const Smem &s) {
    if (threadIdx.x == 0) {
        int n = 0;
        for (int i = 0; i < N; ++i)
            if (s.gL[i] != 0.0) s.rows[n++] = i;
        *s.nrows = n;
    }
}

// rows[0..n) = the modes with gam[i] != 0 (open channels of one lead), ascending.
__device__ inline void open_cols(int N, const Smem &s, const double *gam) {
    if (threadIdx.x == 0) {
        int n = 0;
        for (int i = 0; i < N; ++i)
            if (gam[i] != 0.0) s.rows[n++] = i;
        *s.nrows = n;
    }
}

// out(r, j) = inv(R)(rows[r], j) = R(prow[rows[r]], iprow[j]), r < n.
__device__ inline void unpermute_rows(double2 *__restrict__ out, int ldo, const double2 *__restrict__ R,
                                      int ld, int N, int n, const Smem &s) {
    for (int j = 0; j < N; ++j) {
        const int jc = s.iprow[j];
        for (int r = threadIdx.x; r < n; r += NT) out[r + (size_t)ldo * j] = R[s.prow[s.rows[r]] + (size_t)ld * jc];
    }
}

// ------------------------------------------------------------------ GEMM
// D(8x8) += A(8x4) * B(4x8) on the FP64 tensor cores.  Fragments (PTX ISA,
// mma.m8n8k4 .f64): A row = lane>>2, k = lane&3; B k = lane&3, col = lane>>2;
// C rows lane>>2, cols 2*(lane&3) + {0,1}.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Complex accumulators of one warp tile: 4 x 2 m8n8 tiles, 2 elements each.
struct WarpAcc {
    double re[4][2][2], im[4][2][2];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < 2; ++n)
#pragma unroll
                for (int e = 0; e < 2; ++e) re[m][n][e] = im[m][n][e] = 0.0;
    }
    // acc += A(k-major, lda) * B(k-major, ldb) over 4 k values starting at kb.
    __device__ __forceinline__ void step(const double2 *sA, int lda, int arow, const double2 *sB, int ldb,
                                         int bcol, int kb, int lane) {
        const int kk = kb + (lane & 3), g = lane >> 2;
        double2 a[4], b[2];
#pragma unroll
        for (int m = 0; m < 4; ++m) a[m] = sA[kk * lda + arow + 8 * m + g];
#pragma unroll
        for (int n = 0; n < 2; ++n) b[n] = sB[kk * ldb + bcol + 8 * n + g];
#pragma unroll
        // first the a.re products of all tiles, then the a.im ones, so that
        // the two MMAs into one accumulator are 16 instructions apart
#pragma unroll
        for (int m = 0; m < 4; ++m)
#pragma unroll
            for (int n = 0; n < 2; ++n) {
                dmma(re[m][n][0], re[m][n][1], a[m].x, b[n].x);
                dmma(im[m][n][0], im[m][n][1], a[m].x, b[n].y);
            }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double nai = -a[m].y;
#pragma unroll
            for (int n = 0; n < 2; ++n) {
                dmma(re[m][n][0], re[m][n][1], nai, b[n].y);
                dmma(im[m][n][0], im[m][n][1], a[m].y, b[n].x);
            }
        }
    }
};

// C(i,j) = sum_k A(i, acol[k]) * B(k, bcol[j]) for one CTA, complex FP64.
// acol/bcol == nullptr means identity.  Modes of the epilogue:
enum GemmOut { GEMM_STORE = 0, GEMM_STORE_NEG = 1, GEMM_TAU = 2, GEMM_STORE_ADD_EYE = 3, GEMM_ADD_SCALED = 4 };

struct GemmArgs {
    double2 *C;
    int ldc;
    const double2 *A;
    int lda;
    const int *acol;
    const double2 *B;
    int ldb;
    const int *bcol;
    int M, Ncol, K;
    const int *rowmap;  // GEMM_TAU: row i of C is basis row rowmap[i] (nullptr = identity)
    double2 beta;       // GEMM_ADD_SCALED: C += beta * (A B)
};

// Returns, for GEMM_TAU, this thread's partial sum of
// gL[i] * gR[j] * |(C(i,j)*2)*delta^2|^2 (grid.f90:362-383 after negf.f90:159-165).
__device__ inline double cta_gemm(const GemmArgs &a, const Smem &s, int mode, double delta) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm0 = (warp >> 2) * WM, wn0 = (warp & 3) * WN;
    double2 *sA = s.big;                 // [2][KC][AP]
    double2 *sB = s.big + 2 * KC * AP;   // [2][KC][BP]
    const int ntm = (a.M + CM - 1) / CM, ntn = (a.Ncol + CN - 1) / CN;
    const int nkc = (a.K + KC - 1) / KC;
    double tau = 0.0;
    for (int t = 0; t < ntm * ntn; ++t) {
        const int I0 = (t % ntm) * CM, J0 = (t / ntm) * CN;
        const bool active = (I0 + wm0 < a.M) && (J0 + wn0 < a.Ncol);
        WarpAcc acc;
        acc.zero();
        auto load_stage = [&](int st, int k0) {
            double2 *dA = sA + st * KC * AP;
            double2 *dB = sB + st * KC * BP;
#pragma unroll
            for (int q = 0; q < (KC * CM) / NT; ++q) {
                const int e = tid + NT * q;
                const int kk = e / CM, ii = e % CM;
                const int k = k0 + kk, i = I0 + ii;
                const bool v = (k < a.K) && (i < a.M);
                const int kc = v ? (a.acol ? a.acol[k] : k) : 0;
                cp_async16(dA + kk * AP + ii, a.A + (v ? (i + (size_t)a.lda * kc) : 0), v);
            }
#pragma unroll
            for (int q = 0; q < (KC * CN) / NT; ++q) {
                const int e = tid + NT * q;
                const int kk = e % KC, jj = e / KC;
                const int k = k0 + kk, j = J0 + jj;
                const bool v = (k < a.K) && (j < a.Ncol);
                const int jc = v ? (a.bcol ? a.bcol[j] : j) : 0;
                cp_async16(dB + kk * BP + jj, a.B + (v ? (k + (size_t)a.ldb * jc) : 0), v);
            }
            cp_async_commit();
        };
        load_stage(0, 0);
        for (int c = 0; c < nkc; ++c) {
            if (c + 1 < nkc) {
                load_stage((c + 1) & 1, (c + 1) * KC);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (active) {
                const double2 *cA = sA + (c & 1) * KC * AP;
                const double2 *cB = sB + (c & 1) * KC * BP;
#pragma unroll
                for (int kb = 0; kb < KC; kb += 4) acc.step(cA, AP, wm0, cB, BP, wn0, kb, lane);
            }
            __syncthreads();
        }
        if (active) {
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                const int i = I0 + wm0 + 8 * m + (lane >> 2);
#pragma unroll
                for (int n = 0; n < 2; ++n)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int j = J0 + wn0 + 8 * n + 2 * (lane & 3) + e;
                        if (i < a.M && j < a.Ncol) {
                            double2 v = make_double2(acc.re[m][n][e], acc.im[m][n][e]);
                            if (mode == GEMM_TAU) {
                                const double gx = v.x * 2.0 * (delta * delta), gy = v.y * 2.0 * (delta * delta);
                                const int ib = a.rowmap ? a.rowmap[i] : i;
                                tau += s.gL[ib] * s.gR[j] * (gx * gx + gy * gy);
                            } else {
                                if (mode == GEMM_STORE_NEG) v = make_double2(-v.x, -v.y);
                                if (mode == GEMM_STORE_ADD_EYE && i == j) v.x += 1.0;
                                double2 *cp = a.C + i + (size_t)a.ldc * j;
                                if (mode == GEMM_ADD_SCALED) v = zfma(a.beta, v, *cp);
                                *cp = v;
                            }
                        }
                    }
            }
        }
    }
    return tau;
}

// Block-wide sum of one double per thread; result valid in every thread.
__device__ inline double block_sum(double v, const Smem &s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) s.fred[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) t += s.fred[w];
    __syncthreads();
    return t;
}

// ----------------------------------------------------- Gauss-Jordan inverse
// Rank-nbt update of every column outside the panel [k0, k0+nbt):
//   A(:, j) = mask(A(:, j)) + W * A_old(prow[k0:k0+nbt], j)
// where W = A(:, k0:k0+nbt), the panel after elimination, and mask zeroes the
// panel's pivot rows.  This is the whole effect of the panel's Gauss-Jordan
// steps on the other columns, so one pass over the matrix applies KMAX
// elimination steps.  W tiles are staged from global memory with cp.async;
// W and the gathered pivot rows feed DMMA warp tiles.
template <int KMAX, bool PREFETCH = false>
__device__ inline void trailing_update(double2 *__restrict__ A, int N, int ld, int k0, int nbt,
                                       const Smem &s) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm0 = (warp >> 2) * WM, wn0 = (warp & 3) * WN;
    const int nrest = N - nbt;
    double2 *sB = s.big;               // [KMAX][BP] pivot rows of the column tile
    double2 *sW = s.big + KMAX * BP;   // [KMAX][AP] rows I0.. of the panel
    for (int J0 = 0; J0 < nrest; J0 += CN) {
        // all of a thread's gathers issued before any is stored (loads in flight)
        {
            constexpr int Q = (KMAX * CN) / NT;
            double2 v[Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int e = tid + NT * q;
                const int kk = e / CN, jt = e % CN, jr = J0 + jt;
                v[q] = make_double2(0.0, 0.0);
                if (kk < nbt && jr < nrest) {
                    const int j = jr < k0 ? jr : jr + nbt;
                    v[q] = A[s.prow[k0 + kk] + (size_t)ld * j];
                }
            }
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const int e = tid + NT * q;
                sB[(e / CN) * BP + e % CN] = v[q];
            }
        }
        int col[2][2];
        bool cv[2][2];
#pragma unroll
        for (int n = 0; n < 2; ++n)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int jr = J0 + wn0 + 8 * n + 2 * (lane & 3) + e;
                cv[n][e] = jr < nrest;
                col[n][e] = jr < k0 ? jr : jr + nbt;
            }
        for (int I0 = 0; I0 < N; I0 += CM) {
#pragma unroll
            for (int q = 0; q < (KMAX * CM) / NT; ++q) {
                const int e = tid + NT * q;
                const int kk = e / CM, r = e % CM, i = I0 + r;
                const bool v = (kk < nbt) && (i < N);
                cp_async16(sW + kk * AP + r, A + (v ? (i + (size_t)ld * (k0 + kk)) : 0), v);
            }
            cp_async_commit();
            // large blocks (one CTA per SM): start the warp's C tile on its way
            // from DRAM into L2 while W arrives (slower for the 2-CTA variants)
            if (PREFETCH && (I0 + wm0 < N) && (J0 + wn0 < nrest)) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int i = I0 + wm0 + 8 * m + (lane >> 2);
#pragma unroll
                    for (int n = 0; n < 2; ++n)
#pragma unroll
                        for (int e = 0; e < 2; ++e)
                            if (i < N && cv[n][e])
                                asm volatile("prefetch.global.L2 [%0];" ::"l"(A + i + (size_t)ld * col[n][e]));
                }
            }
            cp_async_wait<0>();
            __syncthreads();
            if ((I0 + wm0 < N) && (J0 + wn0 < nrest)) {
                WarpAcc acc;
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int i = I0 + wm0 + 8 * m + (lane >> 2);
                    const bool rv = (i < N) && !s.inP[i];
#pragma unroll
                    for (int n = 0; n < 2; ++n)
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            double2 c = make_double2(0.0, 0.0);
                            if (rv && cv[n][e]) c = A[i + (size_t)ld * col[n][e]];
                            acc.re[m][n][e] = c.x;
                            acc.im[m][n][e] = c.y;
                        }
                }
#pragma unroll 2
                for (int kb = 0; kb < nbt; kb += 4) acc.step(sW, AP, wm0, sB, BP, wn0, kb, lane);
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int i = I0 + wm0 + 8 * m + (lane >> 2);
                    if (i < N) {
#pragma unroll
                        for (int n = 0; n < 2; ++n)
#pragma unroll
                            for (int e = 0; e < 2; ++e)
                                if (cv[n][e]) A[i + (size_t)ld * col[n][e]] = make_double2(acc.re[m][n][e], acc.im[m][n][e]);
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Gauss-Jordan elimination of the columns [kb, kb+nbe) of a register panel
// w (row tid + NT*r of the block in w[r][.]), with implicit partial pivoting:
// the pivot of each column is the unused row with the largest |re|+|im|
// (lowest index on ties), as zgetf2 chooses.  Pivot rows get inP = tag.
// The step loop is not unrolled: columns are picked out of the register rows
// by predication, which keeps the code size O(NB).  Each step updates the
// next pivot column first and runs its warp-level argmax while the rest of
// the row is updated; the winning lane of each warp computes the reciprocal
// of its candidate before the barrier.
// Warp-level pivot candidate for the column values f: writes the warp's best
// key and the reciprocal of its value into red[buf][warp]; returns, in the
// winning thread, the register row r of the candidate (-1 elsewhere).  That
// thread publishes the candidate's updated row into cand[buf][warp] later.
template <int NB, int RPT>
__device__ inline int warp_pivot(const double2 (&f)[RPT], unsigned used, int buf, const Smem &s) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long key = 0;
    int rbest = -1;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        if (!((used >> r) & 1u)) {
            double v = cabs1(f[r]);
            if (!(v == v)) v = 0.0;  // NaN rows rank as zero pivots
            const unsigned long long k = pivot_key(v, tid + NT * r);
            if (k > key) { key = k; rbest = r; }
        }
    }
    unsigned long long wk = key;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long ok = __shfl_xor_sync(0xffffffffu, wk, o);
        wk = ok > wk ? ok : wk;
    }
    Red *red = s.red + buf * NWARP;
    if (lane == 0) red[warp].key = wk;
    if (wk != 0 && key == wk) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
            if (r == rbest) red[warp].d = zrcp(f[r]);
        return rbest;
    }
    return -1;
}

// Gauss-Jordan elimination of the columns [kb, kb+nbe) of a register panel w
// (row tid + NT*r of the block in w[r][.]) with implicit partial pivoting:
// the pivot of each column is the unused row with the largest |re|+|im|
// (lowest index on ties), as zgetf2 chooses.  Pivot rows get inP = tag.
// One CTA barrier per step: every warp publishes its candidate (key,
// reciprocal, updated row) into a slot double-buffered by step parity, so
// after the barrier all threads read the winner's row directly.  The next
// column is updated first and its warp argmax overlaps the rest of the row.
template <int NB, int RPT>
__device__ inline void factor_subpanel(double2 (&w)[RPT][NB], int kb, int nbe, unsigned &used, int &info,
                                       int tag, const Smem &s) {
    const int tid = threadIdx.x, warp = tid >> 5;
    double2 f[RPT];
#pragma unroll
    for (int r = 0; r < RPT; ++r) f[r] = w[r][0];
    int mine = warp_pivot<NB, RPT>(f, used, 0, s);
    if (mine >= 0) {
#pragma unroll
        for (int r = 0; r < RPT; ++r)
            if (r == mine) {
#pragma unroll
                for (int jj = 0; jj < NB; ++jj) s.cand[warp * 32 + jj] = w[r][jj];
            }
    }
    // fully unrolled: every column index below is a compile-time constant
#pragma unroll
    for (int kk = 0; kk < NB; ++kk) {
        if (kk < nbe) {
            const int buf = kk & 1;
            __syncthreads();
            const Red *red = s.red + buf * NWARP;
            unsigned long long key = red[0].key;
            int q = 0;
#pragma unroll
            for (int j = 1; j < NWARP; ++j) {
                const unsigned long long k = red[j].key;
                if (k > key) { key = k; q = j; }
            }
            const double2 d = red[q].d;
            const double2 *srow = s.cand + (buf * NWARP + q) * 32;
            const int p = 0x7FF - (int)(key & 0x7FFull);
            if ((key >> 11) == 0 && info == 0) info = kb + kk + 1;
#pragma unroll
            for (int r = 0; r < RPT; ++r)
                if (tid + NT * r == p) used |= 1u << r;
            if (tid == 0) { s.prow[kb + kk] = p; s.inP[p] = tag; }
            // column kk+1 first, then its pivot search overlaps the rest of the row
            const bool more = (kk + 1 < NB) && (kk + 1 < nbe);
            double2 gm[RPT];
#pragma unroll
            for (int r = 0; r < RPT; ++r) gm[r] = (tid + NT * r == p) ? make_double2(0.0, 0.0) : zmul(w[r][kk], d);
            if (kk + 1 < NB) {
                double2 fn[RPT];
                const double2 rn = srow[(kk + 1) % NB];
#pragma unroll
                for (int r = 0; r < RPT; ++r)
                    fn[r] = (tid + NT * r == p) ? zmul(rn, d) : zfms(gm[r], rn, w[r][(kk + 1) % NB]);
                mine = more ? warp_pivot<NB, RPT>(fn, used, buf ^ 1, s) : -1;
            } else {
                mine = -1;
            }
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                if (tid + NT * r == p) {
#pragma unroll
                    for (int jj = 0; jj < NB; ++jj) w[r][jj] = (jj == kk) ? d : zmul(srow[jj], d);
                } else {
#pragma unroll
                    for (int jj = 0; jj < NB; ++jj)
                        w[r][jj] = (jj == kk) ? make_double2(-gm[r].x, -gm[r].y) : zfms(gm[r], srow[jj], w[r][jj]);
                }
            }
            if (mine >= 0) {
                double2 *dst = s.cand + ((buf ^ 1) * NWARP + warp) * 32;
#pragma unroll
                for (int r = 0; r < RPT; ++r)
                    if (r == mine) {
#pragma unroll
                        for (int jj = 0; jj < NB; ++jj) dst[jj] = w[r][jj];
                    }
            }
        }
    }
    __syncthreads();
}

// In-place blocked Gauss-Jordan inverse of the N x N block A (leading
// dimension ld) with implicit partial pivoting.  Panels of 2*NB columns are
// eliminated as two register sub-panels a and b:
//   1. eliminate a;  2. bring b up to date with a's steps;  3. eliminate b;
//   4. apply b's steps to a;  5. one rank-2NB trailing update of the rest.
// On return s.prow/s.iprow hold the permutations (inv(A)(r,c) =
// A(prow[r], iprow[c])).  Returns the LAPACK-style info (1-based column of
// the first zero pivot, 0 if none); identical in every thread.
template <int NB, int RPT>
__device__ int gj_invert_pair(double2 *__restrict__ A, int N, int ld, const Smem &s) {
    const int tid = threadIdx.x;
    const int ldw = s.ldw;
    int info = 0;
    unsigned used = 0;
#pragma unroll
    for (int r = 0; r < RPT; ++r)
        if (tid + NT * r >= N) used |= 1u << r;
    for (int i = tid; i < N; i += NT) s.inP[i] = 0;
    __syncthreads();

    for (int k0 = 0; k0 < N; k0 += 2 * NB) {
        const int nba = min(NB, N - k0);
        const int nbb = max(0, min(NB, N - k0 - nba));
        const int nbt = nba + nbb;
        double2 w[RPT][NB];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = tid + NT * r;
#pragma unroll
            for (int jj = 0; jj < NB; ++jj)
                w[r][jj] = (i < N && jj < nba) ? A[i + (size_t)ld * (k0 + jj)] : make_double2(0.0, 0.0);
        }
        double2 *sWa = s.big;              // [NB][ldw] sub-panel a after step 1
        double2 *sX = s.big + NB * ldw;    // [NB][NB]
        const int kbb = k0 + nba;
        // one call site for both sub-panels keeps one copy of the unrolled steps
        for (int half = 0; half < (nbb > 0 ? 2 : 1); ++half) {
            if (half == 1) {
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = tid + NT * r;
                    if (i < ldw) {
#pragma unroll
                        for (int jj = 0; jj < NB; ++jj) sWa[jj * ldw + i] = (i < N) ? w[r][jj] : make_double2(0.0, 0.0);
                    }
                }
                // rows P_a of sub-panel b before a's steps
                for (int e = tid; e < NB * NB; e += NT) {
                    const int kk = e / NB, c = e % NB;
                    sX[e] = (kk < nba && c < nbb) ? A[s.prow[k0 + kk] + (size_t)ld * (kbb + c)] : make_double2(0.0, 0.0);
                }
                __syncthreads();
                // 2. b = mask_a(b) + W_a * b(P_a, :)
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = tid + NT * r;
                    const bool keep = (i < N) && s.inP[i] != 1;
#pragma unroll
                    for (int c = 0; c < NB; ++c)
                        w[r][c] = (keep && c < nbb) ? A[i + (size_t)ld * (kbb + c)] : make_double2(0.0, 0.0);
                    if (i < N) {
#pragma unroll 1
                        for (int kk = 0; kk < nba; ++kk) {
                            const double2 wa = sWa[kk * ldw + i];
#pragma unroll
                            for (int c = 0; c < NB; ++c) w[r][c] = zfma(wa, sX[kk * NB + c], w[r][c]);
                        }
                    }
                }
            }
            // 1. / 3. eliminate the sub-panel
            factor_subpanel<NB, RPT>(w, half ? kbb : k0, half ? nbb : nba, used, info, half + 1, s);
        }
        if (nbb > 0) {
            // rows P_b of sub-panel a after step 1
            for (int e = tid; e < NB * NB; e += NT) {
                const int kk = e / NB, c = e % NB;
                sX[e] = (kk < nbb && c < nba) ? sWa[c * ldw + s.prow[kbb + kk]] : make_double2(0.0, 0.0);
            }
            __syncthreads();
            // 4. a = mask_b(a) + W_b * a(P_b, :); write W = [a | b] back
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = tid + NT * r;
                if (i < N) {
                    const bool keep = s.inP[i] != 2;
                    for (int c = 0; c < nba; ++c) {
                        double2 v = keep ? sWa[c * ldw + i] : make_double2(0.0, 0.0);
#pragma unroll
                        for (int kk = 0; kk < NB; ++kk) v = zfma(w[r][kk], sX[kk * NB + c], v);
                        A[i + (size_t)ld * (k0 + c)] = v;
                    }
#pragma unroll
                    for (int kk = 0; kk < NB; ++kk)
                        if (kk < nbb) A[i + (size_t)ld * (kbb + kk)] = w[r][kk];
                }
            }
        } else {
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = tid + NT * r;
                if (i < N) {
#pragma unroll
                    for (int jj = 0; jj < NB; ++jj)
                        if (jj < nba) A[i + (size_t)ld * (k0 + jj)] = w[r][jj];
                }
            }
        }
        __syncthreads();
        if (nbt < N) trailing_update<2 * NB>(A, N, ld, k0, nbt, s);
        __syncthreads();
        if (tid < nbt) s.inP[s.prow[k0 + tid]] = 0;
        __syncthreads();
    }
    for (int k = tid; k < N; k += NT) s.iprow[s.prow[k]] = k;
    __syncthreads();
    return info;
}

// The same inverse with panels of P sub-panels of NB columns each (one
// rank-P*NB trailing update per panel) for blocks whose sub-panels do not fit
// the shared-memory buffer of gj_invert_pair: the finished sub-panels stay in
// A.  Per sub-panel p: (i) bring its columns up to date with sub-panels < p,
// b = mask_{<p}(b) + W_{<p} b(P_{<p}); (ii) eliminate it in registers; (iii)
// apply its steps to the earlier columns, W_{<p} = mask_p(W_{<p}) +
// W_p W_{<p}(P_p); the trailing update then applies the whole panel at once,
// the single-panel formula of trailing_update with W = A(:, panel).
template <int NB, int RPT, int P>
__device__ int gj_invert_multi(double2 *__restrict__ A, int N, int ld, const Smem &s) {
    const int tid = threadIdx.x;
    const double2 zero = make_double2(0.0, 0.0);
    int info = 0;
    unsigned used = 0;
#pragma unroll
    for (int r = 0; r < RPT; ++r)
        if (tid + NT * r >= N) used |= 1u << r;
    for (int i = tid; i < N; i += NT) s.inP[i] = 0;
    __syncthreads();
    double2 *sX = s.big;                // [P*NB][NB]: rows P_{<p} of sub-panel p before (i)
    double2 *sY = s.big + P * NB * NB;  // [NB][P*NB]: rows P_p of the earlier columns before (iii)
    for (int k0 = 0; k0 < N; k0 += P * NB) {
        const int nbt = min(P * NB, N - k0);
        for (int p = 0; p * NB < nbt; ++p) {
            const int cp = k0 + p * NB, kprev = p * NB;
            const int nbp = min(NB, nbt - kprev);
            if (p > 0) {
                for (int e = tid; e < kprev * NB; e += NT) {
                    const int kk = e / NB, c = e % NB;
                    sX[e] = (c < nbp) ? A[s.prow[k0 + kk] + (size_t)ld * (cp + c)] : zero;
                }
                __syncthreads();
            }
            double2 w[RPT][NB];
#pragma unroll
            for (int r = 0; r < RPT; ++r) {
                const int i = tid + NT * r;
                const bool keep = (i < N) && !(s.inP[i] >= 1 && s.inP[i] <= p);
#pragma unroll
                for (int c = 0; c < NB; ++c) w[r][c] = (keep && c < nbp) ? A[i + (size_t)ld * (cp + c)] : zero;
                if (i < N) {
                    // kprev is a multiple of NB: NB loads of the row in flight per group
#pragma unroll 1
                    for (int kk0 = 0; kk0 < kprev; kk0 += NB) {
                        double2 wa[NB];
#pragma unroll
                        for (int u = 0; u < NB; ++u) wa[u] = A[i + (size_t)ld * (k0 + kk0 + u)];
#pragma unroll
                        for (int u = 0; u < NB; ++u)
#pragma unroll
                            for (int c = 0; c < NB; ++c) w[r][c] = zfma(wa[u], sX[(kk0 + u) * NB + c], w[r][c]);
                    }
                }
            }
            factor_subpanel<NB, RPT>(w, cp, nbp, used, info, p + 1, s);
            if (p > 0) {
                for (int e = tid; e < NB * kprev; e += NT) {
                    const int c = e / kprev, q = e % kprev;
                    sY[e] = (c < nbp) ? A[s.prow[cp + c] + (size_t)ld * (k0 + q)] : zero;
                }
                __syncthreads();
#pragma unroll
                for (int r = 0; r < RPT; ++r) {
                    const int i = tid + NT * r;
                    if (i < N) {
                        const bool keep = s.inP[i] != p + 1;
#pragma unroll 1
                        for (int q0 = 0; q0 < kprev; q0 += NB) {
                            double2 v[NB];
#pragma unroll
                            for (int u = 0; u < NB; ++u) v[u] = keep ? A[i + (size_t)ld * (k0 + q0 + u)] : zero;
#pragma unroll
                            for (int u = 0; u < NB; ++u) {
#pragma unroll
                                for (int c = 0; c < NB; ++c) v[u] = zfma(w[r][c], sY[c * kprev + q0 + u], v[u]);
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
                    for (int c = 0; c < NB; ++c)
                        if (c < nbp) A[i + (size_t)ld * (cp + c)] = w[r][c];
                }
            }
            __syncthreads();
        }
        if (nbt < N) trailing_update<P * NB, (RPT >= 4)>(A, N, ld, k0, nbt, s);
        __syncthreads();
        if (tid < nbt) s.inP[s.prow[k0 + tid]] = 0;
        __syncthreads();
    }
    for (int k = tid; k < N; k += NT) s.iprow[s.prow[k]] = k;
    __syncthreads();
    return info;
}

// The inverse used by the kernels: 16-column sub-panels in pairs through
// shared memory; 8-column sub-panels (the large-N variant) four per panel
// through A, so that every variant applies rank-32 trailing updates.
template <int NB, int RPT>
__device__ int gj_invert(double2 *__restrict__ A, int N, int ld, const Smem &s) {
    if constexpr (NB == 8) return gj_invert_multi<8, RPT, 4>(A, N, ld, s);
    else return gj_invert_pair<NB, RPT>(A, N, ld, s);
}

}  // namespace negf
