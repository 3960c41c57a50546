// negf_engine.cu -- kernels and C ABI of the FP64 RGF engine (sm_100a).
//
// Replaces the per-job drivers of src/negf.f90 and the solver of
// src/math_kernel.f90.  Three kernels carry the hot path:
//   k_transmission  F-mode streaming sweep + transmission epilogue, one CTA
//                   per (E,k) job, O(N^2) state per job (negf.f90:115-174)
//   k_rgf_slab      sweeps that keep every generator block, for the diagonal
//                   (density, LDOS) and first/last-column (tri_solve) blocks
//                   (negf.f90:9-113, 176-236; math_kernel.f90:44-165)
//   k_accumulate    weighted sum of the diagonal blocks over the jobs of a
//                   chunk (the accumulation loops of negf.f90:86-111,226-234)
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "engine_internal.h"
#include "negf_gpu.h"
#include "rgf_device.cuh"

using namespace negf;

namespace {

constexpr double PI = 3.141592653589793;           // global.f90:28
constexpr double HARTREE = 27.211386245988;        // global.f90:24
constexpr double K_B = 8.617333262e-5 / HARTREE;   // global.f90:26

struct RgfJob {
    double e_re, e_im;  // complex energy of the solve, E + i*eta already added
    double e_t;         // real energy of the transmission weights
    int ik;             // k-point
    int pad;
    // WANT_A only: slice k of the output is cd * G_kk + ca * G_k,s Gamma_s G_k,s^H
    // (s = the injecting lead's end slice, Gamma_s its open-channel widths)
    double cd_re, cd_im, ca_re, ca_im;
};

// ------------------------------------------------------------------ kernels
// One F-mode sweep and the transmission trace for the job (E = e + i*eta,
// k-point ik) of problem g, in the workspace A0 (four ld x N blocks).  The
// basis must already be in s.nx / s.ny.  Returns tau in *tau (thread 0) and
// the LAPACK-style info.
template <int NB, int RPT>
__device__ int transmission_job(const Geo &g, const Smem &s, double e, int ik, double2 *A0, double *tau) {
    const int N = g.N, ld = g.ld, Nz = g.Nz;
    double2 *A1 = A0 + (size_t)ld * N;
    double2 *P0 = A1 + (size_t)ld * N;
    double2 *P1 = P0 + (size_t)ld * N;
    const double2 E = make_double2(e, g.eta);
    job_vectors(g, s, E, e, ik);
    __syncthreads();
    open_rows(N, s);
    __syncthreads();
    const int nr = *s.nrows;
    double2 *cur = A0, *oth = A1, *P = P0, *Pn = P1;
    // generator_r(N_z-1) = inv(D_Nz)          math_kernel.f90:82
    form_block(cur, g, s, Nz - 1, E, ik, nullptr, nullptr);
    __syncthreads();
    int info = gj_invert<NB, RPT>(cur, N, ld, s);
    unpermute_rows(P, ld, cur, ld, N, nr, s);
    __syncthreads();
    // generator_r(m) = inv(D_{m+1} - generator_r(m+1)), with the rows of the
    // running product P = gR(Nz-1) ... gR(m) of the first-column chain
    // G_{Nz,1} = (-1)^(Nz-1) gR(Nz-1) ... gR(1) G_11 (math_kernel.f90:83-90,120-128)
    // that the trace reads
    for (int m = Nz - 3; m >= 0; --m) {
        form_block(oth, g, s, m + 1, E, ik, cur, nullptr);
        __syncthreads();
        const int r = gj_invert<NB, RPT>(oth, N, ld, s);
        if (r && !info) info = r;
        GemmArgs ga{Pn, ld, P, ld, s.iprow, oth, ld, s.iprow, nr, N, N, nullptr};
        cta_gemm(ga, s, GEMM_STORE, g.delta);
        __syncthreads();
        double2 *t = cur; cur = oth; oth = t;
        t = P; P = Pn; Pn = t;
    }
    // G_11 = inv(D_1 - generator_r(1))          math_kernel.f90:113-118
    form_block(oth, g, s, 0, E, ik, cur, nullptr);
    __syncthreads();
    const int r = gj_invert<NB, RPT>(oth, N, ld, s);
    if (r && !info) info = r;
    // tau = sum_ij gamma_L,i gamma_R,j |2 dz^2 G_{Nz,1}(i,j)|^2   grid.f90:362-383
    GemmArgs ga{nullptr, 0, P, ld, s.iprow, oth, ld, s.iprow, nr, N, N, s.rows};
    double t = cta_gemm(ga, s, GEMM_TAU, g.delta);
    t = block_sum(t, s);
    *tau = t;
    return info;
}

template <int NB, int RPT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_transmission(Geo g, const double *__restrict__ energies, int nE, int njobs, double2 *ws,
                   size_t wstride, double *tau_jobs, int *info_jobs) {
    extern __shared__ __align__(256) unsigned char smem[];
    Smem s = carve<NB>(smem, g.N);
    for (int i = threadIdx.x; i < g.N; i += NT) { s.nx[i] = g.nx[i]; s.ny[i] = g.ny[i]; }
    __syncthreads();
    double2 *A0 = ws + (size_t)blockIdx.x * wstride;
    for (int job = blockIdx.x; job < njobs; job += gridDim.x) {
        // job -> (energy, k-point), energy fastest: negf.f90:131-133
        const int ie = job % nE, ik = job / nE;
        double t = 0.0;
        const int info = transmission_job<NB, RPT>(g, s, energies[ie], ik, A0, &t);
        if (threadIdx.x == 0) {
            tau_jobs[job] = t;
            if (info_jobs) info_jobs[job] = info;
        }
        __syncthreads();
    }
}

// One (problem, energy, k-point) job of a batch over several problems.
struct BatchJob {
    int prob, ie, ik, pad;
};

// Several problems (each its own basis, V table, slices and k-points) in one
// persistent launch: CTAs take jobs from a counter in the given order
// (largest first), so long and short sweeps balance across the SMs.
template <int NB, int RPT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_transmission_batch(const Geo *__restrict__ geos, const BatchJob *__restrict__ jobs, int njobs,
                         const double *__restrict__ energies, double2 *ws, size_t wstride, double *tau_jobs,
                         int *info_jobs, int *counter) {
    extern __shared__ __align__(256) unsigned char smem[];
    __shared__ int next;
    double2 *A0 = ws + (size_t)blockIdx.x * wstride;
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1);
        __syncthreads();
        const int q = next;
        __syncthreads();
        if (q >= njobs) break;
        const BatchJob jb = jobs[q];
        const Geo g = geos[jb.prob];
        Smem s = carve<NB>(smem, g.N);
        for (int i = threadIdx.x; i < g.N; i += NT) { s.nx[i] = g.nx[i]; s.ny[i] = g.ny[i]; }
        __syncthreads();
        double t = 0.0;
        const int info = transmission_job<NB, RPT>(g, s, energies[jb.ie], jb.ik, A0, &t);
        if (threadIdx.x == 0) {
            tau_jobs[q] = t;
            info_jobs[q] = info;
        }
        __syncthreads();
    }
}

// tau(E) = sum_k w_k tau(E,k)   negf.f90:172
__global__ void k_tau_reduce(const double *__restrict__ tau_jobs, const double *__restrict__ kw, int nE,
                             int nk, double *__restrict__ tau) {
    const int ie = blockIdx.x * blockDim.x + threadIdx.x;
    if (ie >= nE) return;
    double t = 0.0;
    for (int ik = 0; ik < nk; ++ik) t += tau_jobs[(size_t)ik * nE + ie] * kw[ik];
    tau[ie] = t;
}

enum { WANT_D = 1, WANT_F = 2, WANT_L = 4, WANT_A = 8, WANT_MIRROR = 16 };

// One job per CTA.  slab (Nz blocks, leading dimension ld) first receives
// the generator_r blocks; with WANT_D it ends up holding G_kk in block k.
// out_first / out_last (leading dimension N) receive G_k1 / G_kNz.
// WANT_A (with WANT_D): block k becomes cd * G_kk + ca * A_k, where
// A_k = G_k1 Gamma_L G_k1^H is the spectral function injected by the left
// lead, restricted to its open channels: Y_1 = G_11(:, open) sqrt(gamma_L),
// Y_k = -gR(k-1) Y_{k-1}, A_k = Y_k Y_k^H (8 n_open N^2 flop per product).
// WANT_MIRROR runs the same recursions with the slices numbered from the
// right end (left-connected generators; the injecting lead is the right
// one), writing every block at its own slice index.  Workspace: 6 blocks.
template <int NB, int RPT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    k_rgf_slab(Geo g, const RgfJob *__restrict__ jobs, int njobs, const double2 *__restrict__ Dexp,
               double2 *ws, size_t wstride, double2 *slabs, size_t sstride, int want,
               double2 *out_first, double2 *out_last, int *info_jobs) {
    extern __shared__ __align__(256) unsigned char smem[];
    Smem s = carve<NB>(smem, g.N);
    const int N = g.N, ld = g.ld, Nz = g.Nz;
    const size_t NB2 = (size_t)ld * N;  // one workspace block
    const size_t NN = (size_t)N * N;    // one output block
    for (int i = threadIdx.x; i < N; i += NT) { s.nx[i] = g.nx[i]; s.ny[i] = g.ny[i]; }
    __syncthreads();
    const int job = blockIdx.x;
    if (job >= njobs) return;
    double2 *A0 = ws + (size_t)blockIdx.x * wstride;
    double2 *A1 = A0 + NB2, *T0 = A1 + NB2, *T1 = T0 + NB2, *T2 = T1 + NB2, *Zt = T2 + NB2;
    double2 *slab = slabs + (size_t)blockIdx.x * sstride;
    const bool mirror = (want & WANT_MIRROR) != 0;
    // slice of step x, and the slab block that holds it
    auto sl = [&](int x) { return mirror ? Nz - 1 - x : x; };
    auto blk = [&](int x) { return slab + NB2 * sl(x); };
    const RgfJob jb = jobs[job];
    const double2 E = make_double2(jb.e_re, jb.e_im);
    const int ik = jb.ik;
    if (!Dexp) job_vectors(g, s, E, jb.e_t, ik);
    __syncthreads();
    int info = 0, r;
    double2 *cur = A0, *oth = A1;

    if (want & (WANT_D | WANT_F)) {
        // generator_r, math_kernel.f90:81-91
        form_block(cur, g, s, sl(Nz - 1), E, ik, nullptr, Dexp);
        __syncthreads();
        info = gj_invert<NB, RPT>(cur, N, ld, s);
        unpermute(blk(Nz - 2), ld, cur, ld, N, s, 1.0);
        __syncthreads();
        for (int m = Nz - 3; m >= 0; --m) {
            form_block(oth, g, s, sl(m + 1), E, ik, cur, Dexp);
            __syncthreads();
            r = gj_invert<NB, RPT>(oth, N, ld, s);
            if (r && !info) info = r;
            unpermute(blk(m), ld, oth, ld, N, s, 1.0);
            __syncthreads();
            double2 *t = cur; cur = oth; oth = t;
        }
        form_block(oth, g, s, sl(0), E, ik, cur, Dexp);
        __syncthreads();
        r = gj_invert<NB, RPT>(oth, N, ld, s);
        if (r && !info) info = r;
        unpermute(T0, ld, oth, ld, N, s, 1.0);  // T0 = G_11
        __syncthreads();
        if ((want & WANT_F) && out_first) {
            // G_k1 = -gR(k-1) G_{k-1,1}, math_kernel.f90:112-129
            for (int e = threadIdx.x; e < N * N; e += NT) {
                const int i = e % N, j = e / N;
                out_first[e] = T0[i + (size_t)ld * j];
            }
            __syncthreads();
            for (int k = 1; k < Nz; ++k) {
                GemmArgs ga{out_first + NN * k, N, slab + NB2 * (k - 1), ld, nullptr,
                            out_first + NN * (k - 1), N, nullptr, N, N, N, nullptr};
                cta_gemm(ga, s, GEMM_STORE_NEG, g.delta);
                __syncthreads();
            }
        }
        if (want & WANT_D) {
            // G_kk = gR(k-1) (I + G_{k-1,k-1} gR(k-1)), math_kernel.f90:94-109.
            // Block k-1 of the slab is replaced by G_{k-1,k-1} once gR(k-1)
            // has been used for the last time.
            const bool wa = (want & WANT_A) != 0;
            const double2 cd = wa ? make_double2(jb.cd_re, jb.cd_im) : make_double2(1.0, 0.0);
            const double2 ca = make_double2(jb.ca_re, jb.ca_im);
            int nA = 0;
            double2 *Ya = A0, *Yb = A1;  // A0, A1 are free once the sweep is done
            if (wa && (ca.x != 0.0 || ca.y != 0.0)) {
                const double *gam = mirror ? s.gR : s.gL;
                open_cols(N, s, gam);
                __syncthreads();
                nA = *s.nrows;
                for (int e = threadIdx.x; e < N * nA; e += NT) {
                    const int i = e % N, c = e / N, j = s.rows[c];
                    const double sg = sqrt(gam[j]);
                    const double2 v = T0[i + (size_t)ld * j];
                    Ya[e] = make_double2(v.x * sg, v.y * sg);
                }
                __syncthreads();
            }
            // block += ca * Y Y^H, through Zt = Y^H (nA x N)
            auto add_spectral = [&](double2 *dst, const double2 *Y) {
                for (int e = threadIdx.x; e < N * nA; e += NT) {
                    const int i = e % N, c = e / N;
                    Zt[c + (size_t)nA * i] = make_double2(Y[e].x, -Y[e].y);
                }
                __syncthreads();
                GemmArgs ga{dst, ld, Y, N, nullptr, Zt, nA, nullptr, N, N, nA, nullptr, ca};
                cta_gemm(ga, s, GEMM_ADD_SCALED, g.delta);
                __syncthreads();
            };
            double2 *Gc = T0, *Gn = T2;
            for (int k = 1; k < Nz; ++k) {
                double2 *gRk = blk(k - 1);
                if (nA) {
                    GemmArgs gy{Yb, N, gRk, ld, nullptr, Ya, N, nullptr, N, nA, N, nullptr};
                    cta_gemm(gy, s, GEMM_STORE_NEG, g.delta);
                    __syncthreads();
                }
                GemmArgs g1{T1, ld, Gc, ld, nullptr, gRk, ld, nullptr, N, N, N, nullptr};
                cta_gemm(g1, s, GEMM_STORE_ADD_EYE, g.delta);
                __syncthreads();
                GemmArgs g2{Gn, ld, gRk, ld, nullptr, T1, ld, nullptr, N, N, N, nullptr};
                cta_gemm(g2, s, GEMM_STORE, g.delta);
                __syncthreads();
                for (int e = threadIdx.x; e < N * N; e += NT) {
                    const int i = e % N, j = e / N;
                    gRk[i + (size_t)ld * j] = zmul(cd, Gc[i + (size_t)ld * j]);
                }
                __syncthreads();
                if (nA) {
                    add_spectral(gRk, Ya);
                    double2 *t = Ya; Ya = Yb; Yb = t;
                }
                double2 *t = Gc; Gc = Gn; Gn = t;
            }
            double2 *last = blk(Nz - 1);
            for (int e = threadIdx.x; e < N * N; e += NT) {
                const int i = e % N, j = e / N;
                last[i + (size_t)ld * j] = zmul(cd, Gc[i + (size_t)ld * j]);
            }
            __syncthreads();
            if (nA) add_spectral(last, Ya);
        }
    }
    if ((want & WANT_L) && out_last) {
        // generator_l and the last column, math_kernel.f90:132-162; the
        // generator_l blocks reuse slab blocks 0..Nz-2 (D/F are done with it).
        cur = A0; oth = A1;
        form_block(cur, g, s, 0, E, ik, nullptr, Dexp);
        __syncthreads();
        r = gj_invert<NB, RPT>(cur, N, ld, s);
        if (r && !info) info = r;
        unpermute(slab, ld, cur, ld, N, s, 1.0);
        __syncthreads();
        for (int m = 1; m <= Nz - 2; ++m) {
            form_block(oth, g, s, m, E, ik, cur, Dexp);
            __syncthreads();
            r = gj_invert<NB, RPT>(oth, N, ld, s);
            if (r && !info) info = r;
            unpermute(slab + NB2 * m, ld, oth, ld, N, s, 1.0);
            __syncthreads();
            double2 *t = cur; cur = oth; oth = t;
        }
        form_block(oth, g, s, Nz - 1, E, ik, cur, Dexp);
        __syncthreads();
        r = gj_invert<NB, RPT>(oth, N, ld, s);
        if (r && !info) info = r;
        unpermute(out_last + NN * (Nz - 1), N, oth, ld, N, s, 1.0);
        __syncthreads();
        for (int k = 1; k < Nz; ++k) {
            GemmArgs ga{out_last + NN * (Nz - 1 - k), N, slab + NB2 * (Nz - 1 - k), ld, nullptr,
                        out_last + NN * (Nz - k), N, nullptr, N, N, N, nullptr};
            cta_gemm(ga, s, GEMM_STORE_NEG, g.delta);
            __syncthreads();
        }
    }
    if (threadIdx.x == 0 && info_jobs) info_jobs[job] = info;
}

// out[o](i,j,k) (+)= sum_{q<gsz} coef[o*gsz+q] * ((slab_{o*gsz+q}(i,j,k) * 2) * dz^2)
// with out blocks of leading dimension N (negf.f90:78-111, 218-234).
__global__ void k_accumulate(const double2 *__restrict__ slabs, size_t sstride, int ld, int N, int Nz,
                             const double2 *__restrict__ coef, int gsz, int nout, double dz,
                             int accumulate, double2 *__restrict__ out) {
    const size_t per = (size_t)N * N * Nz;
    const size_t total = per * nout;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const int o = (int)(e / per);
        const size_t r = e - (size_t)o * per;
        const int k = (int)(r / ((size_t)N * N));
        const int rem = (int)(r - (size_t)k * N * N);
        const int j = rem / N, i = rem - j * N;
        const size_t off = i + (size_t)ld * j + (size_t)ld * N * k;
        double2 acc = accumulate ? out[e] : make_double2(0.0, 0.0);
        for (int q = 0; q < gsz; ++q) {
            const int b = o * gsz + q;
            const double2 gv = slabs[(size_t)b * sstride + off];
            const double2 gs = make_double2(gv.x * 2.0 * (dz * dz), gv.y * 2.0 * (dz * dz));
            acc = zfma(coef[b], gs, acc);
        }
        out[e] = acc;
    }
}

// ------------------------------------------------- plane wave -> real space
// diag(u,v) = sum_ab G(a,b) e^{+2 pi i ((nx_a-nx_b) u/Nx + (ny_a-ny_b) v/Ny)}, the
// diagonal that the FFT pair of grid.f90:88-133 extracts.  One CTA per slice:
// G is binned on the difference n_a - n_b in shared memory, then transformed
// along x (UC rows of u at a time) and along y.  Writes Im(diag) * scale
// (main.f90:341-351) to dens, or the complex diagonal to cdiag.
constexpr int PT_THREADS = 256;
constexpr int PT_UC = 16;

__global__ void __launch_bounds__(PT_THREADS)
    k_ptor(const double2 *__restrict__ G, int N, int ldg, size_t gstride, const int *__restrict__ nx,
           const int *__restrict__ ny, int mx, int my, int Nx, int Ny, double scale,
           double *__restrict__ dens, double2 *__restrict__ cdiag) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int BX = 4 * mx + 1, BY = 4 * my + 1;
    double2 *bin = (double2 *)smem_raw;                  // [BY][BX]
    double2 *T = bin + (size_t)BX * BY;                  // [PT_UC][BY]
    double2 *twx = T + (size_t)PT_UC * BY;               // [Nx] e^{+2 pi i m/Nx}
    double2 *twy = twx + Nx;                             // [Ny]
    const int k = blockIdx.x;
    const double2 *Gk = G + gstride * k;
    for (int e = threadIdx.x; e < BX * BY; e += PT_THREADS) bin[e] = make_double2(0.0, 0.0);
    for (int m = threadIdx.x; m < Nx; m += PT_THREADS) {
        double sn, cs;
        sincospi(2.0 * m / Nx, &sn, &cs);
        twx[m] = make_double2(cs, sn);
    }
    for (int m = threadIdx.x; m < Ny; m += PT_THREADS) {
        double sn, cs;
        sincospi(2.0 * m / Ny, &sn, &cs);
        twy[m] = make_double2(cs, sn);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < N * N; e += PT_THREADS) {
        const int a = e % N, b = e / N;
        const double2 v = Gk[a + (size_t)ldg * b];
        double2 *t = bin + (nx[a] - nx[b] + 2 * mx) + BX * (ny[a] - ny[b] + 2 * my);
        atomicAdd(&t->x, v.x);
        atomicAdd(&t->y, v.y);
    }
    __syncthreads();
    for (int u0 = 0; u0 < Nx; u0 += PT_UC) {
        // T(u, dy) = sum_dx bin(dx, dy) e^{+2 pi i (dx - 2mx) u / Nx}
        for (int e = threadIdx.x; e < PT_UC * BY; e += PT_THREADS) {
            const int uu = e % PT_UC, dy = e / PT_UC, u = u0 + uu;
            double2 acc = make_double2(0.0, 0.0);
            if (u < Nx)
                for (int dx = 0; dx < BX; ++dx) {
                    int m = ((dx - 2 * mx) * u) % Nx;
                    if (m < 0) m += Nx;
                    acc = zfma(bin[dx + BX * dy], twx[m], acc);
                }
            T[uu + PT_UC * dy] = acc;
        }
        __syncthreads();
        // diag(u, v) = sum_dy T(u, dy) e^{+2 pi i (dy - 2my) v / Ny}
        for (int e = threadIdx.x; e < PT_UC * Ny; e += PT_THREADS) {
            const int uu = e % PT_UC, v = e / PT_UC, u = u0 + uu;
            if (u >= Nx) continue;
            double2 acc = make_double2(0.0, 0.0);
            for (int dy = 0; dy < BY; ++dy) {
                int m = ((dy - 2 * my) * v) % Ny;
                if (m < 0) m += Ny;
                acc = zfma(T[uu + PT_UC * dy], twy[m], acc);
            }
            const size_t o = u + (size_t)Nx * v + (size_t)Nx * Ny * k;
            if (dens) dens[o] = acc.y * scale;
            if (cdiag) cdiag[o] = acc;
        }
        __syncthreads();
    }
}

size_t ptor_smem(int mx, int my, int Nx, int Ny) {
    const size_t BX = 4 * (size_t)mx + 1, BY = 4 * (size_t)my + 1;
    return sizeof(double2) * (BX * BY + PT_UC * BY + Nx + Ny);
}

// LDOS_grid_converter (tools.f90:18-40) applied to one energy's real-space
// diagonal: LDOS(ii,jj,kk) += Im(diag(i,j,k)) * scale * factors (main.f90:510-526).
// LocalPotential_RealToPlanewave + the truncated copy of main.f90:239-247 on
// the GPU, one CTA per slice: V_hat(i,j) = (1/(Nx Ny)) sum_xy V(x,y)
// e^{-2 pi i (x i/Nx + y j/Ny)} on the window |i| <= ngx/2, |j| <= ngy/2 (zero
// elsewhere), as the separable transform of negf_vhat: the slice in shared
// memory, the x transform for i >= 0, the y transform, and V_hat(i,j) =
// conj(V_hat(-i,-j)) for i < 0 (grid.f90:64-68).  tx, ty: e^{-2 pi i m/N}.
constexpr int VH_THREADS = 256;
__global__ void __launch_bounds__(VH_THREADS)
    k_vhat(const double *__restrict__ vreal, int Nx, int Ny, int ngx, int ngy, const double2 *__restrict__ tx,
           const double2 *__restrict__ ty, double2 *__restrict__ vhat) {
    extern __shared__ __align__(16) unsigned char vsm[];
    const int W = 2 * ngx + 1, H = 2 * ngy + 1, hx = ngx / 2, hy = ngy / 2;
    double *v = (double *)vsm;                           // [Ny][Nx]
    double2 *X = (double2 *)(v + (size_t)Nx * Ny);        // [Ny][hx + 1]
    const double *src = vreal + (size_t)Nx * Ny * blockIdx.x;
    for (int e = threadIdx.x; e < Nx * Ny; e += VH_THREADS) v[e] = src[e];
    __syncthreads();
    for (int e = threadIdx.x; e < (hx + 1) * Ny; e += VH_THREADS) {
        const int i = e % (hx + 1), y = e / (hx + 1);
        double2 acc = make_double2(0.0, 0.0);
        int m = 0;  // (x * i) mod Nx
        for (int x = 0; x < Nx; ++x) {
            const double a = v[x + Nx * y];
            const double2 t = tx[m];
            acc.x += a * t.x;
            acc.y += a * t.y;
            m += i;
            if (m >= Nx) m -= Nx;
        }
        X[e] = acc;
    }
    __syncthreads();
    double2 *o = vhat + (size_t)W * H * blockIdx.x;
    const double inv = 1.0 / ((double)Nx * Ny);
    for (int e = threadIdx.x; e < W * H; e += VH_THREADS) {
        const int ii = e % W - ngx, jj = e / W - ngy;
        double2 r = make_double2(0.0, 0.0);
        if (ii >= -hx && ii <= hx && jj >= -hy && jj <= hy) {
            const int i = ii >= 0 ? ii : -ii, j = ii >= 0 ? jj : -jj;
            const int step = ((j % Ny) + Ny) % Ny;
            double2 acc = make_double2(0.0, 0.0);
            int m = 0;  // (y * j) mod Ny
            for (int y = 0; y < Ny; ++y) {
                acc = zfma(X[i + (hx + 1) * y], ty[m], acc);
                m += step;
                if (m >= Ny) m -= Ny;
            }
            r = make_double2(acc.x * inv, ii >= 0 ? acc.y * inv : -(acc.y * inv));
        }
        o[e] = r;
    }
}

__global__ void k_ldos_convert(const double2 *__restrict__ diag, int Nx, int Ny, int Nz, int gx, int gy,
                               int gz, double dx, double dy, double dz, double scale, int Mx, int My,
                               double *__restrict__ out) {
    const size_t tot = (size_t)Nx * Ny * Nz;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % Nx), j = (int)((e / Nx) % Ny), k = (int)(e / ((size_t)Nx * Ny));
        double f = scale;
        int ii = 0, jj = 0, kk = 0;
        // 1-based grid index m selects one point, -1 integrates (x delta), 0 keeps the axis
        if (gx == 0) ii = i; else if (gx == -1) f *= dx; else if (gx != i + 1) f = 0.0;
        if (gy == 0) jj = j; else if (gy == -1) f *= dy; else if (gy != j + 1) f = 0.0;
        if (gz == 0) kk = k; else if (gz == -1) f *= dz; else if (gz != k + 1) f = 0.0;
        if (f != 0.0) atomicAdd(out + ii + (size_t)Mx * (jj + (size_t)My * kk), diag[e].y * f);
    }
}

}  // namespace

// ======================================================================= host
// struct negf_ctx: engine_internal.h

namespace {

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "negf_gpu: %s failed: %s\n", #x, cudaGetErrorString(e_));      \
            return NEGF_ERR_CUDA;                                                          \
        }                                                                                  \
    } while (0)

Geo make_geo(const negf_ctx *c) {
    Geo g;
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

int ensure_ws(negf_ctx *c, size_t bytes) {
    if (bytes <= c->ws_bytes) return 0;
    if (c->d_ws) CK(cudaFree(c->d_ws));
    c->d_ws = nullptr;
    c->ws_bytes = 0;
    if (cudaMalloc(&c->d_ws, bytes) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    c->ws_bytes = bytes;
    return 0;
}

// Grows the per-call arrays.  The capacity is zeroed before the old arrays
// are released, so a failed allocation leaves the context empty (the next
// call retries) rather than holding freed pointers under a stale capacity.
int ensure_jobs(negf_ctx *c, int nE, int njobs) {
    if (nE > c->cap_E) {
        c->cap_E = 0;
        if (c->d_E) CK(cudaFree(c->d_E));
        if (c->d_tau) CK(cudaFree(c->d_tau));
        c->d_E = nullptr;
        c->d_tau = nullptr;
        if (cudaMalloc(&c->d_E, sizeof(double) * nE) != cudaSuccess ||
            cudaMalloc(&c->d_tau, sizeof(double) * nE) != cudaSuccess) {
            cudaGetLastError();
            return NEGF_ERR_NOMEM;
        }
        c->cap_E = nE;
    }
    if (njobs > c->cap_jobs) {
        c->cap_jobs = 0;
        if (c->d_tau_jobs) CK(cudaFree(c->d_tau_jobs));
        if (c->d_info) CK(cudaFree(c->d_info));
        c->d_tau_jobs = nullptr;
        c->d_info = nullptr;
        if (cudaMalloc(&c->d_tau_jobs, sizeof(double) * njobs) != cudaSuccess ||
            cudaMalloc(&c->d_info, sizeof(int) * njobs) != cudaSuccess) {
            cudaGetLastError();
            return NEGF_ERR_NOMEM;
        }
        c->cap_jobs = njobs;
    }
    return 0;
}

// Kernel variants by basis size: (panel width NB, rows per thread RPT,
// CTAs per SM).  Up to 256 plane waves two CTAs share an SM.
enum Variant { V16x1 = 0, V16x2 = 1, V8x4 = 2, V8x1 = 3, VNONE = 4 };
Variant pick_variant(int N) {
    if (N <= NT) return V16x1;
    if (N <= 2 * NT) return V16x2;
    if (N <= 4 * NT) return V8x4;
    return VNONE;
}
bool variant_fits(int v, int N) {
    return (v == V16x1 && N <= NT) || (v == V16x2 && N <= 2 * NT) || (v == V8x4 && N <= 4 * NT) ||
           (v == V8x1 && N <= NT);
}
// Default variant of the transmission kernels: up to 256 plane waves the
// 8-column panels in fours (8 x 1 x 2; at N = 69 7100 vs 5784 solves/s for
// 16 x 1 x 2, at N = 221 194 vs 184).  The slab kernels keep pick_variant:
// their 8 x 1 x 2 build measured slower (N = 221: density 53.9 vs 55.2,
// LDOS 47.3 vs 53.9 jobs/s; N = 69 LDOS 953 vs 1416).
Variant transmission_variant(int N) { return N <= NT ? V8x1 : pick_variant(N); }
Variant ctx_variant(const negf_ctx *c) {
    return (c->variant >= 0 && variant_fits(c->variant, c->N)) ? (Variant)c->variant : transmission_variant(c->N);
}
size_t variant_smem(Variant v, int N) {
    switch (v) {
        case V16x1: return smem_bytes<16>(N);
        case V16x2: return smem_bytes<16>(N);
        case V8x4: return smem_bytes<8>(N);
        case V8x1: return smem_bytes<8>(N);
        default: return 0;
    }
}

template <typename K>
int prep_kernel(K kern, size_t smem, int *occ) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int o = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, NT, smem));
    *occ = o > 0 ? o : 1;
    return 0;
}

// CTAs of the transmission kernel resident per SM for this N.
int resident_ctas(int N) {
    const Variant v = pick_variant(N);
    const size_t smem = variant_smem(v, N);
    int occ = 1;
    switch (v) {
        case V16x1: prep_kernel(k_transmission<16, 1, 2>, smem, &occ); break;
        case V16x2: prep_kernel(k_transmission<16, 2, 1>, smem, &occ); break;
        case V8x4: prep_kernel(k_transmission<8, 4, 1>, smem, &occ); break;
        default: break;
    }
    return occ;
}

int transmission_launch(negf_ctx *c, const double *d_E, int nE, double *d_tau, double *d_tau_jobs,
                        int *d_info, cudaStream_t st) {
    const int njobs = nE * c->nk;
    const Variant v = ctx_variant(c);
    if (v == VNONE) return NEGF_ERR_UNSUPPORTED;
    const size_t smem = variant_smem(v, c->N);
    int occ = 1, rc = 0;
    switch (v) {
        case V16x1: rc = prep_kernel(k_transmission<16, 1, 2>, smem, &occ); break;
        case V16x2: rc = prep_kernel(k_transmission<16, 2, 1>, smem, &occ); break;
        case V8x1: rc = prep_kernel(k_transmission<8, 1, 2>, smem, &occ); break;
        default: rc = prep_kernel(k_transmission<8, 4, 1>, smem, &occ); break;
    }
    if (rc) return rc;
    const int grid = std::min(njobs, c->num_sms * occ);
    const size_t wstride = 4 * (size_t)c->ld * c->N;
    rc = ensure_ws(c, sizeof(double2) * wstride * grid);
    if (rc) return rc;
    Geo g = make_geo(c);
    double2 *ws = (double2 *)c->d_ws;
    switch (v) {
        case V16x1:
            k_transmission<16, 1, 2><<<grid, NT, smem, st>>>(g, d_E, nE, njobs, ws, wstride, d_tau_jobs, d_info);
            break;
        case V16x2:
            k_transmission<16, 2, 1><<<grid, NT, smem, st>>>(g, d_E, nE, njobs, ws, wstride, d_tau_jobs, d_info);
            break;
        case V8x1:
            k_transmission<8, 1, 2><<<grid, NT, smem, st>>>(g, d_E, nE, njobs, ws, wstride, d_tau_jobs, d_info);
            break;
        default:
            k_transmission<8, 4, 1><<<grid, NT, smem, st>>>(g, d_E, nE, njobs, ws, wstride, d_tau_jobs, d_info);
            break;
    }
    CK(cudaGetLastError());
    k_tau_reduce<<<(nE + 127) / 128, 128, 0, st>>>(d_tau_jobs, c->d_kw, nE, c->nk, d_tau);
    CK(cudaGetLastError());
    return 0;
}

int slab_launch(negf_ctx *c, const Geo &g, const RgfJob *d_jobs, int njobs, const double2 *d_D,
                double2 *d_slabs, size_t sstride, int want, double2 *d_first, double2 *d_last,
                int *d_info, cudaStream_t st) {
    const Variant v = pick_variant(g.N);
    if (v == VNONE) return NEGF_ERR_UNSUPPORTED;
    const size_t smem = variant_smem(v, g.N);
    const size_t wstride = 6 * (size_t)g.ld * g.N;
    int rc = ensure_ws(c, sizeof(double2) * wstride * njobs);
    if (rc) return rc;
    double2 *ws = (double2 *)c->d_ws;
    int occ = 1;
    switch (v) {
        case V16x1:
            if ((rc = prep_kernel(k_rgf_slab<16, 1, 2>, smem, &occ))) return rc;
            k_rgf_slab<16, 1, 2><<<njobs, NT, smem, st>>>(g, d_jobs, njobs, d_D, ws, wstride, d_slabs, sstride,
                                                           want, d_first, d_last, d_info);
            break;
        case V16x2:
            if ((rc = prep_kernel(k_rgf_slab<16, 2, 1>, smem, &occ))) return rc;
            k_rgf_slab<16, 2, 1><<<njobs, NT, smem, st>>>(g, d_jobs, njobs, d_D, ws, wstride, d_slabs, sstride,
                                                           want, d_first, d_last, d_info);
            break;
        default:
            if ((rc = prep_kernel(k_rgf_slab<8, 4, 1>, smem, &occ))) return rc;
            k_rgf_slab<8, 4, 1><<<njobs, NT, smem, st>>>(g, d_jobs, njobs, d_D, ws, wstride, d_slabs, sstride,
                                                          want, d_first, d_last, d_info);
            break;
    }
    CK(cudaGetLastError());
    return 0;
}

void fill_stats(negf_stats *st, const std::vector<int> &info, double ms) {
    if (!st) return;
    st->n_jobs = (int)info.size();
    st->n_singular = 0;
    st->first_bad_job = -1;
    st->info = 0;
    for (size_t i = 0; i < info.size(); ++i)
        if (info[i]) {
            if (st->first_bad_job < 0) { st->first_bad_job = (int)i; st->info = info[i]; }
            st->n_singular++;
        }
    st->device_ms = ms;
}

int first_info(const std::vector<int> &info) {
    for (int v : info)
        if (v) return v;
    return 0;
}

// Jobs that fit in device memory at once for the slab kernel.
int slab_jobs_in_flight(negf_ctx *c, size_t per_job_bytes, int njobs) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    free_b += c->ws_bytes;  // the workspace is re-sized for the chunk
    const size_t budget = (size_t)(0.8 * (double)free_b);
    size_t fit = per_job_bytes ? budget / per_job_bytes : (size_t)njobs;
    int b = (int)std::min<size_t>(fit, (size_t)std::min(njobs, c->num_sms * resident_ctas(c->N)));
    return std::max(b, 0);
}

// Runs the D-mode sweeps for `jobs` in chunks and forms the weighted sums of
// their diagonal blocks, 2 dz^2 G_kk scaled by coef[job]:
//   gsz == 0: every job sums into out[0] (density; chunks accumulate);
//   gsz  > 0: jobs [o*gsz, (o+1)*gsz) sum into out[o] (LDOS per energy).
// want selects the slab mode (WANT_D, or WANT_D | WANT_A [| WANT_MIRROR] with
// the per-job cd / ca).
int diag_accumulate(negf_ctx *c, const std::vector<RgfJob> &jobs, const std::vector<double2> &coef,
                    int gsz, double2 *d_out, std::vector<int> &info_all, double &ms_total,
                    int want = WANT_D) {
    const int njobs = (int)jobs.size();
    const int N = c->N, Nz = c->Nz, ld = c->ld;
    const size_t sstride = (size_t)ld * N * Nz;
    const size_t per_job = sizeof(double2) * (sstride + 6 * (size_t)ld * N);
    int b = slab_jobs_in_flight(c, per_job, njobs);
    if (gsz > 0) b = (b / gsz) * gsz;
    if (b < std::max(gsz, 1)) return NEGF_ERR_NOMEM;
    double2 *d_slabs = nullptr, *d_coef = nullptr;
    RgfJob *d_jobs = nullptr;
    int *d_info = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_slabs, sizeof(double2) * sstride * b) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    if (cudaMalloc(&d_coef, sizeof(double2) * b) != cudaSuccess ||
        cudaMalloc(&d_jobs, sizeof(RgfJob) * b) != cudaSuccess ||
        cudaMalloc(&d_info, sizeof(int) * b) != cudaSuccess) {
        cudaFree(d_slabs); cudaFree(d_coef); cudaFree(d_jobs);
        return NEGF_ERR_CUDA;
    }
    Geo g = make_geo(c);
    info_all.assign(njobs, 0);
    ms_total = 0.0;
    for (int j0 = 0; j0 < njobs && !rc; j0 += b) {
        const int nb = std::min(b, njobs - j0);
        const int gs = gsz > 0 ? gsz : nb;
        const int nout = nb / gs;
        const int o0 = gsz > 0 ? j0 / gsz : 0;
        const int acc = gsz > 0 ? 0 : (j0 > 0);
        if (cudaMemcpyAsync(d_jobs, jobs.data() + j0, sizeof(RgfJob) * nb, cudaMemcpyHostToDevice, c->stream) ||
            cudaMemcpyAsync(d_coef, coef.data() + j0, sizeof(double2) * nb, cudaMemcpyHostToDevice, c->stream) ||
            cudaEventRecord(c->ev0, c->stream)) { rc = NEGF_ERR_CUDA; break; }
        rc = slab_launch(c, g, d_jobs, nb, nullptr, d_slabs, sstride, want, nullptr, nullptr, d_info, c->stream);
        if (rc) break;
        const size_t tot = (size_t)N * N * Nz * nout;
        const int blocks = (int)std::min<size_t>((tot + 255) / 256, (size_t)c->num_sms * 8);
        k_accumulate<<<blocks, 256, 0, c->stream>>>(d_slabs, sstride, ld, N, Nz, d_coef, gs, nout,
                                                    c->Lz / Nz, acc, d_out + (size_t)o0 * N * N * Nz);
        float ms = 0.f;
        if (cudaGetLastError() || cudaEventRecord(c->ev1, c->stream) ||
            cudaMemcpyAsync(info_all.data() + j0, d_info, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream) ||
            cudaStreamSynchronize(c->stream) || cudaEventElapsedTime(&ms, c->ev0, c->ev1)) {
            rc = NEGF_ERR_CUDA;
            break;
        }
        ms_total += ms;
    }
    cudaFree(d_slabs);
    cudaFree(d_coef);
    cudaFree(d_jobs);
    cudaFree(d_info);
    return rc;
}

// n-point Gauss-Legendre rule on [-1, 1], nodes ascending.  Newton's method on
// P_n from the guesses cos(pi (i + 3/4) / (n + 1/2)); P_n by the three-term
// recurrence (k P_k = (2k-1) x P_{k-1} - (k-1) P_{k-2}), P_n' = n (x P_n - P_{n-1})
// / (x^2 - 1), weights 2 / ((1 - x^2) P_n'(x)^2).
void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    auto eval = [n](double z, double *dp) {
        double p0 = 1.0, p1 = z;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        *dp = n * (z * p1 - p0) / (z * z - 1.0);
        return p1;
    };
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
        for (int it = 0; it < 100; ++it) {
            const double pn = eval(z, &dp);
            const double step = pn / dp;
            z -= step;
            if (std::fabs(step) <= 1e-15) break;
        }
        eval(z, &dp);
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

int check_problem(const negf_problem *p) {
    if (!p || p->N < 1 || p->Nz < 2 || p->ngx < 0 || p->ngy < 0 || !p->nx || !p->ny || !p->vhat ||
        p->nk < 1 || !p->kpt || !(p->Lx > 0) || !(p->Ly > 0) || !(p->Lz > 0))
        return NEGF_ERR_ARG;
    for (int i = 0; i < p->N; ++i)
        for (int j = 0; j < p->N; ++j) {
            const int dx = p->nx[i] - p->nx[j], dy = p->ny[i] - p->ny[j];
            if (dx < -p->ngx || dx > p->ngx || dy < -p->ngy || dy > p->ngy) return NEGF_ERR_ARG;
        }
    if (pick_variant(p->N) == VNONE) return NEGF_ERR_UNSUPPORTED;
    if (p->lead_model != 0 && p->lead_model != 1) return NEGF_ERR_ARG;
    return 0;
}

}  // namespace

extern "C" {

const char *negf_version(void) { return "negftrans_b200 0.1 (sm_100a, FP64 RGF)"; }

int negf_ctx_create(const negf_problem *p, int32_t device, negf_ctx **out) {
    if (!out) return NEGF_ERR_ARG;
    *out = nullptr;
    int rc = check_problem(p);
    if (rc) return rc;
    negf_ctx *c = new negf_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return NEGF_ERR_CUDA; }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    c->N = p->N; c->Nz = p->Nz; c->ld = round_up(p->N, 8);
    c->ngx = p->ngx; c->ngy = p->ngy; c->nk = p->nk;
    c->Lx = p->Lx; c->Ly = p->Ly; c->Lz = p->Lz;
    c->V_L = p->V_L; c->V_R = p->V_R; c->eta = p->eta;
    c->lead_model = p->lead_model;
    c->kpt.assign(p->kpt, p->kpt + 3 * (size_t)p->nk);
    c->nx.assign(p->nx, p->nx + p->N);
    c->ny.assign(p->ny, p->ny + p->N);
    const size_t nv = (size_t)(2 * p->ngx + 1) * (2 * p->ngy + 1) * p->Nz;
    std::vector<double> ax((size_t)p->nk * p->N), ay((size_t)p->nk * p->N), kw(p->nk);
    for (int k = 0; k < p->nk; ++k) {
        kw[k] = p->kpt[3 * k + 2];
        for (int i = 0; i < p->N; ++i) {
            // (2 * nx_grid(i) * pi / Lx + kx), grid.f90:258
            ax[(size_t)k * p->N + i] = (double)(2 * p->nx[i]) * PI / p->Lx + p->kpt[3 * k];
            ay[(size_t)k * p->N + i] = (double)(2 * p->ny[i]) * PI / p->Ly + p->kpt[3 * k + 1];
        }
    }
#define CKC(x) do { if ((x) != cudaSuccess) { cudaGetLastError(); negf_ctx_destroy(c); return NEGF_ERR_CUDA; } } while (0)
    CKC(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CKC(cudaEventCreate(&c->ev0));
    CKC(cudaEventCreate(&c->ev1));
    CKC(cudaMalloc(&c->d_vhat, sizeof(double2) * nv));
    CKC(cudaMalloc(&c->d_nx, sizeof(int) * p->N));
    CKC(cudaMalloc(&c->d_ny, sizeof(int) * p->N));
    CKC(cudaMalloc(&c->d_ax, sizeof(double) * ax.size()));
    CKC(cudaMalloc(&c->d_ay, sizeof(double) * ay.size()));
    CKC(cudaMalloc(&c->d_kw, sizeof(double) * kw.size()));
    CKC(cudaMemcpy(c->d_vhat, p->vhat, sizeof(double2) * nv, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_nx, p->nx, sizeof(int) * p->N, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_ny, p->ny, sizeof(int) * p->N, cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_ax, ax.data(), sizeof(double) * ax.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_ay, ay.data(), sizeof(double) * ay.size(), cudaMemcpyHostToDevice));
    CKC(cudaMemcpy(c->d_kw, kw.data(), sizeof(double) * kw.size(), cudaMemcpyHostToDevice));
#undef CKC
    *out = c;
    return NEGF_OK;
}

int negf_ctx_destroy(negf_ctx *c) {
    if (!c) return NEGF_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_vhat); cudaFree(c->d_nx); cudaFree(c->d_ny);
    cudaFree(c->d_ax); cudaFree(c->d_ay); cudaFree(c->d_kw);
    cudaFree(c->d_ws); cudaFree(c->d_E); cudaFree(c->d_tau); cudaFree(c->d_tau_jobs); cudaFree(c->d_info);
    cudaFree(c->d_mixed);
    cudaFree(c->d_voff);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return NEGF_OK;
}

int negf_transmission_device(negf_ctx *c, const double *d_energies, int32_t nE, int32_t precision,
                             double *d_tau, double *d_tau_jobs, int32_t *d_info, void *stream) {
    if (!c || !d_energies || !d_tau || nE < 1) return NEGF_ERR_ARG;
    if (precision != NEGF_FP64 && precision != NEGF_MIXED) return NEGF_ERR_UNSUPPORTED;
    if ((int64_t)nE * c->nk > INT32_MAX) return NEGF_ERR_ARG;  // jobs are indexed as int
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int njobs = nE * c->nk;
    if (precision == NEGF_MIXED) {
        // the mixed path schedules FP64 re-runs on the host: wait for the
        // caller's stream, run on the context's, hand the results back
        cudaStream_t cs = (cudaStream_t)stream;
        CK(cudaStreamSynchronize(cs));
        std::vector<double> E(nE), tj(njobs), tau(nE, 0.0);
        std::vector<int> info(njobs);
        CK(cudaMemcpy(E.data(), d_energies, sizeof(double) * nE, cudaMemcpyDeviceToHost));
        double ms = 0;
        int rc = negf_internal_mixed(c, E.data(), d_energies, nE, tj.data(), info.data(), &ms);
        if (rc < 0) return rc;
        for (int ik = 0; ik < c->nk; ++ik)
            for (int ie = 0; ie < nE; ++ie) tau[ie] += tj[(size_t)ik * nE + ie] * c->kpt[3 * ik + 2];
        CK(cudaMemcpyAsync(d_tau, tau.data(), sizeof(double) * nE, cudaMemcpyHostToDevice, cs));
        if (d_tau_jobs) CK(cudaMemcpyAsync(d_tau_jobs, tj.data(), sizeof(double) * njobs, cudaMemcpyHostToDevice, cs));
        if (d_info) CK(cudaMemcpyAsync(d_info, info.data(), sizeof(int) * njobs, cudaMemcpyHostToDevice, cs));
        CK(cudaStreamSynchronize(cs));
        return NEGF_OK;
    }
    int rc = ensure_jobs(c, 1, njobs);
    if (rc) return rc;
    double *tj = d_tau_jobs ? d_tau_jobs : c->d_tau_jobs;
    return transmission_launch(c, d_energies, nE, d_tau, tj, d_info, (cudaStream_t)stream);
}

int negf_transmission(negf_ctx *c, const double *energies, int32_t nE, int32_t precision, double *tau,
                      negf_stats *stats) {
    if (!c || !energies || !tau || nE < 1) return NEGF_ERR_ARG;
    if (precision != NEGF_FP64 && precision != NEGF_MIXED) return NEGF_ERR_UNSUPPORTED;
    if ((int64_t)nE * c->nk > INT32_MAX) return NEGF_ERR_ARG;  // jobs are indexed as int
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int njobs = nE * c->nk;
    int rc = ensure_jobs(c, nE, njobs);
    if (rc) return rc;
    if (precision == NEGF_MIXED) {
        CK(cudaMemcpyAsync(c->d_E, energies, sizeof(double) * nE, cudaMemcpyHostToDevice, c->stream));
        std::vector<double> tj(njobs);
        std::vector<int> info(njobs);
        double ms = 0;
        rc = negf_internal_mixed(c, energies, c->d_E, nE, tj.data(), info.data(), &ms);
        if (rc < 0) return rc;
        // tau(E) = sum_k w_k tau(E,k) in k order (negf.f90:172)
        for (int ie = 0; ie < nE; ++ie) tau[ie] = 0.0;
        for (int ik = 0; ik < c->nk; ++ik)
            for (int ie = 0; ie < nE; ++ie) tau[ie] += tj[(size_t)ik * nE + ie] * c->kpt[3 * ik + 2];
        fill_stats(stats, info, (float)ms);
        return first_info(info);
    }
    CK(cudaMemcpyAsync(c->d_E, energies, sizeof(double) * nE, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    rc = transmission_launch(c, c->d_E, nE, c->d_tau, c->d_tau_jobs, c->d_info, c->stream);
    if (rc) return rc;
    CK(cudaEventRecord(c->ev1, c->stream));
    std::vector<int> info(njobs);
    CK(cudaMemcpyAsync(tau, c->d_tau, sizeof(double) * nE, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(info.data(), c->d_info, sizeof(int) * njobs, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    fill_stats(stats, info, ms);
    return first_info(info);
}

int negf_set_variant(negf_ctx *c, int32_t variant) {
    if (!c || variant < -1 || variant > V8x1) return NEGF_ERR_ARG;
    if (variant >= 0 && !variant_fits(variant, c->N)) return NEGF_ERR_UNSUPPORTED;
    c->variant = variant;
    return NEGF_OK;
}

int negf_autotune(negf_ctx *c, const double *energies, int32_t nE, int32_t *chosen, double *rates) {
    if (!c || !energies || nE < 1) return NEGF_ERR_ARG;
    std::vector<double> tau(nE);
    double best = -1.0;
    int bv = -1;
    const int keep = c->variant;
    for (int v = V16x1; v <= V8x1; ++v) {
        if (rates) rates[v] = 0.0;
        if (!variant_fits(v, c->N)) continue;
        c->variant = v;
        negf_stats st{};
        int rc = negf_transmission(c, energies, nE, NEGF_FP64, tau.data(), &st);  // first use: set-up
        if (rc >= 0) rc = negf_transmission(c, energies, nE, NEGF_FP64, tau.data(), &st);
        if (rc < 0) { c->variant = keep; return rc; }
        const double r = st.device_ms > 0 ? (double)nE * c->nk / (st.device_ms * 1e-3) : 0.0;
        if (rates) rates[v] = r;
        if (r > best) { best = r; bv = v; }
    }
    c->variant = bv;
    if (chosen) *chosen = bv;
    return bv >= 0 ? NEGF_OK : NEGF_ERR_UNSUPPORTED;
}

int negf_density(negf_ctx *c, int32_t n_circle, int32_t n_line, double min_v, double mu, double gap,
                 double temperature, double *dm, negf_stats *stats) {
    if (!c || !dm || n_circle < 2 || n_line < 2) return NEGF_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    // contour of negf.f90:37-65 and weights of negf.f90:86-111
    const double circle_L = min_v - 1.0 / HARTREE, circle_R = mu - gap;
    const double line_L = mu - gap, line_R = mu + gap;
    const double E_c = (circle_R + circle_L) / 2, E_R = (circle_R - circle_L) / 2;
    const int n_int = n_circle + n_line, njobs = n_int * c->nk;
    auto simpson_c = [](int i, int n, double a, double b) {  // math_kernel.f90:167-204
        double cf;
        if (n % 2 == 1) {
            cf = (i == 1 || i == n) ? 1.0 / 3 : (i % 2 == 0 ? 4.0 / 3 : 2.0 / 3);
        } else if (i == 1) cf = 1.0 / 3;
        else if (i == n - 3) cf = 1.0 / 3 + 1.0 * 3 / 8;
        else if (i == n - 2 || i == n - 1) cf = 3.0 * 3 / 8;
        else if (i == n) cf = 1.0 * 3 / 8;
        else cf = (i % 2 == 0) ? 4.0 / 3 : 2.0 / 3;
        return cf * (b - a) / (n - 1);
    };
    auto simpson_x = [](int i, int n, double a, double b) { return (i - 1) * (b - a) / (n - 1) + a; };
    std::vector<RgfJob> jobs(njobs);
    std::vector<double2> coef(njobs);
    for (int job = 0; job < njobs; ++job) {
        const int i_int = 1 + job % n_int, ik = job / n_int;
        const double w = c->kpt[3 * ik + 2];
        RgfJob jb{};
        jb.ik = ik;
        double2 cf;
        if (i_int <= n_circle) {
            const double th = simpson_x(i_int, n_circle, 0.0, PI);
            const double ex = E_c + E_R * std::cos(th), ey = E_R * std::sin(th);
            jb.e_re = ex; jb.e_im = ey + c->eta; jb.e_t = ex;
            // w * 2/pi * c_i * i * E_R * exp(i theta)
            const double s = w * 2.0 / PI * simpson_c(i_int, n_circle, 0.0, PI);
            const double re = 0.0, im = s;  // s * i
            const double re2 = re * E_R, im2 = im * E_R;
            cf.x = re2 * std::cos(th) - im2 * std::sin(th);
            cf.y = re2 * std::sin(th) + im2 * std::cos(th);
        } else {
            const double ex = simpson_x(i_int - n_circle, n_line, line_L, line_R);
            jb.e_re = ex; jb.e_im = c->eta; jb.e_t = ex;
            const double f = 1.0 / (std::exp((ex - mu) / (K_B * temperature)) + 1);
            cf.x = -(w * 2.0 / PI * simpson_c(i_int - n_circle, n_line, line_L, line_R) * f);
            cf.y = 0.0;
        }
        jobs[job] = jb;
        coef[job] = cf;
    }
    const size_t per = (size_t)c->N * c->N * c->Nz;
    double2 *d_out = nullptr;
    if (cudaMalloc(&d_out, sizeof(double2) * per) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    std::vector<int> info;
    double ms = 0;
    int rc = diag_accumulate(c, jobs, coef, 0, d_out, info, ms);
    if (!rc) {
        cudaError_t e = cudaMemcpy(dm, d_out, sizeof(double2) * per, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = NEGF_ERR_CUDA;
    }
    cudaFree(d_out);
    if (rc) return rc;
    fill_stats(stats, info, ms);
    return first_info(info);
}

int negf_density_accumulate(negf_ctx *c, const double *energies, const double *weights, int32_t nE, double *dm,
                            negf_stats *stats) {
    if (!c || !energies || !weights || !dm || nE < 1) return NEGF_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int nk = c->nk;
    std::vector<RgfJob> jobs((size_t)nE * nk);
    std::vector<double2> coef((size_t)nE * nk);
    for (int ik = 0; ik < nk; ++ik) {
        const double wk = c->kpt[3 * ik + 2];
        for (int i = 0; i < nE; ++i) {
            RgfJob jb{};
            jb.e_re = energies[2 * i];
            jb.e_im = energies[2 * i + 1] + c->eta;  // + i*eta as negf.f90:77
            jb.e_t = jb.e_re;
            jb.ik = ik;
            jobs[(size_t)ik * nE + i] = jb;
            coef[(size_t)ik * nE + i] = make_double2(wk * weights[2 * i], wk * weights[2 * i + 1]);
        }
    }
    const size_t per = (size_t)c->N * c->N * c->Nz;
    double2 *d_out = nullptr;
    if (cudaMalloc(&d_out, sizeof(double2) * per) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    std::vector<int> info;
    double ms = 0;
    int rc = diag_accumulate(c, jobs, coef, 0, d_out, info, ms);
    if (!rc && cudaMemcpy(dm, d_out, sizeof(double2) * per, cudaMemcpyDeviceToHost) != cudaSuccess) rc = NEGF_ERR_CUDA;
    cudaFree(d_out);
    if (rc) return rc;
    fill_stats(stats, info, ms);
    return first_info(info);
}

int negf_density_neq(negf_ctx *c, int32_t n_circle, int32_t n_window, double min_v, double mu_L,
                     double mu_R, double gap, double temperature, double *dm, negf_stats *stats) {
    if (!c || !dm || n_circle < 1 || n_window < 1 || !(temperature > 0) || !(gap > 0)) return NEGF_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const double mu_lo = std::min(mu_L, mu_R), mu_hi = std::max(mu_L, mu_R);
    const bool right_injects = mu_R > mu_L;
    const double kT = K_B * temperature, dz = c->Lz / c->Nz;
    // semicircle from below the band bottom (negf.f90:37-41) to mu_lo - gap
    const double circle_L = min_v - 1.0 / HARTREE, circle_R = mu_lo - gap;
    if (!(circle_R > circle_L)) return NEGF_ERR_ARG;
    const double E_c = (circle_R + circle_L) / 2, E_R = (circle_R - circle_L) / 2;
    const double win_L = mu_lo - gap, win_R = mu_hi + gap;
    std::vector<double> xc, wc, xw, ww;
    gauss_legendre(n_circle, xc, wc);
    gauss_legendre(n_window, xw, ww);
    auto fermi = [kT](double e, double mu) { return 1.0 / (std::exp((e - mu) / kT) + 1.0); };
    // One job list (window nodes, then semicircle nodes, per k-point) so that both
    // kinds share the chunks the device memory allows and a short last chunk
    // holds the cheaper semicircle sweeps (no spectral term); every job carries
    // its own cd (and ca) and k_accumulate sums them with unit weight.
    const int nk = c->nk, per_k = n_circle + n_window;
    std::vector<RgfJob> jobs((size_t)per_k * nk);
    for (int ik = 0; ik < nk; ++ik) {
        const double w = c->kpt[3 * ik + 2];
        for (int i = 0; i < n_circle; ++i) {
            const double th = PI / 2 * (xc[i] + 1.0), cth = PI / 2 * wc[i];
            RgfJob jb{};
            jb.e_re = E_c + E_R * std::cos(th);
            jb.e_im = E_R * std::sin(th) + c->eta;
            jb.e_t = jb.e_re;
            jb.ik = ik;
            // w * 2/pi * c_theta * i * E_R * exp(i theta)
            const double sc = w * 2.0 / PI * cth * E_R;
            jb.cd_re = -sc * std::sin(th);
            jb.cd_im = sc * std::cos(th);
            jobs[(size_t)ik * per_k + n_window + i] = jb;
        }
        for (int i = 0; i < n_window; ++i) {
            const double x = (win_L + win_R) / 2 + (win_R - win_L) / 2 * xw[i];
            const double cx = (win_R - win_L) / 2 * ww[i];
            const double flo = fermi(x, mu_lo), fhi = fermi(x, mu_hi);
            RgfJob jb{};
            jb.e_re = x;
            jb.e_im = c->eta;
            jb.e_t = x;
            jb.ik = ik;
            jb.cd_re = -(w * 2.0 / PI * cx * flo);
            jb.ca_im = w / PI * cx * (fhi - flo) * (2.0 * dz * dz);
            jobs[(size_t)ik * per_k + i] = jb;
        }
    }
    const std::vector<double2> unit(jobs.size(), make_double2(1.0, 0.0));
    const size_t per = (size_t)c->N * c->N * c->Nz;
    double2 *d_out = nullptr;
    if (cudaMalloc(&d_out, sizeof(double2) * per) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    std::vector<int> info;
    double ms = 0;
    int rc = diag_accumulate(c, jobs, unit, 0, d_out, info, ms,
                             WANT_D | WANT_A | (right_injects ? WANT_MIRROR : 0));
    if (!rc && cudaMemcpy(dm, d_out, sizeof(double2) * per, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = NEGF_ERR_CUDA;
    cudaFree(d_out);
    if (rc) return rc;
    fill_stats(stats, info, ms);
    return first_info(info);
}

int negf_ldos_matrix(negf_ctx *c, double e_lo, double e_hi, int32_t n_e, int32_t i_e0, int32_t n_chunk,
                     double *ldos, negf_stats *stats) {
    if (!c || !ldos || n_e < 1 || i_e0 < 0 || n_chunk < 1 || i_e0 + n_chunk > n_e) return NEGF_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int nk = c->nk, njobs = n_chunk * nk;
    std::vector<RgfJob> jobs(njobs);
    std::vector<double2> coef(njobs);
    for (int o = 0; o < n_chunk; ++o) {
        // LDOS energy grid, negf.f90:203-204 (last point excluded)
        const int i_energy = i_e0 + o + 1;
        const double e = e_lo + (e_hi - e_lo) * (i_energy - 1) / n_e;
        for (int ik = 0; ik < nk; ++ik) {
            RgfJob jb{};
            jb.e_re = e; jb.e_im = c->eta; jb.e_t = e; jb.ik = ik;
            jobs[o * nk + ik] = jb;
            coef[o * nk + ik] = make_double2(-(c->kpt[3 * ik + 2] * 1.0 / PI), 0.0);  // negf.f90:230-231
        }
    }
    const size_t per = (size_t)c->N * c->N * c->Nz;
    double2 *d_out = nullptr;
    if (cudaMalloc(&d_out, sizeof(double2) * per * n_chunk) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    std::vector<int> info;
    double ms = 0;
    int rc = diag_accumulate(c, jobs, coef, nk, d_out, info, ms);
    if (!rc && cudaMemcpy(ldos, d_out, sizeof(double2) * per * n_chunk, cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = NEGF_ERR_CUDA;
    cudaFree(d_out);
    if (rc) return rc;
    fill_stats(stats, info, ms);
    return first_info(info);
}

int negf_tri_solve(negf_ctx *ctx, const double *D, int32_t N, int32_t Nz, const char *dfl, double *diag,
                   double *first, double *last) {
    if (!D || N < 1 || Nz < 2 || !dfl) return NEGF_ERR_ARG;
    if (pick_variant(N) == VNONE) return NEGF_ERR_UNSUPPORTED;
    const int dev = ctx ? ctx->device : 0;
    if (cudaSetDevice(dev) != cudaSuccess) return NEGF_ERR_CUDA;
    int want = 0;
    if (strpbrk(dfl, "Dd")) want |= WANT_D;
    if (strpbrk(dfl, "Ff")) want |= WANT_F;
    if (strpbrk(dfl, "Ll")) want |= WANT_L;
    const size_t per = (size_t)N * N * Nz;
    const size_t bytes = sizeof(double2) * per;
    // the reference zero-fills every plane (math_kernel.f90:75-77)
    if (diag) memset(diag, 0, bytes);
    if (first) memset(first, 0, bytes);
    if (last) memset(last, 0, bytes);
    negf_ctx local;
    negf_ctx *c = &local;
    c->device = dev;
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, dev);
    Geo g{};
    g.N = N; g.Nz = Nz; g.ld = round_up(N, 8);
    g.delta = 1.0; g.c2 = 1.0;
    g.lead_model = 0;
    double2 *d_D = nullptr, *d_slab = nullptr, *d_first = nullptr, *d_last = nullptr;
    int *d_nx = nullptr, *d_ny = nullptr, *d_info = nullptr;
    int rc = 0, hinfo = 0;
    const size_t sstride = (size_t)g.ld * N * Nz;
    cudaStream_t st = nullptr;
#define CKT(x) do { if ((x) != cudaSuccess) { rc = NEGF_ERR_CUDA; goto done; } } while (0)
    CKT(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CKT(cudaMalloc(&d_D, bytes));
    CKT(cudaMalloc(&d_slab, sizeof(double2) * sstride));
    CKT(cudaMalloc(&d_nx, sizeof(int) * N));
    CKT(cudaMalloc(&d_ny, sizeof(int) * N));
    CKT(cudaMalloc(&d_info, sizeof(int)));
    CKT(cudaMemset(d_nx, 0, sizeof(int) * N));
    CKT(cudaMemset(d_ny, 0, sizeof(int) * N));
    if ((want & WANT_F) && first) CKT(cudaMalloc(&d_first, bytes));
    if ((want & WANT_L) && last) CKT(cudaMalloc(&d_last, bytes));
    CKT(cudaMemcpy(d_D, D, bytes, cudaMemcpyHostToDevice));
    g.nx = d_nx; g.ny = d_ny;
    {
        RgfJob jb{};
        RgfJob *d_job = nullptr;
        int i2 = 0;
        CKT(cudaMalloc(&d_job, sizeof(RgfJob)));
        CKT(cudaMemcpy(d_job, &jb, sizeof(RgfJob), cudaMemcpyHostToDevice));
        // pass 1: generator_r sweep, diagonal and first-column blocks
        int w = want & (WANT_D | WANT_F);
        if (!diag) w &= ~WANT_D;
        if (!first) w &= ~WANT_F;
        if (w) {
            rc = slab_launch(c, g, d_job, 1, d_D, d_slab, sstride, w, d_first, nullptr, d_info, st);
            if (!rc && (cudaStreamSynchronize(st) != cudaSuccess ||
                        cudaMemcpy(&hinfo, d_info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess))
                rc = NEGF_ERR_CUDA;
            if (!rc && (w & WANT_D) &&
                cudaMemcpy2D(diag, sizeof(double2) * N, d_slab, sizeof(double2) * g.ld, sizeof(double2) * N,
                             (size_t)N * Nz, cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = NEGF_ERR_CUDA;
        }
        // pass 2: generator_l sweep and last-column blocks (reuses the slab)
        if (!rc && (want & WANT_L) && last) {
            rc = slab_launch(c, g, d_job, 1, d_D, d_slab, sstride, WANT_L, nullptr, d_last, d_info, st);
            if (!rc && (cudaStreamSynchronize(st) != cudaSuccess ||
                        cudaMemcpy(&i2, d_info, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess))
                rc = NEGF_ERR_CUDA;
            if (!hinfo) hinfo = i2;
        }
        cudaFree(d_job);
        if (rc) goto done;
    }
    if (d_first) CKT(cudaMemcpy(first, d_first, bytes, cudaMemcpyDeviceToHost));
    if (d_last) CKT(cudaMemcpy(last, d_last, bytes, cudaMemcpyDeviceToHost));
#undef CKT
done:
    cudaFree(d_D); cudaFree(d_slab); cudaFree(d_first); cudaFree(d_last);
    cudaFree(d_nx); cudaFree(d_ny); cudaFree(d_info);
    cudaFree(c->d_ws);
    c->d_ws = nullptr;
    if (st) cudaStreamDestroy(st);
    if (rc) return rc;
    return hinfo;
}

}  // extern "C"

// FP64 re-runs for the mixed path: the listed (energy, k-point) jobs of one
// context through the batch kernel.
int negf_internal_fp64_jobs(negf_ctx *c, const double *d_E, const int *ie, const int *ik, int njobs,
                            double *h_tau, int *h_info, float *ms) {
    *ms = 0.f;
    if (njobs <= 0) return 0;
    cudaStream_t st = c->stream;
    const Variant var = ctx_variant(c);
    if (var == VNONE) return NEGF_ERR_UNSUPPORTED;
    std::vector<BatchJob> jobs(njobs);
    for (int q = 0; q < njobs; ++q) jobs[q] = BatchJob{0, ie[q], ik[q], 0};
    const size_t smem = variant_smem(var, c->N);
    int occ = 1, rc = 0;
    switch (var) {
        case V16x1: rc = prep_kernel(k_transmission_batch<16, 1, 2>, smem, &occ); break;
        case V8x1: rc = prep_kernel(k_transmission_batch<8, 1, 2>, smem, &occ); break;
        case V16x2: rc = prep_kernel(k_transmission_batch<16, 2, 1>, smem, &occ); break;
        default: rc = prep_kernel(k_transmission_batch<8, 4, 1>, smem, &occ); break;
    }
    if (rc) return rc;
    const int grid = std::min(njobs, c->num_sms * occ);
    const size_t wstride = 4 * (size_t)c->ld * c->N;
    if ((rc = ensure_ws(c, sizeof(double2) * wstride * grid))) return rc;
    Geo g = make_geo(c);
    Geo *d_geo = nullptr;
    BatchJob *d_jobs = nullptr;
    double *d_tj = nullptr;
    int *d_info = nullptr, *d_counter = nullptr;
    if (cudaMalloc(&d_geo, sizeof(Geo)) != cudaSuccess || cudaMalloc(&d_jobs, sizeof(BatchJob) * njobs) != cudaSuccess ||
        cudaMalloc(&d_tj, sizeof(double) * njobs) != cudaSuccess || cudaMalloc(&d_info, sizeof(int) * njobs) != cudaSuccess ||
        cudaMalloc(&d_counter, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        rc = NEGF_ERR_NOMEM;
    }
    if (!rc && (cudaMemcpyAsync(d_geo, &g, sizeof(Geo), cudaMemcpyHostToDevice, st) ||
                cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(BatchJob) * njobs, cudaMemcpyHostToDevice, st) ||
                cudaMemsetAsync(d_counter, 0, sizeof(int), st) || cudaEventRecord(c->ev0, st)))
        rc = NEGF_ERR_CUDA;
    if (!rc) {
        double2 *ws = (double2 *)c->d_ws;
        switch (var) {
            case V16x1:
                k_transmission_batch<16, 1, 2><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                break;
            case V16x2:
                k_transmission_batch<16, 2, 1><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                break;
            case V8x1:
                k_transmission_batch<8, 1, 2><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                break;
            default:
                k_transmission_batch<8, 4, 1><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                break;
        }
        if (cudaGetLastError() || cudaEventRecord(c->ev1, st) ||
            cudaMemcpyAsync(h_tau, d_tj, sizeof(double) * njobs, cudaMemcpyDeviceToHost, st) ||
            cudaMemcpyAsync(h_info, d_info, sizeof(int) * njobs, cudaMemcpyDeviceToHost, st) ||
            cudaStreamSynchronize(st) || cudaEventElapsedTime(ms, c->ev0, c->ev1))
            rc = NEGF_ERR_CUDA;
    }
    cudaFree(d_geo); cudaFree(d_jobs); cudaFree(d_tj); cudaFree(d_info); cudaFree(d_counter);
    return rc;
}

extern "C" int negf_set_mixed_policy(negf_ctx *c, const negf_mixed_policy *p) {
    if (!c || !p || !(p->threshold_window >= 0) || !(p->eta_fp64_below >= 0) || !(p->tau_tolerance > 0) ||
        p->max_refinements < 1 || p->max_refinements > 16 || p->ctas_per_job < 0 || p->ctas_per_job > 2)
        return NEGF_ERR_ARG;
    c->mixed_policy = *p;
    return NEGF_OK;
}
extern "C" int negf_get_mixed_policy(const negf_ctx *c, negf_mixed_policy *p) {
    if (!c || !p) return NEGF_ERR_ARG;
    *p = c->mixed_policy;
    return NEGF_OK;
}
extern "C" int negf_get_mixed_stats(const negf_ctx *c, negf_mixed_stats *s) {
    if (!c || !s) return NEGF_ERR_ARG;
    *s = c->mixed_stats;
    return NEGF_OK;
}

// ------------------------------------------------------ batches of problems
extern "C" int negf_transmission_batch(negf_ctx *const *ctxs, int32_t nctx, const double *energies, int32_t nE,
                                       double *tau, negf_stats *stats) {
    if (!ctxs || nctx < 1 || !energies || !tau || nE < 1) return NEGF_ERR_ARG;
    for (int p = 0; p < nctx; ++p)
        if (!ctxs[p] || ctxs[p]->device != ctxs[0]->device) return NEGF_ERR_ARG;
    negf_ctx *c0 = ctxs[0];
    if (cudaSetDevice(c0->device) != cudaSuccess) return NEGF_ERR_CUDA;
    cudaStream_t st = c0->stream;
    std::fill(tau, tau + (size_t)nctx * nE, 0.0);
    double *d_E = nullptr;
    if (cudaMalloc(&d_E, sizeof(double) * nE) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    if (cudaMemcpyAsync(d_E, energies, sizeof(double) * nE, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        cudaFree(d_E);
        return NEGF_ERR_CUDA;
    }
    std::vector<int> info_all;
    double ms_all = 0;
    int rc = 0;
    for (int v = V16x1; v <= V8x1 && !rc; ++v) {
        std::vector<int> members;
        for (int p = 0; p < nctx; ++p)
            if (ctx_variant(ctxs[p]) == v) members.push_back(p);
        if (members.empty()) continue;
        std::vector<Geo> geos;
        std::vector<BatchJob> jobs;
        std::vector<double> cost;
        int nmax = 0;
        for (int m = 0; m < (int)members.size(); ++m) {
            negf_ctx *c = ctxs[members[m]];
            geos.push_back(make_geo(c));
            nmax = std::max(nmax, c->N);
            for (int ik = 0; ik < c->nk; ++ik)
                for (int ie = 0; ie < nE; ++ie) {
                    jobs.push_back(BatchJob{m, ie, ik, 0});
                    cost.push_back((double)c->N * c->N * c->N * c->Nz);
                }
        }
        // largest sweeps first, so the last wave holds the short ones
        std::vector<int> order(jobs.size());
        for (size_t q = 0; q < order.size(); ++q) order[q] = (int)q;
        std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        std::vector<BatchJob> sorted(jobs.size());
        for (size_t q = 0; q < order.size(); ++q) sorted[q] = jobs[order[q]];
        const int njobs = (int)sorted.size();
        const Variant var = (Variant)v;
        const size_t smem = variant_smem(var, nmax);
        int occ = 1;
        switch (var) {
            case V16x1: rc = prep_kernel(k_transmission_batch<16, 1, 2>, smem, &occ); break;
            case V8x1: rc = prep_kernel(k_transmission_batch<8, 1, 2>, smem, &occ); break;
            case V16x2: rc = prep_kernel(k_transmission_batch<16, 2, 1>, smem, &occ); break;
            default: rc = prep_kernel(k_transmission_batch<8, 4, 1>, smem, &occ); break;
        }
        if (rc) break;
        const int grid = std::min(njobs, c0->num_sms * occ);
        const size_t wstride = 4 * (size_t)round_up(nmax, 8) * nmax;
        if ((rc = ensure_ws(c0, sizeof(double2) * wstride * grid))) break;
        Geo *d_geo = nullptr;
        BatchJob *d_jobs = nullptr;
        double *d_tj = nullptr;
        int *d_info = nullptr, *d_counter = nullptr;
        if (cudaMalloc(&d_geo, sizeof(Geo) * geos.size()) != cudaSuccess ||
            cudaMalloc(&d_jobs, sizeof(BatchJob) * njobs) != cudaSuccess ||
            cudaMalloc(&d_tj, sizeof(double) * njobs) != cudaSuccess ||
            cudaMalloc(&d_info, sizeof(int) * njobs) != cudaSuccess ||
            cudaMalloc(&d_counter, sizeof(int)) != cudaSuccess) {
            cudaGetLastError();
            rc = NEGF_ERR_NOMEM;
        }
        std::vector<double> tj(njobs);
        std::vector<int> info(njobs);
        float ms = 0.f;
        if (!rc) {
            if (cudaMemcpyAsync(d_geo, geos.data(), sizeof(Geo) * geos.size(), cudaMemcpyHostToDevice, st) ||
                cudaMemcpyAsync(d_jobs, sorted.data(), sizeof(BatchJob) * njobs, cudaMemcpyHostToDevice, st) ||
                cudaMemsetAsync(d_counter, 0, sizeof(int), st) || cudaEventRecord(c0->ev0, st))
                rc = NEGF_ERR_CUDA;
        }
        if (!rc) {
            double2 *ws = (double2 *)c0->d_ws;
            switch (var) {
                case V16x1:
                    k_transmission_batch<16, 1, 2><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                    break;
                case V16x2:
                    k_transmission_batch<16, 2, 1><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                    break;
                case V8x1:
                    k_transmission_batch<8, 1, 2><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                    break;
                default:
                    k_transmission_batch<8, 4, 1><<<grid, NT, smem, st>>>(d_geo, d_jobs, njobs, d_E, ws, wstride, d_tj, d_info, d_counter);
                    break;
            }
            if (cudaGetLastError() || cudaEventRecord(c0->ev1, st) ||
                cudaMemcpyAsync(tj.data(), d_tj, sizeof(double) * njobs, cudaMemcpyDeviceToHost, st) ||
                cudaMemcpyAsync(info.data(), d_info, sizeof(int) * njobs, cudaMemcpyDeviceToHost, st) ||
                cudaStreamSynchronize(st) || cudaEventElapsedTime(&ms, c0->ev0, c0->ev1))
                rc = NEGF_ERR_CUDA;
        }
        cudaFree(d_geo); cudaFree(d_jobs); cudaFree(d_tj); cudaFree(d_info); cudaFree(d_counter);
        if (rc) break;
        ms_all += ms;
        // tau[p][e] = sum_k w_k tau(p, e, k), summed in k order (negf.f90:172)
        std::vector<double> per(jobs.size());
        for (size_t q = 0; q < order.size(); ++q) per[order[q]] = tj[q];
        size_t q = 0;
        for (int m = 0; m < (int)members.size(); ++m) {
            negf_ctx *c = ctxs[members[m]];
            const int pg = members[m];
            for (int ik = 0; ik < c->nk; ++ik)
                for (int ie = 0; ie < nE; ++ie, ++q) tau[(size_t)pg * nE + ie] += per[q] * c->kpt[3 * ik + 2];
        }
        for (size_t qq = 0; qq < order.size(); ++qq) info_all.push_back(info[qq]);
    }
    cudaFree(d_E);
    if (rc) return rc;
    fill_stats(stats, info_all, ms_all);
    return first_info(info_all);
}

// ------------------------------------------------------ real-space outputs
namespace {
int basis_extent(const negf_ctx *c, int *mx, int *my) {
    std::vector<int> nx(c->N), ny(c->N);
    if (cudaMemcpy(nx.data(), c->d_nx, sizeof(int) * c->N, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(ny.data(), c->d_ny, sizeof(int) * c->N, cudaMemcpyDeviceToHost) != cudaSuccess)
        return NEGF_ERR_CUDA;
    *mx = *my = 0;
    for (int a = 0; a < c->N; ++a) {
        *mx = std::max(*mx, std::abs(nx[a]));
        *my = std::max(*my, std::abs(ny[a]));
    }
    return 0;
}

int launch_ptor(negf_ctx *c, const double2 *d_G, int nslices, int Nx, int Ny, double scale, double *d_dens,
                double2 *d_cdiag, cudaStream_t st, int ldg = 0, size_t gstride = 0) {
    int mx, my;
    int rc = basis_extent(c, &mx, &my);
    if (rc) return rc;
    if (2 * mx >= Nx || 2 * my >= Ny) return NEGF_ERR_ARG;  // index nx+Nx/2 must fit (grid.f90:92-94)
    const size_t smem = ptor_smem(mx, my, Nx, Ny);
    if (smem > 200 * 1024) return NEGF_ERR_UNSUPPORTED;
    CK(cudaFuncSetAttribute(k_ptor, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_ptor<<<nslices, PT_THREADS, smem, st>>>(d_G, c->N, ldg ? ldg : c->N, gstride ? gstride : (size_t)c->N * c->N,
                                              c->d_nx, c->d_ny, mx, my, Nx, Ny, scale, d_dens, d_cdiag);
    CK(cudaGetLastError());
    return 0;
}
}  // namespace

extern "C" int negf_density_real(negf_ctx *c, int32_t n_circle, int32_t n_line, double min_v, double mu,
                                 double gap, double temperature, int32_t Nx, int32_t Ny, double scale,
                                 double *density, double *dm, negf_stats *stats) {
    if (!c || !density || Nx < 1 || Ny < 1) return NEGF_ERR_ARG;
    const size_t per = (size_t)c->N * c->N * c->Nz;
    std::vector<double> host_dm;
    double *dmh = dm;
    if (!dmh) { host_dm.resize(2 * per); dmh = host_dm.data(); }
    int rc = negf_density(c, n_circle, n_line, min_v, mu, gap, temperature, dmh, stats);
    if (rc < 0) return rc;
    const int info = rc;
    double2 *d_G = nullptr;
    double *d_dens = nullptr;
    const size_t nd = (size_t)Nx * Ny * c->Nz;
    if (cudaMalloc(&d_G, sizeof(double2) * per) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    if (cudaMalloc(&d_dens, sizeof(double) * nd) != cudaSuccess) { cudaGetLastError(); cudaFree(d_G); return NEGF_ERR_NOMEM; }
    rc = 0;
    if (cudaMemcpyAsync(d_G, dmh, sizeof(double2) * per, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) rc = NEGF_ERR_CUDA;
    if (!rc) rc = launch_ptor(c, d_G, c->Nz, Nx, Ny, scale, d_dens, nullptr, c->stream);
    if (!rc && (cudaMemcpyAsync(density, d_dens, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess))
        rc = NEGF_ERR_CUDA;
    cudaFree(d_G);
    cudaFree(d_dens);
    return rc ? rc : info;
}

extern "C" int negf_vhat_gpu(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx, int32_t ngy,
                             int32_t device, double *vhat) {
    if (!vreal || !vhat || Nx < 1 || Ny < 1 || Nz < 1 || ngx < 0 || ngy < 0) return NEGF_ERR_ARG;
    if (2 * ngx > Nx || 2 * ngy > Ny) return NEGF_ERR_ARG;  // grid.f90:33-37
    if (cudaSetDevice(device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int W = 2 * ngx + 1, H = 2 * ngy + 1, hx = ngx / 2;
    const size_t smem = sizeof(double) * (size_t)Nx * Ny + sizeof(double2) * (size_t)(hx + 1) * Ny;
    if (smem > 200 * 1024) return NEGF_ERR_UNSUPPORTED;
    std::vector<double2> tx(Nx), ty(Ny);  // e^{-2 pi i m/N}, as the host transform
    for (int m = 0; m < Nx; ++m) { const double a = -2.0 * PI * (double)m / Nx; tx[m] = make_double2(std::cos(a), std::sin(a)); }
    for (int m = 0; m < Ny; ++m) { const double a = -2.0 * PI * (double)m / Ny; ty[m] = make_double2(std::cos(a), std::sin(a)); }
    const size_t nv = (size_t)Nx * Ny * Nz, nh = (size_t)W * H * Nz;
    double *d_v = nullptr;
    double2 *d_t = nullptr, *d_h = nullptr;
    cudaStream_t st = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_v, sizeof(double) * nv) != cudaSuccess || cudaMalloc(&d_t, sizeof(double2) * (Nx + Ny)) != cudaSuccess ||
        cudaMalloc(&d_h, sizeof(double2) * nh) != cudaSuccess) {
        cudaGetLastError();
        rc = NEGF_ERR_NOMEM;
    }
    if (!rc && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) rc = NEGF_ERR_CUDA;
    if (!rc && (cudaMemcpyAsync(d_v, vreal, sizeof(double) * nv, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(d_t, tx.data(), sizeof(double2) * Nx, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaMemcpyAsync(d_t + Nx, ty.data(), sizeof(double2) * Ny, cudaMemcpyHostToDevice, st) != cudaSuccess ||
                cudaFuncSetAttribute(k_vhat, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess))
        rc = NEGF_ERR_CUDA;
    if (!rc) {
        k_vhat<<<Nz, VH_THREADS, smem, st>>>(d_v, Nx, Ny, ngx, ngy, d_t, d_t + Nx, d_h);
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(vhat, d_h, sizeof(double2) * nh, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            rc = NEGF_ERR_CUDA;
    }
    if (st) cudaStreamDestroy(st);
    cudaFree(d_v);
    cudaFree(d_t);
    cudaFree(d_h);
    return rc;
}

extern "C" int negf_dm_real(negf_ctx *c, const double *dm, int32_t Nx, int32_t Ny, double scale,
                            double *density) {
    if (!c) return NEGF_ERR_ARG;
    return negf_dm_real_slab(c, dm, c->Nz, Nx, Ny, scale, density);
}

extern "C" int negf_dm_real_slab(negf_ctx *c, const double *dm, int32_t nslices, int32_t Nx, int32_t Ny,
                                 double scale, double *density) {
    if (!c || !dm || !density || Nx < 1 || Ny < 1 || nslices < 1) return NEGF_ERR_ARG;
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const size_t per = (size_t)c->N * c->N * nslices, nd = (size_t)Nx * Ny * nslices;
    double2 *d_G = nullptr;
    double *d_dens = nullptr;
    if (cudaMalloc(&d_G, sizeof(double2) * per) != cudaSuccess) { cudaGetLastError(); return NEGF_ERR_NOMEM; }
    if (cudaMalloc(&d_dens, sizeof(double) * nd) != cudaSuccess) { cudaGetLastError(); cudaFree(d_G); return NEGF_ERR_NOMEM; }
    int rc = 0;
    if (cudaMemcpyAsync(d_G, dm, sizeof(double2) * per, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) rc = NEGF_ERR_CUDA;
    if (!rc) rc = launch_ptor(c, d_G, nslices, Nx, Ny, scale, d_dens, nullptr, c->stream);
    if (!rc && (cudaMemcpyAsync(density, d_dens, sizeof(double) * nd, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess))
        rc = NEGF_ERR_CUDA;
    cudaFree(d_G);
    cudaFree(d_dens);
    return rc;
}

namespace {
// negf_ldos with a single k-point: the LDOS_Matrix of an energy is then one
// job's G_kk times -(w/pi) 2 dz^2, so the slabs go to PtoR directly and no
// (N,N,Nz) matrix per energy is held: as many energies run at once as the
// slabs allow.
int ldos_one_kpoint(negf_ctx *c, double e_lo, double e_hi, int n_e, const int32_t *ldos_grid, int Nx, int Ny,
                    const double *dxyz, double scale, double *ldos, negf_stats *stats) {
    const int N = c->N, Nz = c->Nz, ld = c->ld;
    const int Mx = ldos_grid[0] == 0 ? Nx : 1, My = ldos_grid[1] == 0 ? Ny : 1, Mz = ldos_grid[2] == 0 ? Nz : 1;
    const size_t nreal = (size_t)Nx * Ny * Nz, nout = (size_t)Mx * My * Mz;
    const size_t sstride = (size_t)ld * N * Nz;
    const size_t per_job = sizeof(double2) * (sstride + 6 * (size_t)ld * N + nreal);
    const int b = slab_jobs_in_flight(c, per_job, n_e);
    if (b < 1) return NEGF_ERR_NOMEM;
    double2 *d_slabs = nullptr, *d_diag = nullptr;
    double *d_out = nullptr;
    RgfJob *d_jobs = nullptr;
    int *d_info = nullptr;
    int rc = 0;
    if (cudaMalloc(&d_slabs, sizeof(double2) * sstride * b) != cudaSuccess ||
        cudaMalloc(&d_diag, sizeof(double2) * nreal * b) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(double) * nout * n_e) != cudaSuccess ||
        cudaMalloc(&d_jobs, sizeof(RgfJob) * b) != cudaSuccess || cudaMalloc(&d_info, sizeof(int) * b) != cudaSuccess) {
        cudaGetLastError();
        rc = NEGF_ERR_NOMEM;
    }
    const double f = -(c->kpt[2] / PI) * 2.0 * (c->Lz / Nz) * (c->Lz / Nz);  // negf.f90:230-231, :78
    std::vector<int> info_all(n_e, 0);
    double ms_all = 0;
    Geo g = make_geo(c);
    if (!rc && cudaMemsetAsync(d_out, 0, sizeof(double) * nout * n_e, c->stream) != cudaSuccess) rc = NEGF_ERR_CUDA;
    for (int e0 = 0; e0 < n_e && !rc; e0 += b) {
        const int nb = std::min(b, n_e - e0);
        std::vector<RgfJob> jobs(nb);
        for (int o = 0; o < nb; ++o) {
            const double e = e_lo + (e_hi - e_lo) * (e0 + o) / n_e;  // negf.f90:203-204
            RgfJob jb{};
            jb.e_re = e; jb.e_im = c->eta; jb.e_t = e; jb.ik = 0;
            jobs[o] = jb;
        }
        if (cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(RgfJob) * nb, cudaMemcpyHostToDevice, c->stream) ||
            cudaEventRecord(c->ev0, c->stream)) { rc = NEGF_ERR_CUDA; break; }
        if ((rc = slab_launch(c, g, d_jobs, nb, nullptr, d_slabs, sstride, WANT_D, nullptr, nullptr, d_info, c->stream)))
            break;
        float ms = 0.f;
        if (cudaEventRecord(c->ev1, c->stream) ||
            cudaMemcpyAsync(info_all.data() + e0, d_info, sizeof(int) * nb, cudaMemcpyDeviceToHost, c->stream)) {
            rc = NEGF_ERR_CUDA;
            break;
        }
        if ((rc = launch_ptor(c, d_slabs, nb * Nz, Nx, Ny, 1.0, nullptr, d_diag, c->stream, ld, (size_t)ld * N)))
            break;
        for (int o = 0; o < nb && !rc; ++o) {
            const int blocks = (int)std::min<size_t>((nreal + 255) / 256, (size_t)c->num_sms * 8);
            k_ldos_convert<<<blocks, 256, 0, c->stream>>>(d_diag + nreal * o, Nx, Ny, Nz, ldos_grid[0], ldos_grid[1],
                                                         ldos_grid[2], dxyz[0], dxyz[1], dxyz[2], scale * f, Mx, My,
                                                         d_out + nout * (e0 + o));
            if (cudaGetLastError() != cudaSuccess) rc = NEGF_ERR_CUDA;
        }
        if (!rc && (cudaStreamSynchronize(c->stream) != cudaSuccess || cudaEventElapsedTime(&ms, c->ev0, c->ev1)))
            rc = NEGF_ERR_CUDA;
        ms_all += ms;
    }
    if (!rc && (cudaMemcpyAsync(ldos, d_out, sizeof(double) * nout * n_e, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess))
        rc = NEGF_ERR_CUDA;
    cudaFree(d_slabs); cudaFree(d_diag); cudaFree(d_out); cudaFree(d_jobs); cudaFree(d_info);
    if (rc) return rc;
    fill_stats(stats, info_all, ms_all);
    return first_info(info_all);
}
}  // namespace

extern "C" int negf_ldos(negf_ctx *c, double e_lo, double e_hi, int32_t n_e, const int32_t *ldos_grid,
                         int32_t Nx, int32_t Ny, const double *dxyz, double scale, double *ldos,
                         negf_stats *stats) {
    if (!c || !ldos || !ldos_grid || !dxyz || n_e < 1 || Nx < 1 || Ny < 1) return NEGF_ERR_ARG;
    for (int a = 0; a < 3; ++a)
        if (ldos_grid[a] < -1) return NEGF_ERR_ARG;  // main.f90:125-128
    if (cudaSetDevice(c->device) != cudaSuccess) return NEGF_ERR_CUDA;
    const int Nz = c->Nz, nk = c->nk;
    const int Mx = ldos_grid[0] == 0 ? Nx : 1, My = ldos_grid[1] == 0 ? Ny : 1, Mz = ldos_grid[2] == 0 ? Nz : 1;
    const size_t per = (size_t)c->N * c->N * Nz, nreal = (size_t)Nx * Ny * Nz, nout = (size_t)Mx * My * Mz;
    if (nk == 1) return ldos_one_kpoint(c, e_lo, e_hi, n_e, ldos_grid, Nx, Ny, dxyz, scale, ldos, stats);
    // energies per chunk: LDOS matrices and their real-space diagonals resident at once
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t per_e = sizeof(double2) * (per + nreal);
    int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n_e, (free_b / 4) / std::max<size_t>(per_e, 1)));
    double2 *d_mat = nullptr, *d_diag = nullptr;
    double *d_out = nullptr;
    if (cudaMalloc(&d_mat, sizeof(double2) * per * chunk) != cudaSuccess ||
        cudaMalloc(&d_diag, sizeof(double2) * nreal * chunk) != cudaSuccess ||
        cudaMalloc(&d_out, sizeof(double) * nout * n_e) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_mat); cudaFree(d_diag);
        return NEGF_ERR_NOMEM;
    }
    int rc = cudaMemsetAsync(d_out, 0, sizeof(double) * nout * n_e, c->stream) == cudaSuccess ? 0 : NEGF_ERR_CUDA;
    std::vector<int> info_all;
    double ms_all = 0;
    for (int e0 = 0; e0 < n_e && !rc; e0 += chunk) {
        const int nc = std::min(chunk, n_e - e0);
        std::vector<RgfJob> jobs(nc * nk);
        std::vector<double2> coef(nc * nk);
        for (int o = 0; o < nc; ++o) {
            const int i_energy = e0 + o + 1;  // negf.f90:203-204
            const double e = e_lo + (e_hi - e_lo) * (i_energy - 1) / n_e;
            for (int ik = 0; ik < nk; ++ik) {
                RgfJob jb{};
                jb.e_re = e; jb.e_im = c->eta; jb.e_t = e; jb.ik = ik;
                jobs[o * nk + ik] = jb;
                coef[o * nk + ik] = make_double2(-(c->kpt[3 * ik + 2] * 1.0 / PI), 0.0);
            }
        }
        std::vector<int> info;
        double ms = 0;
        rc = diag_accumulate(c, jobs, coef, nk, d_mat, info, ms);
        if (rc) break;
        info_all.insert(info_all.end(), info.begin(), info.end());
        ms_all += ms;
        rc = launch_ptor(c, d_mat, nc * Nz, Nx, Ny, 1.0, nullptr, d_diag, c->stream);
        for (int o = 0; o < nc && !rc; ++o) {
            const int blocks = (int)std::min<size_t>((nreal + 255) / 256, (size_t)c->num_sms * 8);
            k_ldos_convert<<<blocks, 256, 0, c->stream>>>(d_diag + nreal * o, Nx, Ny, Nz, ldos_grid[0], ldos_grid[1],
                                                         ldos_grid[2], dxyz[0], dxyz[1], dxyz[2], scale, Mx, My,
                                                         d_out + nout * (e0 + o));
            if (cudaGetLastError() != cudaSuccess) rc = NEGF_ERR_CUDA;
        }
    }
    if (!rc && (cudaMemcpyAsync(ldos, d_out, sizeof(double) * nout * n_e, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
                cudaStreamSynchronize(c->stream) != cudaSuccess))
        rc = NEGF_ERR_CUDA;
    cudaFree(d_mat); cudaFree(d_diag); cudaFree(d_out);
    if (rc) return rc;
    fill_stats(stats, info_all, ms_all);
    return first_info(info_all);
}

// ============================================================ no-alloc entry
// negf_transmission_noalloc: the transmission sweep for callers that cannot
// allocate device memory (code running inside another framework's memory
// pool or allocator, or with a fixed memory budget checked at start-up).
// Its scratch is this file-scope array, reserved on every GPU that loads
// the library for as long as the process lives.
static constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)64 << 20;  // 64 MiB
static __device__ __align__(256) double2 g_noalloc_scratch[NOALLOC_SCRATCH_BYTES / sizeof(double2)];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
double2 *g_noalloc_base[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(int dev, double2 **out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return NEGF_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return NEGF_ERR_CUDA;
        }
        g_noalloc_base[dev] = (double2 *)p;
    }
    *out = g_noalloc_base[dev];
    return 0;
}

// ax, ay and the weights of grid.f90:258 / global k-points, into the scratch.
__global__ void k_noalloc_kvectors(const int *__restrict__ nx, const int *__restrict__ ny,
                                   const double *__restrict__ kpt, int N, int nk, double Lx, double Ly,
                                   double *ax, double *ay, double *kw) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nk) kw[t] = kpt[3 * t + 2];
    if (t >= N * nk) return;
    const int k = t / N, i = t - k * N;
    ax[t] = (double)(2 * nx[i]) * PI / Lx + kpt[3 * k];
    ay[t] = (double)(2 * ny[i]) * PI / Ly + kpt[3 * k + 1];
}

// flag = 1 if some pair difference n_i - n_j falls outside the V table.
__global__ void k_noalloc_check(const int *__restrict__ nx, const int *__restrict__ ny, int N, int ngx,
                                int ngy, int *flag) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N * N; t += gridDim.x * blockDim.x) {
        const int i = t % N, j = t / N;
        const int dx = nx[i] - nx[j], dy = ny[i] - ny[j];
        if (dx < -ngx || dx > ngx || dy < -ngy || dy > ngy) *flag = 1;
    }
}
}  // namespace

extern "C" int negf_transmission_noalloc(int32_t N, int32_t Nz, int32_t ngx, int32_t ngy,
                                         const int32_t *d_nx, const int32_t *d_ny, const double *d_vhat,
                                         double Lx, double Ly, double Lz, double V_L, double V_R,
                                         double eta, int32_t nk, const double *d_kpt,
                                         const double *d_energies, int32_t nE, double *d_tau,
                                         int32_t *d_info, void *stream) {
    if (N < 1 || Nz < 2 || ngx < 0 || ngy < 0 || nk < 1 || nE < 1 || !d_nx || !d_ny || !d_vhat ||
        !d_kpt || !d_energies || !d_tau || !(Lx > 0) || !(Ly > 0) || !(Lz > 0))
        return NEGF_ERR_ARG;
    const Variant v = transmission_variant(N);
    if (v == VNONE) return NEGF_ERR_UNSUPPORTED;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NEGF_ERR_CUDA;

    // scratch layout: [flag | ax | ay | kw | tau_jobs] then one workspace per CTA
    const int ld = round_up(N, 8);
    const size_t njobs = (size_t)nE * nk;
    if (njobs > (size_t)INT32_MAX) return NEGF_ERR_ARG;  // the kernels index jobs as int
    const size_t head_doubles = 2 + 2 * (size_t)nk * N + nk + njobs;
    const size_t head_bytes = (head_doubles * sizeof(double) + 255) / 256 * 256;
    const size_t wstride = 4 * (size_t)ld * N;  // double2 per CTA
    if (head_bytes + wstride * sizeof(double2) > NOALLOC_SCRATCH_BYTES) return NEGF_ERR_TOO_LARGE;
    const size_t cap = (NOALLOC_SCRATCH_BYTES - head_bytes) / (wstride * sizeof(double2));

    double2 *base = nullptr;
    int rc = noalloc_scratch(dev, &base);
    if (rc) return rc;
    double *head = (double *)base;
    int *flag = (int *)head;
    double *ax = head + 2, *ay = ax + (size_t)nk * N, *kw = ay + (size_t)nk * N;
    double *tau_jobs = kw + nk;
    double2 *ws = (double2 *)((unsigned char *)base + head_bytes);

    // the pair differences must index inside the V table (the scratch keeps
    // the last call's contents, so the flag is cleared first)
    int hflag = 0;
    CK(cudaMemsetAsync(flag, 0, sizeof(int), st));
    k_noalloc_check<<<64, 256, 0, st>>>(d_nx, d_ny, N, ngx, ngy, flag);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hflag) return NEGF_ERR_ARG;

    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const size_t smem = variant_smem(v, N);
    int occ = 1;
    switch (v) {
        case V16x1: rc = prep_kernel(k_transmission<16, 1, 2>, smem, &occ); break;
        case V16x2: rc = prep_kernel(k_transmission<16, 2, 1>, smem, &occ); break;
        case V8x1: rc = prep_kernel(k_transmission<8, 1, 2>, smem, &occ); break;
        default: rc = prep_kernel(k_transmission<8, 4, 1>, smem, &occ); break;
    }
    if (rc) return rc;
    const int grid = (int)std::min<size_t>(std::min<size_t>(njobs, (size_t)sms * occ), cap);

    const int nkv = std::max(N * nk, nk);
    k_noalloc_kvectors<<<(nkv + 255) / 256, 256, 0, st>>>(d_nx, d_ny, d_kpt, N, nk, Lx, Ly, ax, ay, kw);
    CK(cudaGetLastError());
    Geo g;
    g.N = N; g.Nz = Nz; g.ld = ld;
    g.ngx = ngx; g.ngy = ngy; g.W = 2 * ngx + 1; g.H = 2 * ngy + 1;
    g.nk = nk;
    g.vhat = (const double2 *)d_vhat; g.nx = d_nx; g.ny = d_ny;
    g.ax = ax; g.ay = ay; g.kw = kw;
    g.delta = Lz / Nz;
    g.c2 = 2 * (g.delta * g.delta);
    g.V_L = V_L; g.V_R = V_R; g.eta = eta;
    g.lead_model = 0;
    switch (v) {
        case V16x1:
            k_transmission<16, 1, 2><<<grid, NT, smem, st>>>(g, d_energies, nE, (int)njobs, ws, wstride, tau_jobs, d_info);
            break;
        case V16x2:
            k_transmission<16, 2, 1><<<grid, NT, smem, st>>>(g, d_energies, nE, (int)njobs, ws, wstride, tau_jobs, d_info);
            break;
        case V8x1:
            k_transmission<8, 1, 2><<<grid, NT, smem, st>>>(g, d_energies, nE, (int)njobs, ws, wstride, tau_jobs, d_info);
            break;
        default:
            k_transmission<8, 4, 1><<<grid, NT, smem, st>>>(g, d_energies, nE, (int)njobs, ws, wstride, tau_jobs, d_info);
            break;
    }
    CK(cudaGetLastError());
    k_tau_reduce<<<(nE + 127) / 128, 128, 0, st>>>(tau_jobs, kw, nE, nk, d_tau);
    CK(cudaGetLastError());
    return NEGF_OK;
}
