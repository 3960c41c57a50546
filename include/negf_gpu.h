/*
 * negf_gpu.h -- C ABI of the B200 NEGF engine (libnegfgpu.so).
 *
 * Drop-in for the hot path of NEGFtrans: src/negf.f90 (the per-job drivers)
 * and src/math_kernel.f90 (the RGF solver), called from Fortran through
 * iso_c_binding or from C/C++/Python directly.
 *
 * Conventions
 *  - Plain C types only.  Complex numbers are interleaved (re, im) doubles,
 *    the memory layout of Fortran complex*16 and C double _Complex.
 *  - Arrays are column-major (Fortran order): element (i,j,k) of an
 *    (N,N,Nz) array is at i + N*j + N*N*k, 0-based.  No copies are needed on
 *    the Fortran side.
 *  - Units are the reference's "atomic" units after main.f90:184-205:
 *    energies and potentials in Hartree, lengths in bohr.
 *  - Every entry returns an int status: 0 = NEGF_OK, < 0 = an argument or
 *    CUDA error (never exit()); > 0 = LAPACK-style singular pivot, i.e. a
 *    block had a zero pivot (the 1-based column), results of that job are not
 *    trusted.  The reference ignores INFO (math_kernel.f90:31-32); this
 *    library reports it.
 *  - Ownership: the caller owns every host buffer; a context owns its device
 *    buffers.  One context per host thread; different contexts may be used
 *    concurrently.  Host-pointer entries are synchronous.
 */
#ifndef NEGF_GPU_H
#define NEGF_GPU_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NEGF_OK 0
#define NEGF_ERR_ARG (-1)
#define NEGF_ERR_CUDA (-2)
#define NEGF_ERR_NOMEM (-3)
#define NEGF_ERR_UNSUPPORTED (-4)
#define NEGF_ERR_TOO_LARGE (-5) /* problem needs more than the fixed scratch */

#define NEGF_FP64 0  /* complex128 throughout */
#define NEGF_MIXED 1 /* split-fp16 tensor-core factorization, FP64 residual refinement,
                      * FP64 re-run of the jobs the check rejects (see negf_mixed_policy) */

typedef struct negf_ctx negf_ctx;

/* The inputs that main.f90 hands to the negf.f90 job drivers
 * (V_reciprocal_all, nx_grid, ny_grid, atomic%..., kpoint). */
typedef struct negf_problem {
    int32_t N;            /* plane-wave basis size, size(nx_grid)                */
    int32_t Nz;           /* z slices, size(V_reciprocal_all, 3); must be >= 2   */
    int32_t ngx, ngy;     /* V_reciprocal_all bounds (-ngx:ngx, -ngy:ngy)        */
    const int32_t *nx;    /* [N] nx_grid                                         */
    const int32_t *ny;    /* [N] ny_grid                                         */
    const double *vhat;   /* complex (2ngx+1)*(2ngy+1)*Nz, V_reciprocal_all      */
    double Lx, Ly, Lz;    /* atomic%LX, LY, LZ (bohr)                            */
    double V_L, V_R;      /* atomic%V_L, V_R (Hartree)                           */
    double eta;           /* atomic%ETA (Hartree)                                */
    int32_t nk;           /* size(kpoint)                                        */
    const double *kpt;    /* [nk][3] = kpoint(i)%kx, %ky, %weight                */
    int32_t lead_model;   /* 0: the reference's lead term exp(i q dz) with the
                           * continuum q (grid.f90:284-331) and gamma = sin(q dz)/dz^2
                           * (grid.f90:355-365); 1: the exact surface Green's
                           * function of the discretised flat lead (the fixed point
                           * of Sancho-Rubio decimation, no reference counterpart)  */
} negf_problem;

/* Policy of the NEGF_MIXED path (no reference counterpart: the reference runs
 * LAPACK in complex*16 only, math_kernel.f90:8-42).  Every energy point is
 * either refined from the mixed-precision factorization and accepted, or
 * solved by the FP64 path; none is reported from low precision alone. */
typedef struct negf_mixed_policy {
    double threshold_window; /* Hartree.  Jobs whose energy lies within this distance of
                              * a subband threshold V + |k+G|^2/2 of either lead run in
                              * FP64.  0 = off (the default).                           */
    double eta_fp64_below;   /* Hartree.  If the context's eta is below this, every job
                              * runs in FP64.  0 = off (the default).                   */
    double tau_tolerance;    /* A refined job is accepted when its estimated remaining
                              * error 2 max(tau, 1) (|d_k| / |x|) rho_k is below this:
                              * d_k the k-th refinement correction of G_{Nz,1} on the
                              * open channels, x the refined value, rho_k the measured
                              * contraction (|d_1| / |x| after one step, |d_k| / |d_k-1|
                              * after more).  Default 1e-7.                             */
    int32_t max_refinements; /* refinement steps before a job that has not met the
                              * tolerance is re-run in FP64 (1..16, default 8)          */
    int32_t ctas_per_job;    /* CTAs that sweep one job: 1, 2 (a thread-block cluster
                              * on two SMs), or 0 = automatic (2 when one CTA per job
                              * would leave at least half of the SMs idle, e.g. when
                              * the factor storage bounds the wave)                    */
} negf_mixed_policy;

typedef struct negf_mixed_stats {
    int32_t n_jobs;          /* (E,k) jobs of the last NEGF_MIXED call                  */
    int32_t n_mixed;         /* accepted from the mixed path                            */
    int32_t n_fp64_policy;   /* sent to FP64 by the policy                              */
    int32_t n_fp64_rejected; /* refined, rejected by the check and re-run in FP64       */
    int32_t jobs_per_wave;   /* mixed jobs resident at once (device memory bound)       */
    int32_t ctas_per_job;    /* CTAs per job of the sweep in the last call             */
    double max_correction;   /* largest |d| / |x| among accepted jobs                   */
    double mixed_ms;         /* device time of the mixed part (CUDA events)             */
    double fp64_ms;          /* device time of the FP64 re-runs                         */
} negf_mixed_stats;

typedef struct negf_stats {
    int32_t n_jobs;        /* (E,k) RGF sweeps run                                */
    int32_t n_singular;    /* jobs that met a zero pivot                          */
    int32_t first_bad_job; /* 0-based job index of the first such job, or -1      */
    int32_t info;          /* LAPACK-style info of that job, 0 if none            */
    double device_ms;      /* device time of the sweeps (CUDA events)             */
} negf_stats;

/* ---------------------------------------------------------------- setup
 * Host-side mirrors of the set-up that main.f90 / grid.f90 do once. */

/* PlaneWaveBasis_construction_findsize, grid.f90:387-408 */
int negf_basis_size(double encut, double lx, double ly, int32_t *n);
/* PlaneWaveBasis_construction, grid.f90:410-431; nx, ny have room for n */
int negf_basis(double encut, double lx, double ly, int32_t n, int32_t *nx, int32_t *ny);
/* Basis of one k-point, |k+G|^2/2 <= encut, in the enumeration order of
 * grid.f90:420-429 (a per-k basis; the reference uses the k = 0 set for every
 * k).  *count receives the size; nx, ny (room for n) may be NULL to query it. */
int negf_basis_k(double encut, double lx, double ly, double kx, double ky, int32_t n, int32_t *count,
                 int32_t *nx, int32_t *ny);
/* Kpoint_mesh_construction, grid.f90:433-448; out[3*i] = kx, ky, weight */
int negf_kmesh(int32_t nkx, int32_t nky, double lx, double ly, double *out);
/* LocalPotential_RealToPlanewave per slice + the truncated copy of
 * main.f90:239-247: vreal (Nx,Ny,Nz) Hartree -> vhat (2ngx+1,2ngy+1,Nz)
 * complex, zero where |i|>ngx/2 or |j|>ngy/2 (left uninitialised by the
 * reference).  Errors if 2*ngx > Nx or 2*ngy > Ny (grid.f90:33-37). */
int negf_vhat(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx, int32_t ngy,
              double *vhat);
/* negf_vhat on GPU `device` (one CTA per slice, the same separable sums and
 * twiddles): same arguments and result up to rounding; host pointers, blocks
 * until done.  For set-ups over many potentials (a batch of devices). */
int negf_vhat_gpu(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx, int32_t ngy,
                  int32_t device, double *vhat);

/* -------------------------------------------------------------- context */

/* Uploads V_reciprocal_all, the basis and the k-points to `device`.
 * Replaces the per-job Hamiltonian_construction/E_minus_H_construction
 * inputs of negf.f90:145-150 (blocks are generated on chip). */
int negf_ctx_create(const negf_problem *prob, int32_t device, negf_ctx **ctx);
int negf_ctx_destroy(negf_ctx *ctx);

/* ---------------------------------------------------------- kernel level */

/* GreensFunction_tri_solver(G_inv_D, G_Function, DFL), math_kernel.f90:44-165.
 * D: (N,N,Nz) complex, the scaled E-H blocks with +I couplings.
 * dfl: any of "D", "F", "L"; diag / first / last receive the diagonal, first
 * column and last column blocks ((N,N,Nz) complex each; NULL when not
 * requested; zero-filled like the reference when requested but not in dfl).
 * The reference's t_gfunc array-of-structs becomes three planes. */
int negf_tri_solve(negf_ctx *ctx, const double *D, int32_t N, int32_t Nz, const char *dfl,
                   double *diag, double *first, double *last);

/* ------------------------------------------------------------- job level */

/* Transmission_Coefficient, negf.f90:115-174, for all nE*nk jobs at once
 * (the job loop of main.f90:384-407).  energies[nE] = Transmission(:)%energy
 * (Hartree, real; the solve uses E + i*eta).  On return
 * tau[e] = sum_k weight_k * tau(E_e, k), the reduced Transmission(:)%tau. */
int negf_transmission(negf_ctx *ctx, const double *energies, int32_t nE, int32_t precision,
                      double *tau, negf_stats *stats);

/* The NEGF_MIXED path of negf_transmission / negf_transmission_device.
 * Per job: the Schur complements D_k - gR(k) are formed in FP64 and rounded
 * to complex FP32.  Their inverses use FP32 Gauss-Jordan with pivoting inside
 * each 32 x 32 diagonal block, and trailing updates (rank 32, or rank 64
 * above N = 256) on the tcgen05 tensor cores in split fp16 with FP32
 * accumulation.  Every generator is kept in device memory.  Then refinement
 * steps on the open channels of the right lead: x0 = first block column of G
 * from the stored factors; the residual of the whole block-tridiagonal system
 * in FP64; the correction d from the stored factors; tau (grid.f90:362-383)
 * from x0 + d in FP64.  Jobs rejected by the check of negf_mixed_policy, and
 * jobs the policy sends to FP64, are re-run by the FP64 path, so tau and
 * stats cover all jobs.  Jobs are processed in waves sized to the free device
 * memory (about 7 N^2 N_z bytes per job), one SM per job or, when that would
 * leave half of the SMs idle, a two-SM cluster per job.  With NEGF_MIXED,
 * negf_transmission_device synchronises `stream` once per wave, to schedule
 * the re-runs.  N <= 1023; bases whose sweep state does not fit one SM's
 * shared memory (about N > 890) run in FP64. */
int negf_set_mixed_policy(negf_ctx *ctx, const negf_mixed_policy *policy);
int negf_get_mixed_policy(const negf_ctx *ctx, negf_mixed_policy *policy);
int negf_get_mixed_stats(const negf_ctx *ctx, negf_mixed_stats *stats);

/* negf_transmission for nctx problems at once -- e.g. one per k-point with a
 * per-k basis, or several devices of different length -- on the device of
 * ctxs[0] (all contexts must share it).  One persistent launch per kernel
 * variant takes the (problem, E, k) jobs largest-first from a counter.  The
 * energies are shared; tau[p*nE + e] = sum over the k-points of ctxs[p] of
 * weight * tau.  A multi-problem generalisation of the job loop of
 * main.f90:384-407 (the reference runs one problem per process). */
int negf_transmission_batch(negf_ctx *const *ctxs, int32_t nctx, const double *energies, int32_t nE,
                            double *tau, negf_stats *stats);

/* Transmission kernel variants (no reference counterpart: the reference has
 * one LAPACK path, math_kernel.f90:8-42): panel width x rows per thread x
 * CTAs per SM, 0 = 16 x 1 x 2 (N <= 256), 1 = 16 x 2 x 1 (N <= 512),
 * 2 = 8 x 4 x 1 (N <= 1024), 3 = 8 x 1 x 2 (N <= 256).  By default the
 * variant follows N: 3 up to 256, then 1, then 2.
 * negf_set_variant forces one for this context's negf_transmission[_device]
 * and negf_transmission_batch calls (-1 = back to the default;
 * NEGF_ERR_UNSUPPORTED if it cannot hold N).  negf_autotune times every
 * variant that can hold N on negf_transmission(energies) (each run twice, the
 * second timed), keeps the fastest for this context, returns it in *chosen and
 * the rates (solves/s; 0 for variants that cannot hold N) in rates[4]
 * (optional).  Results are identical across variants up to rounding. */
int negf_set_variant(negf_ctx *ctx, int32_t variant);
int negf_autotune(negf_ctx *ctx, const double *energies, int32_t nE, int32_t *chosen, double *rates);

/* Same computation on device-resident buffers, enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream), no synchronisation.
 * d_tau_jobs (optional, [nk*nE], job order of negf.f90:131-133) receives the
 * unweighted per-job tau; d_info (optional, [nk*nE] int32) the per-job info. */
int negf_transmission_device(negf_ctx *ctx, const double *d_energies, int32_t nE,
                             int32_t precision, double *d_tau, double *d_tau_jobs,
                             int32_t *d_info, void *stream);

/* No counterpart in the reference.  The negf_transmission computation for
 * callers that cannot allocate device memory: code that runs inside another
 * framework's memory pool or allocator, or under a device memory budget that
 * is fixed when the process starts, where a cudaMalloc in the middle of a run
 * is not allowed.  This entry calls no cudaMalloc or cudaFree (and no
 * allocating library routine); everything is passed in as device pointers:
 * d_nx, d_ny [N], d_vhat (2ngx+1)*(2ngy+1)*Nz complex, d_kpt [nk][3],
 * d_energies [nE] in, d_tau [nE] out (sum_k w_k tau), d_info [nk*nE]
 * optional per-job LAPACK-style info.  Scalars as in negf_problem.
 * Its working memory is one fixed 64 MiB array in the library, reserved on
 * every GPU that loads the library until the process exits; problems whose
 * per-job workspace (64 * roundup(N,8) * N bytes) does not fit return
 * NEGF_ERR_TOO_LARGE, and fewer jobs run at once when only a few fit.
 * The first call on a device looks up that array's device address in the
 * device's primary context and keeps it for the life of the process, so the
 * entry assumes the primary context (the CUDA runtime's default) and no
 * cudaDeviceReset between calls.  Every call blocks: it copies a check result
 * to the host (that every basis difference indexes inside the V table) and
 * synchronises `stream` before it enqueues the sweep on `stream` and returns,
 * so it cannot be called while `stream` is being captured into a CUDA graph.
 * nE * nk above INT32_MAX returns NEGF_ERR_ARG.  All calls share the one
 * array, which keeps the last call's contents: calls whose work overlaps on
 * the GPU (other streams, other host threads) race and must be serialised by
 * the caller. */
int negf_transmission_noalloc(int32_t N, int32_t Nz, int32_t ngx, int32_t ngy, const int32_t *d_nx,
                              const int32_t *d_ny, const double *d_vhat, double Lx, double Ly,
                              double Lz, double V_L, double V_R, double eta, int32_t nk,
                              const double *d_kpt, const double *d_energies, int32_t nE,
                              double *d_tau, int32_t *d_info, void *stream);

/* Equilibrium_Density, negf.f90:9-113, for all (N_circle+N_line)*nk jobs
 * (main.f90:258-297).  gap = atomic%GAP (Hartree), min_v = minval(V_real)
 * (Hartree), mu = atomic%MU (Hartree), temperature in K.  dm (N,N,Nz)
 * complex receives Density_Matrix (overwritten, not accumulated). */
int negf_density(negf_ctx *ctx, int32_t n_circle, int32_t n_line, double min_v, double mu,
                 double gap, double temperature, double *dm, negf_stats *stats);

/* The accumulation step of Equilibrium_Density (negf.f90:77-111) for any
 * contour: dm = sum_k w_k sum_i weights[i] * 2 dz^2 G_kk(energies[i] + i*eta)
 * for every slice k (w_k the k-point weights).  energies and weights are
 * complex [nE] (interleaved re, im); dm (N,N,Nz) complex is overwritten.
 * negf_density is this sum over the reference's Simpson contour. */
int negf_density_accumulate(negf_ctx *ctx, const double *energies, const double *weights, int32_t nE,
                            double *dm, negf_stats *stats);

/* Non-equilibrium Density_Matrix under a bias mu_L != mu_R.  No reference
 * counterpart: main.f90:129-132 rejects VDS != 0 and negf.f90:9-113 is
 * equilibrium only.  With mu_lo = min(mu_L, mu_R), mu_hi = max, the lead at
 * mu_hi injecting (s = its end slice, Gamma_s = diag(gamma) of its open
 * channels, the transmission weights of grid.f90:362-365):
 *   dm = (w 2/pi) [ sum over n_circle Gauss-Legendre nodes of theta in (0, pi)
 *                   of c_theta i E_R e^{i theta} G(E_c + E_R e^{i theta})
 *                   (the semicircle of negf.f90:37-65 from min_v - 1 eV to
 *                   mu_lo - gap)
 *                 - sum over n_window Gauss-Legendre nodes x of
 *                   [mu_lo - gap, mu_hi + gap] of c_x f(x - mu_lo) G(x) ]
 *      + i (w/pi) sum_x c_x (f(x - mu_hi) - f(x - mu_lo)) G_ks Gamma_s G_ks^H,
 * every G at energy + i*eta and scaled by 2 dz^2 as in negf.f90:78, the
 * spectral term by (2 dz^2)^2, summed over k-points with weights w.  So
 * Im(PtoR(dm)) * scale is the electron density, as for negf_density; with
 * mu_L == mu_R the spectral term vanishes and dm is the equilibrium
 * Density_Matrix on Gauss-Legendre nodes.  Each window energy is one sweep
 * that forms both terms.  gap, min_v, mu_L, mu_R in Hartree, temperature in
 * K; dm (N,N,Nz) complex is overwritten. */
int negf_density_neq(negf_ctx *ctx, int32_t n_circle, int32_t n_window, double min_v, double mu_L,
                     double mu_R, double gap, double temperature, double *dm, negf_stats *stats);

/* Greensfunction_PlanewaveToReal of any Density_Matrix on the GPU
 * (main.f90:306-351): density (Nx,Ny,Nz) = Im(diag of PtoR(dm slice)) * scale. */
int negf_dm_real(negf_ctx *ctx, const double *dm, int32_t Nx, int32_t Ny, double scale,
                 double *density);
/* negf_dm_real for a slab of nslices consecutive z-slices (any slab of the
 * device, the basis of ctx): dm (N,N,nslices) complex -> density
 * (Nx,Ny,nslices).  The per-rank step after the z reduce-scatter of a
 * multi-GPU density (main.f90:306-340 on each rank's slices). */
int negf_dm_real_slab(negf_ctx *ctx, const double *dm, int32_t nslices, int32_t Nx, int32_t Ny,
                      double scale, double *density);

/* Local_Density_Of_State, negf.f90:176-236, summed over k-points for the
 * energies i_e0 .. i_e0+n_chunk-1 (0-based) of the grid
 * E_i = e_lo + (e_hi-e_lo)*i/n_e.  ldos receives n_chunk consecutive
 * (N,N,Nz) complex LDOS_Matrix arrays (overwritten). */
int negf_ldos_matrix(negf_ctx *ctx, double e_lo, double e_hi, int32_t n_e, int32_t i_e0,
                     int32_t n_chunk, double *ldos, negf_stats *stats);

/* The density of main.f90:258-351 on the GPU: negf_density, then per slice
 * Greensfunction_PlanewaveToReal (grid.f90:71-135) and Density = Im(diag) * scale
 * with scale = N_z/(LX*LY*LZ) in the reference's Angstrom units
 * (main.f90:342-347).  density (Nx,Ny,Nz) receives Angstrom^-3; dm
 * (optional, (N,N,Nz) complex) receives Density_Matrix.  Errors if the basis
 * does not fit the real-space grid (2*max|n| >= N_x). */
int negf_density_real(negf_ctx *ctx, int32_t n_circle, int32_t n_line, double min_v, double mu,
                      double gap, double temperature, int32_t Nx, int32_t Ny, double scale,
                      double *density, double *dm, negf_stats *stats);

/* The LDOS of main.f90:417-554 on the GPU for the grid
 * E_i = e_lo + (e_hi-e_lo)*i/n_e: per energy the k-summed LDOS_Matrix
 * (negf.f90:176-236), Greensfunction_PlanewaveToReal per slice, and the
 * LDOS_grid_converter mapping of tools.f90:6-40 (ldos_grid = LDOS_GRID:
 * 0 keeps the axis, -1 integrates with dxyz[axis] = L/N, m > 0 takes grid
 * point m).  scale = N_z/(LX*LY*LZ)/hartree (main.f90:514).  ldos receives
 * (Mx,My,Mz,n_e) with M = N_axis if LDOS_GRID = 0 else 1. */
int negf_ldos(negf_ctx *ctx, double e_lo, double e_hi, int32_t n_e, const int32_t *ldos_grid,
              int32_t Nx, int32_t Ny, const double *dxyz, double scale, double *ldos,
              negf_stats *stats);

/* Greensfunction_PlanewaveToReal, grid.f90:71-135, for Nz_s slices:
 * g (N,N,Nz_s) complex -> out (Nx,Ny,Nz_s) complex, the unnormalised
 * real-space diagonal.  Computed by binning G(a,b) on n_a-n_b and one 2-D
 * DFT per slice instead of the reference's 2*Nx*Ny 2-D FFTs. */
int negf_ptor(const double *g, const int32_t *nx, const int32_t *ny, int32_t N, int32_t Nz_s,
              int32_t Nx, int32_t Ny, double *out);

/* ------------------------------------------------------------ diagnostics
 * Checks of the tensor-core arithmetic of the mixed-precision path (no
 * reference counterpart; device pointers, complex FP32 interleaved,
 * column-major; block until done; NEGF_ERR_CUDA if a tensor-core wait timed
 * out).
 * negf_tc_product_check: C(M, ncol) = W(:, 0:K) * B(rowmap[0:K], :) with the
 * split-fp16 tensor-core product of the trailing update (K <= 32).
 * negf_tc_inverse_check: the inverses of nmat N x N matrices (A: nmat
 * consecutive N*N blocks, N <= 1023) by the FP32 Gauss-Jordan inverse with
 * tensor-core trailing updates; info[m] as LAPACK's. */
int negf_tc_product_check(const float *d_W, int32_t ldw, const float *d_B, int32_t ldb,
                          const int32_t *d_rowmap, float *d_C, int32_t ldc, int32_t M, int32_t ncol,
                          int32_t K, void *stream);
int negf_tc_inverse_check(const float *d_A, int32_t N, int32_t nmat, float *d_out, int32_t *d_info,
                          void *stream);

/* Library version string. */
const char *negf_version(void);

#ifdef __cplusplus
}
#endif
#endif
