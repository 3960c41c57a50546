/*
 * negf_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of NEGFtrans's hot path (src/negf.f90, src/math_kernel.f90
 * and the parts of src/grid.f90 / src/main.f90 they use), written in plain C
 * with LAPACK/BLAS (zgetrf, zgetri, zgemm) resolved at run time from the
 * ILP64 OpenBLAS that NumPy bundles.  It is the checker the GPU engine is
 * compared against and the CPU baseline that the benchmark times; the product
 * library never links or calls it.
 *
 * Parity status: UNPINNED against the reference build.  The reference ships
 * no golden outputs and cannot be compiled here (no Fortran compiler, no MPI,
 * no FFTW).  The oracle is instead pinned against analytic known answers
 * (flat and z-only potentials, where every plane-wave mode decouples into a
 * scalar three-term recursion solved in extended precision) and against an
 * independent NumPy twin; see tests/test_oracle.py.
 *
 * Conventions: complex values are interleaved (re, im) doubles, i.e. the
 * memory layout of Fortran complex*16; all matrices are column-major with
 * element (i,j,k) of an (N,N,Nz) array at i + N*j + N*N*k (0-based).
 * Energies and potentials are in Hartree, lengths in bohr (the reference's
 * "atomic" units after main.f90:184-205).
 */
#ifndef NEGF_ORACLE_H
#define NEGF_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_problem {
    int32_t N;             /* plane-wave basis size                          */
    int32_t Nz;            /* number of z slices                             */
    int32_t ngx, ngy;      /* V_reciprocal_all bounds: (-ngx:ngx, -ngy:ngy)  */
    const int32_t *nx;     /* [N] basis x indices                            */
    const int32_t *ny;     /* [N] basis y indices                            */
    const double *vhat;    /* complex (2ngx+1)*(2ngy+1)*Nz, column-major     */
    double Lx, Ly, Lz;     /* bohr                                           */
    double V_L, V_R, eta;  /* Hartree                                        */
    int32_t nk;            /* number of k-points                             */
    const double *kpt;     /* [nk][3] = (kx, ky, weight)                     */
} oracle_problem;

/* Load LAPACK/BLAS from the given shared library (ILP64, scipy_ prefix). */
int oracle_init(const char *lapack_path);

/* grid.f90:387-431 */
int32_t oracle_basis_findsize(double encut, double lx, double ly);
void oracle_basis(double encut, double lx, double ly, int32_t *nx, int32_t *ny);
/* grid.f90:433-448; out[3*i] = kx, ky, weight */
void oracle_kmesh(int32_t nkx, int32_t nky, double lx, double ly, double *out);
/* grid.f90:12-69 for one slice: V_reciprocal(-ngx:ngx,-ngy:ngy) */
int oracle_rtop(const double *vreal, int32_t Nx, int32_t Ny, int32_t ngx, int32_t ngy,
                double *vrec);
/* main.f90:239-247 over all slices: truncated V_reciprocal_all, zero outside
 * |i|<=ngx/2, |j|<=ngy/2 (the reference leaves those uninitialised). */
int oracle_vhat_all(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx,
                    int32_t ngy, double *vhat);

/* grid.f90:236-262 -> H (N,N,Nz) complex */
void oracle_hamiltonian(const oracle_problem *p, double kx, double ky, double *H);
/* grid.f90:264-333 -> D (N,N,Nz) complex; energy = E + i*eta already added */
void oracle_e_minus_h(const oracle_problem *p, const double *H, double e_re, double e_im,
                      double kx, double ky, double *D);
/* math_kernel.f90:44-165.  diag/first/last may be NULL when not requested.
 * Returns the largest LAPACK info seen (0 = all pivots nonzero). */
int oracle_tri_solver(const double *D, int32_t N, int32_t Nz, const char *dfl, double *diag,
                      double *first, double *last);
/* grid.f90:335-385; first = G_Function%first_column (N,N,Nz), already rescaled */
double oracle_transmission_solver(const double *first, int32_t N, int32_t Nz, double energy,
                                  const int32_t *nx, const int32_t *ny, double lx, double ly,
                                  double lz, double kx, double ky, double vl, double vr);

/* math_kernel.f90:167-223 */
double oracle_coefficient_simpson(int32_t i, int32_t N, double a, double b);
double oracle_value_simpson(int32_t i, int32_t N, double a, double b);
double oracle_fermi_func(double energy, double mu, double temperature);

/* negf.f90:115-174: one job (1-based i_job), tau[i_energy] += w_k * tau.
 * energies[nE] are Transmission(:)%energy (Hartree). Returns LAPACK info. */
int oracle_transmission_coefficient(const oracle_problem *p, int32_t i_job,
                                    const double *energies, int32_t nE, double *tau);
/* negf.f90:9-113: one job, accumulates into dm (N,N,Nz) complex. */
int oracle_equilibrium_density(const oracle_problem *p, int32_t i_job, int32_t n_circle,
                               int32_t n_line, double min_v, double mu, double gap,
                               double temperature, double *dm);
/* negf.f90:176-236: one (k, E) job, accumulates into ldos (N,N,Nz) complex. */
int oracle_local_density_of_state(const oracle_problem *p, int32_t i_kpoint, int32_t i_energy,
                                  int32_t n_e, double e_lo, double e_hi, double *ldos);

/* grid.f90:71-135 restated as the closed form of its FFT pair:
 * diag(u,v) = sum_ab G(a,b) exp(+2 pi i ((nx_a-nx_b) u / Nx + (ny_a-ny_b) v / Ny)),
 * unnormalised, u,v 0-based.  out is (Nx,Ny) complex. */
void oracle_ptor(const double *G, const int32_t *nx, const int32_t *ny, int32_t N, int32_t Nx,
                 int32_t Ny, double *out);

/* The MPI job loops of main.f90:274-297 and 384-407, with the ranks replaced
 * by `nthreads` OpenMP threads taking jobs round-robin and a sum at the end.
 * jobs [job_lo, job_hi) (0-based) only, for bounded baseline samples.
 * Return the largest LAPACK info. */
int oracle_transmission_jobs(const oracle_problem *p, const double *energies, int32_t nE,
                             int32_t job_lo, int32_t job_hi, int32_t nthreads, double *tau);
int oracle_density_jobs(const oracle_problem *p, int32_t n_circle, int32_t n_line, double min_v,
                        double mu, double gap, double temperature, int32_t job_lo,
                        int32_t job_hi, int32_t nthreads, double *dm);

#ifdef __cplusplus
}
#endif
#endif
