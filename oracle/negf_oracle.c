/*
 * negf_oracle.c -- TEST INFRASTRUCTURE ONLY (see negf_oracle.h).
 *
 * A line-by-line CPU restatement of the algorithms of NEGFtrans's hot path.
 * Each function names the reference lines it follows.  LAPACK/BLAS come from
 * the ILP64 OpenBLAS bundled with NumPy (symbols scipy_zgetrf_64_, ...),
 * loaded with dlopen so that the oracle builds with nothing but gcc.
 *
 * Parity status: unpinned against the reference build (no golden outputs
 * exist, no Fortran toolchain here); pinned against analytic known answers.
 */
#include "negf_oracle.h"

#include <complex.h>
#include <dlfcn.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double _Complex zc;

/* global.f90:24-28 */
static const double HARTREE = 27.211386245988;
static const double K_B = 8.617333262e-5 / 27.211386245988;
static const double PI = 3.141592653589793;

/* ---------------------------------------------------------------- LAPACK */
typedef void (*zgetrf_t)(const int64_t *, const int64_t *, zc *, const int64_t *, int64_t *,
                         int64_t *);
typedef void (*zgetri_t)(const int64_t *, zc *, const int64_t *, const int64_t *, zc *,
                         const int64_t *, int64_t *);
typedef void (*zgemm_t)(const char *, const char *, const int64_t *, const int64_t *,
                        const int64_t *, const zc *, const zc *, const int64_t *, const zc *,
                        const int64_t *, const zc *, zc *, const int64_t *, size_t, size_t);
typedef int64_t (*ilaenv_t)(const int64_t *, const char *, const char *, const int64_t *,
                            const int64_t *, const int64_t *, const int64_t *, size_t, size_t);
typedef void (*setnt_t)(int);

static zgetrf_t p_zgetrf;
static zgetri_t p_zgetri;
static zgemm_t p_zgemm;
static ilaenv_t p_ilaenv;

int oracle_init(const char *lapack_path) {
    if (p_zgetrf) return 0;
    void *h = dlopen(lapack_path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return -1;
    p_zgetrf = (zgetrf_t)dlsym(h, "scipy_zgetrf_64_");
    p_zgetri = (zgetri_t)dlsym(h, "scipy_zgetri_64_");
    p_zgemm = (zgemm_t)dlsym(h, "scipy_zgemm_64_");
    p_ilaenv = (ilaenv_t)dlsym(h, "scipy_ilaenv_64_");
    setnt_t setnt = (setnt_t)dlsym(h, "scipy_openblas_set_num_threads64_");
    if (!p_zgetrf || !p_zgetri || !p_zgemm || !p_ilaenv) return -2;
    /* one BLAS thread per caller: parallelism is over jobs, as in the
     * reference's one-MPI-rank-per-core layout */
    if (setnt) setnt(1);
    return 0;
}

/* math_kernel.f90:8-34 -- copy, zgetrf, zgetri.  Unlike the reference
 * (which drops INFO) the LAPACK info is returned. */
static int64_t inverse(const zc *M, zc *inv, int64_t N, int64_t *ipiv, zc *work, int64_t lwork) {
    memcpy(inv, M, sizeof(zc) * (size_t)N * (size_t)N);
    int64_t info1 = 0, info2 = 0;
    p_zgetrf(&N, &N, inv, &N, ipiv, &info1);
    p_zgetri(&N, inv, &N, ipiv, work, &lwork, &info2);
    return info1 ? info1 : info2;
}

/* math_kernel.f90:36-42 */
static void matrix_product(const zc *A, const zc *B, zc *C, int64_t N) {
    const zc one = 1.0, zero = 0.0;
    p_zgemm("N", "N", &N, &N, &N, &one, A, &N, B, &N, &zero, C, &N, 1, 1);
}

/* math_kernel.f90:44-165 */
int oracle_tri_solver(const double *Dd, int32_t N32, int32_t Nz, const char *dfl, double *diag_d,
                      double *first_d, double *last_d) {
    if (Nz < 2 || N32 < 1) return -1; /* the reference indexes generator(:,:,0) for Nz=1 */
    const int64_t N = N32;
    const size_t NN = (size_t)N * (size_t)N;
    const zc *D = (const zc *)Dd;
    zc *diag = (zc *)diag_d, *first = (zc *)first_d, *last = (zc *)last_d;
    int if_D = strpbrk(dfl, "Dd") != NULL;
    int if_F = strpbrk(dfl, "Ff") != NULL;
    int if_L = strpbrk(dfl, "Ll") != NULL;

    /* the SAVE'd workspace of inverse(), math_kernel.f90:15-23 */
    int64_t ispec = 1, n1 = N, m1 = -1;
    int64_t NB = p_ilaenv(&ispec, "ZGETRI", " ", &n1, &n1, &m1, &m1, 6, 1);
    if (NB < 1) NB = N;
    int64_t lwork = NB * N;
    int64_t *ipiv = (int64_t *)malloc(sizeof(int64_t) * (size_t)N);
    zc *work = (zc *)malloc(sizeof(zc) * (size_t)lwork);
    zc *Mt = (zc *)malloc(sizeof(zc) * NN);
    zc *gR = (if_D || if_F) ? (zc *)malloc(sizeof(zc) * NN * (size_t)(Nz - 1)) : NULL;
    zc *gL = if_L ? (zc *)malloc(sizeof(zc) * NN * (size_t)(Nz - 1)) : NULL;
    int64_t info = 0, r;
#define KEEP(x) do { r = (x); if (r && !info) info = r; } while (0)

    if (diag) memset(diag, 0, sizeof(zc) * NN * (size_t)Nz);
    if (first) memset(first, 0, sizeof(zc) * NN * (size_t)Nz);
    if (last) memset(last, 0, sizeof(zc) * NN * (size_t)Nz);

    /* generator_r, math_kernel.f90:81-91 (0-based slots 0..Nz-2) */
    if (if_D || if_F) {
        KEEP(inverse(D + NN * (size_t)(Nz - 1), gR + NN * (size_t)(Nz - 2), N, ipiv, work, lwork));
        for (int k = 2; k <= Nz - 1; ++k) {
            const zc *Dk = D + NN * (size_t)(Nz - k);
            const zc *gk = gR + NN * (size_t)(Nz - k);
            for (size_t e = 0; e < NN; ++e) Mt[e] = Dk[e] - gk[e];
            KEEP(inverse(Mt, gR + NN * (size_t)(Nz - k - 1), N, ipiv, work, lwork));
        }
    }
    /* diagonal blocks, math_kernel.f90:94-109 */
    if (if_D && diag) {
        for (size_t e = 0; e < NN; ++e) Mt[e] = D[e] - gR[e];
        KEEP(inverse(Mt, diag, N, ipiv, work, lwork));
        for (int k = 1; k < Nz; ++k) {
            matrix_product(diag + NN * (size_t)(k - 1), gR + NN * (size_t)(k - 1), Mt, N);
            for (int64_t i = 0; i < N; ++i) Mt[i + N * i] += 1.0;
            matrix_product(gR + NN * (size_t)(k - 1), Mt, diag + NN * (size_t)k, N);
        }
    }
    /* first column blocks, math_kernel.f90:112-129 */
    if (if_F && first) {
        for (size_t e = 0; e < NN; ++e) Mt[e] = D[e] - gR[e];
        KEEP(inverse(Mt, first, N, ipiv, work, lwork));
        for (int k = 1; k < Nz; ++k) {
            zc *Fk = first + NN * (size_t)k;
            matrix_product(gR + NN * (size_t)(k - 1), first + NN * (size_t)(k - 1), Fk, N);
            for (size_t e = 0; e < NN; ++e) Fk[e] = -Fk[e];
        }
    }
    /* generator_l and last column blocks, math_kernel.f90:132-162 */
    if (if_L) {
        KEEP(inverse(D, gL, N, ipiv, work, lwork));
        for (int m = 1; m <= Nz - 2; ++m) {
            const zc *Dm = D + NN * (size_t)m;
            const zc *gp = gL + NN * (size_t)(m - 1);
            for (size_t e = 0; e < NN; ++e) Mt[e] = Dm[e] - gp[e];
            KEEP(inverse(Mt, gL + NN * (size_t)m, N, ipiv, work, lwork));
        }
        if (last) {
            const zc *Dl = D + NN * (size_t)(Nz - 1);
            const zc *gp = gL + NN * (size_t)(Nz - 2);
            for (size_t e = 0; e < NN; ++e) Mt[e] = Dl[e] - gp[e];
            KEEP(inverse(Mt, last + NN * (size_t)(Nz - 1), N, ipiv, work, lwork));
            for (int k = 1; k < Nz; ++k) {
                zc *Lk = last + NN * (size_t)(Nz - 1 - k);
                matrix_product(gL + NN * (size_t)(Nz - 1 - k), last + NN * (size_t)(Nz - k), Lk, N);
                for (size_t e = 0; e < NN; ++e) Lk[e] = -Lk[e];
            }
        }
    }
#undef KEEP
    free(ipiv); free(work); free(Mt); free(gR); free(gL);
    return (int)info;
}

/* math_kernel.f90:167-204 */
double oracle_coefficient_simpson(int32_t i, int32_t N, double a, double b) {
    double c = 0.0;
    if (N % 2 == 1) {
        if (i == 1 || i == N) c = 1.0 / 3;
        else if (i % 2 == 0) c = 4.0 / 3;
        else c = 2.0 / 3;
    } else {
        if (i == 1) c = 1.0 / 3;
        else if (i == N - 3) c = 1.0 / 3 + 1.0 * 3 / 8;
        else if (i == N - 2 || i == N - 1) c = 3.0 * 3 / 8;
        else if (i == N) c = 1.0 * 3 / 8;
        else if (i % 2 == 0) c = 4.0 / 3;
        else c = 2.0 / 3;
    }
    return c * (b - a) / (N - 1);
}
/* math_kernel.f90:206-216 */
double oracle_value_simpson(int32_t i, int32_t N, double a, double b) {
    return (i - 1) * (b - a) / (N - 1) + a;
}
/* math_kernel.f90:218-223 */
double oracle_fermi_func(double energy, double mu, double temperature) {
    return 1.0 / (exp((energy - mu) / (K_B * temperature)) + 1);
}

/* ------------------------------------------------------------------ grid */
/* grid.f90:387-408 */
int32_t oracle_basis_findsize(double encut, double lx, double ly) {
    int32_t n = 0;
    int32_t nxm = (int32_t)ceil(lx / PI * sqrt(encut / 2));
    int32_t nym = (int32_t)ceil(ly / PI * sqrt(encut / 2));
    for (int32_t j = -nym; j <= nym; ++j)
        for (int32_t i = -nxm; i <= nxm; ++i) {
            double gx = (double)(2 * i) * PI / lx, gy = (double)(2 * j) * PI / ly;
            if ((gx * gx + gy * gy) / 2 <= encut) ++n;
        }
    return n;
}
/* grid.f90:410-431 */
void oracle_basis(double encut, double lx, double ly, int32_t *nx, int32_t *ny) {
    int32_t n = 0;
    int32_t nxm = (int32_t)ceil(lx / PI * sqrt(encut / 2));
    int32_t nym = (int32_t)ceil(ly / PI * sqrt(encut / 2));
    for (int32_t j = -nym; j <= nym; ++j)
        for (int32_t i = -nxm; i <= nxm; ++i) {
            double gx = (double)(2 * i) * PI / lx, gy = (double)(2 * j) * PI / ly;
            if ((gx * gx + gy * gy) / 2 <= encut) { nx[n] = i; ny[n] = j; ++n; }
        }
}
/* grid.f90:433-448 */
void oracle_kmesh(int32_t nkx, int32_t nky, double lx, double ly, double *out) {
    for (int32_t j = 1; j <= nky; ++j)
        for (int32_t i = 1; i <= nkx; ++i) {
            int32_t idx = (j - 1) * nkx + (i - 1);
            out[3 * idx + 0] = (i - (1 + nkx) / 2.0) / nkx * (2 * PI / lx);
            out[3 * idx + 1] = (j - (1 + nky) / 2.0) / nky * (2 * PI / ly);
            out[3 * idx + 2] = 1.0 / (nkx * nky);
        }
}

/* grid.f90:12-69: multiply by (-1)^(j-1), r2c 2-D DFT (restated as a direct
 * separable DFT instead of FFTW), divide by Nx*Ny, fill i>=0 and mirror. */
int oracle_rtop(const double *vreal, int32_t Nx, int32_t Ny, int32_t ngx, int32_t ngy,
                double *vrec_d) {
    if (2 * ngx > Nx || 2 * ngy > Ny) return -1; /* grid.f90:33-37 */
    zc *vrec = (zc *)vrec_d;
    const int32_t W = 2 * ngx + 1;
    const double nprod = (double)(Nx * Ny);
    /* X(u, y) = sum_x work(x,y) e^{-2 pi i x u / Nx}, u = 0..ngx */
    zc *X = (zc *)malloc(sizeof(zc) * (size_t)(ngx + 1) * (size_t)Ny);
    for (int32_t y = 0; y < Ny; ++y) {
        double sgn = (y % 2 == 0) ? 1.0 : -1.0; /* (-1)**(j-1), j = y+1 */
        for (int32_t u = 0; u <= ngx; ++u) {
            zc s = 0.0;
            for (int32_t x = 0; x < Nx; ++x) {
                int64_t m = ((int64_t)x * u) % Nx;
                double ang = -2.0 * PI * (double)m / Nx;
                s += vreal[x + (size_t)Nx * y] * sgn * (cos(ang) + I * sin(ang));
            }
            X[u + (size_t)(ngx + 1) * y] = s;
        }
    }
    /* out(u, v) = sum_y X(u,y) e^{-2 pi i y v / Ny}, v = j + Ny/2 */
    for (int32_t u = 0; u <= ngx; ++u)
        for (int32_t j = -ngy; j <= ngy; ++j) {
            int32_t v = j + Ny / 2;
            zc s = 0.0;
            for (int32_t y = 0; y < Ny; ++y) {
                int64_t m = ((int64_t)y * v) % Ny;
                double ang = -2.0 * PI * (double)m / Ny;
                s += X[u + (size_t)(ngx + 1) * y] * (cos(ang) + I * sin(ang));
            }
            vrec[(u + ngx) + (size_t)W * (j + ngy)] = s / nprod;
        }
    for (int32_t i = -ngx; i <= -1; ++i)
        for (int32_t j = -ngy; j <= ngy; ++j)
            vrec[(i + ngx) + (size_t)W * (j + ngy)] = conj(vrec[(-i + ngx) + (size_t)W * (-j + ngy)]);
    free(X);
    return 0;
}

/* main.f90:239-247 */
int oracle_vhat_all(const double *vreal, int32_t Nx, int32_t Ny, int32_t Nz, int32_t ngx,
                    int32_t ngy, double *vhat_d) {
    const int32_t W = 2 * ngx + 1, H = 2 * ngy + 1;
    zc *vhat = (zc *)vhat_d;
    zc *slice = (zc *)malloc(sizeof(zc) * (size_t)W * H);
    memset(vhat, 0, sizeof(zc) * (size_t)W * H * Nz);
    for (int32_t k = 0; k < Nz; ++k) {
        int rc = oracle_rtop(vreal + (size_t)Nx * Ny * k, Nx, Ny, ngx, ngy, (double *)slice);
        if (rc) { free(slice); return rc; }
        for (int32_t j = -ngy / 2; j <= ngy / 2; ++j)
            for (int32_t i = -ngx / 2; i <= ngx / 2; ++i)
                vhat[(i + ngx) + (size_t)W * ((j + ngy) + (size_t)H * k)] =
                    slice[(i + ngx) + (size_t)W * (j + ngy)];
    }
    free(slice);
    return 0;
}

static inline double kin_x(int32_t n, double L, double k) { return (double)(2 * n) * PI / L + k; }

/* grid.f90:236-262 */
void oracle_hamiltonian(const oracle_problem *p, double kx, double ky, double *H_d) {
    const int32_t N = p->N, W = 2 * p->ngx + 1, Hh = 2 * p->ngy + 1;
    const size_t NN = (size_t)N * N;
    const zc *vhat = (const zc *)p->vhat;
    zc *H = (zc *)H_d;
    for (int32_t k = 0; k < p->Nz; ++k) {
        for (int32_t j = 0; j < N; ++j)
            for (int32_t i = 0; i < N; ++i) {
                int32_t dx = p->nx[i] - p->nx[j], dy = p->ny[i] - p->ny[j];
                zc v = 0.0;
                if (dx >= -p->ngx && dx <= p->ngx && dy >= -p->ngy && dy <= p->ngy)
                    v = vhat[(dx + p->ngx) + (size_t)W * ((dy + p->ngy) + (size_t)Hh * k)];
                H[i + (size_t)N * j + NN * k] = v;
            }
        for (int32_t i = 0; i < N; ++i) {
            double ax = kin_x(p->nx[i], p->Lx, kx), ay = kin_x(p->ny[i], p->Ly, ky);
            H[i + (size_t)N * i + NN * k] += (ax * ax + ay * ay) / 2;
        }
    }
}

/* grid.f90:264-333 */
void oracle_e_minus_h(const oracle_problem *p, const double *H_d, double e_re, double e_im,
                      double kx, double ky, double *D_d) {
    const int32_t N = p->N, Nz = p->Nz;
    const size_t NN = (size_t)N * N;
    const zc *H = (const zc *)H_d;
    zc *D = (zc *)D_d;
    const zc energy = e_re + I * e_im;
    const double delta = p->Lz / Nz;
    const double c2 = 2 * (delta * delta);
    zc *QR = (zc *)malloc(sizeof(zc) * (size_t)N), *QT = (zc *)malloc(sizeof(zc) * (size_t)N);
    for (int32_t i = 0; i < N; ++i) {
        double ax = kin_x(p->nx[i], p->Lx, kx), ay = kin_x(p->ny[i], p->Ly, ky);
        QR[i] = csqrt(2 * (energy - p->V_L) - ax * ax - ay * ay);
        QT[i] = csqrt(2 * (energy - p->V_R) - ax * ax - ay * ay);
    }
    for (size_t e = 0; e < NN * (size_t)Nz; ++e) D[e] = -H[e];
    for (int32_t k = 0; k < Nz; ++k)
        for (int32_t i = 0; i < N; ++i) D[i + (size_t)N * i + NN * k] += energy;
    for (size_t e = 0; e < NN * (size_t)Nz; ++e) D[e] = D[e] * c2;
    for (int32_t k = 0; k < Nz; ++k)
        for (int32_t i = 0; i < N; ++i) D[i + (size_t)N * i + NN * k] -= 2.0;
    for (int32_t i = 0; i < N; ++i) D[i + (size_t)N * i] += cexp(I * QR[i] * delta);
    for (int32_t i = 0; i < N; ++i)
        D[i + (size_t)N * i + NN * (size_t)(Nz - 1)] += cexp(I * QT[i] * delta);
    free(QR); free(QT);
}

/* grid.f90:335-385 */
double oracle_transmission_solver(const double *first_d, int32_t N, int32_t Nz, double energy,
                                  const int32_t *nx, const int32_t *ny, double lx, double ly,
                                  double lz, double kx, double ky, double vl, double vr) {
    const zc *G = (const zc *)first_d + (size_t)N * N * (size_t)(Nz - 1);
    const double delta = lz / Nz;
    double *sL = (double *)malloc(sizeof(double) * (size_t)N);
    double *sR = (double *)malloc(sizeof(double) * (size_t)N);
    for (int32_t i = 0; i < N; ++i) {
        double ax = kin_x(nx[i], lx, kx), ay = kin_x(ny[i], ly, ky);
        double qr = sqrt(fmax(2 * (energy - vl) - ax * ax - ay * ay, 0.0));
        double qt = sqrt(fmax(2 * (energy - vr) - ax * ax - ay * ay, 0.0));
        sL[i] = sin(qr * delta) / (delta * delta);
        sR[i] = sin(qt * delta) / (delta * delta);
    }
    zc sum = 0.0;
    for (int32_t j = 0; j < N; ++j)
        for (int32_t i = 0; i < N; ++i) {
            zc a = sL[i] * G[i + (size_t)N * j];           /* Matrix_A(i,j) */
            zc b = sR[j] * conj(G[i + (size_t)N * j]);     /* Matrix_B(j,i) */
            sum += a * b;
        }
    free(sL); free(sR);
    return creal(sum);
}

/* ------------------------------------------------------------------ negf */
static void rescale(zc *G, size_t n, double lz, int32_t Nz) {
    double d = lz / Nz;
    for (size_t e = 0; e < n; ++e) G[e] = G[e] * 2.0 * (d * d);
}

/* negf.f90:115-174 */
int oracle_transmission_coefficient(const oracle_problem *p, int32_t i_job,
                                    const double *energies, int32_t nE, double *tau) {
    const int32_t N = p->N, Nz = p->Nz;
    const size_t n = (size_t)N * N * (size_t)Nz;
    int32_t i_energy = 1 + (i_job - 1) % nE;
    int32_t i_kpoint = 1 + (i_job - 1) / nE;
    double kx = p->kpt[3 * (i_kpoint - 1)], ky = p->kpt[3 * (i_kpoint - 1) + 1];
    double w = p->kpt[3 * (i_kpoint - 1) + 2];
    double energy = energies[i_energy - 1];
    double *H = (double *)malloc(sizeof(zc) * n);
    double *D = (double *)malloc(sizeof(zc) * n);
    double *F = (double *)malloc(sizeof(zc) * n);
    oracle_hamiltonian(p, kx, ky, H);
    oracle_e_minus_h(p, H, energy, p->eta, kx, ky, D);
    free(H);
    int info = oracle_tri_solver(D, N, Nz, "F", NULL, F, NULL);
    free(D);
    rescale((zc *)F, n, p->Lz, Nz);
    double t = oracle_transmission_solver(F, N, Nz, energy, p->nx, p->ny, p->Lx, p->Ly, p->Lz, kx,
                                          ky, p->V_L, p->V_R);
    free(F);
    tau[i_energy - 1] += t * w;
    return info;
}

/* negf.f90:9-113 */
int oracle_equilibrium_density(const oracle_problem *p, int32_t i_job, int32_t n_circle,
                               int32_t n_line, double min_v, double mu, double gap,
                               double temperature, double *dm_d) {
    const int32_t N = p->N, Nz = p->Nz;
    const size_t n = (size_t)N * N * (size_t)Nz;
    const int32_t n_int = n_circle + n_line;
    int32_t i_int = 1 + (i_job - 1) % n_int;
    int32_t i_kpoint = 1 + (i_job - 1) / n_int;
    double circle_L = min_v - 1.0 / HARTREE, circle_R = mu - gap;
    double line_L = mu - gap, line_R = mu + gap;
    double E_c = (circle_R + circle_L) / 2, E_R = (circle_R - circle_L) / 2;
    double kx = p->kpt[3 * (i_kpoint - 1)], ky = p->kpt[3 * (i_kpoint - 1) + 1];
    double w = p->kpt[3 * (i_kpoint - 1) + 2];
    zc energy;
    double theta = 0.0;
    if (i_int <= n_circle) {
        theta = oracle_value_simpson(i_int, n_circle, 0.0, PI);
        energy = E_c + E_R * cexp(I * theta);
    } else {
        energy = oracle_value_simpson(i_int - n_circle, n_line, line_L, line_R);
    }
    double *H = (double *)malloc(sizeof(zc) * n);
    double *D = (double *)malloc(sizeof(zc) * n);
    double *G = (double *)malloc(sizeof(zc) * n);
    oracle_hamiltonian(p, kx, ky, H);
    zc e2 = energy + I * p->eta;
    oracle_e_minus_h(p, H, creal(e2), cimag(e2), kx, ky, D);
    free(H);
    int info = oracle_tri_solver(D, N, Nz, "D", G, NULL, NULL);
    free(D);
    zc *Gz = (zc *)G, *dm = (zc *)dm_d;
    rescale(Gz, n, p->Lz, Nz);
    if (i_int <= n_circle) {
        zc c = w * 2.0 / PI * oracle_coefficient_simpson(i_int, n_circle, 0.0, PI) * I * E_R *
               cexp(I * theta);
        for (size_t e = 0; e < n; ++e) dm[e] = dm[e] + c * Gz[e];
    } else {
        double c = w * 2.0 / PI * oracle_coefficient_simpson(i_int - n_circle, n_line, line_L, line_R) *
                   oracle_fermi_func(creal(energy), mu, temperature);
        for (size_t e = 0; e < n; ++e) dm[e] = dm[e] - c * Gz[e];
    }
    free(G);
    return info;
}

/* negf.f90:176-236 */
int oracle_local_density_of_state(const oracle_problem *p, int32_t i_kpoint, int32_t i_energy,
                                  int32_t n_e, double e_lo, double e_hi, double *ldos_d) {
    const int32_t N = p->N, Nz = p->Nz;
    const size_t n = (size_t)N * N * (size_t)Nz;
    double kx = p->kpt[3 * (i_kpoint - 1)], ky = p->kpt[3 * (i_kpoint - 1) + 1];
    double w = p->kpt[3 * (i_kpoint - 1) + 2];
    double energy = e_lo + (e_hi - e_lo) * (i_energy - 1) / n_e;
    double *H = (double *)malloc(sizeof(zc) * n);
    double *D = (double *)malloc(sizeof(zc) * n);
    double *G = (double *)malloc(sizeof(zc) * n);
    oracle_hamiltonian(p, kx, ky, H);
    oracle_e_minus_h(p, H, energy, p->eta, kx, ky, D);
    free(H);
    int info = oracle_tri_solver(D, N, Nz, "D", G, NULL, NULL);
    free(D);
    zc *Gz = (zc *)G, *ld = (zc *)ldos_d;
    rescale(Gz, n, p->Lz, Nz);
    double c = w * 1.0 / PI;
    for (size_t e = 0; e < n; ++e) ld[e] = ld[e] - c * Gz[e];
    free(G);
    return info;
}

/* grid.f90:71-135 as the closed form of its FFT pair (see header). */
void oracle_ptor(const double *G_d, const int32_t *nx, const int32_t *ny, int32_t N, int32_t Nx,
                 int32_t Ny, double *out_d) {
    const zc *G = (const zc *)G_d;
    zc *out = (zc *)out_d;
    for (int32_t v = 0; v < Ny; ++v)
        for (int32_t u = 0; u < Nx; ++u) {
            zc s = 0.0;
            for (int32_t b = 0; b < N; ++b)
                for (int32_t a = 0; a < N; ++a) {
                    int64_t mx = ((int64_t)(nx[a] - nx[b]) * u) % Nx;
                    int64_t my = ((int64_t)(ny[a] - ny[b]) * v) % Ny;
                    double ang = 2.0 * PI * ((double)mx / Nx + (double)my / Ny);
                    s += G[a + (size_t)N * b] * (cos(ang) + I * sin(ang));
                }
            out[u + (size_t)Nx * v] = s;
        }
}

/* ------------------------------------------------ MPI job loops -> OpenMP */
int oracle_transmission_jobs(const oracle_problem *p, const double *energies, int32_t nE,
                             int32_t job_lo, int32_t job_hi, int32_t nthreads, double *tau) {
    if (nthreads < 1) nthreads = 1;
    double *part = (double *)calloc((size_t)nthreads * (size_t)nE, sizeof(double));
    int info = 0;
#pragma omp parallel num_threads(nthreads) reduction(max : info)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        for (int32_t j = job_lo + t; j < job_hi; j += nthreads) {
            int r = oracle_transmission_coefficient(p, j + 1, energies, nE, part + (size_t)t * nE);
            if (r > info) info = r;
        }
    }
    for (int t = 0; t < nthreads; ++t)
        for (int32_t e = 0; e < nE; ++e) tau[e] += part[(size_t)t * nE + e];
    free(part);
    return info;
}

int oracle_density_jobs(const oracle_problem *p, int32_t n_circle, int32_t n_line, double min_v,
                        double mu, double gap, double temperature, int32_t job_lo,
                        int32_t job_hi, int32_t nthreads, double *dm) {
    if (nthreads < 1) nthreads = 1;
    const size_t n = 2 * (size_t)p->N * p->N * (size_t)p->Nz;
    double *part = (double *)calloc((size_t)nthreads * n, sizeof(double));
    int info = 0;
#pragma omp parallel num_threads(nthreads) reduction(max : info)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        for (int32_t j = job_lo + t; j < job_hi; j += nthreads) {
            int r = oracle_equilibrium_density(p, j + 1, n_circle, n_line, min_v, mu, gap,
                                               temperature, part + (size_t)t * n);
            if (r > info) info = r;
        }
    }
    for (int t = 0; t < nthreads; ++t)
        for (size_t e = 0; e < n; ++e) dm[e] += part[(size_t)t * n + e];
    free(part);
    return info;
}
