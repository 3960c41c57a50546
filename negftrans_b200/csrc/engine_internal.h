// engine_internal.h -- the context shared by the FP64 engine (negf_engine.cu)
// and the mixed-precision path (negf_mixed.cu).  Host-side only.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "negf_gpu.h"

struct negf_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int N = 0, Nz = 0, ld = 0, ngx = 0, ngy = 0, nk = 0;
    double Lx = 0, Ly = 0, Lz = 0, V_L = 0, V_R = 0, eta = 0;
    int lead_model = 0;
    int variant = -1;         // transmission kernel variant forced by negf_set_variant /
                              // negf_autotune; -1 = chosen by N
    std::vector<double> kpt;  // nk x 3
    std::vector<int> nx, ny;  // host copy of the basis
    double2 *d_vhat = nullptr;
    int *d_nx = nullptr, *d_ny = nullptr;
    double *d_ax = nullptr, *d_ay = nullptr, *d_kw = nullptr;
    // scratch grown on demand
    void *d_ws = nullptr;
    size_t ws_bytes = 0;
    double *d_E = nullptr, *d_tau = nullptr, *d_tau_jobs = nullptr;
    int *d_info = nullptr;
    int cap_E = 0, cap_jobs = 0;
    // mixed-precision path
    negf_mixed_policy mixed_policy{0.0, 0.0, 1e-7, 8, 0};
    negf_mixed_stats mixed_stats{};
    void *d_mixed = nullptr;  // per-wave factor storage and scratch
    size_t mixed_bytes = 0;
    // -c2 V(G_i - G_j) of every slice (energy- and k-independent part of D_k),
    // complex FP64 [Nz][N][ld] column-major, built on the first mixed call
    double2 *d_voff = nullptr;
};

// FP64 sweeps of the listed jobs (energy index ie[q] into d_E, k-point ik[q])
// of context c through the batch kernel: h_tau[q] the unweighted tau of job q,
// h_info[q] its info; *ms the device time.  Synchronous on c->stream.
int negf_internal_fp64_jobs(negf_ctx *c, const double *d_E, const int *ie, const int *ik, int njobs,
                            double *h_tau, int *h_info, float *ms);

// The NEGF_MIXED transmission of all nE * nk jobs (job = ik * nE + ie, the
// order of negf.f90:131-133): h_E host energies, d_E the same on the device.
// h_tau_jobs[job] unweighted tau, h_info[job] info.  Synchronous.
int negf_internal_mixed(negf_ctx *c, const double *h_E, const double *d_E, int nE, double *h_tau_jobs,
                        int *h_info, double *device_ms);
