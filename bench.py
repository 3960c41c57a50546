#!/usr/bin/env python
"""Benchmark of the RGF hot path: (E,k) energy-point solves per second,
mixed precision against FP64 on one B200.

Workload (default): qpc_disorder_n797 -- the large-block configuration the
mixed-vs-FP64 metric is quoted on: N = 797 plane waves (33x33 G grid, circular
cutoff), N_z = 400 slices of 1 nm, Gamma point, a QPC (V_g = 60 meV, w = 20 nm)
with 2 meV / 10 nm disorder, energies from the 1024-point grid on [0, 50) meV.
`--workload qpc_disorder_n221` is the medium case (N = 221, N_z = 800, 2048
energies on [0, 40) meV).

--precision mixed (default): one step = negf_transmission(NEGF_MIXED) on
`--batch` energies (default: whole mixed waves, about one SM per job; at
N = 797 device memory bounds a wave to ~61 jobs on two SMs each): split-fp16
tensor-core factorization, FP64 residual refinement, FP64 re-run of rejected
jobs -- every job of the step, whatever path it takes.  `value` = jobs / the
device time of the call (CUDA events on the context's stream); `e2e` = jobs /
the wall time of the same host-buffer call.  Outside the timed region the
FP64 path runs every timed energy (at its best batch, two CTAs per SM):
`fp64_value`, `mixed_over_fp64` and `max_abs_dT` over all of them.
--precision fp64: the FP64 path alone (device-resident inputs, L2 flushed).

Output: one JSON line (rank 0).  `--impl reference` times the CPU
restatement of the reference's algorithm (LAPACK zgetrf/zgetri + zgemm per
block, one job per host thread) instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RGF energy-point solves/s, mixed vs FP64 on 1 B200 at max|ΔT|≤1e-6"  # the headline metric, verbatim
# ncu dram bytes (read + write) of k_transmission per job-slice at N = 221, measured on a
# 296-job, 16-slice launch (same per-slice work as the full workload)
TRAFFIC_PER_JOB_SLICE_N221 = 66.423e9 / (296 * 16)
UNIT = "solves/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="qpc_disorder_n797")
    ap.add_argument("--batch", type=int, default=0,
                    help="energies per step and GPU (0: whole mixed waves, about the SM count; 2x the SM count for fp64)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="mixed: NEGF_MIXED headline with the FP64 rate and max|dT| beside it")
    ap.add_argument("--nz", type=int, default=0,
                    help="profiling only: rebuild the workload with this many slices (same dz)")
    ap.add_argument("--cpu-threads", type=int, default=0, help="0 = all host cores (as many as host memory holds)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--density", action="store_true", help="also time the density contour once")
    ap.add_argument("--ldos", action="store_true", help="also time one LDOS pass (LDOS_GRID = -1 -1 0)")
    return ap.parse_args()


def host_threads(req, per_job_bytes=0):
    """Host threads for the CPU arm: all cores (or --cpu-threads), fewer only if
    that many concurrent jobs (per_job_bytes each) would not fit in 60 % of the
    available host memory."""
    n = os.cpu_count() or 1
    t = min(req or n, n)
    if per_job_bytes:
        try:
            import psutil
            avail = psutil.virtual_memory().available
            t = min(t, max(1, int(0.6 * avail // per_job_bytes)))
        except Exception:
            pass
    return max(1, t)


def flops_per_solve(N, Nz):
    """Flops of one transmission (F-mode) sweep in the reference's algorithm:
    N_z inverses and N_z-1 complex block products at 8 N^3 real flops each
    (math_kernel.f90:81-128)."""
    return 8.0 * N ** 3 * Nz + 8.0 * N ** 3 * (Nz - 1)


def open_channels(pr, energies):
    """Per energy and k-point, the rows of G_{Nz,1} the trace reads: modes with
    2(E - V_L) > |k+G|^2 (gamma_L != 0, grid.f90:355-365)."""
    a = pr.atomic
    out = []
    for kx, ky, _ in pr.kpoint:
        ax = (2.0 * pr.nx) * np.pi / a.LX + kx
        ay = (2.0 * pr.ny) * np.pi / a.LY + ky
        q2 = 2 * (np.asarray(energies)[:, None] - a.V_L) - ax[None, :] ** 2 - ay[None, :] ** 2
        out.append((q2 > 0).sum(axis=1))
    return np.concatenate(out)


def executed_flops(N, Nz, n_open):
    """Flops this engine executes per sweep: N_z inverses (8 N^3) and N_z-1
    chain products restricted to the n_open rows the trace reads (8 n N^2)."""
    return 8.0 * N ** 3 * Nz + 8.0 * n_open * N ** 2 * (Nz - 1)


def oracle_inputs(w):
    """The inputs of workload w built by the oracle's own restatement of the
    set-up (grid.f90:387-448 basis and k-mesh, grid.f90:12-69 + main.f90:239-249
    V table), so that the reference arm runs no code of libnegfgpu.so.  The
    deck's unit conversion (main.f90:184-205) is plain Python arithmetic."""
    from negftrans_b200 import prepare as P
    from oracle import oracle as O
    d = w.deck
    a = P.to_atomic(d)
    ngx, ngy = P.ngrid(P.scaled_deck(d))
    vh = np.asfortranarray(w.V_eV, dtype=np.float64) * P.scaled_deck_factor(d) / P.HARTREE
    kp = O.kmesh(d.NKX, d.NKY, a.LX, a.LY)
    nx, ny = O.basis(a.ENCUT, a.LX, a.LY)
    vhat = O.vhat_all(vh, ngx, ngy)
    p = O.Problem(nx, ny, vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, kp)
    return p, P.transmission_energies(a, w.n_energy)


def cpu_rate_problem(p, energies, nthreads, reps=1):
    """Solves/s of the oracle on problem p with `nthreads` host threads (one job each)."""
    from oracle import oracle as O
    E = np.asarray(energies[:nthreads], np.float64)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        O.transmission_jobs(p, E, nthreads=nthreads)
        times.append(time.perf_counter() - t0)
    return len(E) / statistics.mean(times), times


# one CPU sweep of a bounded sample should take about this long (seconds per job)
CPU_SAMPLE_S = 10.0


def cpu_sample_nz(N, Nz):
    """Slices of the CPU sample sweep: the whole device when one oracle sweep
    takes under ~3 CPU_SAMPLE_S (16 N^3 N_z flop at ~20 GFLOP/s per core, the
    LAPACK/BLAS rates measured for these block sizes), else a device of the same
    basis and slice thickness cut to fewer slices.  The oracle's work per slice
    (one zgetrf+zgetri and one zgemm of N x N) does not depend on the potential,
    so the full sweep's rate is the sample's times (2 nz - 1) / (2 N_z - 1)."""
    est = 16.0 * N ** 3 * Nz / 20e9
    if est <= 3 * CPU_SAMPLE_S:
        return Nz
    return max(8, int(Nz * CPU_SAMPLE_S / est))


def sweep_scale(nz, Nz):
    """Work of a sweep of nz slices over one of Nz slices (nz inverses, nz - 1 products)."""
    return (2.0 * nz - 1.0) / (2.0 * Nz - 1.0)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return None
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 7:
                    continue
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    continue
        os.unlink(self.f.name)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def fp64_peak_tflops(torch, dev):
    """Measured FP64 GEMM rate (cuBLAS DGEMM 8192^3, best of 5): the FP64 roofline."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def sample_problem(name, nz_full):
    """The oracle's problem for the CPU sample of workload `name`: the whole
    device, or (cpu_sample_nz) the same basis and slice thickness over fewer
    slices; its inputs come from the oracle's own set-up."""
    from negftrans_b200 import workloads as W
    w = W.config(name)
    p, E = oracle_inputs(w)
    nz = cpu_sample_nz(p.N, nz_full)
    if nz != nz_full:
        p, E = oracle_inputs(W.config(name, nz=nz))
    return w, p, E


def cpu_baseline(args, N, Nz):
    """cpu_baseline of this implementation's line: the oracle port on every host
    core (one sweep per thread) over the bounded sample of sample_problem."""
    _, p, E = sample_problem(args.workload, Nz)
    nth = host_threads(args.cpu_threads, 4 * 16 * p.N * p.N * p.Nz)
    r, t = cpu_rate_problem(p, E[::7], nth)
    rate = r * sweep_scale(p.Nz, Nz)
    what = "sweeps of this workload" if p.Nz == Nz else \
        f"sweeps over {p.Nz} of the {Nz} slices (same basis, blocks and slice thickness; the rate is scaled by the work per sweep)"
    return {"value": rate, "unit": UNIT, "cores": nth, "kind": "port",
            "sample": f"{nth} {what}, one per thread, {t[0]:.1f} s"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from negftrans_b200 import workloads as W
    w = W.config(args.workload)
    Nz_full = w.V_eV.shape[2]
    w, p, E = sample_problem(args.workload, Nz_full)
    scale = sweep_scale(p.Nz, Nz_full)
    nth = host_threads(args.cpu_threads, 4 * 16 * p.N * p.N * p.Nz)
    for _ in range(args.warmup):
        cpu_rate_problem(p, E, nth)
    times = []
    for s in range(args.steps):
        sample = np.roll(E, -s * nth)
        r, t = cpu_rate_problem(p, sample, nth)
        times.append(t[0])
    # a step is nth full sweeps; with a shortened device its time is the sample's / scale
    ms = 1e3 * statistics.mean(times) / scale
    value = nth / (ms * 1e-3)
    if p.Nz == Nz_full:
        sample = f"{nth} (E,k) sweeps per step, one per host thread (N={p.N}, Nz={p.Nz})"
    else:
        sample = (f"{nth} (E,k) sweeps per step, one per host thread, each over {p.Nz} of the {Nz_full} slices "
                  f"(N={p.N}, same slice thickness; time scaled by the work per sweep, {scale:.4f})")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": workload_config(args.workload, p.N, Nz_full, w.n_energy, len(p.kpt)),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nth, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Fortran+MPI+FFTW+LAPACK) cannot be built on this image; its "
                "algorithm is timed as the C restatement with LAPACK from OpenBLAS 0.3.30",
    }
    print(json.dumps(line), flush=True)


def run_ours_fp64(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # under torchrun (any world size) the ranks meet in an NCCL process group
    distributed = "RANK" in os.environ and "MASTER_ADDR" in os.environ
    if distributed:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    from negftrans_b200 import prepare as P, workloads as W
    from negftrans_b200.negf import Engine

    w = W.config(args.workload, nz=args.nz or None)
    pr = P.prepare(w.deck, w.V_eV)
    E_all = P.transmission_energies(pr.atomic, w.n_energy)
    B = args.batch or 2 * torch.cuda.get_device_properties(dev).multi_processor_count
    nk = len(pr.kpoint)
    eng = Engine(*pr.engine_args(), device=local)

    # every step's energies resident on the device before timing
    # batches are consecutive chunks of a seeded permutation of the energy grid, so every
    # step samples the whole grid (the work per energy grows with the open channels)
    n_batches = args.warmup + args.steps
    perm = np.random.default_rng(2024).permutation(len(E_all))
    idx = [perm[((s * world + rank) * B + np.arange(B)) % len(E_all)] for s in range(n_batches)]
    d_E = [torch.from_numpy(E_all[i].copy()).to(dev) for i in idx]
    d_tau = torch.zeros(B, dtype=torch.float64, device=dev)
    d_tj = torch.zeros(B * nk, dtype=torch.float64, device=dev)
    d_info = torch.zeros(B * nk, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    stream = torch.cuda.current_stream(dev)

    def step(s):
        eng.transmission_device(d_E[s].data_ptr(), B, d_tau.data_ptr(), d_tj.data_ptr(),
                                d_info.data_ptr(), stream=stream.cuda_stream)

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize(dev)
    if distributed:
        dist.barrier()
    torch.cuda.synchronize(dev)
    evs = []
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(args.warmup + s)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize(dev)
    if distributed:
        dist.barrier()
    torch.cuda.synchronize(dev)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.mean(step_ms)
    if distributed:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    info_bad = int((d_info != 0).sum().item())
    jobs_per_step = B * nk * world
    value = jobs_per_step / (ms * 1e-3)

    # correctness spot check of the last batch against the host API
    tau_dev = d_tau.cpu().numpy()

    line = None
    if rank == 0:
        N, Nz = pr.N, pr.Nz
        # flops of the timed batches (rank 0's; every rank's batch is the same size)
        nopen = np.concatenate([open_channels(pr, E_all[idx[args.warmup + s]]) for s in range(args.steps)])
        fl = float(np.sum(executed_flops(N, Nz, nopen))) / args.steps
        fl_ref = flops_per_solve(N, Nz) * B * nk
        peak = fp64_peak_tflops(torch, dev)
        achieved = fl / (ms * 1e-3) / 1e12
        cs = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": workload_config(args.workload, N, Nz, w.n_energy, nk),
            "step": {"energies_per_gpu": B, "precision": "fp64", "parallelism": f"energy-sharded x{world}",
                     "l2": "256 MB buffer written between timed steps; per-job workspace "
                           f"{4 * ((N + 7) // 8 * 8) * N * 16 * min(B * nk, 148) / 1e6:.0f} MB > L2"},
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak,
                         # ncu dram read+write of this kernel per job-slice at N = 221 (a 296-job,
                         # 16-slice capture), scaled by the job-slices of one launch
                         "traffic": (TRAFFIC_PER_JOB_SLICE_N221 * B * nk * Nz
                                     if N == 221 and args.nz in (0, Nz) else None),
                         "traffic_unit": "bytes per launch",
                         "peak_source": "measured in-run: cuBLAS FP64 GEMM 8192^3 (MEASURED_PEAKS.json "
                                        "has no FP64 figure)",
                         "flops_per_launch": fl,
                         "kernel": ("k_transmission<8,1,2>" if N <= 256 else
                                    "k_transmission<16,2,1>" if N <= 512 else "k_transmission<8,4,1>"),
                         "flops_note": "executed: 8N^3 per inverse + 8 n_open N^2 per chain product "
                                       "(rows of G_{Nz,1} with gamma_L != 0); the reference's "
                                       "16 N^3 N_z per sweep is reported as reference_equiv_tflops",
                         "reference_equiv_tflops": fl_ref / (ms * 1e-3) / 1e12,
                         "mean_open_channels": float(np.mean(nopen))},
            "gpu_launches": 2 * args.steps,
            "clocks": cs,
            "singular_jobs": info_bad,
        }
    if distributed:
        dist.barrier()

    # end to end through the C ABI with host buffers (copies in the timed region)
    if not args.no_e2e:
        E_host = [np.ascontiguousarray(E_all[i]) for i in idx]
        for s in range(min(args.warmup, 2)):
            eng.transmission(E_host[s])
        torch.cuda.synchronize(dev)
        if distributed:
            dist.barrier()
        t0 = time.perf_counter()
        for s in range(args.steps):
            tau_h, _ = eng.transmission(E_host[args.warmup + s])
        el = time.perf_counter() - t0
        if distributed:
            t = torch.tensor([el], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        if rank == 0:
            line["e2e"] = {"value": jobs_per_step * args.steps / el, "unit": UNIT,
                           "h2d_bytes_per_step": 8 * B, "d2h_bytes_per_step": 8 * B + 4 * B * nk,
                           "api": "negf_transmission (host pointers)"}
            line["e2e_matches_device"] = bool(np.allclose(tau_h, tau_dev, rtol=1e-12, atol=1e-14))

    if rank == 0 and not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args, pr.N, pr.Nz)
    if args.density:
        # the density path (D mode + contour, negf.f90:9-113) on the same device, as
        # information beside the headline: contour jobs per second
        a = pr.atomic
        nl = P.n_line(a, w.deck.N_line_per_eV)
        nc = w.deck.N_circle
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _, info_d = eng.equilibrium_density(nc, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
        el = time.perf_counter() - t0
        if rank == 0:
            njd = (nc + nl) * nk
            line["density"] = {"jobs": njd, "seconds": el, "jobs_per_s": njd / el,
                               "device_ms": eng.last_stats.device_ms,
                               "flops_per_job": 24.0 * pr.N ** 3 * pr.Nz, "info": info_d}
        # the biased density of the same configuration: 48-point Gauss-Legendre
        # semicircle + 256-point real-axis window, 1 mV bias (left lead injecting)
        from negftrans_b200 import HARTREE
        vb = W.MSTAR * 1e-3 / HARTREE
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _, info_n = eng.density_neq(nc, 256, pr.min_V, a.MU + vb, a.MU, a.GAP, a.TEMPERATURE)
        el = time.perf_counter() - t0
        if rank == 0:
            njn = (nc + 256) * nk
            line["density_neq"] = {"jobs": njn, "circle": nc, "window": 256, "bias_V": 1e-3,
                                   "seconds": el, "jobs_per_s": njn / el,
                                   "device_ms": eng.last_stats.device_ms, "info": info_n}
    if args.ldos:
        # LDOS (main.f90:417-554) on B energies of the transmission window, integrated over
        # x and y (LDOS_GRID = -1 -1 0): D-mode sweeps + PtoR per slice on the GPU
        a = pr.atomic
        Nx, Ny, Nz_ = pr.shape
        e_hi = float(E_all[-1])
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        _, info_l = eng.ldos(0.0, e_hi, B, (-1, -1, 0), Nx, Ny, w.deck.LX, w.deck.LY, w.deck.LZ)
        el = time.perf_counter() - t0
        if rank == 0:
            line["ldos"] = {"jobs": B * nk, "seconds": el, "jobs_per_s": B * nk / el,
                            "device_ms": eng.last_stats.device_ms, "info": info_l}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if distributed:
        dist.destroy_process_group()


def workload_config(name, N, Nz, n_energy, nk):
    """The workload identity, the same dict for this implementation and the reference arm."""
    return {"workload": name, "N": N, "Nz": Nz, "energies": n_energy, "kpoints": nk}


def mixed_mma_flops(N, Nz):
    """Tensor-core flops (fp16 MMAs) the mixed sweep executes per solve: per
    Gauss-Jordan panel of 32 columns, 24 MMAs (3 split products x 4 real
    products x 2 K-steps of 16) per 128 x 32 output tile of the rows x the
    columns outside the panel."""
    ntr = -(-N // 128)
    f = 0.0
    for k0 in range(0, N, 32):
        nbt = min(32, N - k0)
        nrest = N - nbt
        if nrest <= 0:
            continue
        f += ntr * (-(-nrest // 32)) * 24 * 2.0 * 128 * 32 * 16
    return f * Nz


def run_ours(args):
    if args.precision == "fp64":
        return run_ours_fp64(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    distributed = "RANK" in os.environ and "MASTER_ADDR" in os.environ
    if distributed:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    from negftrans_b200 import prepare as P, workloads as W
    from negftrans_b200._lib import NEGF_FP64, NEGF_MIXED
    from negftrans_b200.negf import Engine

    w = W.config(args.workload, nz=args.nz or None)
    pr = P.prepare(w.deck, w.V_eV)
    E_all = P.transmission_energies(pr.atomic, w.n_energy)
    nk = len(pr.kpoint)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    eng = Engine(*pr.engine_args(), device=local)
    # set-up call (allocations) on one SM count of energies spread over the grid,
    # its last point included; it also reports how many jobs a mixed wave holds on
    # this device (one job per SM, or fewer on two SMs each when device memory
    # bounds the wave: a wave's memory grows with the open channels of its highest
    # energy), so a step is whole waves
    E_setup = E_all[np.linspace(0, len(E_all) - 1, min(sms, len(E_all))).round().astype(int)]
    eng.transmission(np.ascontiguousarray(E_setup), precision=NEGF_MIXED)
    wave = max(1, eng.mixed_stats()["jobs_per_wave"])
    B = args.batch or wave * max(1, round(sms / wave))
    n_steps = args.warmup + args.steps
    perm = np.random.default_rng(2024).permutation(len(E_all))
    # a step is B energies per GPU: every rank holds the step's whole batch and the
    # product multi-GPU layer splits it (contiguous slices, all-gather of tau)
    idx = [perm[(s * world * B + np.arange(world * B)) % len(E_all)] for s in range(n_steps)]
    E_host = [np.ascontiguousarray(E_all[i]) for i in idx]
    if distributed:
        from negftrans_b200.multigpu import ShardedEngine
        solver = ShardedEngine(eng, pr.Nz, device=dev)
    else:
        solver = eng

    def step(s):
        t0 = time.perf_counter()
        tau, info = solver.transmission(E_host[s], precision=NEGF_MIXED)
        wall = time.perf_counter() - t0
        return tau, info, wall, eng.last_stats.device_ms, eng.mixed_stats()

    for s in range(args.warmup):
        step(s)
    torch.cuda.synchronize(dev)
    if distributed:
        dist.barrier()
    torch.cuda.synchronize(dev)
    dev_ms, walls, taus, infos, stats = [], [], [], [], []
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            tau, info, wall, ms, st = step(args.warmup + s)
            dev_ms.append(ms)
            walls.append(wall)
            taus.append(tau)
            infos.append(info)
            stats.append(st)
    torch.cuda.synchronize(dev)
    if distributed:
        dist.barrier()
    ms = statistics.mean(dev_ms)
    wall = statistics.mean(walls)
    if distributed:
        t = torch.tensor([ms, wall], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, wall = float(t[0]), float(t[1])
    jobs_per_step = B * nk * world
    value = jobs_per_step / (ms * 1e-3)

    # the FP64 path on the same energies, outside the timed region: its rate at
    # its best batch (two CTAs per SM) and max|dT| of every timed mixed energy
    timed_E = np.concatenate([E_host[args.warmup + s] for s in range(args.steps)])
    timed_tau = np.concatenate(taus)
    if world > 1:
        # each rank checks its own share of the timed energies
        from negftrans_b200.shard import energy_shard
        lo, hi = energy_shard(len(timed_E), rank, world)
        timed_E, timed_tau = timed_E[lo:hi], timed_tau[lo:hi]
    F = 2 * sms
    fp_ms, fp_jobs, tau64 = [], [], np.zeros_like(timed_tau)
    eng.transmission(timed_E[:8], precision=NEGF_FP64)  # warm-up (kernel variant chosen, workspace)
    for c0 in range(0, len(timed_E), F):
        chunk = timed_E[c0:c0 + F]
        t64, _ = eng.transmission(chunk, precision=NEGF_FP64)
        tau64[c0:c0 + len(chunk)] = t64
        if len(chunk) == F:
            fp_ms.append(eng.last_stats.device_ms)
            fp_jobs.append(len(chunk) * nk)
    fp64_value = (sum(fp_jobs) / (sum(fp_ms) * 1e-3)) if fp_ms else None
    dT = np.abs(timed_tau - tau64)
    if distributed:
        t = torch.tensor([fp64_value or 0.0, float(dT.max()) if len(dT) else 0.0], dtype=torch.float64, device=dev)
        fv = t[:1].clone()
        dist.all_reduce(fv, op=dist.ReduceOp.SUM)   # whole-job FP64 rate
        dm_ = t[1:].clone()
        dist.all_reduce(dm_, op=dist.ReduceOp.MAX)
        fp64_value, dmax = float(fv.item()), float(dm_.item())
    else:
        dmax = float(dT.max()) if len(dT) else 0.0

    line = None
    if rank == 0:
        N, Nz = pr.N, pr.Nz
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        tc_peak = peaks.get("bf16_tflops", 1590.0)
        fp64_peak = fp64_peak_tflops(torch, dev)
        n_mixed = sum(s_["n_mixed"] for s_ in stats)
        n_rej = sum(s_["n_fp64_rejected"] for s_ in stats)
        n_pol = sum(s_["n_fp64_policy"] for s_ in stats)
        waves = sum(-(-(s_["n_jobs"] - s_["n_fp64_policy"]) // max(1, s_["jobs_per_wave"])) for s_ in stats)
        pol = eng.mixed_policy()["max_refinements"]
        mma = mixed_mma_flops(N, Nz) * n_mixed / args.steps
        mixed_ms = statistics.mean(s_["mixed_ms"] for s_ in stats)
        cs = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64 (split-fp16 tensor products, f32 accumulate) + f64 refinement",
            "data": "synthetic",
            "config": workload_config(args.workload, N, Nz, w.n_energy, nk),
            "step": {"energies_per_gpu": B, "jobs_per_wave": wave,
                     "ctas_per_job": stats[-1].get("ctas_per_job"), "precision": "mixed (NEGF_MIXED)",
                     "parallelism": f"energy-sharded x{world}",
                     "l2": f"per-job factor storage ~{8 * N * N * Nz / 1e6:.0f} MB > L2 (inputs larger than L2)"},
            "fp64_value": fp64_value,
            "mixed_over_fp64": (value / fp64_value) if fp64_value else None,
            "max_abs_dT": dmax, "dT_energies": int(len(dT)) * world,
            "energies_covered": int(len(np.unique(timed_E))),
            "accepted_mixed": n_mixed, "fp64_rejected": n_rej, "fp64_policy": n_pol,
            "roofline": {"bound": "tensor", "kernel": "k_mixed_sweep (tcgen05 kind::f16 trailing updates)",
                         "achieved": mma / (mixed_ms * 1e-3) / 1e12, "peak": tc_peak, "unit": "TFLOP/s",
                         "frac": mma / (mixed_ms * 1e-3) / 1e12 / tc_peak, "traffic": None,
                         "peak_source": "MEASURED_PEAKS.json bf16_tflops (dense fp16 runs at the bf16 rate)",
                         "flops_note": "executed fp16 MMA flops of the sweep's trailing updates per step "
                                       "(3 split products x 4 real products) over the mixed device time",
                         "reference_equiv_tflops": flops_per_solve(N, Nz) * jobs_per_step / (ms * 1e-3) / 1e12,
                         "fp64_peak_tflops": fp64_peak},
            "gpu_launches": waves * (2 + 3 * pol) + (args.steps if n_rej else 0),
            "clocks": cs,
            "e2e": {"value": jobs_per_step / wall, "unit": UNIT, "h2d_bytes_per_step": 8 * B,
                    "d2h_bytes_per_step": 8 * B, "api": "negf_transmission(NEGF_MIXED) with host buffers"},
            "singular_jobs": int(sum(1 for i in infos if i)),
        }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        line["cpu_baseline"] = cpu_baseline(args, pr.N, pr.Nz)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if distributed:
        dist.destroy_process_group()


def run_batched(args):
    """Uneven batch: one problem per (device, k-point) of a 4x4 mesh with per-k
    bases, devices of 300/600/1200 slices; a step = --batch energies for every
    problem through negf_transmission_batch (one persistent launch)."""
    import torch

    from negftrans_b200 import workloads as W
    from negftrans_b200.negf import Engine, transmission_batch
    probs = W.batched_uneven(n_range=(180, 260))  # per-k cutoffs: bases of 180-263 plane waves
    engines = [Engine(*p["args"]) for p in probs]
    E_all = np.linspace(0.0, W.MSTAR * 0.030 / 27.211386245988, 1024, endpoint=False)
    # tile shapes by the autotuner: per basis size, time the variants on a full
    # wave (296 energies) of the shortest device of that size and use the winner
    # for all of them
    tuned = {}
    for N in sorted({p["N"] for p in probs}):
        idx = min((i for i, p in enumerate(probs) if p["N"] == N), key=lambda i: probs[i]["Nz"])
        v, rates = engines[idx].autotune(E_all[:296])
        tuned[N] = {"variant": v, "solves_per_s": [round(float(r), 2) for r in rates]}
        for i, p in enumerate(probs):
            if p["N"] == N:
                engines[i].set_variant(v)
    perm = np.random.default_rng(2024).permutation(len(E_all))
    B = args.batch or 32
    batches = [E_all[perm[(s * B + np.arange(B)) % len(E_all)]] for s in range(args.warmup + args.steps)]
    for s in range(args.warmup):
        transmission_batch(engines, batches[s])
    times, dev_ms = [], []
    for s in range(args.steps):
        t0 = time.perf_counter()
        _, info, st = transmission_batch(engines, batches[args.warmup + s])
        times.append(time.perf_counter() - t0)
        dev_ms.append(st.device_ms)
    njobs = B * len(probs)
    ms = statistics.mean(dev_ms)
    flops = sum(8.0 * p["N"] ** 3 * p["Nz"] for p in probs) * B
    line = {"metric": METRIC, "value": njobs / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic",
            "config": {"workload": "batched_uneven", "problems": len(probs),
                       "N_range": [min(p["N"] for p in probs), max(p["N"] for p in probs)],
                       "Nz": sorted({p["Nz"] for p in probs}), "energies_per_step": B,
                       "tuned_variants": tuned},
            "inverse_tflops": flops / (ms * 1e-3) / 1e12, "e2e_seconds_per_step": statistics.mean(times),
            "singular": info}
    print(json.dumps(line), flush=True)
    for e in engines:
        e.close()


def run_surrogate(args):
    """Surrogate-guided energy sampling on seeded QPC + disorder devices (N = 69,
    100 slices of 1 nm): RGF training data (T and the probe LDOS), GPU training
    of the 4 x 256 GELU network, then per unseen device the RGF solves needed for the integral of
    T over [0, 30) meV to 1e-4 with uniform nodes and with surrogate-placed
    nodes (every node an RGF solve)."""
    from negftrans_b200 import surrogate as S
    n_train, n_test, n_e = 512, 32, 256
    t0 = time.perf_counter()
    train = S.sample_devices(n_train, seed=11, nz=100)
    e_train = S.training_energies(n_e)
    T, L = S.training_set(train, n_e)
    t1 = time.perf_counter()
    sur = S.Surrogate(seed=0)
    steps, batch = (3000, 1500), 4096
    hist = sur.fit(train, e_train, T, L, steps=steps, lr=(1e-3, 2e-4), batch=batch)
    t2 = time.perf_counter()
    test = S.sample_devices(n_test, seed=99, nz=100)
    rows = S.compare(sur, test, tol=1e-4)
    t3 = time.perf_counter()
    # probe LDOS of 4 unseen devices: the network against RGF (median relative error)
    errs = []
    for d in test[:4]:
        rgf = S.RGF(d)
        try:
            ref = rgf.ldos_probes(n_e)
        finally:
            rgf.close()
        pred = sur.predict_ldos(d.desc, e_train)
        errs.append(np.median(np.abs(pred - ref) / np.maximum(ref, 1e-30)))
    ldos_err = float(np.median(errs))
    sur.close()
    w = S.WIDTHS
    # forward + backward ~ 3x the forward MACs, 2 flop each
    flop_step = 6.0 * batch * sum(a * b for a, b in zip(w[:-1], w[1:]))
    n_u = [r["uniform"] for r in rows]
    n_a = [r["adaptive"] for r in rows]
    ok = [i for i in range(len(rows)) if n_u[i] and n_a[i]]
    line = {"metric": "RGF solves for the T(E) integral to 1e-4 (uniform / surrogate-placed)",
            "value": (sum(n_u[i] for i in ok) / sum(n_a[i] for i in ok)) if ok else None,
            "unit": "ratio", "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "qpc_disorder_surrogate", "N": 69, "Nz": 100, "train_devices": n_train,
                       "energies_per_device": n_e, "test_devices": n_test, "network": w,
                       "precision": "bf16 operands, fp32 accumulate, fp32 Adam"},
            "uniform_solves_mean": float(np.mean([n_u[i] for i in ok])) if ok else None,
            "surrogate_solves_mean": float(np.mean([n_a[i] for i in ok])) if ok else None,
            "surrogate_max_abs_err_median": float(np.median([r["surrogate_max_abs_err"] for r in rows])),
            "train": {"steps": sum(steps), "batch": batch, "seconds": t2 - t1,
                      "tflops": flop_step * sum(steps) / (t2 - t1) / 1e12,
                      "loss_first": float(hist[:50].mean()), "loss_last": float(hist[-50:].mean())},
            "ldos_probe_median_rel_err": ldos_err,
            "datagen_seconds": t1 - t0, "datagen_solves": n_train * n_e * 2, "eval_seconds": t3 - t2,
            "unreached": len(rows) - len(ok)}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched_uneven":
        run_batched(args)
    elif args.workload == "surrogate":
        run_surrogate(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
