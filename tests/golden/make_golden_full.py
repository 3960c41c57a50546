"""Oracle fixtures at the full sizes of the benchmark workloads.

The CPU oracle (the C restatement of src/negf.f90 + src/math_kernel.f90) is run
on the same seeded inputs the GPU tests and bench.py build:

* qpc_disorder_n221 (N = 221, N_z = 800, QPC + 2 meV disorder): tau at 16
  energies of the workload's 2048-point grid -- the grid points nearest to
  eight subband thresholds of the leads (|E - eps_c| < 0.02 meV, where the
  new channel's self-energy e^{iq dz} is closest to 1 and gamma to 0), points
  just below a threshold, the band bottom, and plain points;
* qpc_disorder_n797 (N = 797, N_z = 400, V_g = 60 meV): tau at 6 energies of
  its 1024-point grid chosen the same way (16 GB of oracle memory per job, so
  three jobs run at a time);
* qpc_n69 (N = 69, N_z = 200): the equilibrium density contour of the
  workload's deck (N_circle = 48, N_line from N_line_per_eV) and the LDOS at 8
  energies of its 512-point grid with LDOS_GRID = -1 -1 0.  A full
  Density_Matrix is 15 MB, so the fixture keeps per-slice fingerprints:
  Tr(DM_k) and u^H DM_k v for two seeded random vectors, plus the real-space
  density summed over x and y per slice.

The inputs are not stored (the N = 797 V table alone is 30 MB): the tests
rebuild them from the seeded workload and check input fingerprints first.
Run:  python tests/golden/make_golden_full.py [n221] [n797] [n69]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from negftrans_b200 import prepare as P, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def input_fingerprint(pr):
    """Cheap checksums of the prepared inputs (basis and V table)."""
    v = np.asarray(pr.vhat)
    return np.array([pr.N, pr.Nz, float(np.sum(pr.nx * 3 + pr.ny * 7)), float(np.sum(np.abs(v))),
                     float(np.sum(v.real)), float(np.sum(v.imag))])


def thresholds(pr):
    """Subband thresholds of the (flat, V_L) left lead: V_L + |k+G|^2/2 (Hartree)."""
    a = pr.atomic
    kx, ky, _ = pr.kpoint[0]
    ax = 2.0 * pr.nx * np.pi / a.LX + kx
    ay = 2.0 * pr.ny * np.pi / a.LY + ky
    return np.unique(np.round(a.V_L + 0.5 * (ax ** 2 + ay ** 2), 15))


def pick_energies(pr, grid, n_above, n_below, n_plain, seed):
    """Indices into grid: nearest point above each of the first thresholds,
    nearest point below some others, plus seeded plain points."""
    th = thresholds(pr)
    th = th[(th > grid[0]) & (th < grid[-1])]
    idx = []
    for t in th[:n_above]:
        idx.append(int(np.searchsorted(grid, t)))           # first point >= threshold
    for t in th[n_above:n_above + n_below]:
        idx.append(int(np.searchsorted(grid, t)) - 1)       # last point < threshold
    idx.append(1)                                            # band bottom (E = 0 is point 0)
    rng = np.random.default_rng(seed)
    rest = np.setdiff1d(np.arange(len(grid)), idx)
    idx += list(rng.choice(rest, n_plain, replace=False))
    return np.array(sorted(set(idx)), np.int64)


def oracle_problem(pr):
    a = pr.atomic
    return O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)


def make_tau(name, n_above, n_below, n_plain, nthreads):
    w = W.config(name)
    pr = P.prepare(w.deck, w.V_eV)
    grid = P.transmission_energies(pr.atomic, w.n_energy)
    idx = pick_energies(pr, grid, n_above, n_below, n_plain, seed=7)
    t0 = time.time()
    tau, info = O.transmission_jobs(oracle_problem(pr), grid[idx], nthreads=nthreads)
    assert info == 0, info
    th = thresholds(pr)
    dist = np.array([np.min(np.abs(th - e)) for e in grid[idx]])
    out = os.path.join(HERE, f"oracle_{name}.npz")
    np.savez_compressed(out, workload=name, inputs=input_fingerprint(pr), grid_size=w.n_energy,
                        idx=idx, energies=grid[idx], tau=tau, threshold_distance=dist)
    print(out, f"N={pr.N} Nz={pr.Nz} jobs={len(idx)} {time.time() - t0:.0f}s", tau)


def fingerprints(dm, u, v):
    """Per slice: Tr(DM_k) and u^H DM_k v."""
    tr = np.einsum("iik->k", dm)
    uv = np.einsum("i,ijk,j->k", u.conj(), dm, v)
    return tr, uv


def make_density_ldos(nthreads):
    w = W.config("qpc_n69")
    pr = P.prepare(w.deck, w.V_eV)
    a = pr.atomic
    nl = P.n_line(a, w.deck.N_line_per_eV)
    nc = w.deck.N_circle
    p = oracle_problem(pr)
    t0 = time.time()
    dm, info = O.density_jobs(p, nc, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE, nthreads=nthreads)
    assert info == 0, info
    rng = np.random.default_rng(31)
    u = rng.standard_normal(pr.N) + 1j * rng.standard_normal(pr.N)
    v = rng.standard_normal(pr.N) + 1j * rng.standard_normal(pr.N)
    tr, uv = fingerprints(dm, u, v)
    Nx, Ny, Nz = pr.shape
    d = w.deck
    dens = O.density_from_matrix(dm, pr.nx, pr.ny, Nx, Ny, d.LX, d.LY, d.LZ)
    dens_z = dens.sum(axis=(0, 1))
    # LDOS on the 512-point grid [0, e_hi) of the transmission window, LDOS_GRID = -1 -1 0:
    # Im(PtoR) * N_z/(LX LY LZ)/hartree integrated over x and y (tools.f90:6-40)
    e_hi = float(P.transmission_energies(a, w.n_energy)[-1])
    n_e = 512
    le = np.array([3, 40, 97, 150, 211, 300, 388, 470])
    ldos = np.zeros((len(le), Nz))
    scale = Nz / (d.LX * d.LY * d.LZ) / O.HARTREE * (d.LX / Nx) * (d.LY / Ny)
    for r, ie in enumerate(le):
        mat = np.zeros((pr.N, pr.N, Nz), np.complex128, order="F")
        for ik in range(len(pr.kpoint)):
            assert O.local_density_of_state(p, ik + 1, int(ie) + 1, n_e, 0.0, e_hi, mat) == 0
        for k in range(Nz):
            ldos[r, k] = O.ptor(mat[:, :, k], pr.nx, pr.ny, Nx, Ny).imag.sum() * scale
    out = os.path.join(HERE, "oracle_qpc_n69_density_ldos.npz")
    np.savez_compressed(out, inputs=input_fingerprint(pr), n_circle=nc, n_line=nl, u=u, v=v,
                        dm_trace=tr, dm_uv=uv, dm_norm=np.linalg.norm(dm), density_z=dens_z,
                        ldos_e_hi=e_hi, ldos_n_e=n_e, ldos_idx=le, ldos_z=ldos)
    print(out, f"N={pr.N} Nz={Nz} density jobs={nc + nl} {time.time() - t0:.0f}s")


def main():
    what = sys.argv[1:] or ["n69", "n221", "n797"]
    if "n69" in what:
        make_density_ldos(nthreads=8)
    if "n221" in what:
        make_tau("qpc_disorder_n221", n_above=8, n_below=3, n_plain=4, nthreads=8)
    if "n797" in what:
        make_tau("qpc_disorder_n797", n_above=3, n_below=1, n_plain=1, nthreads=3)


if __name__ == "__main__":
    main()
