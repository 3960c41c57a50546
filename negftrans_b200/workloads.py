"""Seeded synthetic workloads (no dataset is involved).

A split-gate quantum point contact in a 100 x 100 nm periodic cell,
    V(x, z) = V_g exp(-z^2 / 2 s_z^2) (1 - exp(-x^2 / 2 w^2)),
x and z measured from the cell centre (x_i = (i - N_x/2) dx, z_k = (k + 1/2 - N_z/2) dz
for 0-based i, k), plus optional Gaussian-correlated disorder (white noise
filtered by exp(-q^2 l^2 / 4), normalised to an RMS of sigma).  GaAs
(m* = 0.067) is emulated in the reference's free-electron units by scaling the
INPUT: V' = m* V, E' = m* E, eta' = m* eta, T' = m* T; tau is unchanged.
ENCUT' values give the circular cutoffs with N = 69 / 221 / 797 plane waves.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .constants import HARTREE
from .prepare import InputDeck

MSTAR = 0.067


def qpc_potential(Nx, Ny, Nz, L_nm, Lz_nm, Vg, w_nm, sz_nm, disorder=0.0, corr_nm=10.0, seed=1000):
    """Potential in eV (unscaled), shape (Nx, Ny, Nz), Fortran order."""
    dx = L_nm / Nx
    dz = Lz_nm / Nz
    x = (np.arange(Nx) - Nx / 2) * dx
    z = (np.arange(Nz) + 0.5 - Nz / 2) * dz
    gate = 1.0 - np.exp(-x ** 2 / (2 * w_nm ** 2))
    env = np.exp(-z ** 2 / (2 * sz_nm ** 2))
    V = Vg * gate[:, None, None] * env[None, None, :] * np.ones((1, Ny, 1))
    if disorder > 0:
        rng = np.random.Generator(np.random.PCG64(seed))
        noise = rng.standard_normal((Nx, Ny, Nz))
        qx = 2 * np.pi * np.fft.fftfreq(Nx, d=dx)
        qy = 2 * np.pi * np.fft.fftfreq(Ny, d=L_nm / Ny)
        qz = 2 * np.pi * np.fft.fftfreq(Nz, d=dz)
        q2 = qx[:, None, None] ** 2 + qy[None, :, None] ** 2 + qz[None, None, :] ** 2
        filt = np.exp(-q2 * corr_nm ** 2 / 4)
        d = np.real(np.fft.ifftn(np.fft.fftn(noise) * filt))
        d *= disorder / np.sqrt(np.mean(d ** 2))
        V = V + d
    return np.asfortranarray(V)


@dataclass
class Workload:
    name: str
    deck: InputDeck
    V_eV: np.ndarray         # POTENTIAL (already m*-scaled), eV
    n_energy: int
    notes: str = ""


def _deck(Lz_A, encut, e_max_meV, n_e, nk=1, mu_meV=20.0, t_K=1.1605, n_circle=48, n_line=256):
    # N_line = IDNINT(N_line_per_eV * 2 * GAP[eV]) with GAP = 6 k_B T' (main.f90:193,261)
    kT_eV = 8.617333262e-5 * MSTAR * t_K
    per_eV = int(round(n_line / (12 * kT_eV)))
    return InputDeck(
        if_transmission=True, if_density=True, LX=1000.0, LY=1000.0, LZ=Lz_A, ENCUT=encut,
        ETA=MSTAR * 1e-6 / HARTREE, NKX=nk, NKY=nk, TEMPERATURE=MSTAR * t_K, MU=MSTAR * mu_meV * 1e-3,
        TRANSMISSION_GRID=(0.0, MSTAR * e_max_meV * 1e-3, float(n_e)), N_circle=n_circle,
        N_line_per_eV=per_eV)


def config(name: str, nz: int | None = None) -> Workload:
    """Named workloads with the shapes of the benchmark configurations.

    nz (profiling only) rebuilds the device with that many slices of the same
    thickness, which scales the sweep length and nothing else."""
    if name == "qpc_n69":
        # 69 plane waves, 200 slices of 1 nm, 512 energies on [0, 30) meV, Gamma only
        nz = nz or 200
        V = MSTAR * qpc_potential(64, 64, nz, 100.0, nz * 1.0, 0.050, 15.0, 20.0)
        return Workload(name, _deck(nz * 10.0, 0.0033091, 30.0, 512), V, 512)
    if name == "qpc_disorder_n221":
        # 221 plane waves, 800 slices of 0.5 nm, 2048 energies on [0, 40) meV, disorder 2 meV / 10 nm
        nz = nz or 800
        V = MSTAR * qpc_potential(64, 64, nz, 100.0, nz * 0.5, 0.050, 15.0, 20.0, disorder=0.002)
        return Workload(name, _deck(nz * 5.0, 0.0105288, 40.0, 2048), V, 2048)
    if name == "qpc_disorder_n797":
        # 797 plane waves (128x128 grid), 400 slices of 1 nm, 1024 energies on [0, 50) meV
        nz = nz or 400
        V = MSTAR * qpc_potential(128, 128, nz, 100.0, nz * 1.0, 0.060, 20.0, 20.0, disorder=0.002)
        return Workload(name, _deck(nz * 10.0, 0.0385807, 50.0, 1024), V, 1024)
    if name.startswith("small"):
        # test-sized QPC: small basis and few slices, same physics
        # small:<encut_meV>:<Nz>  (e.g. small:1.2:16)
        _, enc, nz = name.split(":")
        nz = int(nz)
        V = MSTAR * qpc_potential(32, 32, nz, 100.0, nz * 1.0, 0.050, 15.0, nz / 10.0, disorder=0.002)
        return Workload(name, _deck(nz * 10.0, float(enc) * 1e-3, 30.0, 16), V, 16)
    raise KeyError(name)


def _encut_for_size(n_target, L, kx, ky, hi):
    """Smallest cutoff (Hartree) whose basis |k+G|^2/2 <= ENCUT at (kx, ky) has
    at least n_target plane waves (the count is monotone in the cutoff)."""
    from .grid import PlaneWaveBasis_k
    lo = 0.0
    for _ in range(60):
        mid = 0.5 * (lo + hi)
        if len(PlaneWaveBasis_k(mid, L, L, kx, ky)[0]) >= n_target:
            hi = mid
        else:
            lo = mid
    return hi


def batched_uneven(nkx=4, nzs=(300, 600, 1200), encut_eV=0.0105288, grid=64, seed=4000, n_range=None):
    """Problems of the uneven batch: one per (device, k-point) of an nkx x nkx
    Monkhorst-Pack mesh, each with its own basis |k+G| <= G_c, devices of N_z
    slices of 1 nm with seeded V_g ~ U[20, 80] meV and w ~ U[8, 25] nm (+ GaAs
    scaling).  With one G_c (n_range None) the k shifts change the basis size
    by a few plane waves only; n_range = (lo, hi) gives k-point i its own cutoff
    so that the sizes spread evenly over [lo, hi].  Returns a list of dicts
    holding the Engine arguments ('args'), 'N', 'Nz' and the device index."""
    from .grid import Kpoint_mesh_construction, PlaneWaveBasis_k, V_reciprocal_all
    from .constants import A_0
    rng = np.random.Generator(np.random.PCG64(seed))
    L = 1000.0 / A_0
    enc = encut_eV / HARTREE
    kp = Kpoint_mesh_construction(nkx, nkx, L, L)
    if n_range is None:
        bases = [PlaneWaveBasis_k(enc, L, L, kx, ky) for kx, ky, _ in kp]
    else:
        targets = np.rint(np.linspace(n_range[0], n_range[1], len(kp))).astype(int)
        bases = [PlaneWaveBasis_k(_encut_for_size(int(t), L, kx, ky, 20.0 * enc), L, L, kx, ky)
                 for t, (kx, ky, _) in zip(targets, kp)]
    nmax = max(int(np.max(np.abs(np.concatenate([b[0], b[1]])))) for b in bases)
    # the reference's NGX (main.f90:94-100), raised so that every pair
    # difference of a shifted basis indexes inside the table; the table keeps
    # the reference's window |dn| <= NGX/2 (main.f90:242-244)
    from .prepare import InputDeck, ngrid
    ng = max(max(ngrid(InputDeck(LX=1000.0, LY=1000.0, ENCUT=encut_eV))), 2 * nmax)
    out = []
    for d, nz in enumerate(nzs):
        vg = rng.uniform(0.020, 0.080)
        w = rng.uniform(8.0, 25.0)
        V = MSTAR * qpc_potential(grid, grid, nz, 100.0, nz * 1.0, vg, w, 20.0)
        vhat = V_reciprocal_all(V / HARTREE, ng, ng)
        lz = nz * 10.0 / A_0
        for (kx, ky, wk), (nx, ny) in zip(kp, bases):
            out.append({"device": d, "Nz": nz, "N": len(nx),
                        "args": (nx, ny, vhat, L, L, lz, 0.0, 0.0, MSTAR * 1e-6 / HARTREE,
                                 np.array([[kx, ky, wk]]))})
    return out
