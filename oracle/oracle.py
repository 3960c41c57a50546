"""ctypes front end of the C oracle, plus two independent checks of it.

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, by ``__graft_entry__.smoke``
and by the CPU-baseline leg of ``bench.py``; never by the product package.

* ``C*`` functions call ``liboracle.so`` (the restatement of src/negf.f90,
  src/math_kernel.f90 and src/grid.f90; see negf_oracle.c for line cites).
* ``dense_blocks`` inverts the whole block-tridiagonal matrix with NumPy, an
  algorithm unrelated to RGF, to check the recursions of
  math_kernel.f90:81-162.
* ``closed_form_*`` solve potentials that depend on z only.  Then H is
  diagonal in the plane-wave basis and every mode is a scalar tridiagonal
  system; its Green's function follows from the three-term determinant
  recursion, evaluated here in 80-bit long double.  These are the analytic
  known answers that pin the oracle (the reference ships no golden outputs).

Parity status: unpinned against the reference build (see negf_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

HARTREE = 27.211386245988          # global.f90:24
K_B = 8.617333262e-5 / HARTREE     # global.f90:26
A_0 = 0.529177210903               # global.f90:27
PI = 3.141592653589793             # global.f90:28

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class _Problem(C.Structure):
    _fields_ = [("N", C.c_int32), ("Nz", C.c_int32), ("ngx", C.c_int32), ("ngy", C.c_int32),
                ("nx", _ip), ("ny", _ip), ("vhat", _dp), ("Lx", C.c_double), ("Ly", C.c_double),
                ("Lz", C.c_double), ("V_L", C.c_double), ("V_R", C.c_double), ("eta", C.c_double),
                ("nk", C.c_int32), ("kpt", _dp)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        rc = L.oracle_init(_build.lapack_path().encode())
        if rc != 0:
            raise RuntimeError(f"oracle_init failed ({rc})")
        L.oracle_basis_findsize.restype = C.c_int32
        L.oracle_basis_findsize.argtypes = [C.c_double] * 3
        for name in ("oracle_coefficient_simpson", "oracle_value_simpson"):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double]
        L.oracle_fermi_func.restype = C.c_double
        L.oracle_fermi_func.argtypes = [C.c_double] * 3
        L.oracle_transmission_solver.restype = C.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Problem:
    """The inputs of one hot-path run in the reference's atomic units.

    vhat is V_reciprocal_all(-ngx:ngx, -ngy:ngy, 1:Nz) as a complex
    Fortran-ordered array (already truncated to |i|<=ngx/2, |j|<=ngy/2).
    kpt is an (nk, 3) array of (kx, ky, weight).
    """

    def __init__(self, nx, ny, vhat, Lx, Ly, Lz, V_L, V_R, eta, kpt):
        self.nx = np.ascontiguousarray(nx, dtype=np.int32)
        self.ny = np.ascontiguousarray(ny, dtype=np.int32)
        self.vhat = np.asfortranarray(vhat, dtype=np.complex128)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.V_L, self.V_R, self.eta = float(V_L), float(V_R), float(eta)
        self.kpt = np.ascontiguousarray(kpt, dtype=np.float64).reshape(-1, 3)
        self.N = len(self.nx)
        self.ngx = (self.vhat.shape[0] - 1) // 2
        self.ngy = (self.vhat.shape[1] - 1) // 2
        self.Nz = self.vhat.shape[2]

    def c(self):
        s = _Problem()
        s.N, s.Nz, s.ngx, s.ngy = self.N, self.Nz, self.ngx, self.ngy
        s.nx, s.ny = _i(self.nx), _i(self.ny)
        s.vhat = self.vhat.ctypes.data_as(_dp)
        s.Lx, s.Ly, s.Lz = self.Lx, self.Ly, self.Lz
        s.V_L, s.V_R, s.eta = self.V_L, self.V_R, self.eta
        s.nk = len(self.kpt)
        s.kpt = _d(self.kpt)
        self._keep = s
        return C.byref(s)


# ------------------------------------------------------------ grid.f90 mirror
def basis(encut, lx, ly):
    L = lib()
    n = L.oracle_basis_findsize(encut, lx, ly)
    nx = np.zeros(n, np.int32)
    ny = np.zeros(n, np.int32)
    L.oracle_basis(C.c_double(encut), C.c_double(lx), C.c_double(ly), _i(nx), _i(ny))
    return nx, ny


def basis_k(encut, lx, ly, kx, ky):
    """Per-k basis |k+G|^2/2 <= encut in the j-outer / i-inner order of
    grid.f90:420-429 (restated in Python; the engine's is C++)."""
    gc = np.sqrt(2 * encut)
    i0 = int(np.floor((-gc - kx) * lx / (2 * PI))) - 2
    i1 = int(np.ceil((gc - kx) * lx / (2 * PI))) + 2
    j0 = int(np.floor((-gc - ky) * ly / (2 * PI))) - 2
    j1 = int(np.ceil((gc - ky) * ly / (2 * PI))) + 2
    nx, ny = [], []
    for j in range(j0, j1 + 1):
        for i in range(i0, i1 + 1):
            gx = (2.0 * i) * PI / lx + kx
            gy = (2.0 * j) * PI / ly + ky
            if (gx * gx + gy * gy) / 2 <= encut:
                nx.append(i)
                ny.append(j)
    return np.array(nx, np.int32), np.array(ny, np.int32)


def kmesh(nkx, nky, lx, ly):
    out = np.zeros((nkx * nky, 3))
    lib().oracle_kmesh(C.c_int32(nkx), C.c_int32(nky), C.c_double(lx), C.c_double(ly), _d(out))
    return out


def rtop(vreal2d, ngx, ngy):
    v = np.asfortranarray(vreal2d, dtype=np.float64)
    out = np.zeros((2 * ngx + 1, 2 * ngy + 1), np.complex128, order="F")
    rc = lib().oracle_rtop(_d(v), C.c_int32(v.shape[0]), C.c_int32(v.shape[1]), C.c_int32(ngx),
                           C.c_int32(ngy), out.ctypes.data_as(_dp))
    if rc:
        raise ValueError("V_reciprocal larger than the real-space grid (grid.f90:33-37)")
    return out


def vhat_all(vreal3d, ngx, ngy):
    v = np.asfortranarray(vreal3d, dtype=np.float64)
    Nx, Ny, Nz = v.shape
    out = np.zeros((2 * ngx + 1, 2 * ngy + 1, Nz), np.complex128, order="F")
    rc = lib().oracle_vhat_all(_d(v), C.c_int32(Nx), C.c_int32(Ny), C.c_int32(Nz), C.c_int32(ngx),
                               C.c_int32(ngy), out.ctypes.data_as(_dp))
    if rc:
        raise ValueError("V_reciprocal larger than the real-space grid (grid.f90:33-37)")
    return out


def hamiltonian(p: Problem, kx, ky):
    H = np.zeros((p.N, p.N, p.Nz), np.complex128, order="F")
    lib().oracle_hamiltonian(p.c(), C.c_double(kx), C.c_double(ky), H.ctypes.data_as(_dp))
    return H


def e_minus_h(p: Problem, H, energy, kx, ky):
    H = np.asfortranarray(H, dtype=np.complex128)
    D = np.zeros_like(H, order="F")
    e = complex(energy)
    lib().oracle_e_minus_h(p.c(), H.ctypes.data_as(_dp), C.c_double(e.real), C.c_double(e.imag),
                           C.c_double(kx), C.c_double(ky), D.ctypes.data_as(_dp))
    return D


def tri_solver(D, dfl):
    D = np.asfortranarray(D, dtype=np.complex128)
    N, _, Nz = D.shape
    outs = {}
    ptrs = []
    for key in "DFL":
        if key in dfl.upper():
            outs[key] = np.zeros_like(D, order="F")
            ptrs.append(outs[key].ctypes.data_as(_dp))
        else:
            ptrs.append(None)
    info = lib().oracle_tri_solver(D.ctypes.data_as(_dp), C.c_int32(N), C.c_int32(Nz),
                                   dfl.encode(), *ptrs)
    if info < 0:
        raise ValueError("tri_solver needs N >= 1 and Nz >= 2")
    return outs, info


def transmission_solver(p: Problem, first, energy, kx, ky):
    first = np.asfortranarray(first, dtype=np.complex128)
    return lib().oracle_transmission_solver(
        first.ctypes.data_as(_dp), C.c_int32(p.N), C.c_int32(p.Nz), C.c_double(energy), _i(p.nx),
        _i(p.ny), C.c_double(p.Lx), C.c_double(p.Ly), C.c_double(p.Lz), C.c_double(kx),
        C.c_double(ky), C.c_double(p.V_L), C.c_double(p.V_R))


def coefficient_simpson(i, N, a, b):
    return lib().oracle_coefficient_simpson(i, N, a, b)


def value_simpson(i, N, a, b):
    return lib().oracle_value_simpson(i, N, a, b)


def fermi_func(e, mu, t):
    return lib().oracle_fermi_func(e, mu, t)


# ------------------------------------------------------------ negf.f90 mirror
def transmission_coefficient(p: Problem, i_job, energies, tau):
    """negf.f90:115-174 for one 1-based job; accumulates into tau in place."""
    energies = np.ascontiguousarray(energies, dtype=np.float64)
    assert tau.dtype == np.float64 and tau.flags.c_contiguous
    return lib().oracle_transmission_coefficient(p.c(), C.c_int32(i_job), _d(energies),
                                                 C.c_int32(len(energies)), _d(tau))


def transmission_jobs(p: Problem, energies, job_lo=0, job_hi=None, nthreads=1):
    """main.f90:384-407 job loop (ranks -> threads) -> tau[nE] = sum_k w_k tau."""
    energies = np.ascontiguousarray(energies, dtype=np.float64)
    nE = len(energies)
    if job_hi is None:
        job_hi = nE * len(p.kpt)
    tau = np.zeros(nE)
    info = lib().oracle_transmission_jobs(p.c(), _d(energies), C.c_int32(nE), C.c_int32(job_lo),
                                          C.c_int32(job_hi), C.c_int32(nthreads), _d(tau))
    return tau, info


def equilibrium_density(p: Problem, i_job, n_circle, n_line, min_v, mu, gap, temperature, dm):
    return lib().oracle_equilibrium_density(
        p.c(), C.c_int32(i_job), C.c_int32(n_circle), C.c_int32(n_line), C.c_double(min_v),
        C.c_double(mu), C.c_double(gap), C.c_double(temperature), dm.ctypes.data_as(_dp))


def density_jobs(p: Problem, n_circle, n_line, min_v, mu, gap, temperature, job_lo=0,
                 job_hi=None, nthreads=1):
    if job_hi is None:
        job_hi = (n_circle + n_line) * len(p.kpt)
    dm = np.zeros((p.N, p.N, p.Nz), np.complex128, order="F")
    info = lib().oracle_density_jobs(
        p.c(), C.c_int32(n_circle), C.c_int32(n_line), C.c_double(min_v), C.c_double(mu),
        C.c_double(gap), C.c_double(temperature), C.c_int32(job_lo), C.c_int32(job_hi),
        C.c_int32(nthreads), dm.ctypes.data_as(_dp))
    return dm, info


def local_density_of_state(p: Problem, i_kpoint, i_energy, n_e, e_lo, e_hi, ldos):
    return lib().oracle_local_density_of_state(
        p.c(), C.c_int32(i_kpoint), C.c_int32(i_energy), C.c_int32(n_e), C.c_double(e_lo),
        C.c_double(e_hi), ldos.ctypes.data_as(_dp))


def ptor(G, nx, ny, Nx, Ny):
    G = np.asfortranarray(G, dtype=np.complex128)
    out = np.zeros((Nx, Ny), np.complex128, order="F")
    lib().oracle_ptor(G.ctypes.data_as(_dp), _i(np.ascontiguousarray(nx, np.int32)),
                      _i(np.ascontiguousarray(ny, np.int32)), C.c_int32(G.shape[0]),
                      C.c_int32(Nx), C.c_int32(Ny), out.ctypes.data_as(_dp))
    return out


def density_from_matrix(dm, nx, ny, N_x, N_y, LX_A, LY_A, LZ_A):
    """main.f90:306-351: PtoR per slice (oracle_ptor), Density = Im(.) * N_z/(LX*LY*LZ)."""
    Nz = dm.shape[2]
    out = np.zeros((N_x, N_y, Nz))
    for k in range(Nz):
        out[:, :, k] = ptor(dm[:, :, k], nx, ny, N_x, N_y).imag * (Nz / (LX_A * LY_A * LZ_A))
    return out


def _grid_converter(i, m, delta, rescale):
    """tools.f90:18-40 (i 1-based); returns (ii 1-based, rescale)."""
    ii = i if m == 0 else 1
    if m == 0:
        pass
    elif m == -1:
        rescale = rescale * delta
    elif m == i:
        pass
    else:
        rescale = 0.0
    return ii, rescale


def ldos_from_matrix(ldos_mat, nx, ny, N_x, N_y, LX_A, LY_A, LZ_A, LDOS_GRID):
    """main.f90:479-526 for one energy: PtoR per slice and the grid conversion."""
    Nz = ldos_mat.shape[2]
    size = lambda m, n: n if m == 0 else 1      # tools.f90:6-16
    out = np.zeros((size(LDOS_GRID[0], N_x), size(LDOS_GRID[1], N_y), size(LDOS_GRID[2], Nz)))
    real = np.stack([ptor(ldos_mat[:, :, k], nx, ny, N_x, N_y) for k in range(Nz)], axis=2)
    for k in range(1, Nz + 1):
        for j in range(1, N_y + 1):
            for i in range(1, N_x + 1):
                r = Nz / (LX_A * LY_A * LZ_A) / HARTREE
                ii, r = _grid_converter(i, LDOS_GRID[0], LX_A / N_x, r)
                jj, r = _grid_converter(j, LDOS_GRID[1], LY_A / N_y, r)
                kk, r = _grid_converter(k, LDOS_GRID[2], LZ_A / Nz, r)
                out[ii - 1, jj - 1, kk - 1] += real[i - 1, j - 1, k - 1].imag * r
    return out


# ----------------------------------------------------- independent checkers
def dense_blocks(D):
    """All blocks of inv(tridiag(I, D_k, I)) by one dense NumPy inverse."""
    N, _, Nz = D.shape
    A = np.zeros((N * Nz, N * Nz), np.complex128)
    for k in range(Nz):
        A[k * N:(k + 1) * N, k * N:(k + 1) * N] = D[:, :, k]
        if k + 1 < Nz:
            A[k * N:(k + 1) * N, (k + 1) * N:(k + 2) * N] = np.eye(N)
            A[(k + 1) * N:(k + 2) * N, k * N:(k + 1) * N] = np.eye(N)
    G = np.linalg.inv(A)
    diag = np.stack([G[k * N:(k + 1) * N, k * N:(k + 1) * N] for k in range(Nz)], axis=2)
    first = np.stack([G[k * N:(k + 1) * N, 0:N] for k in range(Nz)], axis=2)
    last = np.stack([G[k * N:(k + 1) * N, (Nz - 1) * N:] for k in range(Nz)], axis=2)
    return diag, first, last


def _kin(n, L, k):
    return (2.0 * n) * PI / L + k


def closed_form_modes(nx, ny, vz, Lx, Ly, Lz, V_L, V_R, eta, energy, kx, ky, lattice=False):
    """Scalar three-term recursion per plane-wave mode for a z-only potential.

    vz[k] is V_reciprocal(0,0,k) (the xy-average of slice k, Hartree).  Returns
    (G_first[N] = G_{Nz,1}, G_diag[N, Nz] = G_{kk}) rescaled by 2*Delta^2 as in
    negf.f90:159-165, computed in long double, plus sL, sR of grid.f90:355-365.
    lattice=True replaces the lead term e^{iq dz} by -g, g the |g|<1 root of
    g^2 - d g + 1 = 0 for the lead block d (the exact semi-infinite discretised
    lead), and gamma by sqrt(1 - d^2/4)/dz^2 for |d| < 2 at the real energy.
    """
    ld = np.longdouble
    Nz = len(vz)
    delta = ld(Lz) / Nz
    c2 = 2 * delta * delta
    e = complex(energy)
    N = len(nx)
    G_first = np.zeros(N, np.complex128)
    G_diag = np.zeros((N, Nz), np.complex128)
    sL = np.zeros(N)
    sR = np.zeros(N)
    vz = np.asarray(vz)
    for i in range(N):
        ax = ld(_kin(int(nx[i]), Lx, kx))
        ay = ld(_kin(int(ny[i]), Ly, ky))
        eps = (ax * ax + ay * ay) / 2
        qL = np.sqrt(np.clongdouble(2 * (np.clongdouble(e) - ld(V_L) + 1j * ld(eta)) - 2 * eps))
        qR = np.sqrt(np.clongdouble(2 * (np.clongdouble(e) - ld(V_R) + 1j * ld(eta)) - 2 * eps))
        d = np.empty(Nz, np.clongdouble)
        for k in range(Nz):
            d[k] = c2 * (np.clongdouble(e) + 1j * ld(eta) - ld(vz[k].real) - 1j * ld(vz[k].imag)
                         - eps) - 2
        if lattice:
            for idx, V in ((0, V_L), (Nz - 1, V_R)):
                dl = c2 * (np.clongdouble(e) + 1j * ld(eta) - ld(V) - eps) - 2
                disc = np.sqrt(np.clongdouble(dl * dl - 4))
                g1, g2 = (dl + disc) / 2, (dl - disc) / 2
                d[idx] -= g1 if abs(g1) <= abs(g2) else g2
        else:
            d[0] += np.exp(1j * qL * delta)
            d[-1] += np.exp(1j * qR * delta)
        # theta_k = det of leading k x k, phi_k = det of trailing block from k
        th = np.empty(Nz + 1, np.clongdouble)
        th[0] = 1
        th[1] = d[0]
        for k in range(2, Nz + 1):
            th[k] = d[k - 1] * th[k - 1] - th[k - 2]
        ph = np.empty(Nz + 2, np.clongdouble)
        ph[Nz + 1] = 1
        ph[Nz] = d[Nz - 1]
        for k in range(Nz - 1, 0, -1):
            ph[k] = d[k - 1] * ph[k + 1] - ph[k + 2]
        det = th[Nz]
        G_first[i] = complex(((-1) ** (Nz - 1)) / det * c2)
        for k in range(1, Nz + 1):
            G_diag[i, k - 1] = complex(th[k - 1] * ph[k + 1] / det * c2)
        if lattice:
            for arr, V in ((sL, V_L), (sR, V_R)):
                dr = c2 * (ld(e.real) - ld(V) - eps) - 2
                arr[i] = float(np.sqrt(1 - dr * dr / 4) / (delta * delta)) if abs(dr) < 2 else 0.0
        else:
            qr = np.sqrt(max(2 * (ld(e.real) - ld(V_L)) - 2 * eps, ld(0)))
            qt = np.sqrt(max(2 * (ld(e.real) - ld(V_R)) - 2 * eps, ld(0)))
            sL[i] = float(np.sin(qr * delta) / (delta * delta))
            sR[i] = float(np.sin(qt * delta) / (delta * delta))
    return G_first, G_diag, sL, sR


def closed_form_tau(nx, ny, vz, Lx, Ly, Lz, V_L, V_R, eta, energy, kx, ky, lattice=False):
    """tau of grid.f90:335-385 for a z-only potential (G diagonal in modes)."""
    Gf, _, sL, sR = closed_form_modes(nx, ny, vz, Lx, Ly, Lz, V_L, V_R, eta, energy, kx, ky, lattice)
    return float(np.sum(sL * sR * np.abs(Gf) ** 2))


lapack_path = _build.lapack_path
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "liboracle.so")


# ------------------------------------------- non-equilibrium density (no reference counterpart)
def lead_gammas(p: Problem, energy, kx, ky):
    """gamma_L, gamma_R = sin(q dz)/dz^2 of grid.f90:355-365 at a real energy."""
    delta = p.Lz / p.Nz
    ax = _kin(p.nx.astype(np.float64), p.Lx, kx)
    ay = _kin(p.ny.astype(np.float64), p.Ly, ky)
    qL = np.sqrt(np.maximum(2 * (energy - p.V_L) - ax * ax - ay * ay, 0.0))
    qR = np.sqrt(np.maximum(2 * (energy - p.V_R) - ax * ax - ay * ay, 0.0))
    return np.sin(qL * delta) / (delta * delta), np.sin(qR * delta) / (delta * delta)


def density_neq_contour(p: Problem, n_circle, n_window, min_v, mu_L, mu_R, gap, temperature):
    """The jobs of the biased density: list of (kind, energy, kx, ky, c_D, c_A).

    Semicircle (negf.f90:37-65 geometry) from min_v - 1 eV to mu_lo - gap with
    Gauss-Legendre nodes in theta, coefficient w 2/pi c_theta i E_R e^{i theta};
    real-axis window [mu_lo - gap, mu_hi + gap] with Gauss-Legendre nodes x:
    c_D = -w 2/pi c_x f(x - mu_lo) on G and c_A = i w/pi c_x (f(x - mu_hi) -
    f(x - mu_lo)) (2 dz^2) on G_ks Gamma_s G_ks^H (s = the lead at mu_hi).
    Both are then scaled by 2 dz^2 like every G of negf.f90:78."""
    mu_lo, mu_hi = min(mu_L, mu_R), max(mu_L, mu_R)
    kT = K_B * temperature
    dz = p.Lz / p.Nz
    cl, cr = min_v - 1.0 / HARTREE, mu_lo - gap
    E_c, E_R = (cr + cl) / 2, (cr - cl) / 2
    wl, wr = mu_lo - gap, mu_hi + gap
    xc, wc = np.polynomial.legendre.leggauss(n_circle)
    xw, ww = np.polynomial.legendre.leggauss(n_window)
    fermi = lambda e, mu: 1.0 / (np.exp((e - mu) / kT) + 1.0)
    jobs = []
    for kx, ky, w in p.kpt:
        for x, c in zip(xc, wc):
            th, cth = PI / 2 * (x + 1), PI / 2 * c
            z = E_c + E_R * np.exp(1j * th)
            jobs.append(("circle", z, kx, ky, w * 2 / PI * cth * 1j * E_R * np.exp(1j * th), 0.0))
        for x, c in zip(xw, ww):
            e = (wl + wr) / 2 + (wr - wl) / 2 * x
            cx = (wr - wl) / 2 * c
            flo, fhi = fermi(e, mu_lo), fermi(e, mu_hi)
            jobs.append(("window", complex(e), kx, ky, -(w * 2 / PI * cx * flo),
                         1j * w / PI * cx * (fhi - flo) * (2 * dz * dz)))
    return jobs


def density_neq(p: Problem, n_circle, n_window, min_v, mu_L, mu_R, gap, temperature):
    """Density_Matrix (N, N, Nz) under a bias, from the oracle's tri_solver
    (math_kernel.f90:44-165: D blocks, and the F or L column for the injecting
    lead) per job of density_neq_contour."""
    dz = p.Lz / p.Nz
    right = mu_R > mu_L
    dm = np.zeros((p.N, p.N, p.Nz), np.complex128, order="F")
    info_all = 0
    for kind, z, kx, ky, cd, ca in density_neq_contour(p, n_circle, n_window, min_v, mu_L, mu_R,
                                                       gap, temperature):
        H = hamiltonian(p, kx, ky)
        D = e_minus_h(p, H, z + 1j * p.eta, kx, ky)
        want = "D" + (("L" if right else "F") if ca != 0 else "")
        outs, info = tri_solver(D, want)
        info_all = info_all or info
        term = cd * outs["D"]
        if ca != 0:
            gL, gR = lead_gammas(p, z.real, kx, ky)
            gam = gR if right else gL
            C = outs["L" if right else "F"]
            for k in range(p.Nz):
                term[:, :, k] += ca * (C[:, :, k] * gam[None, :]) @ C[:, :, k].conj().T
        dm += term * (2 * dz * dz)
    return dm, info_all


def density_accumulate(p: Problem, energies, weights):
    """sum_k w_k sum_i weights[i] 2 dz^2 G_kk(E_i + i eta), with G_kk from the
    restated tri_solver (D mode, math_kernel.f90:94-109): the accumulation of
    negf.f90:77-111 for an arbitrary contour."""
    dz = p.Lz / p.Nz
    dm = np.zeros((p.N, p.N, p.Nz), np.complex128, order="F")
    info_all = 0
    for kx, ky, wk in p.kpt:
        H = hamiltonian(p, kx, ky)
        for e, w in zip(np.asarray(energies, np.complex128), np.asarray(weights, np.complex128)):
            outs, info = tri_solver(e_minus_h(p, H, e + 1j * p.eta, kx, ky), "D")
            info_all = info_all or info
            dm += (wk * w * 2 * dz * dz) * outs["D"]
    return dm, info_all
