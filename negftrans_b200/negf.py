"""The job-level drivers of src/negf.f90 and the solver of src/math_kernel.f90,
run on the GPU through libnegfgpu.so.

``Engine`` holds one negf_ctx (the V table, basis and k-points resident on the
device).  Its methods take whole batches of jobs, which is how the MPI job
loops of src/main.f90 call the reference drivers one job at a time:

=====================================  =====================================
reference                              here
=====================================  =====================================
Transmission_Coefficient (negf:115)    Engine.transmission(energies)
Equilibrium_Density (negf:9)           Engine.equilibrium_density(...)
Local_Density_Of_State (negf:176)      Engine.ldos_matrix(...)
GreensFunction_tri_solver (mk:44)      GreensFunction_tri_solver(D, DFL)
=====================================  =====================================
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import NEGF_FP64, NEGF_MIXED, MixedPolicy, MixedStats, Problem, Stats, _dp, _ip, check, lib


class Engine:
    """A device-resident problem (negf_ctx).

    nx_grid, ny_grid: basis; V_reciprocal_all: (2NGX+1, 2NGY+1, N_z) complex;
    Lx, Ly, Lz (bohr); V_L, V_R, ETA (Hartree); kpoint: (nk, 3) of (kx, ky, w).
    """

    def __init__(self, nx_grid, ny_grid, V_reciprocal_all, Lx, Ly, Lz, V_L, V_R, ETA, kpoint,
                 device=0, lead_model=0):
        self.nx = np.ascontiguousarray(nx_grid, np.int32)
        self.ny = np.ascontiguousarray(ny_grid, np.int32)
        self.vhat = np.asfortranarray(V_reciprocal_all, np.complex128)
        self.kpt = np.ascontiguousarray(kpoint, np.float64).reshape(-1, 3)
        self.N = len(self.nx)
        self.Nz = self.vhat.shape[2]
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.V_L, self.V_R, self.eta = float(V_L), float(V_R), float(ETA)
        p = Problem()
        p.N, p.Nz = self.N, self.Nz
        p.ngx = (self.vhat.shape[0] - 1) // 2
        p.ngy = (self.vhat.shape[1] - 1) // 2
        p.nx = self.nx.ctypes.data_as(_ip)
        p.ny = self.ny.ctypes.data_as(_ip)
        p.vhat = self.vhat.ctypes.data_as(_dp)
        p.Lx, p.Ly, p.Lz = self.Lx, self.Ly, self.Lz
        p.V_L, p.V_R, p.eta = self.V_L, self.V_R, self.eta
        p.nk = len(self.kpt)
        p.kpt = self.kpt.ctypes.data_as(_dp)
        p.lead_model = int(lead_model)   # 0 reference lead term, 1 exact lattice surface GF
        self._ctx = C.c_void_p()
        check("negf_ctx_create", lib().negf_ctx_create(C.byref(p), device, C.byref(self._ctx)))
        self.device = device
        self.last_stats = Stats()

    def close(self):
        if self._ctx:
            lib().negf_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._ctx

    # negf.f90:115-174 over all (E, k) jobs
    def transmission(self, energies, precision=NEGF_FP64):
        """Transmission(:)%tau after the job loop and reduction of main.f90:384-407.

        energies: Transmission(:)%energy in Hartree.  Returns (tau[nE], info) where
        info > 0 flags a zero pivot in some job (see last_stats)."""
        e = np.ascontiguousarray(energies, np.float64)
        tau = np.zeros(len(e))
        st = Stats()
        rc = check("negf_transmission", lib().negf_transmission(
            self._ctx, e.ctypes.data_as(_dp), len(e), precision, tau.ctypes.data_as(_dp), C.byref(st)))
        self.last_stats = st
        return tau, rc

    def set_mixed_policy(self, threshold_window=None, eta_fp64_below=None, tau_tolerance=None,
                         max_refinements=None, ctas_per_job=None):
        """Policy of the NEGF_MIXED path (Hartree): energies within threshold_window of a
        lead subband threshold run in FP64; eta below eta_fp64_below sends every job to
        FP64; a refined job is accepted when its estimated remaining |dtau| is below
        tau_tolerance after at most max_refinements steps (else it is re-run in FP64).
        ctas_per_job: 1 or 2 CTAs sweep one job (0 = automatic).
        Unset arguments keep their current values."""
        p = MixedPolicy()
        check("negf_get_mixed_policy", lib().negf_get_mixed_policy(self._ctx, C.byref(p)))
        if threshold_window is not None:
            p.threshold_window = float(threshold_window)
        if eta_fp64_below is not None:
            p.eta_fp64_below = float(eta_fp64_below)
        if tau_tolerance is not None:
            p.tau_tolerance = float(tau_tolerance)
        if max_refinements is not None:
            p.max_refinements = int(max_refinements)
        if ctas_per_job is not None:
            p.ctas_per_job = int(ctas_per_job)
        check("negf_set_mixed_policy", lib().negf_set_mixed_policy(self._ctx, C.byref(p)))

    def mixed_policy(self):
        """The current NEGF_MIXED policy (dict)."""
        p = MixedPolicy()
        check("negf_get_mixed_policy", lib().negf_get_mixed_policy(self._ctx, C.byref(p)))
        return {k: getattr(p, k) for k, _ in p._fields_}

    def mixed_stats(self):
        """Counts and device times of the last NEGF_MIXED call (dict)."""
        s = MixedStats()
        check("negf_get_mixed_stats", lib().negf_get_mixed_stats(self._ctx, C.byref(s)))
        return s.as_dict()

    def set_variant(self, variant):
        """Force the transmission kernel variant (0, 1, 2, 3; -1 = chosen by N)."""
        check("negf_set_variant", lib().negf_set_variant(self._ctx, int(variant)))

    def autotune(self, energies):
        """Time every variant that holds N on these energies and keep the fastest;
        returns (variant, rates[4] in solves/s)."""
        e = np.ascontiguousarray(energies, np.float64)
        v = C.c_int32(-1)
        rates = np.zeros(4)
        check("negf_autotune", lib().negf_autotune(self._ctx, e.ctypes.data_as(_dp), len(e), C.byref(v),
                                                   rates.ctypes.data_as(_dp)))
        return v.value, rates

    def transmission_device(self, d_energies, nE, d_tau, d_tau_jobs=None, d_info=None, stream=None,
                            precision=NEGF_FP64):
        """Enqueue on device pointers (ints); no synchronisation."""
        check("negf_transmission_device", lib().negf_transmission_device(
            self._ctx, C.c_void_p(d_energies), nE, precision, C.c_void_p(d_tau),
            C.c_void_p(d_tau_jobs or 0), C.c_void_p(d_info or 0), C.c_void_p(stream or 0)))

    # negf.f90:9-113 over all contour jobs
    def equilibrium_density(self, N_circle, N_line, min_V, MU, GAP, TEMPERATURE):
        """Density_Matrix (N, N, N_z) complex after main.f90:272-297."""
        dm = np.zeros((self.N, self.N, self.Nz), np.complex128, order="F")
        st = Stats()
        rc = check("negf_density", lib().negf_density(
            self._ctx, N_circle, N_line, min_V, MU, GAP, TEMPERATURE, dm.ctypes.data_as(_dp),
            C.byref(st)))
        self.last_stats = st
        return dm, rc

    def density_real(self, N_circle, N_line, min_V, MU, GAP, TEMPERATURE, N_x, N_y, LX_A, LY_A, LZ_A):
        """Density (N_x, N_y, N_z) in Angstrom^-3 after main.f90:258-351 (all on the GPU);
        returns (density, Density_Matrix, info)."""
        dens = np.zeros((N_x, N_y, self.Nz), np.float64, order="F")
        dm = np.zeros((self.N, self.N, self.Nz), np.complex128, order="F")
        scale = self.Nz / (LX_A * LY_A * LZ_A)
        st = Stats()
        rc = check("negf_density_real", lib().negf_density_real(
            self._ctx, N_circle, N_line, min_V, MU, GAP, TEMPERATURE, N_x, N_y, scale,
            dens.ctypes.data_as(_dp), dm.ctypes.data_as(_dp), C.byref(st)))
        self.last_stats = st
        return dens, dm, rc

    def density_accumulate(self, energies, weights):
        """Density_Matrix of any contour: sum_k w_k sum_i weights[i] 2 dz^2 G_kk(E_i + i eta)
        (the accumulation of negf.f90:77-111); energies, weights complex (Hartree)."""
        e = np.ascontiguousarray(energies, np.complex128)
        w = np.ascontiguousarray(weights, np.complex128)
        assert e.shape == w.shape and e.ndim == 1
        dm = np.zeros((self.N, self.N, self.Nz), np.complex128, order="F")
        st = Stats()
        rc = check("negf_density_accumulate", lib().negf_density_accumulate(
            self._ctx, e.ctypes.data_as(_dp), w.ctypes.data_as(_dp), len(e), dm.ctypes.data_as(_dp),
            C.byref(st)))
        self.last_stats = st
        return dm, rc

    def density_neq(self, n_circle, n_window, min_V, MU_L, MU_R, GAP, TEMPERATURE):
        """Non-equilibrium Density_Matrix (N, N, N_z) under a bias MU_L != MU_R: a
        Gauss-Legendre semicircle up to min(MU) - GAP plus a real-axis window
        [min(MU) - GAP, max(MU) + GAP] whose sweeps also form the spectral
        function injected by the higher lead (no reference counterpart)."""
        dm = np.zeros((self.N, self.N, self.Nz), np.complex128, order="F")
        st = Stats()
        rc = check("negf_density_neq", lib().negf_density_neq(
            self._ctx, n_circle, n_window, min_V, MU_L, MU_R, GAP, TEMPERATURE, dm.ctypes.data_as(_dp),
            C.byref(st)))
        self.last_stats = st
        return dm, rc

    def dm_real(self, dm, N_x, N_y, LX_A, LY_A, LZ_A):
        """Density (N_x, N_y, N_z) in Angstrom^-3 of any Density_Matrix (main.f90:306-351, GPU)."""
        dm = np.asfortranarray(dm, dtype=np.complex128)
        dens = np.zeros((N_x, N_y, self.Nz), np.float64, order="F")
        check("negf_dm_real", lib().negf_dm_real(self._ctx, dm.ctypes.data_as(_dp), N_x, N_y,
                                                 self.Nz / (LX_A * LY_A * LZ_A), dens.ctypes.data_as(_dp)))
        return dens

    def dm_real_slab(self, dm_slab, N_x, N_y, LX_A, LY_A, LZ_A):
        """Density (N_x, N_y, n) in Angstrom^-3 of n consecutive slices of a Density_Matrix
        (N, N, n) (the GPU PtoR of main.f90:306-351 on one slab)."""
        dm = np.asfortranarray(dm_slab, dtype=np.complex128)
        n = dm.shape[2]
        dens = np.zeros((N_x, N_y, n), np.float64, order="F")
        check("negf_dm_real_slab", lib().negf_dm_real_slab(
            self._ctx, dm.ctypes.data_as(_dp), n, N_x, N_y, self.Nz / (LX_A * LY_A * LZ_A),
            dens.ctypes.data_as(_dp)))
        return dens

    def ldos(self, e_lo, e_hi, N_E, LDOS_GRID, N_x, N_y, LX_A, LY_A, LZ_A):
        """LDOS (M_x, M_y, M_z, N_E) after main.f90:417-554 (Angstrom^-n eV^-1)."""
        from .constants import HARTREE
        g = np.ascontiguousarray(LDOS_GRID, np.int32)
        M = [N_x if g[0] == 0 else 1, N_y if g[1] == 0 else 1, self.Nz if g[2] == 0 else 1]
        out = np.zeros((M[0], M[1], M[2], N_E), np.float64, order="F")
        dxyz = np.array([LX_A / N_x, LY_A / N_y, LZ_A / self.Nz])
        scale = self.Nz / (LX_A * LY_A * LZ_A) / HARTREE
        st = Stats()
        rc = check("negf_ldos", lib().negf_ldos(
            self._ctx, e_lo, e_hi, N_E, g.ctypes.data_as(_ip), N_x, N_y, dxyz.ctypes.data_as(_dp), scale,
            out.ctypes.data_as(_dp), C.byref(st)))
        self.last_stats = st
        return out, rc

    # negf.f90:176-236 summed over k-points, for a range of LDOS energies
    def ldos_matrix(self, e_lo, e_hi, N_E, i_e0=0, n_chunk=None):
        """LDOS_Matrix per energy: (n_chunk, N, N, N_z) complex (each Fortran-ordered)."""
        if n_chunk is None:
            n_chunk = N_E - i_e0
        out = np.zeros((n_chunk, self.Nz, self.N, self.N), np.complex128)
        st = Stats()
        rc = check("negf_ldos_matrix", lib().negf_ldos_matrix(
            self._ctx, e_lo, e_hi, N_E, i_e0, n_chunk, out.ctypes.data_as(_dp), C.byref(st)))
        self.last_stats = st
        # memory is [o][k][j][i] -> expose (o, i, j, k)
        return np.transpose(out, (0, 3, 2, 1)), rc


def transmission_batch(engines, energies):
    """tau (n_problems, nE) for several Engines on one device in one persistent
    launch per kernel variant (largest sweeps first)."""
    e = np.ascontiguousarray(energies, np.float64)
    arr = (C.c_void_p * len(engines))(*[eng.handle.value for eng in engines])
    tau = np.zeros((len(engines), len(e)))
    st = Stats()
    rc = check("negf_transmission_batch", lib().negf_transmission_batch(
        arr, len(engines), e.ctypes.data_as(_dp), len(e), tau.ctypes.data_as(_dp), C.byref(st)))
    return tau, rc, st


def GreensFunction_tri_solver(G_inv_D, DFL, engine: Engine | None = None):
    """math_kernel.f90:44-165 on the GPU.

    G_inv_D: (N, N, N_z) complex.  Returns ({'D': diag, 'F': first, 'L': last}
    for the letters in DFL, each (N, N, N_z) complex), info)."""
    D = np.asfortranarray(G_inv_D, np.complex128)
    N, _, Nz = D.shape
    outs, ptrs = {}, []
    for key in "DFL":
        if key in DFL.upper():
            outs[key] = np.zeros_like(D, order="F")
            ptrs.append(outs[key].ctypes.data_as(_dp))
        else:
            ptrs.append(None)
    rc = check("negf_tri_solve", lib().negf_tri_solve(
        engine.handle if engine else None, D.ctypes.data_as(_dp), N, Nz, DFL.encode(), *ptrs))
    return outs, rc
