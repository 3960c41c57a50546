"""Set-up routines of src/grid.f90 (and the V table copy of src/main.f90),
with the reference's names and argument meaning, computed by libnegfgpu.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import _dp, _ip, check, lib


def PlaneWaveBasis_construction_findsize(ENCUT, Lx, Ly):
    """grid.f90:387-408: size N of the |G|^2/2 <= ENCUT basis (atomic units)."""
    n = C.c_int32(0)
    check("negf_basis_size", lib().negf_basis_size(ENCUT, Lx, Ly, C.byref(n)))
    return n.value


def PlaneWaveBasis_construction(ENCUT, Lx, Ly):
    """grid.f90:410-431: (nx_grid, ny_grid), j outer / i inner order."""
    n = PlaneWaveBasis_construction_findsize(ENCUT, Lx, Ly)
    nx = np.zeros(n, np.int32)
    ny = np.zeros(n, np.int32)
    check("negf_basis", lib().negf_basis(ENCUT, Lx, Ly, n, nx.ctypes.data_as(_ip),
                                          ny.ctypes.data_as(_ip)))
    return nx, ny


def Kpoint_mesh_construction(NKX, NKY, Lx, Ly):
    """grid.f90:433-448: (NKX*NKY, 3) array of (kx, ky, weight)."""
    out = np.zeros((NKX * NKY, 3))
    check("negf_kmesh", lib().negf_kmesh(NKX, NKY, Lx, Ly, out.ctypes.data_as(_dp)))
    return out


def V_reciprocal_all(V_real, NGX, NGY):
    """LocalPotential_RealToPlanewave (grid.f90:12-69) on every slice plus the
    truncated copy of main.f90:239-247.

    V_real: (N_x, N_y, N_z) real potential in Hartree.  Returns the complex
    (2NGX+1, 2NGY+1, N_z) Fortran-ordered table, zero where |i| > NGX/2 or
    |j| > NGY/2 (entries the reference leaves uninitialised).
    """
    v = np.asfortranarray(V_real, dtype=np.float64)
    Nx, Ny, Nz = v.shape
    out = np.zeros((2 * NGX + 1, 2 * NGY + 1, Nz), np.complex128, order="F")
    rc = lib().negf_vhat(v.ctypes.data_as(_dp), Nx, Ny, Nz, NGX, NGY, out.ctypes.data_as(_dp))
    if rc:
        raise ValueError("'The size of V_reciprocal minus one' must not exceed the real-space grid "
                         "(grid.f90:33-37)")
    return out


def V_reciprocal_all_gpu(V_real, NGX, NGY, device=0):
    """V_reciprocal_all computed on GPU `device` (negf_vhat_gpu): same table up to rounding."""
    v = np.asfortranarray(V_real, dtype=np.float64)
    Nx, Ny, Nz = v.shape
    out = np.zeros((2 * NGX + 1, 2 * NGY + 1, Nz), np.complex128, order="F")
    check("negf_vhat_gpu", lib().negf_vhat_gpu(v.ctypes.data_as(_dp), Nx, Ny, Nz, NGX, NGY, device,
                                               out.ctypes.data_as(_dp)))
    return out


def Greensfunction_PlanewaveToReal(subGreenFunc, nx_grid, ny_grid, N_x, N_y):
    """grid.f90:71-135 for one or more slices: (N,N[,Nz]) -> (N_x,N_y[,Nz]) complex."""
    g = np.asfortranarray(subGreenFunc, dtype=np.complex128)
    squeeze = g.ndim == 2
    if squeeze:
        g = g[:, :, None]
    N, _, nzs = g.shape
    out = np.zeros((N_x, N_y, nzs), np.complex128, order="F")
    check("negf_ptor", lib().negf_ptor(
        g.ctypes.data_as(_dp), np.ascontiguousarray(nx_grid, np.int32).ctypes.data_as(_ip),
        np.ascontiguousarray(ny_grid, np.int32).ctypes.data_as(_ip), N, nzs, N_x, N_y,
        out.ctypes.data_as(_dp)))
    return out[:, :, 0] if squeeze else out


def PlaneWaveBasis_k(ENCUT, Lx, Ly, kx, ky):
    """Per-k basis |k+G|^2/2 <= ENCUT in the reference's enumeration order."""
    n = C.c_int32(0)
    check("negf_basis_k", lib().negf_basis_k(ENCUT, Lx, Ly, kx, ky, 0, C.byref(n), None, None))
    nx = np.zeros(n.value, np.int32)
    ny = np.zeros(n.value, np.int32)
    cnt = C.c_int32(0)
    check("negf_basis_k", lib().negf_basis_k(ENCUT, Lx, Ly, kx, ky, n.value, C.byref(cnt),
                                              nx.ctypes.data_as(_ip), ny.ctypes.data_as(_ip)))
    return nx, ny
