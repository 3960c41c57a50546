"""The once-per-run preparation of src/main.f90 (lines 26-54, 94-100, 184-249,
261, 369-375): INPUT defaults, NGX/NGY sizing, unit conversion, k-mesh, basis,
the V table, and the energy grids.  Inputs are in the reference's INPUT units
(eV, Angstrom, K; ETA in Hartree)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .constants import A_0, HARTREE, K_B, PI
from .grid import Kpoint_mesh_construction, PlaneWaveBasis_construction, V_reciprocal_all


@dataclass
class InputDeck:
    """The &INPUT namelist with the defaults of main.f90:26-50."""
    if_density: bool = False
    if_transmission: bool = False
    if_LDOS: bool = False
    V_L: float = 0.0            # eV
    V_R: float = 0.0            # eV
    MU: float = 5.568           # eV
    ETA: float = 1e-5           # Hartree (not converted, main.f90:187)
    TEMPERATURE: float = 20.0   # K
    LX: float = 0.0             # Angstrom
    LY: float = 0.0
    LZ: float = 0.0
    ENCUT: float = 100.0        # eV
    GAP: float = 6.0            # k_B T
    VDS: float = 0.0            # eV
    TRANSMISSION_GRID: tuple = (0.0, 0.0, 0.0)
    LDOS_ENERGY_GRID: tuple = (0.0, 0.0, 0.0)
    LDOS_GRID: tuple = (-10, -10, -10)
    NGX: int = 0
    NGY: int = 0
    NKX: int = 0
    NKY: int = 0
    N_circle: int = 40
    N_line_per_eV: int = 500
    # Engine key with no reference counterpart: effective mass m*/m_e.  The
    # reference's kinetic term is |k+G|^2/2 (m* = 1, grid.f90:258); EMASS = m*
    # is applied as the exact scaling E' = m* E, V' = m* V, eta' = m* eta,
    # T' = m* T, ENCUT' = m* ENCUT, under which tau and the density are
    # unchanged and the LDOS per eV scales by 1/m*.
    EMASS: float = 1.0


def validate(d: InputDeck):
    """main.f90:102-132; returns the list of error lines (empty when valid)."""
    err = []
    if d.LX == 0 or d.LY == 0 or d.LZ == 0:
        err.append("ERROR: LX, LY, LZ must be specified in INPUT")
    if d.NKX == 0 or d.NKY == 0:
        err.append("ERROR: NKX, NKY must be specified in INPUT")
    if not (d.if_density or d.if_transmission or d.if_LDOS):
        err.append("ERROR: At least one of (if_xxxxx) be .true.   Nothing to do...")
    if d.if_transmission and d.TRANSMISSION_GRID[2] == 0:
        err.append("ERROR: TRANSMISSION_GRID must be specified for (if_transmission = .true.)")
    if d.if_LDOS and d.LDOS_ENERGY_GRID[2] == 0:
        err.append("ERROR: LDOS_ENERGY_GRID must be specified for (if_LDOS = .true.)")
    if d.if_LDOS and min(d.LDOS_GRID) < -1:
        err.append("ERROR: LDOS_GRID must be specified for (if_LDOS = .true.)")
    if d.VDS != 0:
        err.append("ERROR: VDS must be zero in this version, please upgrade to higher version.")
    return err


def ngrid(d: InputDeck):
    """NGX, NGY after main.f90:94-100 (the NGX test reads LY, as the reference does)."""
    s = math.sqrt(d.ENCUT / HARTREE / 2)
    ngx, ngy = d.NGX, d.NGY
    if ngx <= math.ceil((d.LY / A_0) / PI * s * 2):
        ngx = math.ceil((d.LX / A_0) / PI * s * 2) + 1
    if ngy <= math.ceil((d.LY / A_0) / PI * s * 2):
        ngy = math.ceil((d.LY / A_0) / PI * s * 2) + 1
    return ngx, ngy


@dataclass
class Atomic:
    """t_parameters after the unit conversion of main.f90:184-198."""
    V_L: float
    V_R: float
    MU: float
    ETA: float
    TEMPERATURE: float
    LX: float
    LY: float
    LZ: float
    ENCUT: float
    GAP: float
    VDS: float
    TRANSMISSION_GRID: tuple
    LDOS_ENERGY_GRID: tuple


@dataclass
class Prepared:
    atomic: Atomic
    nx: np.ndarray
    ny: np.ndarray
    kpoint: np.ndarray
    vhat: np.ndarray
    NGX: int
    NGY: int
    min_V: float            # minval(V_real) in Hartree
    shape: tuple            # (N_x, N_y, N_z)
    extra: dict = field(default_factory=dict)

    @property
    def N(self):
        return len(self.nx)

    @property
    def Nz(self):
        return self.vhat.shape[2]

    def engine_args(self):
        a = self.atomic
        return (self.nx, self.ny, self.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, self.kpoint)


def scaled_deck(d: InputDeck) -> InputDeck:
    """The m* = 1 deck equivalent to d (EMASS folded into the energy scale)."""
    import dataclasses
    m = d.EMASS
    if m == 1.0:
        return d
    if not m > 0:
        raise ValueError("EMASS must be positive")
    return dataclasses.replace(
        d, V_L=m * d.V_L, V_R=m * d.V_R, MU=m * d.MU, ETA=m * d.ETA, TEMPERATURE=m * d.TEMPERATURE,
        ENCUT=m * d.ENCUT, VDS=m * d.VDS,
        TRANSMISSION_GRID=(m * d.TRANSMISSION_GRID[0], m * d.TRANSMISSION_GRID[1], d.TRANSMISSION_GRID[2]),
        LDOS_ENERGY_GRID=(m * d.LDOS_ENERGY_GRID[0], m * d.LDOS_ENERGY_GRID[1], d.LDOS_ENERGY_GRID[2]),
        N_line_per_eV=int(math.floor(d.N_line_per_eV / m + 0.5)), EMASS=1.0)


def to_atomic(d: InputDeck) -> Atomic:
    d = scaled_deck(d)
    return Atomic(
        V_L=d.V_L / HARTREE, V_R=d.V_R / HARTREE, MU=d.MU / HARTREE, ETA=d.ETA,
        TEMPERATURE=d.TEMPERATURE, LX=d.LX / A_0, LY=d.LY / A_0, LZ=d.LZ / A_0,
        ENCUT=d.ENCUT / HARTREE, GAP=d.GAP * K_B * d.TEMPERATURE, VDS=d.VDS / HARTREE,
        TRANSMISSION_GRID=(d.TRANSMISSION_GRID[0] / HARTREE, d.TRANSMISSION_GRID[1] / HARTREE),
        LDOS_ENERGY_GRID=(d.LDOS_ENERGY_GRID[0] / HARTREE, d.LDOS_ENERGY_GRID[1] / HARTREE))


def prepare(d: InputDeck, V_real_eV) -> Prepared:
    """main.f90:94-249 for a deck and a POTENTIAL array (N_x, N_y, N_z) in eV."""
    v = np.asfortranarray(V_real_eV, dtype=np.float64) * scaled_deck_factor(d)
    Nx, Ny, Nz = v.shape
    if Nx % 2 or Ny % 2:
        raise ValueError("The number of grid point in x & y direction must be even number")
    a = to_atomic(d)
    ngx, ngy = ngrid(scaled_deck(d))
    vh = v / HARTREE
    kp = Kpoint_mesh_construction(d.NKX, d.NKY, a.LX, a.LY)
    nx, ny = PlaneWaveBasis_construction(a.ENCUT, a.LX, a.LY)
    vhat = V_reciprocal_all(vh, ngx, ngy)
    return Prepared(a, nx, ny, kp, vhat, ngx, ngy, float(vh.min()), (Nx, Ny, Nz))


def scaled_deck_factor(d: InputDeck) -> float:
    """Factor applied to POTENTIAL values by EMASS (1 for the reference)."""
    return float(d.EMASS)


def transmission_energies(atomic: Atomic, n_e: int):
    """main.f90:369-375: E_i = E1 + (E2-E1)(i-1)/N_E, last point excluded (Hartree)."""
    e1, e2 = atomic.TRANSMISSION_GRID
    return np.array([e1 + (e2 - e1) * i / n_e for i in range(n_e)])


def n_line(atomic: Atomic, N_line_per_eV: int) -> int:
    """main.f90:261: IDNINT(N_line_per_eV * 2 * GAP[eV])."""
    x = N_line_per_eV * ((2 * atomic.GAP) * HARTREE)
    return int(math.floor(x + 0.5)) if x >= 0 else -int(math.floor(-x + 0.5))
