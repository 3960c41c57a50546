"""Surrogate-guided adaptive energy sampling for the transmission integral.

No counterpart in the reference: NEGFtrans evaluates T(E) on the uniform grid
E_i = E1 + (E2 - E1)(i - 1)/N_E (main.f90:369-375) and every point costs one
RGF sweep.  Here a small network, trained on the GPU by this package's own
kernels (include/negf_mlp.h) on RGF outputs of seeded QPC + disorder
devices, predicts log T(E) and the LDOS at 8 probe sites of the constriction
plane for an unseen device from 16 descriptors of its potential; the
prediction only decides WHERE the RGF is evaluated (node density from the
predicted curvature), and every reported point, as well as the integral,
comes from RGF solves.

Devices: the split-gate QPC of ``workloads.qpc_potential`` in the 100 x 100 nm
cell (GaAs by input scaling), V_g ~ U[20, 80] meV, w ~ U[8, 25] nm, 2 meV /
10 nm disorder with its own seed, N = 69 plane waves, N_z slices of 1 nm.
Descriptors: |V^(m, n)| of the constriction plane (z = 0) for the 14 lowest
2-D Fourier modes (meV), V_g (meV) and w (nm).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from . import prepare as P
from .constants import A_0, HARTREE
from .negf import Engine
from .workloads import MSTAR, _deck, qpc_potential

ENCUT_N69 = 0.0033091          # eV (m*-scaled INPUT): 69 plane waves in the 1000 A cell
E_MAX_MEV = 30.0               # energy window [0, E_MAX_MEV) meV
T_FLOOR = 0.01                 # the network predicts log(T + T_FLOOR)
MODES = [(0, 0), (1, 0), (0, 1), (1, 1), (2, 0), (0, 2), (2, 1), (1, 2), (2, 2), (3, 0), (0, 3), (3, 1),
         (1, 3), (4, 0)]
N_PROBES = 8
WIDTHS = [17, 256, 256, 256, 256, 1 + N_PROBES]  # energy + 16 descriptors -> 4 GELU layers -> log T, log LDOS
LDOS_FLOOR = 1e-3              # the network predicts log(LDOS / LDOS_ref + LDOS_FLOOR)
GRID = 64                      # real-space grid of the POTENTIAL (x, y)


def probe_sites(grid=GRID):
    """(x, y) grid indices of the 8 LDOS probes: along x from the channel axis
    outwards (0 ... 22 nm in steps of 3.1 nm) at the cell's centre line in y."""
    return [(grid // 2 + 2 * i, grid // 2) for i in range(N_PROBES)]
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)


# ------------------------------------------------------------------ network
class MLP:
    """The C-ABI network (negf_mlp_*): BF16 products, FP32 accumulation and
    FP32 Adam master weights, all on the GPU."""

    def __init__(self, widths, max_batch=8192, device=0, seed=0):
        self.widths = [int(w) for w in widths]
        h = C.c_void_p()
        arr = (C.c_int32 * len(self.widths))(*self.widths)
        _lib.check("negf_mlp_create", _lib.lib().negf_mlp_create(len(self.widths) - 1, arr, max_batch, device,
                                                               C.byref(h)))
        self._h = h
        self.max_batch = max_batch
        self.n_params = int(_lib.lib().negf_mlp_param_count(h))
        self.params = self.init_params(seed)

    def init_params(self, seed):
        """Uniform(-a, a) weights with a = sqrt(6 / fan_in) (scaled for GELU), zero biases."""
        rng = np.random.Generator(np.random.PCG64(seed))
        parts = []
        for a, b in zip(self.widths[:-1], self.widths[1:]):
            lim = np.sqrt(6.0 / a) * (1.0 if b != self.widths[-1] else 0.5)
            parts += [rng.uniform(-lim, lim, a * b), np.zeros(b)]
        return np.concatenate(parts).astype(np.float32)

    @property
    def params(self):
        out = np.empty(self.n_params, np.float32)
        _lib.check("negf_mlp_get_params", _lib.lib().negf_mlp_get_params(self._h, out.ctypes.data_as(_fp)))
        return out

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        _lib.check("negf_mlp_set_params", _lib.lib().negf_mlp_set_params(self._h, p.ctypes.data_as(_fp)))

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.empty((x.shape[0], self.widths[-1]), np.float32)
        _lib.check("negf_mlp_forward", _lib.lib().negf_mlp_forward(self._h, x.ctypes.data_as(_fp), x.shape[0],
                                                                 y.ctypes.data_as(_fp)))
        return y

    def grad(self, x, t, w):
        x, t, w = (np.ascontiguousarray(a, np.float32) for a in (x, t, w))
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        _lib.check("negf_mlp_grad", _lib.lib().negf_mlp_grad(
            self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), w.ctypes.data_as(_fp), x.shape[0],
            C.byref(loss), g.ctypes.data_as(_fp)))
        return loss.value, g

    def train(self, x, t, w, steps, batch=4096, lr=1e-3, seed=0):
        x, t, w = (np.ascontiguousarray(a, np.float32) for a in (x, t, w))
        losses = np.zeros(max(steps, 1))
        _lib.check("negf_mlp_train", _lib.lib().negf_mlp_train(
            self._h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp), w.ctypes.data_as(_fp), x.shape[0],
            min(batch, self.max_batch), steps, lr, seed, losses.ctypes.data_as(_dp)))
        return losses[:steps]

    def close(self):
        if self._h:
            _lib.lib().negf_mlp_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ devices
@dataclass
class QPCDevice:
    Vg: float        # eV (physical)
    w: float         # nm
    seed: int        # disorder seed
    nz: int
    V_eV: np.ndarray  # POTENTIAL (m*-scaled), eV
    desc: np.ndarray  # 16 descriptors


def descriptors(V_eV, Vg, w):
    """14 lowest-mode |V^| of the constriction plane (physical meV), V_g (meV), w (nm)."""
    plane = np.asarray(V_eV)[:, :, V_eV.shape[2] // 2] / MSTAR
    F = np.fft.fft2(plane) / plane.size
    nx, ny = plane.shape
    d = [abs(F[m % nx, n % ny]) * 1e3 for m, n in MODES]
    return np.array(d + [Vg * 1e3, w], np.float64)


def sample_devices(n, seed, nz=100, grid=64, disorder=0.002, sz_nm=15.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        vg = rng.uniform(0.020, 0.080)
        w = rng.uniform(8.0, 25.0)
        ds = int(rng.integers(1, 2 ** 31 - 1))
        V = MSTAR * qpc_potential(grid, grid, nz, 100.0, nz * 1.0, vg, w, sz_nm, disorder=disorder, seed=ds)
        out.append(QPCDevice(vg, w, ds, nz, V, descriptors(V, vg, w)))
    return out


def energies_hartree(e_mev):
    return MSTAR * np.asarray(e_mev, np.float64) * 1e-3 / HARTREE


class RGF:
    """RGF transmission of one device on the GPU (the ground truth of every point)."""

    def __init__(self, dev: QPCDevice, device=0):
        deck = _deck(dev.nz * 10.0, ENCUT_N69, E_MAX_MEV, 16)
        self.pr = P.prepare(deck, dev.V_eV)
        self.eng = Engine(*self.pr.engine_args(), device=device)
        self.solves = 0

    def T(self, e_mev):
        e = energies_hartree(e_mev)
        tau, info = self.eng.transmission(e)
        self.solves += len(e)
        if info:
            raise RuntimeError(f"zero pivot in the RGF sweep (info {info})")
        return np.asarray(tau)

    def ldos_probes(self, n_e):
        """LDOS (Angstrom^-3 eV^-1, physical units) at the probe sites of the
        constriction slice z = N_z/2 on the grid E_i = E_MAX i / n_e, i < n_e
        (main.f90:417-554 with LDOS_GRID = 0 0 N_z/2+1): shape (n_e, 8)."""
        a = self.pr.atomic
        Nx, Ny, Nz = self.pr.shape
        L = self.eng.ldos(0.0, float(energies_hartree(E_MAX_MEV)), n_e, (0, 0, Nz // 2 + 1), Nx, Ny,
                          a.LX * A_0, a.LY * A_0, a.LZ * A_0)[0]
        self.solves += n_e * len(self.pr.kpoint)
        # LDOS per scaled eV -> per physical eV (E' = m* E)
        return np.stack([L[x, y, 0, :] for x, y in probe_sites(Nx)], axis=1) * MSTAR

    def close(self):
        self.eng.close()


# ------------------------------------------------------------------ surrogate
class Surrogate:
    """Normalisation + network: (E, descriptors) -> log(T + T_FLOOR) and
    log(LDOS / LDOS_ref + LDOS_FLOOR) at the probe sites."""

    def __init__(self, device=0, seed=0, widths=WIDTHS, max_batch=8192):
        self.net = MLP(widths, max_batch=max_batch, device=device, seed=seed)
        self.mu = None
        self.sd = None
        self.ldos_ref = 1.0

    def features(self, desc, e_mev):
        e = np.asarray(e_mev, np.float64)
        d = np.broadcast_to((desc - self.mu) / self.sd, (len(e), len(desc)))
        return np.concatenate([(e[:, None] / E_MAX_MEV) * 2 - 1, d], axis=1).astype(np.float32)

    def fit(self, devices, e_mev, T, ldos=None, steps=(2000, 1000), lr=(1e-3, 2e-4), batch=4096, seed=0):
        """T[i, j] = RGF transmission of devices[i] at e_mev[j], ldos[i, j, p] the
        probe LDOS there (None: the LDOS outputs get zero weight); returns the
        loss history."""
        D = np.stack([d.desc for d in devices])
        self.mu, self.sd = D.mean(axis=0), D.std(axis=0) + 1e-9
        X = np.concatenate([self.features(d.desc, e_mev) for d in devices])
        yt = np.log(np.asarray(T, np.float64).reshape(-1, 1) + T_FLOOR)
        n_out = self.net.widths[-1]
        if ldos is not None and n_out > 1:
            L = np.asarray(ldos, np.float64).reshape(-1, n_out - 1)
            self.ldos_ref = float(np.median(L[L > 0])) if np.any(L > 0) else 1.0
            yl = np.log(np.maximum(L, 0.0) / self.ldos_ref + LDOS_FLOOR)
            Wt = np.ones((len(yt), n_out), np.float32)
        else:
            yl = np.zeros((len(yt), n_out - 1))
            Wt = np.zeros((len(yt), n_out), np.float32)
            Wt[:, 0] = 1.0
        Y = np.concatenate([yt, yl], axis=1).astype(np.float32)
        hist = []
        for s, (n, r) in enumerate(zip(steps, lr)):
            hist.append(self.net.train(X, Y, Wt, n, batch=batch, lr=r, seed=seed + s))
        return np.concatenate(hist)

    def predict(self, desc, e_mev):
        y = self.net.forward(self.features(desc, e_mev))[:, 0].astype(np.float64)
        return np.maximum(np.exp(y) - T_FLOOR, 0.0)

    def predict_ldos(self, desc, e_mev):
        """Probe LDOS (n_e, 8) in the units of RGF.ldos_probes."""
        y = self.net.forward(self.features(desc, e_mev))[:, 1:].astype(np.float64)
        return np.maximum(np.exp(y) - LDOS_FLOOR, 0.0) * self.ldos_ref

    def close(self):
        self.net.close()


# ------------------------------------------------------------------ sampling
def trapezoid(e, t):
    e, t = np.asarray(e), np.asarray(t)
    return float(np.sum(0.5 * (t[1:] + t[:-1]) * np.diff(e)))


def simpson(e, t):
    """Composite Simpson on an odd number of equally spaced points."""
    t = np.asarray(t)
    h = (e[-1] - e[0]) / (len(e) - 1)
    return float(h / 3 * (t[0] + t[-1] + 4 * t[1:-1:2].sum() + 2 * t[2:-1:2].sum()))


def uniform_nodes(n, e_lo=0.0, e_hi=E_MAX_MEV):
    return np.linspace(e_lo, e_hi, n)


def curvature_nodes(e_dense, t_dense, n, floor=0.05):
    """n nodes (ends included) equidistributing the trapezoid error: density
    proportional to (|T''| + floor * mean |T''|)^(1/3) of the predicted curve."""
    h = e_dense[1] - e_dense[0]
    d2 = np.zeros_like(t_dense)
    d2[1:-1] = np.abs(t_dense[2:] - 2 * t_dense[1:-1] + t_dense[:-2]) / h ** 2
    d2[0], d2[-1] = d2[1], d2[-2]
    k = np.ones(9) / 9
    d2 = np.convolve(d2, k, mode="same")
    # floor: a share of the mean curvature, and a tiny absolute term so that a
    # straight line (curvature at rounding level) gives uniform nodes
    tiny = 1e-6 * (np.max(np.abs(t_dense)) + 1e-30) / (e_dense[-1] - e_dense[0]) ** 2
    rho = (d2 + floor * d2.mean() + tiny) ** (1.0 / 3.0)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (rho[1:] + rho[:-1]) * np.diff(e_dense))])
    cdf /= cdf[-1]
    nodes = np.interp(np.linspace(0.0, 1.0, n), cdf, e_dense)
    nodes[0], nodes[-1] = e_dense[0], e_dense[-1]
    return np.unique(nodes)


CANDIDATES = (9, 13, 17, 25, 33, 49, 65, 97, 129, 193, 257, 385, 513, 769, 1025, 1537, 2049)


def solves_to_tolerance(rgf: RGF, i_ref, node_fn, tol, candidates=CANDIDATES):
    """Smallest candidate n whose grid (node_fn(n)) gives |I - I_ref| <= tol * |I_ref|
    for it and every larger candidate tried; every grid point is an RGF solve.
    Returns (n, relative errors per candidate)."""
    errs = []
    for n in candidates:
        e = node_fn(n)
        errs.append(abs(trapezoid(e, rgf.T(e)) - i_ref) / abs(i_ref))
    errs = np.array(errs)
    ok = errs <= tol
    for j in range(len(candidates)):
        if ok[j:].all():
            return candidates[j], errs
    return None, errs


def reference_integral(rgf: RGF, n_fine=4097):
    e = uniform_nodes(n_fine)
    return simpson(e, rgf.T(e))


def compare(sur: Surrogate, devices, tol=1e-4, n_dense=4096, device=0):
    """Per unseen device: RGF solves needed for the integral tolerance with
    uniform nodes and with surrogate-placed nodes, and the surrogate's own
    error at the adaptive nodes."""
    rows = []
    e_dense = np.linspace(0.0, E_MAX_MEV, n_dense)
    for dev in devices:
        rgf = RGF(dev, device=device)
        try:
            i_ref = reference_integral(rgf)
            n_u, err_u = solves_to_tolerance(rgf, i_ref, uniform_nodes, tol)
            t_pred = sur.predict(dev.desc, e_dense)
            n_a, err_a = solves_to_tolerance(rgf, i_ref, lambda n: curvature_nodes(e_dense, t_pred, n), tol)
            e_chk = curvature_nodes(e_dense, t_pred, 65)
            t_chk = rgf.T(e_chk)
            surr_err = float(np.max(np.abs(sur.predict(dev.desc, e_chk) - t_chk)))
            rows.append({"Vg_meV": dev.Vg * 1e3, "w_nm": dev.w, "integral": i_ref, "uniform": n_u,
                         "adaptive": n_a, "surrogate_max_abs_err": surr_err})
        finally:
            rgf.close()
    return rows


def training_energies(n_e):
    """The grid E_i = E_MAX i / n_e (i < n_e) of both training targets (meV)."""
    return E_MAX_MEV * np.arange(n_e) / n_e


def training_set(devices, n_e, device=0, with_ldos=True):
    """RGF transmission (n_dev, n_e) and probe LDOS (n_dev, n_e, 8) on training_energies(n_e)."""
    e_mev = training_energies(n_e)
    T = np.zeros((len(devices), n_e))
    L = np.zeros((len(devices), n_e, N_PROBES)) if with_ldos else None
    for i, dev in enumerate(devices):
        rgf = RGF(dev, device=device)
        try:
            T[i] = rgf.T(e_mev)
            if with_ldos:
                L[i] = rgf.ldos_probes(n_e)
        finally:
            rgf.close()
    return T, L
