"""FP64 parity at the full sizes of the benchmark workloads.

The fixtures under tests/golden/ were made by tests/golden/make_golden_full.py
from the CPU oracle on the same seeded inputs:

* qpc_disorder_n221 (N = 221, N_z = 800): tau at 15 energies of the 2048-point
  grid, most within 0.02 meV of a lead subband threshold;
* qpc_disorder_n797 (N = 797, N_z = 400): tau at 6 energies of the 1024-point
  grid chosen the same way;
* qpc_n69 (N = 69, N_z = 200): the equilibrium density contour of the deck
  (per-slice fingerprints of Density_Matrix and the density summed over x, y)
  and the LDOS (LDOS_GRID = -1 -1 0) at 8 energies of a 512-point grid.

Tolerance: 1e-9 relative (tau elementwise with a 1e-12 absolute floor;
per-slice fingerprints normwise).
"""
import os

import numpy as np
import pytest

from negftrans_b200 import prepare as P
from negftrans_b200 import workloads as W
from negftrans_b200.negf import Engine

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
RTOL = 1e-9


def _load(name):
    return np.load(os.path.join(HERE, name), allow_pickle=False)


def _inputs(name, ref):
    from golden.make_golden_full import input_fingerprint
    w = W.config(name)
    pr = P.prepare(w.deck, w.V_eV)
    np.testing.assert_allclose(input_fingerprint(pr), ref["inputs"], rtol=1e-12)
    return w, pr


@pytest.mark.parametrize("name", ["qpc_disorder_n221", "qpc_disorder_n797"])
def test_transmission_matches_oracle_at_full_size(name):
    ref = _load(f"oracle_{name}.npz")
    w, pr = _inputs(name, ref)
    grid = P.transmission_energies(pr.atomic, int(ref["grid_size"]))
    E = grid[ref["idx"]]
    np.testing.assert_array_equal(E, ref["energies"])
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    np.testing.assert_allclose(tau, ref["tau"], rtol=RTOL, atol=1e-12)


def test_density_and_ldos_match_oracle_at_full_size():
    from golden.make_golden_full import fingerprints
    ref = _load("oracle_qpc_n69_density_ldos.npz")
    w, pr = _inputs("qpc_n69", ref)
    a, d = pr.atomic, w.deck
    Nx, Ny, Nz = pr.shape
    with Engine(*pr.engine_args()) as eng:
        dens, dm, info = eng.density_real(int(ref["n_circle"]), int(ref["n_line"]), pr.min_V, a.MU, a.GAP,
                                          a.TEMPERATURE, Nx, Ny, d.LX, d.LY, d.LZ)
        assert info == 0
        tr, uv = fingerprints(dm, ref["u"], ref["v"])
        for got, want in ((tr, ref["dm_trace"]), (uv, ref["dm_uv"])):
            assert np.linalg.norm(got - want) <= RTOL * np.linalg.norm(want)
        assert abs(np.linalg.norm(dm) - float(ref["dm_norm"])) <= RTOL * float(ref["dm_norm"])
        dz = dens.sum(axis=(0, 1))
        assert np.linalg.norm(dz - ref["density_z"]) <= RTOL * np.linalg.norm(ref["density_z"])
        ldos, info = eng.ldos(0.0, float(ref["ldos_e_hi"]), int(ref["ldos_n_e"]), (-1, -1, 0), Nx, Ny,
                              d.LX, d.LY, d.LZ)
        assert info == 0
    got = ldos[0, 0, :, ref["ldos_idx"]]            # (n_idx, Nz)
    want = ref["ldos_z"]
    for r in range(len(want)):
        assert np.linalg.norm(got[r] - want[r]) <= RTOL * np.linalg.norm(want[r]), r
