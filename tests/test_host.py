"""Host-side mirror of the reference set-up (CPU): basis, k-mesh, V table,
PtoR, unit conversion and INPUT checks, against the oracle and the formulas
of src/main.f90."""
import math

import numpy as np
import pytest

from negftrans_b200 import A_0, HARTREE, K_B, PI
from negftrans_b200 import grid as G
from negftrans_b200 import prepare as P
from negftrans_b200 import workloads as W


@pytest.fixture(scope="module", autouse=True)
def _lib(built_lib):
    return built_lib


@pytest.mark.parametrize("encut,l", [(0.0033091, 1000.0), (0.0105288, 1000.0), (0.0385807, 1000.0),
                                     (100.0, 8.0), (3.0, 18.0)])
def test_basis_matches_oracle(oracle, encut, l):
    e, lx, ly = encut / HARTREE, l / A_0, 1.3 * l / A_0
    nx, ny = G.PlaneWaveBasis_construction(e, lx, ly)
    onx, ony = oracle.basis(e, lx, ly)
    assert G.PlaneWaveBasis_construction_findsize(e, lx, ly) == len(onx)
    assert np.array_equal(nx, onx) and np.array_equal(ny, ony)


def test_kmesh_matches_oracle(oracle):
    for nkx, nky in ((1, 1), (4, 4), (1, 6), (3, 2)):
        np.testing.assert_array_equal(G.Kpoint_mesh_construction(nkx, nky, 10.0, 7.0),
                                      oracle.kmesh(nkx, nky, 10.0, 7.0))


@pytest.mark.parametrize("shape,ng", [((16, 12, 3), (6, 5)), ((32, 32, 4), (11, 11)), ((50, 90, 2), (20, 40))])
def test_vhat_matches_oracle(oracle, shape, ng):
    rng = np.random.default_rng(sum(shape))
    v = np.asfortranarray(rng.standard_normal(shape))
    got = G.V_reciprocal_all(v, *ng)
    ref = oracle.vhat_all(v, *ng)
    assert np.max(np.abs(got - ref)) < 1e-14 * np.max(np.abs(ref))
    # zero outside the |i| <= NGX/2, |j| <= NGY/2 window (main.f90:242-244)
    hx, hy = ng[0] // 2, ng[1] // 2
    mask = np.ones(got.shape[:2], bool)
    mask[ng[0] - hx:ng[0] + hx + 1, ng[1] - hy:ng[1] + hy + 1] = False
    assert np.all(got[mask] == 0)


def test_vhat_rejects_oversized_table():
    with pytest.raises(ValueError):
        G.V_reciprocal_all(np.zeros((8, 8, 1)), 5, 2)


@pytest.mark.parametrize("Nx,Ny", [(8, 6), (16, 16)])
def test_ptor_matches_oracle(oracle, Nx, Ny):
    nx, ny = oracle.basis(0.6, 2 * PI, 2 * PI)
    N = len(nx)
    rng = np.random.default_rng(N)
    g = np.asfortranarray(rng.standard_normal((N, N, 2)) + 1j * rng.standard_normal((N, N, 2)))
    got = G.Greensfunction_PlanewaveToReal(g, nx, ny, Nx, Ny)
    for k in range(2):
        ref = oracle.ptor(g[:, :, k], nx, ny, Nx, Ny)
        assert np.max(np.abs(got[:, :, k] - ref)) < 1e-12 * np.max(np.abs(ref))


def test_units_and_ngrid():
    d = P.InputDeck(LX=8.0, LY=18.0, LZ=40.0, ENCUT=100.0, NKX=1, NKY=6, if_transmission=True,
                    TRANSMISSION_GRID=(4.0, 20.0, 200), ETA=1e-6, TEMPERATURE=20.0, GAP=6.0, MU=5.568)
    a = P.to_atomic(d)
    assert a.LX == 8.0 / A_0 and a.LZ == 40.0 / A_0
    assert a.ETA == 1e-6                       # already Hartree (main.f90:187)
    assert a.ENCUT == 100.0 / HARTREE
    assert a.GAP == 6.0 * K_B * 20.0
    assert a.TRANSMISSION_GRID == (4.0 / HARTREE, 20.0 / HARTREE)
    s = math.sqrt(100.0 / HARTREE / 2)
    # main.f90:95-100: NGX is sized from LX but tested against LY
    assert P.ngrid(d) == (math.ceil(8.0 / A_0 / PI * s * 2) + 1, math.ceil(18.0 / A_0 / PI * s * 2) + 1)
    d2 = P.InputDeck(LX=8.0, LY=18.0, ENCUT=100.0, NGX=25, NGY=60)
    lim = math.ceil(18.0 / A_0 / PI * s * 2)
    assert 25 <= lim                      # so NGX=25 is overridden because of LY
    assert P.ngrid(d2)[0] == math.ceil(8.0 / A_0 / PI * s * 2) + 1
    assert P.ngrid(d2)[1] == 60


def test_energy_grid_excludes_endpoint():
    # Manual.tex: TRANSMISSION_GRID = 0.0 2.0 4 -> 0.0, 0.5, 1.0, 1.5
    a = P.to_atomic(P.InputDeck(TRANSMISSION_GRID=(0.0, 2.0, 4)))
    np.testing.assert_allclose(P.transmission_energies(a, 4) * HARTREE, [0.0, 0.5, 1.0, 1.5])


def test_n_line_rounding():
    a = P.to_atomic(P.InputDeck(TEMPERATURE=20.0, GAP=6.0))
    x = 500 * (2 * a.GAP * HARTREE)
    assert P.n_line(a, 500) == int(math.floor(x + 0.5))


def test_validation_messages():
    err = P.validate(P.InputDeck())
    assert any("LX, LY, LZ" in e for e in err) and any("NKX, NKY" in e for e in err)
    assert any("Nothing to do" in e for e in err)
    err = P.validate(P.InputDeck(LX=1, LY=1, LZ=1, NKX=1, NKY=1, if_transmission=True, VDS=0.1))
    assert any("TRANSMISSION_GRID" in e for e in err) and any("VDS" in e for e in err)
    assert P.validate(P.InputDeck(LX=1, LY=1, LZ=1, NKX=1, NKY=1, if_transmission=True,
                                  TRANSMISSION_GRID=(0, 1, 4))) == []


def test_prepare_rejects_odd_grid():
    with pytest.raises(ValueError):
        P.prepare(P.InputDeck(LX=10, LY=10, LZ=10, NKX=1, NKY=1), np.zeros((7, 8, 2)))


def test_workload_shapes():
    for name, n in (("qpc_n69", 69), ("qpc_disorder_n221", 221)):
        w = W.config(name)
        pr = P.prepare(w.deck, w.V_eV)
        assert pr.N == n
        # every pair difference is inside the V table (the engine's precondition)
        assert np.max(np.abs(pr.nx[:, None] - pr.nx[None, :])) <= pr.NGX


def test_uneven_batch_spreads_the_basis_sizes(oracle):
    """cfg 4 with per-k cutoffs: 16 k-points x 3 devices, bases spread over
    180-263 plane waves; every per-k basis is the oracle's basis at its own
    cutoff and k, and the V table covers every pair difference."""
    probs = W.batched_uneven(n_range=(180, 260))
    assert len(probs) == 48 and sorted({p["Nz"] for p in probs}) == [300, 600, 1200]
    sizes = sorted({p["N"] for p in probs})
    assert len(sizes) == 16 and 180 <= sizes[0] <= 185 and 256 < sizes[-1] <= 270
    for p in probs[:16]:
        nx, ny, vhat = p["args"][:3]
        ngx = (vhat.shape[0] - 1) // 2
        assert np.max(np.abs(np.subtract.outer(nx, nx))) <= ngx
        assert np.max(np.abs(np.subtract.outer(ny, ny))) <= (vhat.shape[1] - 1) // 2


def test_disorder_statistics():
    V = W.qpc_potential(32, 32, 64, 100.0, 64.0, 0.0, 15.0, 20.0, disorder=0.002, seed=7)
    assert abs(np.sqrt(np.mean(V ** 2)) - 0.002) < 1e-12
    V2 = W.qpc_potential(32, 32, 64, 100.0, 64.0, 0.0, 15.0, 20.0, disorder=0.002, seed=7)
    assert np.array_equal(V, V2)


def test_emass_key_is_the_input_scaling():
    """EMASS = m* equals the m*-scaled deck with m* = 1 (same table, basis, energies)."""
    import dataclasses
    V = W.qpc_potential(32, 32, 8, 100.0, 8.0, 0.05, 15.0, 1.0, disorder=0.002)
    phys = P.InputDeck(if_transmission=True, LX=1000.0, LY=1000.0, LZ=80.0, ENCUT=1.2e-3 / 0.067,
                       ETA=1e-6 / HARTREE, NKX=1, NKY=2, TEMPERATURE=1.0, MU=0.02,
                       TRANSMISSION_GRID=(0.0, 0.03, 16), EMASS=0.067)
    scaled = dataclasses.replace(phys, ENCUT=1.2e-3, ETA=0.067e-6 / HARTREE, TEMPERATURE=0.067,
                                 MU=0.067 * 0.02, TRANSMISSION_GRID=(0.0, 0.067 * 0.03, 16), EMASS=1.0)
    a = P.prepare(phys, V)
    b = P.prepare(scaled, 0.067 * V)
    assert np.array_equal(a.nx, b.nx) and np.array_equal(a.ny, b.ny)
    assert np.max(np.abs(a.vhat - b.vhat)) <= 1e-15 * np.max(np.abs(b.vhat))
    np.testing.assert_allclose(P.transmission_energies(a.atomic, 16),
                               P.transmission_energies(b.atomic, 16), rtol=1e-15)
    assert math.isclose(a.atomic.ETA, b.atomic.ETA, rel_tol=1e-15)
    assert math.isclose(a.atomic.MU, b.atomic.MU, rel_tol=1e-15)
    assert math.isclose(a.atomic.GAP, b.atomic.GAP, rel_tol=1e-15)
    with pytest.raises(ValueError):
        P.to_atomic(dataclasses.replace(phys, EMASS=-1.0))
