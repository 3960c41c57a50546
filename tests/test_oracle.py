"""Pins of the CPU oracle (CPU only).

The reference ships no golden outputs and cannot be built here, so the oracle
is pinned against known answers that follow from the algorithm itself:
a dense inverse of the block-tridiagonal matrix, the closed-form mode
recursion for z-only potentials, exact quadrature rules, and the QPC
testcase's generator arithmetic; plus the committed fixtures in tests/golden.
"""
import os

import numpy as np
import pytest

from negftrans_b200 import HARTREE, A_0, PI

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("N,Nz", [(1, 2), (3, 2), (4, 5), (7, 9)])
def test_tri_solver_matches_dense_inverse(oracle, N, Nz):
    rng = np.random.default_rng(N * 10 + Nz)
    D = rng.standard_normal((N, N, Nz)) + 1j * rng.standard_normal((N, N, Nz))
    outs, info = oracle.tri_solver(D, "DFL")
    dg, fc, lc = oracle.dense_blocks(D)
    assert info == 0
    assert rel(outs["D"], dg) < 1e-12
    assert rel(outs["F"], fc) < 1e-12
    assert rel(outs["L"], lc) < 1e-12


def test_tri_solver_rejects_single_slice(oracle):
    with pytest.raises(ValueError):
        oracle.tri_solver(np.ones((2, 2, 1), complex), "F")


def test_tri_solver_reports_singular(oracle):
    D = np.zeros((3, 3, 3), complex)
    _, info = oracle.tri_solver(D, "F")
    assert info > 0


def _zonly_problem(oracle, nz=20, grid=16, nk=(1, 1), vl=0.0, vr=0.0):
    lx = ly = 400 / A_0
    lz = nz * 10 / A_0
    encut = 0.05 / HARTREE
    nx, ny = oracle.basis(encut, lx, ly)
    z = np.arange(nz) + 0.5 - nz / 2
    vz = 0.03 / HARTREE * np.exp(-z ** 2 / 20.0)
    vreal = np.asfortranarray(np.broadcast_to(vz[None, None, :], (grid, grid, nz)))
    ng = 5
    vh = oracle.vhat_all(vreal, ng, ng)
    kp = oracle.kmesh(nk[0], nk[1], lx, ly)
    p = oracle.Problem(nx, ny, vh, lx, ly, lz, vl, vr, 1e-6 / HARTREE, kp)
    return p, vh[ng, ng, :]


@pytest.mark.parametrize("nk", [(1, 1), (2, 3)])
def test_transmission_closed_form_zonly(oracle, nk):
    p, vz00 = _zonly_problem(oracle, nk=nk)
    E = np.array([0.005, 0.02, 0.035, 0.06]) / HARTREE
    tau, info = oracle.transmission_jobs(p, E, nthreads=2)
    assert info == 0
    cf = np.zeros(len(E))
    for kx, ky, w in p.kpt:
        cf += w * np.array([oracle.closed_form_tau(p.nx, p.ny, vz00, p.Lx, p.Ly, p.Lz, p.V_L, p.V_R,
                                                   p.eta, e, kx, ky) for e in E])
    np.testing.assert_allclose(tau, cf, rtol=1e-10, atol=1e-13)


def test_transmission_closed_form_unequal_leads(oracle):
    p, vz00 = _zonly_problem(oracle, vl=0.002 / HARTREE, vr=0.004 / HARTREE)
    E = np.array([0.01, 0.03]) / HARTREE
    tau, _ = oracle.transmission_jobs(p, E)
    cf = [oracle.closed_form_tau(p.nx, p.ny, vz00, p.Lx, p.Ly, p.Lz, p.V_L, p.V_R, p.eta, e, 0, 0)
          for e in E]
    np.testing.assert_allclose(tau, cf, rtol=1e-10)


def test_diag_closed_form_zonly(oracle):
    p, vz00 = _zonly_problem(oracle, nz=12)
    e = 0.02 / HARTREE
    H = oracle.hamiltonian(p, 0.0, 0.0)
    D = oracle.e_minus_h(p, H, e + 1j * p.eta, 0.0, 0.0)
    outs, _ = oracle.tri_solver(D, "DF")
    dz = p.Lz / p.Nz
    _, gd, _, _ = oracle.closed_form_modes(p.nx, p.ny, vz00, p.Lx, p.Ly, p.Lz, p.V_L, p.V_R, p.eta,
                                           e, 0, 0)
    diag = np.array([np.diag(outs["D"][:, :, k]) for k in range(p.Nz)]).T * 2 * dz ** 2
    np.testing.assert_allclose(diag, gd, rtol=1e-10)
    # off-diagonal elements vanish: H is diagonal in the plane-wave basis
    off = outs["D"].copy()
    for k in range(p.Nz):
        np.fill_diagonal(off[:, :, k], 0)
    assert np.max(np.abs(off)) < 1e-12 * np.max(np.abs(outs["D"]))


def test_transmission_bounded_by_open_channels(oracle):
    p, _ = _zonly_problem(oracle)
    E = np.linspace(0.001, 0.06, 7) / HARTREE
    tau, _ = oracle.transmission_jobs(p, E)
    for e, t in zip(E, tau):
        eps = ((2.0 * p.nx * PI / p.Lx) ** 2 + (2.0 * p.ny * PI / p.Ly) ** 2) / 2
        assert -1e-12 <= t <= np.sum(eps < e) + 1e-9


def test_simpson_rules(oracle):
    for n in (3, 5, 9, 41):      # odd: composite 1/3, exact for cubics
        c = [oracle.coefficient_simpson(i, n, 0.0, 2.0) for i in range(1, n + 1)]
        x = [oracle.value_simpson(i, n, 0.0, 2.0) for i in range(1, n + 1)]
        assert abs(sum(c) - 2.0) < 1e-14
        assert abs(np.dot(c, np.array(x) ** 3) - 4.0) < 1e-12
    for n in (6, 8, 256):        # even: 1/3 up to N-3 plus a 3/8 tail, exact for cubics
        c = [oracle.coefficient_simpson(i, n, 0.0, 2.0) for i in range(1, n + 1)]
        x = [oracle.value_simpson(i, n, 0.0, 2.0) for i in range(1, n + 1)]
        assert abs(sum(c) - 2.0) < 1e-13
        assert abs(np.dot(c, np.array(x) ** 3) - 4.0) < 1e-11
    # N = 4: i == 1 takes the first branch, so the weights are 1/3, 9/8, 9/8, 3/8
    c4 = [oracle.coefficient_simpson(i, 4, 0.0, 3.0) for i in range(1, 5)]
    np.testing.assert_allclose(c4, [1 / 3, 9 / 8, 9 / 8, 3 / 8])


def test_fermi(oracle):
    assert oracle.fermi_func(0.1, 0.1, 300.0) == 0.5
    kT = 8.617333262e-5 / HARTREE * 300.0
    assert abs(oracle.fermi_func(0.1 + kT, 0.1, 300.0) - 1 / (np.e + 1)) < 1e-15


def test_basis_sizes_and_order(oracle):
    lx = ly = 1000 / A_0
    for enc, n in ((0.0033091, 69), (0.0105288, 221), (0.0385807, 797)):
        nx, ny = oracle.basis(enc / HARTREE, lx, ly)
        assert len(nx) == n
        # j outer, i inner (grid.f90:420-429)
        key = ny.astype(np.int64) * 100000 + nx
        assert np.all(np.diff(key) > 0)


def test_kmesh(oracle):
    lx, ly = 10.0, 20.0
    k = oracle.kmesh(2, 3, lx, ly)
    assert k.shape == (6, 3)
    np.testing.assert_allclose(k[:, 2], 1 / 6)
    np.testing.assert_allclose(k[0, :2], [(1 - 1.5) / 2 * 2 * PI / lx, (1 - 2.0) / 3 * 2 * PI / ly])
    np.testing.assert_allclose(k[5, :2], [(2 - 1.5) / 2 * 2 * PI / lx, (3 - 2.0) / 3 * 2 * PI / ly])


def test_rtop_known_potentials(oracle):
    Nx, Ny = 16, 12
    v = np.full((Nx, Ny), 0.3)
    vr = oracle.rtop(v, 4, 3)
    assert abs(vr[4, 3] - 0.3) < 1e-15
    vr[4, 3] = 0
    assert np.max(np.abs(vr)) < 1e-15
    x = np.arange(Nx)
    y = np.arange(Ny)
    v = 0.2 * np.cos(2 * PI * x / Nx)[:, None] + 0.1 * np.sin(2 * PI * 2 * y / Ny)[None, :]
    vr = oracle.rtop(v, 4, 3)
    assert abs(vr[4 + 1, 3] - 0.1) < 1e-15 and abs(vr[4 - 1, 3] - 0.1) < 1e-15
    # sin(2 pi 2 y / Ny) = (e^{+i..} - e^{-i..}) / 2i -> V(0, 2) = 0.1/(2i)
    assert abs(vr[4, 3 + 2] - 0.1 / 2j) < 1e-15 and abs(vr[4, 3 - 2] + 0.1 / 2j) < 1e-15
    with pytest.raises(ValueError):
        oracle.rtop(v, 9, 3)   # 2*NGX > N_x (grid.f90:33-37)


def test_ptor_identity(oracle):
    nx = np.array([0, 1, -1, 0], np.int32)
    ny = np.array([0, 0, 0, 1], np.int32)
    out = oracle.ptor(np.eye(4, dtype=complex), nx, ny, 8, 6)
    np.testing.assert_allclose(out, 4.0, atol=1e-13)


def test_qpc_testcase_generator_levels():
    """testcase/potential_QPC.f90:34-39 prints the plateau onsets
    E = gap_x/2 + gap_y (n_y + 1/2) eV for n_x = 1; restated."""
    gap_x, gap_y = 12.0, 2.0
    levels = [gap_x * 0.5 + gap_y * (i + 0.5) for i in range(7)]
    assert levels == [7.0, 9.0, 11.0, 13.0, 15.0, 17.0, 19.0]


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLD, "oracle_small.npz")),
                    reason="golden fixtures not generated")
def test_golden_fixtures(oracle):
    """The committed fixtures (tests/golden/make_golden.py) are reproduced."""
    g = np.load(os.path.join(GOLD, "oracle_small.npz"))
    p = oracle.Problem(g["nx"], g["ny"], g["vhat"], *g["params"], g["kpt"])
    tau, _ = oracle.transmission_jobs(p, g["energies"])
    np.testing.assert_allclose(tau, g["tau"], rtol=1e-12, atol=1e-15)
    outs, _ = oracle.tri_solver(g["D"], "DFL")
    for k in "DFL":
        assert rel(outs[k], g["tri_" + k]) < 1e-12
    dm, _ = oracle.density_jobs(p, int(g["n_circle"]), int(g["n_line"]), float(g["min_v"]),
                                float(g["mu"]), float(g["gap"]), float(g["temperature"]))
    assert rel(dm, g["dm"]) < 1e-12


def test_lattice_leads_closed_form_is_unitary(oracle):
    """With the exact lattice lead term a flat device transmits every open
    lattice channel fully: tau = number of modes with |d| < 2 (pins the closed
    form used to check the engine's lead_model = 1)."""
    lx = ly = 400 / A_0
    nz = 12
    lz = nz * 10 / A_0
    nx, ny = oracle.basis(0.05 / HARTREE, lx, ly)
    vz = np.zeros(nz)
    dz = lz / nz
    for e in (0.004 / HARTREE, 0.03 / HARTREE):
        t = oracle.closed_form_tau(nx, ny, vz, lx, ly, lz, 0.0, 0.0, 1e-12, e, 0.0, 0.0, lattice=True)
        eps = ((2.0 * nx * PI / lx) ** 2 + (2.0 * ny * PI / ly) ** 2) / 2
        d = 2 * dz * dz * (e - eps) - 2
        assert abs(t - np.sum(np.abs(d) < 2)) < 1e-4   # eta absorbs a little near band edges
        # the reference's continuum lead term reflects a little at the ends
        t_ref = oracle.closed_form_tau(nx, ny, vz, lx, ly, lz, 0.0, 0.0, 1e-12, e, 0.0, 0.0)
        assert t_ref <= t + 1e-9


def _xy_problem(oracle, nz=6, eta=1e-6 / HARTREE, symmetric=True, vl=0.0, vr=0.0, nk=(1, 2)):
    """A small device whose potential varies in x, y and z (plane-wave blocks are dense);
    symmetric=True makes it even under slice reversal."""
    lx = ly = 400 / A_0
    lz = nz * 10 / A_0
    nx, ny = oracle.basis(0.03 / HARTREE, lx, ly)
    g = 16
    x = (np.arange(g) - g / 2) / g
    z = np.arange(nz) + 0.5 - nz / 2 if symmetric else np.arange(nz) * 0.7 - 1.0
    V = (0.02 / HARTREE * (1 - np.exp(-x[:, None, None] ** 2 / 0.02)) * np.exp(-z[None, None, :] ** 2 / 4.0)
         * (1 + 0.3 * np.cos(2 * PI * x[None, :, None])))
    vh = oracle.vhat_all(np.asfortranarray(V), 5, 5)
    kp = oracle.kmesh(nk[0], nk[1], lx, ly)
    return oracle.Problem(nx, ny, vh, lx, ly, lz, vl, vr, eta, kp)


def test_spectral_functions_sum_to_the_diagonal(oracle):
    """i (G_kk - G_kk^H) = 2 dz^2 (G_k1 Gamma_L G_k1^H + G_kNz Gamma_R G_kNz^H) as eta -> 0:
    the spectral-function term of density_neq has the right lead widths and scale."""
    p = _xy_problem(oracle, nz=5, eta=1e-13, symmetric=False, vl=0.001 / HARTREE)
    assert p.N > 4
    dz = p.Lz / p.Nz
    for e in (0.004 / HARTREE, 0.012 / HARTREE):
        kx, ky, _ = p.kpt[1]
        D = oracle.e_minus_h(p, oracle.hamiltonian(p, kx, ky), e + 1j * p.eta, kx, ky)
        outs, info = oracle.tri_solver(D, "DFL")
        assert info == 0
        gL, gR = oracle.lead_gammas(p, e, kx, ky)
        assert np.count_nonzero(gL) > 0
        for k in range(p.Nz):
            G, F, L = outs["D"][:, :, k], outs["F"][:, :, k], outs["L"][:, :, k]
            lhs = 1j * (G - G.conj().T)
            rhs = 2 * dz * dz * ((F * gL) @ F.conj().T + (L * gR) @ L.conj().T)
            assert np.max(np.abs(lhs - rhs)) <= 1e-7 * np.max(np.abs(lhs)), k


def test_density_neq_mirror_symmetry(oracle):
    """On a device even under slice reversal, swapping mu_L and mu_R mirrors the
    density matrix in z (left-injected F column vs right-injected L column)."""
    p = _xy_problem(oracle, nz=6)
    mu = 0.008 / HARTREE
    T = 0.5
    gap = 6 * (8.617333262e-5 / HARTREE) * T
    a, _ = oracle.density_neq(p, 6, 10, 0.0, mu + 0.002 / HARTREE, mu, gap, T)
    b, _ = oracle.density_neq(p, 6, 10, 0.0, mu, mu + 0.002 / HARTREE, gap, T)
    assert np.max(np.abs(a - b[:, :, ::-1])) <= 1e-9 * np.max(np.abs(a))
    # the bias term is present: differs from the zero-bias matrix
    c, _ = oracle.density_neq(p, 6, 10, 0.0, mu, mu, gap, T)
    assert np.max(np.abs(a - c)) > 1e-4 * np.max(np.abs(a))


def test_mlp_oracle_bf16_rounding():
    from oracle import mlp_oracle as M
    x = np.array([1.0, 1 + 2.0 ** -8, 1 + 3 * 2.0 ** -8, -2.5, 3.0e-5, 1 + 2.0 ** -9])
    np.testing.assert_array_equal(M.bf16(x), [1.0, 1.0, 1 + 2.0 ** -6, -2.5, M.bf16(3.0e-5), 1.0])
    assert abs(M.bf16(3.0e-5) - 3.0e-5) <= 2.0 ** -9 * 3.0e-5


def test_mlp_oracle_gradient_finite_differences():
    """The FP64 network's backward pass against central differences of its loss."""
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(7)
    widths = [5, 7, 6, 3]
    n = sum(a * b + b for a, b in zip(widths[:-1], widths[1:]))
    p = rng.standard_normal(n) * 0.5
    x = rng.standard_normal((9, 5))
    t = rng.standard_normal((9, 3))
    w = rng.uniform(0.5, 1.5, (9, 3))
    _, g = M.loss_and_grad(p, widths, x, t, w, bf16_ops=False)
    eps = 1e-6
    fd = np.empty(n)
    for i in range(n):
        e = np.zeros(n)
        e[i] = eps
        fd[i] = (M.loss_and_grad(p + e, widths, x, t, w, False)[0]
                 - M.loss_and_grad(p - e, widths, x, t, w, False)[0]) / (2 * eps)
    assert np.max(np.abs(fd - g)) <= 1e-7 * max(1.0, np.max(np.abs(g)))
