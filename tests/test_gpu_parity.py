"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerance: FP64 mode must match within 1e-9 relative (normwise for matrices,
elementwise with a 1e-12 absolute floor for tau).
"""
import numpy as np
import pytest

from negftrans_b200 import HARTREE, workloads as W
from negftrans_b200 import prepare as P
from negftrans_b200.negf import Engine, GreensFunction_tri_solver

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def rel_err(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def oracle_problem(O, pr):
    a = pr.atomic
    return O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)


def small_problem(encut_meV=1.2, nz=16, nk=1, grid=32, V_L=0.0, V_R=0.0, seed=1000):
    V = W.MSTAR * W.qpc_potential(grid, grid, nz, 100.0, nz * 1.0, 0.050, 15.0, nz / 10.0,
                                  disorder=0.002, seed=seed)
    d = W._deck(nz * 10.0, encut_meV * 1e-3, 30.0, 16, nk=nk)
    d.V_L, d.V_R = V_L, V_R
    return P.prepare(d, V)


def random_blocks(N, Nz, seed, shift=4.0):
    rng = np.random.default_rng(seed)
    D = rng.standard_normal((N, N, Nz)) + 1j * rng.standard_normal((N, N, Nz))
    for k in range(Nz):
        D[:, :, k] += shift * np.sqrt(N) * np.eye(N)
    return np.asfortranarray(D)


@pytest.mark.parametrize("N,Nz", [(1, 2), (5, 2), (5, 7), (33, 3), (64, 4), (70, 5), (129, 3)])
def test_tri_solve_random(oracle, N, Nz):
    D = random_blocks(N, Nz, seed=N * 100 + Nz)
    ref, rinfo = oracle.tri_solver(D, "DFL")
    got, info = GreensFunction_tri_solver(D, "DFL")
    assert info == rinfo == 0
    for k in "DFL":
        assert rel_err(got[k], ref[k]) < RTOL, k


@pytest.mark.parametrize("N,Nz", [(300, 3), (600, 2)])
def test_tri_solve_wide_variants(oracle, N, Nz):
    """N > 256 runs the 2- and 4-rows-per-thread kernel variants."""
    D = random_blocks(N, Nz, seed=N)
    ref, _ = oracle.tri_solver(D, "DF")
    got, info = GreensFunction_tri_solver(D, "DF")
    assert info == 0
    for k in "DF":
        assert rel_err(got[k], ref[k]) < RTOL, k


def test_tri_solve_partial_dfl_zero_fills(oracle):
    D = random_blocks(6, 4, seed=3)
    got, _ = GreensFunction_tri_solver(D, "F")
    ref, _ = oracle.tri_solver(D, "F")
    assert set(got) == {"F"}
    assert rel_err(got["F"], ref["F"]) < RTOL


def test_tri_solve_singular_reports_info():
    D = random_blocks(4, 3, seed=5)
    D[:, :, 2] = 0.0  # inv(D_Nz) of a zero block
    _, info = GreensFunction_tri_solver(D, "F")
    assert info > 0


def test_tri_solve_physical_blocks(oracle):
    pr = small_problem()
    p = oracle_problem(oracle, pr)
    H = oracle.hamiltonian(p, 0.0, 0.0)
    D = oracle.e_minus_h(p, H, 0.067 * 0.012 / HARTREE + 1j * pr.atomic.ETA, 0.0, 0.0)
    ref, _ = oracle.tri_solver(D, "DFL")
    got, info = GreensFunction_tri_solver(D, "DFL")
    assert info == 0
    for k in "DFL":
        assert rel_err(got[k], ref[k]) < RTOL, k


@pytest.mark.parametrize("nk", [1, 2])
def test_transmission_small(oracle, nk):
    pr = small_problem(nk=nk)
    E = P.transmission_energies(pr.atomic, 16)
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=4)
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)


def test_transmission_device_entry(oracle):
    """negf_transmission_device on device buffers and the caller's stream: the
    same tau as the host entry, the per-job tau in k-major order summing to it
    with the k weights, the per-job info; the optional outputs may be omitted."""
    torch = pytest.importorskip("torch")
    pr = small_problem(nk=2)
    E = P.transmission_energies(pr.atomic, 16)
    nE = len(E)
    kpt = np.asarray(pr.kpoint, np.float64).reshape(-1, 3)
    nk = len(kpt)
    assert nk > 1
    dev = torch.device("cuda", 0)
    d_E = torch.from_numpy(np.ascontiguousarray(E)).to(dev)
    d_tau = torch.full((nE,), float("nan"), dtype=torch.float64, device=dev)
    d_tj = torch.full((nk * nE,), float("nan"), dtype=torch.float64, device=dev)
    d_info = torch.full((nk * nE,), -7, dtype=torch.int32, device=dev)
    d_tau2 = torch.full((nE,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(device=dev)
    with Engine(*pr.engine_args()) as eng:
        tau_host, info_host = eng.transmission(E)
        eng.transmission_device(d_E.data_ptr(), nE, d_tau.data_ptr(), d_tj.data_ptr(), d_info.data_ptr(),
                                stream.cuda_stream)
        stream.synchronize()
        eng.transmission_device(d_E.data_ptr(), nE, d_tau2.data_ptr())
        torch.cuda.synchronize(dev)
    assert info_host == 0
    tau, tau2 = d_tau.cpu().numpy(), d_tau2.cpu().numpy()
    tj = d_tj.cpu().numpy().reshape(nk, nE)
    np.testing.assert_array_equal(tau, tau_host)
    np.testing.assert_array_equal(tau2, tau_host)
    assert (d_info.cpu().numpy() == 0).all()
    np.testing.assert_allclose(kpt[:, 2] @ tj, tau, rtol=1e-14, atol=1e-15)
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=4)
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)


def test_transmission_leads_differ(oracle):
    """V_L != V_R exercises the gamma_L-on-rows quirk of grid.f90:363-374."""
    pr = small_problem(V_L=0.067 * 0.002, V_R=0.067 * 0.005)
    E = P.transmission_energies(pr.atomic, 16)
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=4)
    with Engine(*pr.engine_args()) as eng:
        tau, _ = eng.transmission(E)
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)


def test_transmission_n69_subset(oracle):
    w = W.config("qpc_n69")
    pr = P.prepare(w.deck, w.V_eV)
    E = P.transmission_energies(pr.atomic, 512)[::64]
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=8)
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)


def test_transmission_closed_form(oracle):
    """z-only potential: every mode decouples (long-double three-term recursion)."""
    nz, grid = 24, 32
    z = (np.arange(nz) + 0.5 - nz / 2)
    vz = 0.067 * 0.02 * np.exp(-z ** 2 / 18.0)
    V = np.asfortranarray(np.broadcast_to(vz[None, None, :], (grid, grid, nz)))
    d = W._deck(nz * 10.0, 1.2e-3, 30.0, 16)
    pr = P.prepare(d, V)
    a = pr.atomic
    E = P.transmission_energies(a, 16)
    with Engine(*pr.engine_args()) as eng:
        tau, _ = eng.transmission(E)
    vz00 = pr.vhat[pr.NGX, pr.NGY, :]
    cf = [oracle.closed_form_tau(pr.nx, pr.ny, vz00, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, e, 0, 0)
          for e in E]
    np.testing.assert_allclose(tau, cf, rtol=1e-9, atol=1e-12)


def test_transmission_many_jobs_and_determinism(oracle):
    """More jobs than SMs (persistent loop) and bitwise repeatability."""
    pr = small_problem(encut_meV=0.6, nz=6)
    E = P.transmission_energies(pr.atomic, 16)
    E = np.linspace(E[0], 0.067 * 0.03 / HARTREE, 333)
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=8)
    with Engine(*pr.engine_args()) as eng:
        t1, _ = eng.transmission(E)
        t2, _ = eng.transmission(E)
    np.testing.assert_allclose(t1, tau_ref, rtol=RTOL, atol=1e-12)
    assert np.array_equal(t1, t2)


def test_density_small(oracle):
    pr = small_problem(nz=8, nk=2)
    a = pr.atomic
    n_c, n_l = 6, 5
    dm_ref, _ = oracle.density_jobs(oracle_problem(oracle, pr), n_c, n_l, pr.min_V, a.MU, a.GAP,
                                    a.TEMPERATURE, nthreads=4)
    with Engine(*pr.engine_args()) as eng:
        dm, info = eng.equilibrium_density(n_c, n_l, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
    assert info == 0
    assert rel_err(dm, dm_ref) < RTOL


def test_ldos_small(oracle):
    pr = small_problem(nz=8, nk=2)
    p = oracle_problem(oracle, pr)
    e_lo, e_hi, n_e = 0.0, 0.067 * 0.03 / HARTREE, 5
    with Engine(*pr.engine_args()) as eng:
        got, info = eng.ldos_matrix(e_lo, e_hi, n_e, i_e0=1, n_chunk=3)
    assert info == 0
    for o in range(3):
        ref = np.zeros((pr.N, pr.N, pr.Nz), np.complex128, order="F")
        for ik in range(len(pr.kpoint)):
            oracle.local_density_of_state(p, ik + 1, o + 2, n_e, e_lo, e_hi, ref)
        assert rel_err(got[o], ref) < RTOL


@pytest.mark.parametrize("encut_meV,grid", [(14.5, 64), (29.0, 96)])
def test_transmission_wide_basis(oracle, encut_meV, grid):
    """N > 256 and N > 512: the 2- and 4-rows-per-thread kernel variants."""
    nz = 5
    V = W.MSTAR * W.qpc_potential(grid, grid, nz, 100.0, nz * 1.0, 0.050, 15.0, 1.0, disorder=0.002)
    d = W._deck(nz * 10.0, encut_meV * 1e-3, 30.0, 16)
    pr = P.prepare(d, V)
    assert pr.N > 256
    E = P.transmission_energies(pr.atomic, 16)[::3]
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=8)
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)


def test_density_real_space(oracle):
    """Density (main.f90:258-351): contour, G_kk sum, PtoR and scale on the GPU."""
    pr = small_problem(nz=6, nk=1)
    a, d = pr.atomic, None
    Nx, Ny = 32, 32
    LX, LY, LZ = 1000.0, 1000.0, pr.Nz * 10.0
    n_c, n_l = 5, 4
    with Engine(*pr.engine_args()) as eng:
        dens, dm, info = eng.density_real(n_c, n_l, pr.min_V, a.MU, a.GAP, a.TEMPERATURE, Nx, Ny, LX, LY, LZ)
    assert info == 0
    dm_ref, _ = oracle.density_jobs(oracle_problem(oracle, pr), n_c, n_l, pr.min_V, a.MU, a.GAP,
                                    a.TEMPERATURE)
    assert rel_err(dm, dm_ref) < RTOL
    ref = oracle.density_from_matrix(dm_ref, pr.nx, pr.ny, Nx, Ny, LX, LY, LZ)
    assert rel_err(dens, ref) < RTOL


@pytest.mark.parametrize("grid", [(0, 0, 0), (-1, -1, 0), (-1, 5, -1), (3, 0, 2)])
def test_ldos_real_space(oracle, grid):
    """LDOS (main.f90:417-554) incl. every LDOS_GRID mode of tools.f90:6-40."""
    pr = small_problem(nz=4, nk=2)
    p = oracle_problem(oracle, pr)
    Nx, Ny = 32, 32
    LX, LY, LZ = 1000.0, 1000.0, pr.Nz * 10.0
    e_lo, e_hi, n_e = 0.0, 0.067 * 0.03 / HARTREE, 3
    with Engine(*pr.engine_args()) as eng:
        got, info = eng.ldos(e_lo, e_hi, n_e, grid, Nx, Ny, LX, LY, LZ)
    assert info == 0
    for ie in range(n_e):
        mat = np.zeros((pr.N, pr.N, pr.Nz), np.complex128, order="F")
        for ik in range(len(pr.kpoint)):
            oracle.local_density_of_state(p, ik + 1, ie + 1, n_e, e_lo, e_hi, mat)
        ref = oracle.ldos_from_matrix(mat, pr.nx, pr.ny, Nx, Ny, LX, LY, LZ, grid)
        assert got.shape[:3] == ref.shape
        assert rel_err(got[..., ie], ref) < RTOL


def test_transmission_batch_uneven(oracle):
    """Per-k bases and devices of different length in one persistent launch per
    kernel variant, each problem against the oracle; one problem has N > 256
    (second variant)."""
    from negftrans_b200.negf import transmission_batch
    probs = W.batched_uneven(nkx=2, nzs=(4, 7), encut_eV=1.2e-3, grid=32)
    V = W.MSTAR * W.qpc_potential(64, 64, 3, 100.0, 3.0, 0.05, 15.0, 1.0, disorder=0.002)
    big = P.prepare(W._deck(30.0, 14.5e-3, 30.0, 16), V)
    probs.append({"device": 2, "Nz": 3, "N": big.N, "args": big.engine_args()})
    assert len({p["N"] for p in probs}) > 1 and max(p["N"] for p in probs) > 256
    E = np.linspace(0.0, 0.067 * 0.03 / HARTREE, 6, endpoint=False)
    engines = [Engine(*p["args"]) for p in probs]
    try:
        tau, info, _ = transmission_batch(engines, E)
    finally:
        for e in engines:
            e.close()
    assert info == 0
    for p, t in zip(probs, tau):
        nx, ny, vhat, lx, ly, lz, vl, vr, eta, kp = p["args"]
        ref, _ = oracle.transmission_jobs(oracle.Problem(nx, ny, vhat, lx, ly, lz, vl, vr, eta, kp), E,
                                          nthreads=8)
        np.testing.assert_allclose(t, ref, rtol=RTOL, atol=1e-12)


def test_transmission_batch_uneven_spread(oracle):
    """The uneven batch of the benchmark's shape at reduced length: per-k
    cutoffs spreading the bases over 180-263 plane waves (both kernel
    variants), devices of 4 and 7 slices, one persistent launch per variant,
    every problem against the oracle."""
    from negftrans_b200.negf import transmission_batch
    probs = W.batched_uneven(nkx=2, nzs=(4, 7), n_range=(180, 260))
    sizes = sorted({p["N"] for p in probs})
    assert sizes[0] <= 185 and sizes[-1] >= 256 and len(sizes) == 4
    E = np.linspace(0.0, 0.067 * 0.03 / HARTREE, 5, endpoint=False)
    engines = [Engine(*p["args"]) for p in probs]
    try:
        tau, info, _ = transmission_batch(engines, E)
    finally:
        for e in engines:
            e.close()
    assert info == 0
    for p, t in zip(probs, tau):
        nx, ny, vhat, lx, ly, lz, vl, vr, eta, kp = p["args"]
        ref, _ = oracle.transmission_jobs(oracle.Problem(nx, ny, vhat, lx, ly, lz, vl, vr, eta, kp), E,
                                          nthreads=8)
        np.testing.assert_allclose(t, ref, rtol=RTOL, atol=1e-12)


@pytest.mark.parametrize("flat", [True, False])
def test_lattice_lead_model(oracle, flat):
    """lead_model = 1 (exact lattice surface Green's function of the leads)
    against the closed form; a flat device transmits open channels fully."""
    nz, grid = 20, 32
    z = np.arange(nz) + 0.5 - nz / 2
    vz = np.zeros(nz) if flat else 0.067 * 0.02 * np.exp(-z ** 2 / 18.0)
    V = np.asfortranarray(np.broadcast_to(vz[None, None, :], (grid, grid, nz)))
    d = W._deck(nz * 10.0, 1.2e-3, 30.0, 16)
    d.ETA = 1e-13      # eta absorbs slow near-edge modes; keep it small for the unitarity check
    pr = P.prepare(d, V)
    a = pr.atomic
    E = P.transmission_energies(a, 16)
    with Engine(*pr.engine_args(), lead_model=1) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    vz00 = pr.vhat[pr.NGX, pr.NGY, :]
    cf = [oracle.closed_form_tau(pr.nx, pr.ny, vz00, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, e, 0, 0,
                                 lattice=True) for e in E]
    np.testing.assert_allclose(tau, cf, rtol=1e-9, atol=1e-12)
    if flat:
        dz = a.LZ / nz
        eps = ((2.0 * pr.nx * np.pi / a.LX) ** 2 + (2.0 * pr.ny * np.pi / a.LY) ** 2) / 2
        n_open = [np.sum(np.abs(2 * dz * dz * (e - eps) - 2) < 2) for e in E]
        np.testing.assert_allclose(tau, n_open, atol=1e-4)


@pytest.mark.parametrize("bias", ["left", "right", "none"])
def test_density_neq_small(oracle, bias):
    """Biased density matrix (Gauss-Legendre semicircle + real-axis window with the
    spectral function of the injecting lead) against the oracle's tri_solver
    restatement; 'right' runs the mirrored sweep."""
    pr = small_problem(nz=8, nk=2)
    a = pr.atomic
    vb = W.MSTAR * 1e-3 / HARTREE  # 1 mV
    mu_L, mu_R = {"left": (a.MU + vb, a.MU), "right": (a.MU, a.MU + vb), "none": (a.MU, a.MU)}[bias]
    n_c, n_w = 6, 10
    dm_ref, _ = oracle.density_neq(oracle_problem(oracle, pr), n_c, n_w, pr.min_V, mu_L, mu_R, a.GAP,
                                   a.TEMPERATURE)
    with Engine(*pr.engine_args()) as eng:
        dm, info = eng.density_neq(n_c, n_w, pr.min_V, mu_L, mu_R, a.GAP, a.TEMPERATURE)
        assert info == 0
        assert rel_err(dm, dm_ref) < RTOL
        if bias == "left":
            Nx = Ny = 32
            dens = eng.dm_real(dm, Nx, Ny, 1000.0, 1000.0, pr.Nz * 10.0)
            ref = oracle.density_from_matrix(dm_ref, pr.nx, pr.ny, Nx, Ny, 1000.0, 1000.0, pr.Nz * 10.0)
            assert rel_err(dens, ref) < RTOL


def test_density_neq_wide_basis(oracle):
    """N > 256 (the 2-rows-per-thread slab variant) with many open channels."""
    nz = 4
    V = W.MSTAR * W.qpc_potential(64, 64, nz, 100.0, nz * 1.0, 0.050, 15.0, 1.0, disorder=0.002)
    pr = P.prepare(W._deck(nz * 10.0, 14.5e-3, 30.0, 16), V)
    assert pr.N > 256
    a = pr.atomic
    vb = W.MSTAR * 1e-3 / HARTREE
    dm_ref, _ = oracle.density_neq(oracle_problem(oracle, pr), 2, 3, pr.min_V, a.MU + vb, a.MU, a.GAP,
                                   a.TEMPERATURE)
    with Engine(*pr.engine_args()) as eng:
        dm, info = eng.density_neq(2, 3, pr.min_V, a.MU + vb, a.MU, a.GAP, a.TEMPERATURE)
    assert info == 0
    assert rel_err(dm, dm_ref) < RTOL


@pytest.mark.gpu
def test_every_variant_and_the_autotuner(oracle):
    """Each transmission kernel variant that can hold N (forced per context)
    matches the oracle; the autotuner keeps the fastest of them."""
    pr = small_problem(nz=8, nk=2)
    E = P.transmission_energies(pr.atomic, 16)[::2]
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=4)
    with Engine(*pr.engine_args()) as eng:
        for v in (0, 1, 2, 3):
            eng.set_variant(v)
            tau, info = eng.transmission(E)
            assert info == 0
            np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)
        v, rates = eng.autotune(E)
        assert v in (0, 1, 2, 3) and rates[v] == rates.max() > 0
        tau, _ = eng.transmission(E)
        np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)
        eng.set_variant(-1)


@pytest.mark.parametrize("grid,ng,nz", [(64, 9, 5), (64, 17, 3), (128, 34, 2), (32, 3, 4)])
@pytest.mark.gpu
def test_vhat_gpu_matches_host(grid, ng, nz):
    """The V table computed on the GPU against the host transform (and its
    conjugate symmetry and zero window) on a seeded disordered QPC."""
    from negftrans_b200.grid import V_reciprocal_all, V_reciprocal_all_gpu
    V = W.MSTAR * W.qpc_potential(grid, grid, nz, 100.0, nz * 1.0, 0.05, 15.0, 1.0, disorder=0.002) / HARTREE
    ref = V_reciprocal_all(V, ng, ng)
    got = V_reciprocal_all_gpu(V, ng, ng)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    h = ng // 2
    assert np.all(got[: ng - h] == 0) and np.all(got[ng + h + 1:] == 0)
    np.testing.assert_allclose(got[ng - h:ng + h + 1, ng - h:ng + h + 1][::-1, ::-1],
                               np.conj(got[ng - h:ng + h + 1, ng - h:ng + h + 1]), rtol=0, atol=1e-14 * np.max(np.abs(ref)))


@pytest.mark.gpu
def test_transmission_near_the_maximum_basis(oracle):
    """N = 997 (the largest variant holds N <= 1024), two slices; and N = 1041
    is refused with NEGF_ERR_UNSUPPORTED rather than run."""
    from negftrans_b200._lib import NEGF_ERR_UNSUPPORTED, NegfError
    nz = 2
    V = W.MSTAR * W.qpc_potential(128, 128, nz, 100.0, nz * 1.0, 0.050, 15.0, 1.0, disorder=0.002)
    pr = P.prepare(W._deck(nz * 10.0, 0.048, 30.0, 16), V)
    assert pr.N == 997
    E = P.transmission_energies(pr.atomic, 16)[::5]
    tau_ref, _ = oracle.transmission_jobs(oracle_problem(oracle, pr), E, nthreads=8)
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E)
    assert info == 0
    np.testing.assert_allclose(tau, tau_ref, rtol=RTOL, atol=1e-12)
    big = P.prepare(W._deck(nz * 10.0, 0.05, 30.0, 16), V)
    assert big.N == 1041
    with pytest.raises(NegfError) as exc:
        Engine(*big.engine_args())
    assert exc.value.code == NEGF_ERR_UNSUPPORTED


@pytest.mark.gpu
def test_density_accumulate_any_contour(oracle):
    """Arbitrary complex energies and weights against the oracle; and the
    reference's own Simpson contour through this entry equals negf_density."""
    pr = small_problem(nz=8, nk=2)
    a = pr.atomic
    rng = np.random.default_rng(7)
    E = a.MU * rng.uniform(0.2, 1.2, 6) + 1j * a.MU * rng.uniform(0.0, 0.5, 6)
    w = rng.standard_normal(6) + 1j * rng.standard_normal(6)
    ref, _ = oracle.density_accumulate(oracle_problem(oracle, pr), E, w)
    with Engine(*pr.engine_args()) as eng:
        dm, info = eng.density_accumulate(E, w)
        assert info == 0
        assert rel_err(dm, ref) < RTOL
        # negf.f90:37-65 contour and weights restated here (Simpson, n_circle = 6, n_line = 5)
        n_c, n_l = 6, 5
        cl, cr = pr.min_V - 1.0 / HARTREE, a.MU - a.GAP
        Ec, ER = (cr + cl) / 2, (cr - cl) / 2
        sx = lambda i, n, lo, hi: (i - 1) * (hi - lo) / (n - 1) + lo
        EE, WW = [], []
        for i in range(1, n_c + 1):
            th = sx(i, n_c, 0.0, np.pi)
            EE.append(Ec + ER * np.exp(1j * th))
            WW.append(2 / np.pi * oracle.coefficient_simpson(i, n_c, 0.0, np.pi) * 1j * ER * np.exp(1j * th))
        for i in range(1, n_l + 1):
            x = sx(i, n_l, a.MU - a.GAP, a.MU + a.GAP)
            EE.append(x)
            WW.append(-2 / np.pi * oracle.coefficient_simpson(i, n_l, a.MU - a.GAP, a.MU + a.GAP)
                      * oracle.fermi_func(x, a.MU, a.TEMPERATURE))
        dm2, _ = eng.density_accumulate(np.array(EE), np.array(WW))
        dm_ref, _ = eng.equilibrium_density(n_c, n_l, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
        assert rel_err(dm2, dm_ref) < RTOL
