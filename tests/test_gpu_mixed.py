"""Tensor-core arithmetic of the mixed-precision path, against NumPy FP64.

* The split-fp16 complex product of the trailing update (tcgen05 MMAs, FP32
  accumulation in tensor memory, one power-of-two exponent per row of W and
  per column of B): normwise relative error below 2e-6 (three split products
  keep ~2^-21), on operands whose rows and columns span 1e-15 .. 1e15.
* The FP32 blocked Gauss-Jordan inverse (32-column panels, pivoting inside
  each diagonal block, rank-32 tensor-core trailing updates):
  ||X A - I|| / (||X|| ||A||) below 1e-6 for N from 5 to 797 (FP32 rounding
  of A itself is ~6e-8) on Schur-complement-like blocks whose rows are
  shuffled inside each 32-row block and whose first pivot is zero.
"""
import numpy as np
import pytest

from negftrans_b200 import _lib

pytestmark = pytest.mark.gpu


def _c64(torch, a):
    a = np.asfortranarray(a, np.complex64)
    return torch.from_numpy(a.ravel(order="F").view(np.float32).copy()).cuda()


@pytest.mark.parametrize("M,ncol,K", [(128, 64, 32), (221, 150, 32), (300, 7, 19), (5, 3, 1)])
def test_split_fp16_product(M, ncol, K):
    import torch

    rng = np.random.default_rng(M + ncol + K)
    W = rng.standard_normal((M, 32)) + 1j * rng.standard_normal((M, 32))
    Bfull = rng.standard_normal((64, ncol)) + 1j * rng.standard_normal((64, ncol))
    # rows of W and columns of B over 30 decades (products stay inside the
    # FP32 range): the per-row / per-column exponents keep each of them at
    # full relative accuracy
    W *= 10.0 ** rng.uniform(-15, 15, M)[:, None]
    Bfull *= 10.0 ** rng.uniform(-15, 15, ncol)[None, :]
    W = W.astype(np.complex64)
    Bfull = Bfull.astype(np.complex64)
    rowmap = rng.permutation(64)[:K].astype(np.int32)
    dW, dB = _c64(torch, W), _c64(torch, Bfull)
    dC = torch.zeros(2 * M * ncol, dtype=torch.float32, device="cuda")
    dmap = torch.from_numpy(rowmap).cuda()
    rc = _lib.lib().negf_tc_product_check(dW.data_ptr(), M, dB.data_ptr(), 64, dmap.data_ptr(), dC.data_ptr(),
                                          M, M, ncol, K, None)
    assert rc == _lib.NEGF_OK
    C = dC.cpu().numpy().view(np.complex64).reshape((M, ncol), order="F").astype(np.complex128)
    ref = W[:, :K].astype(np.complex128) @ Bfull[rowmap].astype(np.complex128)
    # relative error of every element against |W_i| |B_j| (the normwise bound)
    bound = np.abs(W[:, :K]).astype(float) @ np.abs(Bfull[rowmap]).astype(float)
    err = np.abs(C - ref) / bound
    assert err.max() < 2e-6, err.max()


@pytest.mark.parametrize("N", [5, 37, 69, 221, 300, 797])
def test_fp32_gauss_jordan_inverse(N):
    import torch

    rng = np.random.default_rng(N)
    # Schur-complement-like blocks: -2 + small on the diagonal, weak dense coupling
    A = (-2.0 + 0.3 * rng.standard_normal(N) + 0.01j) * np.eye(N)
    A = A + 0.05 * (rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))) / np.sqrt(N)
    # rows that need pivoting inside each diagonal block, and a zero first pivot
    perm = np.concatenate([k0 + rng.permutation(min(32, N - k0)) for k0 in range(0, N, 32)])
    A = A[perm]
    if N > 1:
        A[[0, 1]] = A[[1, 0]]
        A[0, 0] = 0.0
    A = A.astype(np.complex64)
    nmat = 3
    As = np.stack([A, A * (1 + 0.5j), A.T], axis=0)
    dA = torch.from_numpy(np.ascontiguousarray(
        np.concatenate([m.ravel(order="F") for m in As])).view(np.float32)).cuda()
    dOut = torch.zeros_like(dA)
    dInfo = torch.full((nmat,), -7, dtype=torch.int32, device="cuda")
    rc = _lib.lib().negf_tc_inverse_check(dA.data_ptr(), N, nmat, dOut.data_ptr(), dInfo.data_ptr(), None)
    assert rc == _lib.NEGF_OK
    assert (dInfo.cpu().numpy() == 0).all()
    out = dOut.cpu().numpy().view(np.complex64)
    for m in range(nmat):
        X = out[m * N * N:(m + 1) * N * N].reshape((N, N), order="F").astype(np.complex128)
        Am = As[m].astype(np.complex128)
        res = np.linalg.norm(X @ Am - np.eye(N)) / (np.linalg.norm(X) * np.linalg.norm(Am))
        assert res < 1e-6, (m, res)
        Xr = np.linalg.inv(Am)
        assert np.linalg.norm(X - Xr) / np.linalg.norm(Xr) < 1e-5


# ------------------------------------------------------ mixed transmission
# NEGF_MIXED: split-fp16 tensor-core factorization + FP64 residual refinement
# + FP64 re-run of rejected jobs.  The bar of the headline metric: every
# energy within max|dT| <= 1e-6 of the FP64 oracle.
TOL_MIXED = 1e-6


def _oracle(pr, E, nthreads=8):
    from oracle import oracle as O
    a = pr.atomic
    p = O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    tau, info = O.transmission_jobs(p, E, nthreads=nthreads)
    assert info == 0
    return tau


def _prepared(name, nz=None):
    from negftrans_b200 import prepare as P, workloads as W
    w = W.config(name, nz=nz)
    return w, P.prepare(w.deck, w.V_eV)


@pytest.mark.parametrize("name,ne,nk", [("small:1.2:16", 16, 1), ("qpc_n69", 48, 1)])
def test_mixed_transmission_matches_oracle(name, ne, nk):
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_MIXED
    from negftrans_b200.negf import Engine
    w, pr = _prepared(name)
    grid = P.transmission_energies(pr.atomic, w.n_energy)
    E = np.ascontiguousarray(grid[:: max(1, len(grid) // ne)][:ne])
    ref = _oracle(pr, E)
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E, precision=NEGF_MIXED)
        st = eng.mixed_stats()
    assert info == 0
    assert st["n_jobs"] == len(E) * nk
    assert st["n_mixed"] + st["n_fp64_policy"] + st["n_fp64_rejected"] == st["n_jobs"]
    assert st["n_mixed"] >= 0.8 * st["n_jobs"], st
    assert np.max(np.abs(tau - ref)) <= TOL_MIXED, np.max(np.abs(tau - ref))


@pytest.mark.parametrize("name", ["qpc_disorder_n221", "qpc_disorder_n797"])
def test_mixed_transmission_matches_full_size_fixture(name):
    import os
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_MIXED
    from negftrans_b200.negf import Engine
    ref = np.load(os.path.join(os.path.dirname(__file__), "golden", f"oracle_{name}.npz"))
    w, pr = _prepared(name)
    E = P.transmission_energies(pr.atomic, int(ref["grid_size"]))[ref["idx"]]
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E, precision=NEGF_MIXED)
        st = eng.mixed_stats()
    assert info == 0
    assert np.max(np.abs(tau - ref["tau"])) <= TOL_MIXED, (np.abs(tau - ref["tau"]), st)


def test_mixed_policy_routes_jobs_to_fp64():
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_FP64, NEGF_MIXED
    from negftrans_b200.negf import Engine
    w, pr = _prepared("qpc_n69", nz=40)
    E = P.transmission_energies(pr.atomic, w.n_energy)[::16]
    a = pr.atomic
    with Engine(*pr.engine_args()) as eng:
        t64, _ = eng.transmission(E, precision=NEGF_FP64)
        # eta below the bound: every job runs the FP64 path, bit for bit
        eng.set_mixed_policy(eta_fp64_below=2 * a.ETA)
        tm, _ = eng.transmission(E, precision=NEGF_MIXED)
        st = eng.mixed_stats()
        assert st["n_fp64_policy"] == len(E) and st["n_mixed"] == 0
        np.testing.assert_array_equal(tm, t64)
        # threshold window: exactly the energies near a lead threshold go to FP64
        eng.set_mixed_policy(eta_fp64_below=0.0, threshold_window=1e-3 * 0.067 / 27.211386245988)
        tm, _ = eng.transmission(E, precision=NEGF_MIXED)
        st = eng.mixed_stats()
    kx = 2.0 * pr.nx * np.pi / a.LX
    ky = 2.0 * pr.ny * np.pi / a.LY
    th = 0.5 * (kx ** 2 + ky ** 2)
    near = sum(bool(np.any(np.abs(e - th) < 1e-3 * 0.067 / 27.211386245988)) for e in E)
    assert st["n_fp64_policy"] == near
    assert np.max(np.abs(tm - t64)) <= TOL_MIXED


@pytest.mark.parametrize("name,nz,ne", [("qpc_n69", 40, 24), ("qpc_disorder_n221", 48, 12), ("qpc_disorder_n797", 12, 4)])
def test_mixed_one_and_two_ctas_per_job(name, nz, ne):
    """The sweep on one CTA per job and on a two-CTA cluster per job (rows,
    panel products and trailing tiles split between two SMs) both meet the
    bar against the oracle, and the call reports which one ran."""
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_MIXED
    from negftrans_b200.negf import Engine
    w, pr = _prepared(name, nz=nz)
    grid = P.transmission_energies(pr.atomic, w.n_energy)
    E = np.ascontiguousarray(grid[:: max(1, len(grid) // ne)][:ne])
    ref = _oracle(pr, E)
    out = {}
    with Engine(*pr.engine_args()) as eng:
        for cpj in (1, 2):
            eng.set_mixed_policy(ctas_per_job=cpj)
            tau, info = eng.transmission(E, precision=NEGF_MIXED)
            st = eng.mixed_stats()
            assert info == 0
            assert st["ctas_per_job"] == cpj, st
            assert np.max(np.abs(tau - ref)) <= TOL_MIXED, (cpj, np.abs(tau - ref), st)
            out[cpj] = tau
    assert np.max(np.abs(out[1] - out[2])) <= TOL_MIXED


def test_mixed_accepts_energies_without_a_trace_term():
    """At the band bottom (E = 0, flat leads at V = 0) no channel of the left
    lead is open, so every gamma_L vanishes and tau is exactly 0 (grid.f90:355-383)
    whatever G_{Nz,1} holds.  The mixed path accepts such a job at once instead of
    sending it to an FP64 re-run."""
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_MIXED
    from negftrans_b200.negf import Engine
    w, pr = _prepared("qpc_n69", nz=40)
    grid = P.transmission_energies(pr.atomic, w.n_energy)
    E = np.ascontiguousarray(np.concatenate([[0.0], grid[1::64]]))
    ref = _oracle(pr, E)
    assert ref[0] == 0.0
    with Engine(*pr.engine_args()) as eng:
        tau, info = eng.transmission(E, precision=NEGF_MIXED)
        st = eng.mixed_stats()
    assert info == 0
    assert tau[0] == 0.0
    assert st["n_fp64_rejected"] == 0 and st["n_mixed"] == len(E), st
    assert np.max(np.abs(tau - ref)) <= TOL_MIXED


def test_mixed_device_entry_matches_host_entry():
    """negf_transmission_device with NEGF_MIXED on device buffers and the
    caller's stream gives the host entry's tau bit for bit (the mixed path is
    deterministic: fixed-order reductions, order-free column maxima), and the
    per-job tau in k-major order sums to it with the k weights."""
    import torch
    from negftrans_b200 import prepare as P
    from negftrans_b200._lib import NEGF_MIXED
    from negftrans_b200.negf import Engine
    w, pr = _prepared("small:1.2:16")
    E = P.transmission_energies(pr.atomic, 16)
    nE = len(E)
    kpt = np.asarray(pr.kpoint, np.float64).reshape(-1, 3)
    nk = len(kpt)
    dev = torch.device("cuda", 0)
    d_E = torch.from_numpy(np.ascontiguousarray(E)).to(dev)
    d_tau = torch.full((nE,), float("nan"), dtype=torch.float64, device=dev)
    d_tj = torch.full((nk * nE,), float("nan"), dtype=torch.float64, device=dev)
    d_info = torch.full((nk * nE,), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    with Engine(*pr.engine_args()) as eng:
        tau_host, info_host = eng.transmission(E, precision=NEGF_MIXED)
        eng.transmission_device(d_E.data_ptr(), nE, d_tau.data_ptr(), d_tj.data_ptr(), d_info.data_ptr(),
                                stream.cuda_stream, precision=NEGF_MIXED)
        stream.synchronize()
    assert info_host == 0
    np.testing.assert_array_equal(d_tau.cpu().numpy(), tau_host)
    assert (d_info.cpu().numpy() == 0).all()
    tj = d_tj.cpu().numpy().reshape(nk, nE)
    np.testing.assert_allclose(kpt[:, 2] @ tj, tau_host, rtol=1e-14, atol=1e-15)
    ref = _oracle(pr, E)
    assert np.max(np.abs(tau_host - ref)) <= TOL_MIXED
