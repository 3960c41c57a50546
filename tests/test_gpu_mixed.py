"""Tensor-core arithmetic of the mixed-precision path, against NumPy FP64.

* The split-fp16 complex product of the trailing update (tcgen05 MMAs, FP32
  accumulation in tensor memory, one power-of-two exponent per row of W and
  per column of B): normwise relative error below 2e-6 (three split products
  keep ~2^-21), on operands whose rows and columns span 1e-15 .. 1e15.
* The FP32 blocked Gauss-Jordan inverse with partial pivoting and rank-32
  tensor-core trailing updates: ||X A - I|| / (||X|| ||A||) below 1e-6 for
  N from 5 to 797 (FP32 rounding of A itself is ~6e-8).
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
    # and some rows that need pivoting
    perm = rng.permutation(N)
    A = A[perm].astype(np.complex64)
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
