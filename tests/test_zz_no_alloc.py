"""The allocation-free transmission entry (negf_transmission_noalloc).

It is for callers that may not allocate device memory themselves -- code
running inside another framework's memory pool or under a device-memory
budget fixed at start-up -- so everything is handed in as device pointers and
the library works in one fixed scratch array.  The test allocates its own
buffers with torch (the caller's memory), then checks, on two calls in a row,
that the entry reproduces both the CPU oracle and the context-based
negf_transmission within the FP64 tolerance of the other parity tests.  It
also covers a basis so large that only one job fits in the scratch at a time,
a call without the optional info array, and the refusals (a problem larger
than the scratch, a basis difference outside the V table).  This file is
collected last.
"""
import numpy as np
import pytest

from negftrans_b200 import _lib
from negftrans_b200 import prepare as P
from negftrans_b200 import workloads as W
from negftrans_b200.negf import Engine

pytestmark = pytest.mark.gpu

RTOL = 1e-9


def _call(pr, d, E, tau, info, stream):
    a = pr.atomic
    return _lib.lib().negf_transmission_noalloc(
        pr.N, pr.Nz, pr.NGX, pr.NGY, d["nx"].data_ptr(), d["ny"].data_ptr(), d["vhat"].data_ptr(),
        a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, len(pr.kpoint), d["kpt"].data_ptr(), E.data_ptr(),
        E.numel(), tau.data_ptr(), info.data_ptr() if info is not None else None, stream)


def _device_inputs(torch, pr):
    dev = torch.device("cuda", 0)
    return {
        "nx": torch.from_numpy(pr.nx.astype(np.int32)).to(dev),
        "ny": torch.from_numpy(pr.ny.astype(np.int32)).to(dev),
        # V table in its Fortran memory order, complex as interleaved doubles
        "vhat": torch.from_numpy(np.ascontiguousarray(pr.vhat.ravel(order="F")).view(np.float64)).to(dev),
        "kpt": torch.from_numpy(np.ascontiguousarray(pr.kpoint, np.float64)).to(dev),
    }


def _problem(name, nz, ne, nk):
    if name == "small":
        V = W.MSTAR * W.qpc_potential(32, 32, nz, 100.0, nz * 1.0, 0.05, 15.0, 1.2, disorder=0.002)
        pr = P.prepare(W._deck(nz * 10.0, 1.2e-3, 30.0, ne, nk=nk), V)
        return pr, P.transmission_energies(pr.atomic, ne)
    w = W.config(name, nz=nz)
    pr = P.prepare(w.deck, w.V_eV)
    # every n-th point of the workload's own grid, so the batch spans its window
    E = P.transmission_energies(pr.atomic, w.n_energy)
    return pr, np.ascontiguousarray(E[:: max(1, len(E) // ne)][:ne])


def _oracle_tau(pr, E):
    from oracle import oracle as O
    a = pr.atomic
    p = O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    tau, info = O.transmission_jobs(p, E, nthreads=8)
    assert info == 0
    return tau


# "qpc_disorder_n797": one job's workspace (64 * 800 * 797 bytes) leaves room
# for a single job in the 64 MiB scratch, so the persistent loop runs on one CTA
@pytest.mark.parametrize("name,nz,ne,nk", [("small", 12, 40, 2), ("qpc_disorder_n221", 16, 24, 1),
                                           ("qpc_disorder_n797", 4, 3, 1)])
def test_noalloc_matches_oracle_and_context_entry_twice(name, nz, ne, nk):
    import torch

    pr, E_host = _problem(name, nz, ne, nk)
    ref = _oracle_tau(pr, E_host)
    with Engine(*pr.engine_args()) as eng:
        ctx_tau, info_ctx = eng.transmission(E_host)
    assert info_ctx == 0
    np.testing.assert_allclose(ctx_tau, ref, rtol=RTOL, atol=1e-12)

    d = _device_inputs(torch, pr)
    E = torch.from_numpy(np.ascontiguousarray(E_host)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        tau = torch.full((len(E_host),), float("nan"), dtype=torch.float64, device="cuda")
        info = torch.full((len(E_host) * len(pr.kpoint),), -7, dtype=torch.int32, device="cuda")
        assert _call(pr, d, E, tau, info, stream) == _lib.NEGF_OK
        torch.cuda.synchronize()
        got = tau.cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=1e-12)
        np.testing.assert_allclose(got, ctx_tau, rtol=RTOL, atol=1e-12)
        assert int((info != 0).sum()) == 0


def test_noalloc_without_info_array():
    import torch

    pr, E_host = _problem("small", 8, 12, 1)
    ref = _oracle_tau(pr, E_host)
    d = _device_inputs(torch, pr)
    E = torch.from_numpy(np.ascontiguousarray(E_host)).cuda()
    tau = torch.full((len(E_host),), float("nan"), dtype=torch.float64, device="cuda")
    assert _call(pr, d, E, tau, None, torch.cuda.current_stream().cuda_stream) == _lib.NEGF_OK
    torch.cuda.synchronize()
    np.testing.assert_allclose(tau.cpu().numpy(), ref, rtol=RTOL, atol=1e-12)


def test_noalloc_rejects_oversized_problem():
    import torch

    # N = 1024 needs 64 MiB of workspace for one job, more than the scratch holds
    z = torch.zeros(16, dtype=torch.float64, device="cuda")
    zi = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = _lib.lib().negf_transmission_noalloc(
        1024, 4, 40, 40, zi.data_ptr(), zi.data_ptr(), z.data_ptr(), 1.0, 1.0, 1.0, 0.0, 0.0, 1e-9,
        1, z.data_ptr(), z.data_ptr(), 1, z.data_ptr(), None, None)
    assert rc == _lib.NEGF_ERR_TOO_LARGE


def test_noalloc_rejects_basis_outside_table():
    import torch

    # n_x spans 0..5 but the table only holds differences |dn_x| <= 2: the
    # check kernel flags it before any sweep is enqueued
    nx = torch.tensor([0, 1, 5, 0], dtype=torch.int32, device="cuda")
    ny = torch.zeros(4, dtype=torch.int32, device="cuda")
    vhat = torch.zeros(2 * 5 * 1 * 4, dtype=torch.float64, device="cuda")  # (5, 1, 4) complex
    kpt = torch.tensor([0.0, 0.0, 1.0], dtype=torch.float64, device="cuda")
    E = torch.tensor([1e-4], dtype=torch.float64, device="cuda")
    tau = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _lib.lib().negf_transmission_noalloc(
        4, 4, 2, 0, nx.data_ptr(), ny.data_ptr(), vhat.data_ptr(), 100.0, 100.0, 100.0, 0.0, 0.0, 1e-9,
        1, kpt.data_ptr(), E.data_ptr(), 1, tau.data_ptr(), None, torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.NEGF_ERR_ARG
