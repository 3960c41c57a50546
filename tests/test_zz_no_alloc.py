"""The allocation-free transmission entry (negf_transmission_noalloc).

It is for callers that may not allocate device memory themselves -- code
running inside another framework's memory pool or under a device-memory
budget fixed at start-up -- so everything is handed in as device pointers and
the library works in one fixed scratch array.  The test allocates its own
buffers with torch (the caller's memory), then checks, on two calls in a row,
that the entry reproduces the context-based negf_transmission within the
FP64 tolerance of the other parity tests.  This file is collected last.
"""
import ctypes as C

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


@pytest.mark.parametrize("name,nz,ne,nk", [("small", 12, 40, 2), ("qpc_disorder_n221", 16, 24, 1)])
def test_noalloc_matches_context_entry_twice(name, nz, ne, nk):
    import torch

    if name == "small":
        V = W.MSTAR * W.qpc_potential(32, 32, nz, 100.0, nz * 1.0, 0.05, 15.0, 1.2, disorder=0.002)
        pr = P.prepare(W._deck(nz * 10.0, 1.2e-3, 30.0, ne, nk=nk), V)
    else:
        w = W.config(name, nz=nz)
        pr = P.prepare(w.deck, w.V_eV)
    E_host = P.transmission_energies(pr.atomic, 2048)[:ne] if name != "small" else \
        P.transmission_energies(pr.atomic, ne)
    with Engine(*pr.engine_args()) as eng:
        ref, info_ref = eng.transmission(E_host)
    assert info_ref == 0

    d = _device_inputs(torch, pr)
    E = torch.from_numpy(np.ascontiguousarray(E_host)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        tau = torch.full((ne,), float("nan"), dtype=torch.float64, device="cuda")
        info = torch.full((ne * len(pr.kpoint),), -7, dtype=torch.int32, device="cuda")
        assert _call(pr, d, E, tau, info, stream) == _lib.NEGF_OK
        torch.cuda.synchronize()
        np.testing.assert_allclose(tau.cpu().numpy(), ref, rtol=RTOL, atol=1e-12)
        assert int((info != 0).sum()) == 0


def test_noalloc_rejects_oversized_problem():
    import torch

    # N = 1024 needs 64 MiB of workspace for one job, more than the scratch holds
    z = torch.zeros(16, dtype=torch.float64, device="cuda")
    zi = torch.zeros(16, dtype=torch.int32, device="cuda")
    rc = _lib.lib().negf_transmission_noalloc(
        1024, 4, 40, 40, zi.data_ptr(), zi.data_ptr(), z.data_ptr(), 1.0, 1.0, 1.0, 0.0, 0.0, 1e-9,
        1, z.data_ptr(), z.data_ptr(), 1, z.data_ptr(), None, None)
    assert rc == _lib.NEGF_ERR_TOO_LARGE
