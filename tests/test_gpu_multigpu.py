"""The multi-GPU layer (negftrans_b200.multigpu.ShardedEngine) on the GPU with
the Engine as the per-rank solver, in a one-rank NCCL group (every run here
gets one GPU): transmission (mixed and FP64) and the density through the
z-slab reduce-scatter, slab PtoR on the GPU and the density all-gather must
reproduce the single-process engine entries.  The exchange logic itself is
tested with two gloo ranks in test_dist.py."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.fixture(scope="module")
def nccl_group():
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60),
                            device_id=torch.device("cuda", 0))
    yield
    dist.destroy_process_group()


def test_sharded_engine_one_rank_matches_engine(nccl_group):
    import torch

    from negftrans_b200 import prepare as P, workloads as W
    from negftrans_b200._lib import NEGF_FP64, NEGF_MIXED
    from negftrans_b200.multigpu import ShardedEngine
    from negftrans_b200.negf import Engine
    w = W.config("qpc_n69", nz=40)
    pr = P.prepare(w.deck, w.V_eV)
    a, d = pr.atomic, w.deck
    Nx, Ny, Nz = pr.shape
    E = P.transmission_energies(a, w.n_energy)[::8]
    with Engine(*pr.engine_args()) as eng:
        sh = ShardedEngine(eng, pr.Nz, device=torch.device("cuda", 0))
        for prec in (NEGF_FP64, NEGF_MIXED):
            tau, info = sh.transmission(E, precision=prec)
            ref, info_ref = eng.transmission(E, precision=prec)
            assert info == info_ref == 0
            np.testing.assert_allclose(tau, ref, rtol=1e-12, atol=1e-14)
        nl = P.n_line(a, d.N_line_per_eV)
        dens, dm_slab, info = sh.density(d.N_circle, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE, Nx, Ny, d.LX, d.LY,
                                         d.LZ)
        dens_ref, dm_ref, info_ref = eng.density_real(d.N_circle, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE, Nx, Ny,
                                                      d.LX, d.LY, d.LZ)
    assert info == info_ref == 0
    assert np.max(np.abs(dm_slab - dm_ref)) <= 1e-10 * np.max(np.abs(dm_ref))
    assert np.max(np.abs(dens - dens_ref)) <= 1e-10 * np.max(np.abs(dens_ref))
