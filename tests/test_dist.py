"""Multi-process sharding on CPU (gloo, world_size 2): the job split and the
tau / density exchange that replace the MPI loops and reductions of
src/main.f90.  The per-rank compute is the oracle (CPU), so no GPU is used."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from negftrans_b200.shard import energy_shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_energy_shard_partition():
    for n in (1, 7, 16, 2048):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = energy_shard(n, r, world)
                seen.extend(range(lo, hi))
            assert seen == list(range(n))
            sizes = [energy_shard(n, r, world)[1] - energy_shard(n, r, world)[0] for r in range(world)]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        energy_shard(4, 2, 2)


def _problem():
    from negftrans_b200 import prepare as P, workloads as W
    from oracle import oracle as O
    V = W.MSTAR * W.qpc_potential(16, 16, 6, 100.0, 6.0, 0.05, 15.0, 1.0, disorder=0.002)
    d = W._deck(60.0, 0.6e-3, 30.0, 9, nk=2)
    pr = P.prepare(d, V)
    a = pr.atomic
    p = O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    return pr, p


def _worker(rank, world, port, q, mode):
    import datetime

    import torch.distributed as dist

    from negftrans_b200.shard import density_sharded, transmission_sharded
    from negftrans_b200 import prepare as P
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        pr, p = _problem()
        E = P.transmission_energies(pr.atomic, 9)
        if mode == "fail" and rank == 1:
            raise SystemExit(3)   # this rank dies before the exchange
        tau = transmission_sharded(lambda e: O.transmission_jobs(p, e)[0], E)
        a = pr.atomic
        n_jobs = (4 + 5) * len(pr.kpoint)
        dm = density_sharded(lambda lo, hi: O.density_jobs(p, 4, 5, pr.min_V, a.MU, a.GAP, a.TEMPERATURE,
                                                           job_lo=lo, job_hi=hi)[0], n_jobs)
        q.put((rank, "ok", tau, dm))
    except SystemExit:
        q.put((rank, "exit", None, None))
    except Exception as e:  # the surviving rank must see an error, not hang
        q.put((rank, "error:" + type(e).__name__, None, None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(mode):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q, mode)) for r in range(2)]
    for pr_ in ps:
        pr_.start()
    out = {}
    for _ in ps:
        r, status, tau, dm = q.get(timeout=120)
        out[r] = (status, tau, dm)
    for pr_ in ps:
        pr_.join(timeout=60)
        if pr_.is_alive():
            pr_.kill()
    return out


def test_sharded_transmission_and_density_match_single_process(oracle):
    from negftrans_b200 import prepare as P
    out = _run("ok")
    pr, p = _problem()
    E = P.transmission_energies(pr.atomic, 9)
    tau_ref, _ = oracle.transmission_jobs(p, E)
    a = pr.atomic
    dm_ref, _ = oracle.density_jobs(p, 4, 5, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
    for r in (0, 1):
        status, tau, dm = out[r]
        assert status == "ok"
        np.testing.assert_allclose(tau, tau_ref, rtol=1e-13, atol=1e-16)
        assert np.max(np.abs(dm - dm_ref)) < 1e-12 * np.max(np.abs(dm_ref))


def test_rank_loss_is_reported_not_hung():
    out = _run("fail")
    assert out[1][0] == "exit"
    assert out[0][0].startswith("error:")
