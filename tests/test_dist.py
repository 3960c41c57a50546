"""Multi-process sharding on CPU (gloo, world_size 2): the product
multi-GPU layer (negftrans_b200.multigpu.ShardedEngine) -- the job split, the
all-gather of tau, the reduce-scatter of Density_Matrix by z-slab, the
per-slab PtoR and the all-gather of the density -- that replaces the MPI
loops and collectives of src/main.f90.  Only the per-rank solver is a CPU
stand-in (the oracle behind the Engine's method names), so no GPU is used."""
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


def test_contour_matches_oracle_quadrature(oracle):
    """The host contour of the multi-GPU density against the oracle's Simpson
    and Fermi restatement (math_kernel.f90:167-223)."""
    from negftrans_b200 import contour as Ct
    for n in (2, 3, 4, 5, 8, 9, 48):
        for i in range(1, n + 1):
            assert Ct.coefficient_simpson(i, n, 0.1, 2.3) == pytest.approx(oracle.coefficient_simpson(i, n, 0.1, 2.3),
                                                                            rel=1e-15)
            assert Ct.value_simpson(i, n, 0.1, 2.3) == pytest.approx(oracle.value_simpson(i, n, 0.1, 2.3), rel=1e-15)
    assert Ct.fermi_func(1e-3, 2e-3, 300.0) == pytest.approx(oracle.fermi_func(1e-3, 2e-3, 300.0), rel=1e-14)
    E, w = Ct.equilibrium_contour(6, 5, -0.01, 0.02, 1e-3, 50.0)
    # the semicircle starts at min(V) - 1 eV and ends at mu - GAP; the line spans mu +- GAP
    assert E[0].real == pytest.approx(0.02 - 1e-3, rel=1e-12) and abs(E[0].imag) < 1e-15
    assert E[5].real == pytest.approx(-0.01 - 1 / 27.211386245988, rel=1e-12)
    assert E[6] == pytest.approx(0.02 - 1e-3) and E[-1] == pytest.approx(0.02 + 1e-3)


def _problem():
    from negftrans_b200 import prepare as P, workloads as W
    from oracle import oracle as O
    V = W.MSTAR * W.qpc_potential(16, 16, 7, 100.0, 7.0, 0.05, 15.0, 1.0, disorder=0.002)
    d = W._deck(70.0, 0.6e-3, 30.0, 9, nk=2)
    pr = P.prepare(d, V)
    a = pr.atomic
    p = O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    return pr, p, d


class OracleSolver:
    """The Engine's per-rank methods computed by the CPU oracle (test stand-in)."""

    def __init__(self, p):
        from oracle import oracle as O
        self.O, self.p, self.N = O, p, p.N

    def transmission(self, E, precision=0):
        return self.O.transmission_jobs(self.p, E)

    def density_accumulate(self, E, w):
        return self.O.density_accumulate(self.p, E, w)

    def dm_real_slab(self, dm_slab, Nx, Ny, LX_A, LY_A, LZ_A):
        scale = self.p.Nz / (LX_A * LY_A * LZ_A)
        return np.stack([self.O.ptor(dm_slab[:, :, k], self.p.nx, self.p.ny, Nx, Ny).imag * scale
                         for k in range(dm_slab.shape[2])], axis=2)


def _worker(rank, world, port, q, mode):
    import datetime

    import torch.distributed as dist

    from negftrans_b200 import prepare as P
    from negftrans_b200.multigpu import ShardedEngine
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        pr, p, d = _problem()
        E = P.transmission_energies(pr.atomic, 9)
        if mode == "fail" and rank == 1:
            raise SystemExit(3)   # this rank dies before the exchange
        eng = ShardedEngine(OracleSolver(p), pr.Nz)
        tau, info = eng.transmission(E)
        a = pr.atomic
        Nx, Ny, _ = pr.shape
        dens, dm_slab, info_d = eng.density(4, 5, pr.min_V, a.MU, a.GAP, a.TEMPERATURE, Nx, Ny, d.LX, d.LY, d.LZ)
        q.put((rank, "ok", tau, (dens, dm_slab, eng.z_slab(), info + info_d)))
    except SystemExit:
        q.put((rank, "exit", None, None))
    except Exception as e:  # the surviving rank must see an error, not hang
        q.put((rank, "error:" + type(e).__name__, None, None))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q, mode)) for r in range(world)]
    for pr_ in ps:
        pr_.start()
    out = {}
    for _ in ps:
        r, status, tau, rest = q.get(timeout=180)
        out[r] = (status, tau, rest)
    for pr_ in ps:
        pr_.join(timeout=60)
        if pr_.is_alive():
            pr_.kill()
    return out


def test_sharded_transmission_and_density_match_single_process(oracle):
    from negftrans_b200 import prepare as P
    out = _run("ok")
    pr, p, d = _problem()
    E = P.transmission_energies(pr.atomic, 9)
    tau_ref, _ = oracle.transmission_jobs(p, E)
    a = pr.atomic
    Nx, Ny, Nz = pr.shape
    dm_ref, _ = oracle.density_jobs(p, 4, 5, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
    dens_ref = oracle.density_from_matrix(dm_ref, pr.nx, pr.ny, Nx, Ny, d.LX, d.LY, d.LZ)
    for r in (0, 1):
        status, tau, (dens, dm_slab, (lo, hi), info) = out[r]
        assert status == "ok" and info == 0
        np.testing.assert_allclose(tau, tau_ref, rtol=1e-13, atol=1e-16)
        # the rank's slab of the summed Density_Matrix, and the whole density on every rank
        assert np.max(np.abs(dm_slab - dm_ref[:, :, lo:hi])) < 1e-12 * np.max(np.abs(dm_ref))
        assert np.max(np.abs(dens - dens_ref)) < 1e-12 * np.max(np.abs(dens_ref))
    # the two slabs partition the device
    assert out[0][2][2] == (0, 4) and out[1][2][2] == (4, 7)


def test_rank_loss_is_reported_not_hung():
    out = _run("fail")
    assert out[1][0] == "exit"
    assert out[0][0].startswith("error:")
