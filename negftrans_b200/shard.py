"""Multi-GPU sharding of the (E, k) job space: one process per GPU.

Replaces the MPI job loops of src/main.f90 (round-robin i_job = rank+1,
+mpi_size at lines 274-282 and 385-391) and the MPI_Reduce of tau
(main.f90:401-407) and of Density_Matrix (main.f90:291-297).  Every (E,k)
solve is independent, so each rank takes a contiguous slice of the energy
grid (all k-points of those energies stay on one rank, so the k-sum of
negf.f90:172 is local) and the only exchange is one collective at the end:
an all-gather of tau, or an all-reduce of the density matrix.

The compute callable is injected, so the same code runs with the GPU engine
(NCCL) and, in tests, with a CPU stand-in (gloo).
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def energy_shard(n_e: int, rank: int, world: int):
    """Contiguous slice [lo, hi) of the energy grid owned by `rank`.

    The first n_e % world ranks take one extra energy, so slices differ in
    length by at most one."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_e, world)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def transmission_sharded(solve: Callable[[np.ndarray], np.ndarray], energies, group=None,
                         device=None):
    """tau over the whole grid; `solve(E_slice) -> tau_slice` runs on this rank.

    torch.distributed must be initialised; the result is identical on every
    rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    energies = np.asarray(energies, np.float64)
    n_e = len(energies)
    lo, hi = energy_shard(n_e, rank, world)
    local = np.asarray(solve(energies[lo:hi]), np.float64) if hi > lo else np.zeros(0)
    # pad to the longest slice so all ranks exchange equal-sized buffers
    width = energy_shard(n_e, 0, world)[1]
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[: hi - lo] = torch.from_numpy(local).to(buf.device)
    out = torch.zeros(world * width, dtype=torch.float64, device=device)
    dist.all_gather_into_tensor(out, buf, group=group)
    out = out.cpu().numpy().reshape(world, width)
    tau = np.empty(n_e)
    for r in range(world):
        a, b = energy_shard(n_e, r, world)
        tau[a:b] = out[r, : b - a]
    return tau


def density_sharded(solve_jobs: Callable[[int, int], np.ndarray], n_jobs: int, group=None,
                    device=None):
    """Density_Matrix summed over all jobs; `solve_jobs(lo, hi)` returns the
    partial (N, N, N_z) complex sum of jobs [lo, hi) on this rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    lo, hi = energy_shard(n_jobs, rank, world)
    part = np.asarray(solve_jobs(lo, hi), np.complex128)
    t = torch.from_numpy(np.ascontiguousarray(part).view(np.float64)).to(device)
    dist.all_reduce(t, group=group)
    return t.cpu().numpy().view(np.complex128).reshape(part.shape)
