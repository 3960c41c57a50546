"""Multi-GPU execution of the hot path: one process per GPU, torch.distributed
(NCCL between GPUs) for the exchanges.

What it replaces in src/main.f90:
* the (E, k) job loops with round-robin ranks (lines 274-282, 385-391): each
  rank takes a contiguous slice of the energy grid or of the density contour
  (with every k-point of those energies, so the k-sum of negf.f90:172 and
  86-111 stays local);
* MPI_Reduce of tau (lines 401-407): one all-gather of the tau slices;
* MPI_Reduce of Density_Matrix + MPI_Scatter of z-slices (lines 291-321):
  one reduce-scatter of the partial Density_Matrix by z-slab, so each rank
  receives the summed slices it converts;
* Greensfunction_PlanewaveToReal per slice (lines 326-334): on the rank's own
  slab, on its GPU;
* MPI_Gather of the real-space slices (lines 339-340) and the scaling of
  lines 341-351: one all-gather of the density slabs.

The per-rank solver is an Engine on the rank's device (or, in CPU tests, an
object with the same four methods).  Collectives run on `device` tensors:
CUDA tensors over NCCL on GPUs, CPU tensors over gloo in tests.
"""
from __future__ import annotations

import numpy as np

from .contour import equilibrium_contour
from .shard import energy_shard


def _dist():
    import torch.distributed as dist
    return dist


class ShardedEngine:
    """The hot path of one problem split over the ranks of a process group.

    backend: this rank's solver, with transmission(E, precision) -> (tau, info),
    density_accumulate(E, w) -> (dm, info) and dm_real_slab(dm_slab, Nx, Ny,
    LX_A, LY_A, LZ_A) -> density slab (an Engine).  Nz: slices of the device."""

    def __init__(self, backend, Nz: int, group=None, device=None):
        self.backend = backend
        self.Nz = int(Nz)
        self.group = group
        self.device = device
        dist = _dist()
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)

    # ---------------------------------------------------------- transmission
    def transmission(self, energies, precision=0):
        """tau(E) = sum_k w_k tau(E, k) on the whole grid, on every rank, and the
        largest info of any rank's jobs."""
        import torch
        dist = _dist()
        E = np.ascontiguousarray(energies, np.float64)
        n_e = len(E)
        lo, hi = energy_shard(n_e, self.rank, self.world)
        if hi > lo:
            local, info = self.backend.transmission(E[lo:hi], precision=precision)
        else:
            local, info = np.zeros(0), 0
        width = energy_shard(n_e, 0, self.world)[1]   # the longest slice
        buf = torch.zeros(width + 1, dtype=torch.float64, device=self.device)
        buf[: hi - lo] = torch.from_numpy(np.asarray(local, np.float64)).to(buf.device)
        buf[width] = float(info)
        out = torch.empty(self.world * (width + 1), dtype=torch.float64, device=self.device)
        dist.all_gather_into_tensor(out, buf, group=self.group)
        out = out.cpu().numpy().reshape(self.world, width + 1)
        tau = np.empty(n_e)
        for r in range(self.world):
            a, b = energy_shard(n_e, r, self.world)
            tau[a:b] = out[r, : b - a]
        return tau, int(out[:, width].max())

    # ----------------------------------------------------------------- density
    def z_slab(self, rank=None):
        """Slices [lo, hi) whose density `rank` converts (balanced to one slice)."""
        return energy_shard(self.Nz, self.rank if rank is None else rank, self.world)

    def density(self, n_circle, n_line, min_v, mu, gap, temperature, Nx, Ny, LX_A, LY_A, LZ_A):
        """The equilibrium density (Nx, Ny, Nz) in Angstrom^-3 (main.f90:258-351)
        on every rank, the rank's summed Density_Matrix slab (N, N, hi-lo) and the
        largest info."""
        import torch
        dist = _dist()
        E, w = equilibrium_contour(n_circle, n_line, min_v, mu, gap, temperature)
        lo, hi = energy_shard(len(E), self.rank, self.world)
        if hi > lo:
            dm, info = self.backend.density_accumulate(E[lo:hi], w[lo:hi])
        else:
            dm, info = None, 0
        N = dm.shape[0] if dm is not None else self._basis_size()
        Nz, world = self.Nz, self.world
        slab = energy_shard(Nz, 0, world)[1]           # the widest slab
        # partial Density_Matrix as world equal blocks of `slab` slices (z-major,
        # padded), summed and scattered in one collective
        send = np.zeros((world, slab, N, N), np.complex128)
        if dm is not None:
            dmz = np.transpose(np.asarray(dm), (2, 1, 0))  # [z][j][i]: slice z contiguous, Fortran (i,j)
            for r in range(world):
                a, b = energy_shard(Nz, r, world)
                send[r, : b - a] = dmz[a:b]
        st = torch.from_numpy(send.view(np.float64).reshape(-1)).to(self.device)
        rt = torch.empty(slab * N * N * 2, dtype=torch.float64, device=self.device)
        dist.reduce_scatter_tensor(rt, st, group=self.group)
        mine = rt.cpu().numpy().view(np.complex128).reshape(slab, N, N)
        a, b = self.z_slab()
        dm_slab = np.asfortranarray(np.transpose(mine[: b - a], (2, 1, 0)))   # (N, N, b-a)
        dens_slab = np.zeros((Nx, Ny, slab))
        if b > a:
            dens_slab[:, :, : b - a] = self.backend.dm_real_slab(dm_slab, Nx, Ny, LX_A, LY_A, LZ_A)
        # gather the real-space slabs
        gs = torch.from_numpy(np.ascontiguousarray(np.transpose(dens_slab, (2, 1, 0))).reshape(-1)).to(self.device)
        gr = torch.empty(world * gs.numel(), dtype=torch.float64, device=self.device)
        dist.all_gather_into_tensor(gr, gs, group=self.group)
        allz = gr.cpu().numpy().reshape(world, slab, Ny, Nx)
        density = np.zeros((Nx, Ny, Nz), order="F")
        for r in range(world):
            ra, rb = energy_shard(Nz, r, world)
            density[:, :, ra:rb] = np.transpose(allz[r, : rb - ra], (2, 1, 0))
        it = torch.tensor([float(info)], dtype=torch.float64, device=self.device)
        dist.all_reduce(it, op=dist.ReduceOp.MAX, group=self.group)
        return density, dm_slab, int(it.item())

    def _basis_size(self):
        n = getattr(self.backend, "N", None)
        if n is None:
            raise RuntimeError("a rank without contour points needs backend.N")
        return int(n)
