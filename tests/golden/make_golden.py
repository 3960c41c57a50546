"""Generate tests/golden/oracle_small.npz from the CPU oracle.

The reference publishes no outputs and cannot be built in this image, so
these fixtures are oracle outputs on a small seeded problem: they pin the
oracle against regressions and let the GPU tests compare against committed
numbers.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from negftrans_b200 import prepare as P, workloads as W  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main():
    V = W.MSTAR * W.qpc_potential(16, 16, 8, 100.0, 8.0, 0.05, 15.0, 1.0, disorder=0.002, seed=1234)
    d = W._deck(80.0, 0.6e-3, 30.0, 12, nk=2)
    pr = P.prepare(d, V)
    a = pr.atomic
    p = O.Problem(pr.nx, pr.ny, pr.vhat, a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA, pr.kpoint)
    E = P.transmission_energies(a, 12)
    tau, _ = O.transmission_jobs(p, E)
    rng = np.random.default_rng(99)
    D = rng.standard_normal((4, 4, 3)) + 1j * rng.standard_normal((4, 4, 3))
    tri, _ = O.tri_solver(D, "DFL")
    nc, nl = 4, 5
    dm, _ = O.density_jobs(p, nc, nl, pr.min_V, a.MU, a.GAP, a.TEMPERATURE)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle_small.npz")
    np.savez_compressed(
        out, nx=pr.nx, ny=pr.ny, vhat=pr.vhat, kpt=pr.kpoint,
        params=np.array([a.LX, a.LY, a.LZ, a.V_L, a.V_R, a.ETA]), energies=E, tau=tau, D=D,
        tri_D=tri["D"], tri_F=tri["F"], tri_L=tri["L"], n_circle=nc, n_line=nl, min_v=pr.min_V,
        mu=a.MU, gap=a.GAP, temperature=a.TEMPERATURE, dm=dm)
    print(out, "N", pr.N, "Nz", pr.Nz, "tau", tau)


if __name__ == "__main__":
    main()
