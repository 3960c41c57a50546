"""The equilibrium-density energy contour of src/negf.f90 (lines 37-65, 86-111)
with the quadrature of src/math_kernel.f90 (lines 167-223), on the host.

Equilibrium_Density integrates G over a semicircle from min(V) - 1 eV to
mu - GAP (angles on a Simpson grid over [0, pi]) and over the real line
[mu - GAP, mu + GAP] (Simpson nodes weighted by the Fermi function).  The
points and weights here are the ones negf_density uses on the GPU; with them,
negf_density_accumulate (any contour) reproduces it.  The multi-GPU density
splits these points between ranks.
"""
from __future__ import annotations

import math

import numpy as np

from .constants import HARTREE, K_B, PI


def coefficient_simpson(i: int, n: int, a: float, b: float) -> float:
    """Weight of node i (1-based) of n on [a, b] (math_kernel.f90:167-204):
    composite Simpson 1/3 for odd n; for even n, Simpson 1/3 up to node n-3
    and the 3/8 rule over the last four nodes."""
    if n % 2 == 1:
        c = 1.0 / 3 if i in (1, n) else (4.0 / 3 if i % 2 == 0 else 2.0 / 3)
    elif i == 1:
        c = 1.0 / 3
    elif i == n - 3:
        c = 1.0 / 3 + 1.0 * 3 / 8
    elif i in (n - 2, n - 1):
        c = 3.0 * 3 / 8
    elif i == n:
        c = 1.0 * 3 / 8
    else:
        c = 4.0 / 3 if i % 2 == 0 else 2.0 / 3
    return c * (b - a) / (n - 1)


def value_simpson(i: int, n: int, a: float, b: float) -> float:
    """Node i (1-based) of n uniform nodes on [a, b] (math_kernel.f90:206-216)."""
    return (i - 1) * (b - a) / (n - 1) + a


def fermi_func(energy: float, mu: float, temperature: float) -> float:
    """1 / (exp((E - mu) / k_B T) + 1), Hartree and K (math_kernel.f90:218-223)."""
    return 1.0 / (math.exp((energy - mu) / (K_B * temperature)) + 1.0)


def equilibrium_contour(n_circle: int, n_line: int, min_v: float, mu: float, gap: float, temperature: float):
    """Complex energies E_i (without the i*eta of the solve) and weights w_i,
    i = 1 .. n_circle + n_line, such that
        Density_Matrix = sum_k w_k sum_i w_i 2 dz^2 G_kk(E_i + i eta)
    is the accumulation of negf.f90:86-111.  Energies in Hartree."""
    if n_circle < 2 or n_line < 2:
        raise ValueError("the contour needs at least two circle and two line points")
    circle_l, circle_r = min_v - 1.0 / HARTREE, mu - gap          # negf.f90:37-44
    e_c, e_r = (circle_r + circle_l) / 2, (circle_r - circle_l) / 2
    E = np.zeros(n_circle + n_line, np.complex128)
    w = np.zeros(n_circle + n_line, np.complex128)
    for i in range(1, n_circle + 1):
        th = value_simpson(i, n_circle, 0.0, PI)
        E[i - 1] = complex(e_c + e_r * math.cos(th), e_r * math.sin(th))
        # (2/pi) c_i * i E_R e^{i theta}                            negf.f90:88-97
        w[i - 1] = 2.0 / PI * coefficient_simpson(i, n_circle, 0.0, PI) * 1j * e_r * complex(math.cos(th),
                                                                                          math.sin(th))
    lo, hi = mu - gap, mu + gap
    for i in range(1, n_line + 1):
        x = value_simpson(i, n_line, lo, hi)
        E[n_circle + i - 1] = x
        # -(2/pi) c_i f(x)                                          negf.f90:99-110
        w[n_circle + i - 1] = -2.0 / PI * coefficient_simpson(i, n_line, lo, hi) * fermi_func(x, mu, temperature)
    return E, w
