"""Initial conditions, generated once on the host in FP64 and uploaded unchanged.

Every state array uses the reference's layout: ``vars(3, -1:m_xi+2, -1:m_eta+2)`` in
column-major order, i.e. a C-contiguous numpy array of shape ``(m_eta+4, m_xi+4, 3)`` indexed
``[j+1, i+1, me]``.  Ghost cells are set too, as the reference sets them
(``examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:33-46`` loops over the
padded block); the first ghost fill overwrites all but the four corner blocks.

Cell centres follow ``domain/SMOD_mesh_manipulation.f90:50-51``:
``xi(i) = (xi_min + (i-1)*d_xi) + d_xi/2`` with ``d_xi = (xi_max - xi_min)/m_xi``; the
identity mapping makes them the physical coordinates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Tuple

import numpy as np


def cell_centres(m_xi: int, m_eta: int, xi_min=-1.0, xi_max=1.0, eta_min=-1.0, eta_max=1.0
                 ) -> Tuple[np.ndarray, np.ndarray]:
    """Cell-centre coordinates (length m+4 vectors over i, j = -1 .. m+2)."""
    d_xi = (xi_max - xi_min) / m_xi
    d_eta = (eta_max - eta_min) / m_eta
    i = np.arange(-1, m_xi + 3, dtype=np.float64)
    j = np.arange(-1, m_eta + 3, dtype=np.float64)
    x = (xi_min + (i - 1.0) * d_xi) + d_xi / 2
    y = (eta_min + (j - 1.0) * d_eta) + d_eta / 2
    return x, y


def empty_state(m_xi: int, m_eta: int) -> np.ndarray:
    return np.zeros((m_eta + 4, m_xi + 4, 3), dtype=np.float64)


def circular_dam(m_xi: int, m_eta: int, radius: float = 0.5, h_in: float = 2.0, h_out: float = 1.0,
                 x0: float = 0.0, y0: float = 0.0, domain=(-1.0, 1.0, -1.0, 1.0)) -> np.ndarray:
    """Dam break: h = h_in where sqrt(x^2 + y^2) < radius (strict), else h_out; u = v = 0.

    With the defaults this is the reference example's IC
    (examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:34-46): the same
    expression ``sqrt(x**2 + y**2) < 0.5`` evaluated without contraction.  A non-zero centre
    shifts x and y first.
    """
    x, y = cell_centres(m_xi, m_eta, *domain)
    xs = x - x0 if x0 != 0.0 else x
    ys = y - y0 if y0 != 0.0 else y
    r = np.sqrt(xs[None, :] * xs[None, :] + ys[:, None] * ys[:, None])
    q = empty_state(m_xi, m_eta)
    q[..., 0] = np.where(r < radius, h_in, h_out)
    return q


@dataclass
class DamParams:
    radius: float
    h_in: float
    h_out: float
    x0: float
    y0: float


def seeded_dam_params(seed: int, offset: float = 0.0) -> DamParams:
    """Seeded dam: radius ~ U(0.2, 0.6), h_in/h_out ~ U(1.5, 5) with h_out = 1, and a centre
    offset ~ U(-offset, offset)^2."""
    rng = np.random.Generator(np.random.PCG64(seed))
    radius = float(rng.uniform(0.2, 0.6))
    ratio = float(rng.uniform(1.5, 5.0))
    x0, y0 = (float(v) for v in rng.uniform(-offset, offset, size=2)) if offset > 0 else (0.0, 0.0)
    return DamParams(radius=radius, h_in=ratio, h_out=1.0, x0=x0, y0=y0)


def seeded_dam(m: int, seed: int, offset: float = 0.0) -> np.ndarray:
    p = seeded_dam_params(seed, offset)
    return circular_dam(m, m, p.radius, p.h_in, p.h_out, p.x0, p.y0)


@dataclass
class Bump:
    amplitude: float
    width: float
    cx: float
    cy: float


def gaussian_bump_params(seed: int, n: int = 16, domain=(-1.0, 1.0, -1.0, 1.0)) -> List[Bump]:
    """16 bumps: amplitude ~ U(0.1, 1.0), width ~ U(0.02, 0.1), centre uniform in the domain."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.uniform(0.1, 1.0, size=n)
    w = rng.uniform(0.02, 0.1, size=n)
    cx = rng.uniform(domain[0], domain[1], size=n)
    cy = rng.uniform(domain[2], domain[3], size=n)
    return [Bump(float(a[k]), float(w[k]), float(cx[k]), float(cy[k])) for k in range(n)]


def gaussian_bumps(m_xi: int, m_eta: int, seed: int = 0, n: int = 16,
                   domain=(-1.0, 1.0, -1.0, 1.0)) -> np.ndarray:
    """h = 1 + sum_k A_k exp(-(x-cx_k)^2/(2 w_k^2)) exp(-(y-cy_k)^2/(2 w_k^2)), u = v = 0.

    The product of two 1D Gaussians equals the 2D bump; evaluating it as an outer product
    fixes the bits (this generator defines them) and keeps 8192^2 grids cheap to build.
    """
    x, y = cell_centres(m_xi, m_eta, *domain)
    h = np.ones((m_eta + 4, m_xi + 4), dtype=np.float64)
    for b in gaussian_bump_params(seed, n, domain):
        s = 2.0 * b.width * b.width
        gx = np.exp(-((x - b.cx) ** 2) / s)
        gy = np.exp(-((y - b.cy) ** 2) / s)
        h += b.amplitude * np.outer(gy, gx)
    q = empty_state(m_xi, m_eta)
    q[..., 0] = h
    return q


def lake_at_rest(m_xi: int, m_eta: int, h: float = 1.0) -> np.ndarray:
    q = empty_state(m_xi, m_eta)
    q[..., 0] = h
    return q


def log_uniform_sides(n: int, lo: int, hi: int, multiple: int, seed: int) -> List[int]:
    """Square grid sides drawn log-uniform in [lo, hi], rounded to a multiple, clamped."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = rng.uniform(math.log(lo), math.log(hi), size=n)
    sides = [int(min(max(multiple * round(math.exp(v) / multiple), lo), hi)) for v in u]
    return sides
