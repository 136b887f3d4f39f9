"""Mapped (curvilinear) grids: the reference's mesh metrics from a coordinate mapping.

The reference maps each cell's corners through the user routine map_to_physical_coordinates
(user_subroutines/SMOD_coordinate_mapping.f90:35-43) and keeps, per cell, the capacity (physical
area over computational area) and the length ratios of its lower xi and eta faces
(domain/SMOD_mesh_manipulation.f90:129-176).  The step reads only those three arrays, so a mapped
grid is a uniform computational grid plus them (pcl_set_mesh_metrics).  ``metrics`` computes them
through the C ABI (pcl_compute_mesh_metrics), evaluating a Python mapping at every corner.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Tuple

import numpy as np

from . import _lib
from .control import ControlSettings
from .solver import to_c_control

Mapping = Callable[[float, float], Tuple[float, float]]


def metrics(control: ControlSettings, mapping: Optional[Mapping] = None) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(capacity, length_ratio_xi, length_ratio_eta), each shaped (m_eta+4, m_xi+4), for the grid of
    `control` under `mapping(xi, eta) -> (x, y)` (None: the identity)."""
    L = _lib.load()
    c = to_c_control(control)
    shape = (control.m_eta + 4, control.m_xi + 4)
    out = [np.empty(shape, dtype=np.float64) for _ in range(3)]
    cb = None
    if mapping is not None:
        def trampoline(xi, eta, xp, yp, _user):
            x, y = mapping(xi, eta)
            xp[0] = float(x)
            yp[0] = float(y)
        cb = _lib.MapFn(trampoline)
    fn = C.cast(cb, C.c_void_p) if cb is not None else None
    _lib.check(L.pcl_compute_mesh_metrics(C.byref(c), fn, None, *(a.ctypes.data for a in out)), "pcl_compute_mesh_metrics")
    return out[0], out[1], out[2]


def cell_centres(control: ControlSettings, mapping: Optional[Mapping] = None) -> Tuple[np.ndarray, np.ndarray]:
    """Physical cell centres (x, y) of the padded grid: the computational centre
    xi_min + (i-1) d_xi + d_xi/2 (SMOD_mesh_manipulation.f90:50-51) mapped like the corners."""
    mx, my = control.m_xi, control.m_eta
    dxi = (control.xi_max - control.xi_min) / mx
    deta = (control.eta_max - control.eta_min) / my
    i = np.arange(-1, mx + 3, dtype=np.float64)
    j = np.arange(-1, my + 3, dtype=np.float64)
    xi = control.xi_min + (i - 1) * dxi + dxi / 2
    eta = control.eta_min + (j - 1) * deta + deta / 2
    X, Y = np.meshgrid(xi, eta)
    if mapping is None:
        return X, Y
    xs = np.empty_like(X)
    ys = np.empty_like(Y)
    for jj in range(X.shape[0]):
        for ii in range(X.shape[1]):
            xs[jj, ii], ys[jj, ii] = mapping(X[jj, ii], Y[jj, ii])
    return xs, ys


def stretch(ax: float, ay: float) -> Mapping:
    """Linear stretching x = ax*xi, y = ay*eta (the reference's cartesian_stretching example uses
    4 and 2, examples/2D_dam_break/cartesian_stretching/SMOD_coordinate_mapping.f90:35-43)."""
    return lambda xi, eta: (ax * xi, ay * eta)


def dam(control: ControlSettings, mapping: Optional[Mapping], radius: float = 0.5, h_in: float = 2.0,
        h_out: float = 1.0) -> np.ndarray:
    """Dam break on the physical cell centres (the stretching example's set_initial_conditions:
    h = h_in where sqrt(x^2 + y^2) < radius, else h_out; hu = hv = 0)."""
    x, y = cell_centres(control, mapping)
    q = np.zeros(x.shape + (3,), dtype=np.float64)
    q[..., 0] = np.where(np.sqrt(x ** 2 + y ** 2) < radius, h_in, h_out)
    return q
