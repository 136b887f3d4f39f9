"""Mapped grids, host side: the C ABI's mesh metrics (pcl_compute_mesh_metrics) against the
oracle's mesh for the identity mapping, the exact values of the reference's stretching example,
and a line-by-line restatement of finalize_mesh for a skewed curvilinear mapping."""
import dataclasses
import math

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import mesh


def _restated(control, mapping):
    """domain/SMOD_mesh_manipulation.f90:14-56 and :129-176, written out independently."""
    mx, my = control.m_xi, control.m_eta
    dxi = (control.xi_max - control.xi_min) / mx
    deta = (control.eta_max - control.eta_min) / my
    kap = np.empty((my + 4, mx + 4))
    lrx = np.empty_like(kap)
    lry = np.empty_like(kap)

    def norm2(a, b):
        if b == 0.0:
            return abs(a)
        if a == 0.0:
            return abs(b)
        return math.sqrt(a * a + b * b)

    for j in range(-1, my + 3):
        for i in range(-1, mx + 3):
            x1 = control.xi_min + (i - 1) * dxi
            y1 = control.eta_min + (j - 1) * deta
            xi = [None, x1, x1 + dxi, x1 + dxi, x1, x1]
            eta = [None, y1, y1, y1 + deta, y1 + deta, y1]
            pts = [None] + [mapping(xi[m], eta[m]) for m in range(1, 6)]
            x = [None] + [p[0] for p in pts[1:]]
            y = [None] + [p[1] for p in pts[1:]]
            lrx[j + 1, i + 1] = norm2(x[4] - x[1], y[4] - y[1]) / deta
            lry[j + 1, i + 1] = norm2(x[2] - x[1], y[2] - y[1]) / dxi
            area = 0.0
            for m in range(1, 5):
                area = area + (0.5 * (y[m] + y[m + 1])) * (x[m] - x[m + 1])
            kap[j + 1, i + 1] = area / (dxi * deta)
    return kap, lrx, lry


def skewed(xi, eta):
    return xi + 0.1 * math.sin(math.pi * eta), eta + 0.08 * xi * xi


def test_identity_matches_oracle_mesh(oracle_lib):
    from oracle.oracle import Oracle
    c = dataclasses.replace(ctl.dam_break_control(37), m_eta=23)
    kap, lrx, lry = mesh.metrics(c)
    o = Oracle(c)
    m = o.mesh()
    o.close()
    assert np.array_equal(kap, m["kappa"]) and np.array_equal(lrx, m["lr_xi"]) and np.array_equal(lry, m["lr_eta"])


def test_stretching_example_is_exact():
    c = ctl.dam_break_control(64)
    kap, lrx, lry = mesh.metrics(c, mesh.stretch(4.0, 2.0))
    assert np.all(kap == 8.0) and np.all(lrx == 2.0) and np.all(lry == 4.0)


@pytest.mark.parametrize("mapping", [skewed, mesh.stretch(3.0, 0.5)])
def test_metrics_match_restated_finalize_mesh(mapping):
    c = dataclasses.replace(ctl.dam_break_control(12), m_eta=9)
    got = mesh.metrics(c, mapping)
    want = _restated(c, mapping)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)
    assert np.all(got[0] > 0)


def test_skewed_metrics_vary_per_cell():
    c = ctl.dam_break_control(16)
    kap, lrx, lry = mesh.metrics(c, skewed)
    assert np.unique(kap).size > 100 and np.unique(lrx).size > 10 and np.unique(lry).size > 10
