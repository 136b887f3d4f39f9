"""Mapped (curvilinear) grids on the FP64 path: with the per-cell capacity and face length ratios
of a coordinate mapping (pcl_set_mesh_metrics), the CUDA sweeps reproduce the oracle bit for bit:
state, dt sequence and accept/reject flags."""
import dataclasses
import math

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import mesh
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu


def skewed(xi, eta):
    return xi + 0.1 * math.sin(math.pi * eta), eta + 0.08 * xi * xi


CASES = [
    # name, mapping, (mx, my), limiter, bc, time_final
    ("stretch_4x2_mc_bc2", mesh.stretch(4.0, 2.0), (64, 48), 4, 2, 0.08),
    ("skewed_minmod_bc3", skewed, (40, 56), 1, 3, 0.05),
    ("skewed_superbee_wall", skewed, (33, 29), 2, 1, 0.05),
    ("stretch_3x05_vanleer_bc2", mesh.stretch(3.0, 0.5), (50, 50), 3, 2, 0.04),
]


@pytest.mark.parametrize("name,mapping,grid,lim,bc,tf", CASES)
def test_mapped_run_matches_oracle(pcl, oracle_lib, name, mapping, grid, lim, bc, tf):
    from oracle.oracle import Oracle
    mx, my = grid
    c = dataclasses.replace(ctl.dam_break_control(mx, limiter=lim, bc=bc, time_final=tf), m_eta=my)
    kap, lrx, lry = mesh.metrics(c, mapping)
    q = mesh.dam(c, mapping, radius=0.5 if mapping is skewed else 1.2)
    s = Solver(c)
    s.set_mesh_metrics(kap, lrx, lry)
    o = Oracle(c)
    o.set_mesh(kap, lrx, lry)
    s.upload(q)
    s.update_rank_boundaries()
    o.set_state(q)
    o.update_rank_boundaries()
    st = s.advance()
    lo = o.run()
    lg = s.step_log()
    assert lo.status == 0 and st.status == 0 and st.accepted > 5
    assert np.array_equal(lg.dt, lo.dt) and np.array_equal(lg.ierr, lo.ierr)
    a, b = s.download(), o.state()
    s.close()
    o.close()
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ, max {np.abs(a - b).max():.3e}"


def test_mapped_metrics_change_the_solution(pcl):
    """The metrics reach the kernels: a stretched grid gives a different state than the same
    computational grid without them."""
    c = ctl.dam_break_control(32, limiter=1, time_final=0.02)
    q = mesh.dam(c, None)
    out = []
    for mapping in (None, mesh.stretch(4.0, 2.0)):
        s = Solver(c)
        if mapping is not None:
            s.set_mesh_metrics(*mesh.metrics(c, mapping))
        s.upload(q)
        s.update_rank_boundaries()
        s.advance()
        out.append(s.download())
        s.close()
    assert not np.array_equal(out[0], out[1])


def test_mixed_context_rejects_mapped_metrics(pcl):
    c = ctl.dam_break_control(16)
    s = Solver(c, precision=ctl.PRECISION_MIXED)
    with pytest.raises(_lib.PclError):
        s.set_mesh_metrics(*mesh.metrics(c))
    s.close()
