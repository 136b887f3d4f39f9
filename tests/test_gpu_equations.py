"""Equation modules on the FP64 path: the generic sweeps run the reference's step for a module's
Jacobian (flux J(q).q in dgemv order, HLL on the largest |eigenvalue|).  The dam-break module
through the generic path equals the specialised kernels bit for bit, and linear acoustics equals
the oracle running the same module bit for bit."""
import dataclasses

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic, mesh
from paraclaws_b200.solver import Solver, run_host_loop

pytestmark = pytest.mark.gpu


def pulse(mx, my, w=0.15):
    x, y = np.meshgrid(*ic.cell_centres(mx, my))
    q = np.zeros((my + 4, mx + 4, 3))
    q[..., 0] = np.exp(-((x - 0.1) ** 2 + (y + 0.05) ** 2) / (w * w))
    return q


@pytest.mark.parametrize("device_loop", [False, True])
def test_generic_shallow_water_equals_specialised(pcl, device_loop):
    c = dataclasses.replace(ctl.dam_break_control(70, limiter=4, bc=2, time_final=0.08), m_eta=54)
    q = ic.gaussian_bumps(70, 54, seed=2)
    out = []
    for module in (ctl.EQ_SHALLOW_WATER, ctl.EQ_SHALLOW_WATER_GENERIC):
        s = Solver(c)
        s.set_equation(module)
        s.upload(q)
        s.update_rank_boundaries()
        if device_loop:
            s.advance()
            dt = s.step_log().dt
        else:
            dt = run_host_loop(s).dt
        out.append((s.download(), dt))
        s.close()
    assert len(out[0][1]) > 10 and np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("lim,bc", [(1, 2), (4, 1), (2, 3), (3, 2)])
def test_acoustics_matches_oracle(pcl, oracle_lib, lim, bc):
    from oracle.oracle import Oracle
    c = dataclasses.replace(ctl.dam_break_control(48, limiter=lim, bc=bc, time_final=0.3), m_eta=40)
    q = pulse(48, 40)
    s = Solver(c)
    s.set_equation(ctl.EQ_ACOUSTICS, (2.0, 0.5))
    s.upload(q)
    s.update_rank_boundaries()
    st = s.advance()
    o = Oracle(c)
    o.set_equation(ctl.EQ_ACOUSTICS, 2.0, 0.5)
    o.set_state(q)
    o.update_rank_boundaries()
    lo = o.run()
    assert st.status == 0 and lo.status == 0 and st.accepted > 10
    assert np.array_equal(s.step_log().dt, lo.dt)
    a, b = s.download(), o.state()
    s.close()
    o.close()
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ"
    assert np.abs(a[2:-2, 2:-2, 1]).max() > 1e-3  # the pulse radiated


def test_equation_module_rejections(pcl):
    c = ctl.dam_break_control(16)
    s = Solver(c, precision=ctl.PRECISION_MIXED)
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0, 1.0))
    s.close()
    s = Solver(c)
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0,))        # needs K and rho
    with pytest.raises(_lib.PclError):
        s.set_equation(7)
    s.set_mesh_metrics(*mesh.metrics(c, mesh.stretch(2.0, 2.0)))
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0, 1.0))    # mapped grids take the shallow-water module
    s.close()
