"""Equation modules on the oracle (CPU): the acoustics module's closed-form eigenvalues agree
with LAPACK dgeev on its Jacobian (the reference's calculateEigenSolution), and the shallow-water
module through the shared module header reproduces the oracle's own restatement."""
import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic


def pulse(m, w=0.15):
    x, y = np.meshgrid(*ic.cell_centres(m, m))
    q = np.zeros((m + 4, m + 4, 3))
    q[..., 0] = np.exp(-(x ** 2 + y ** 2) / (w * w))
    return q


def _run(c, q, module, prm, mode):
    from oracle.oracle import Oracle
    o = Oracle(c, eigen_mode=mode)
    o.set_equation(module, *prm)
    o.set_state(q)
    o.update_rank_boundaries()
    log = o.run()
    out = o.state()
    o.close()
    return log, out


def test_acoustics_closed_form_matches_dgeev(oracle_lib):
    from oracle import oracle
    if not oracle.load_lapack():
        pytest.skip("no LAPACK for dgeev mode")
    c = ctl.dam_break_control(24, limiter=4, bc=2, time_final=0.05)
    q = pulse(24)
    l0, s0 = _run(c, q, ctl.EQ_ACOUSTICS, (2.0, 0.5), 0)
    l1, s1 = _run(c, q, ctl.EQ_ACOUSTICS, (2.0, 0.5), 1)
    assert l0.status == 0 and l1.status == 0
    assert len(l0.dt) == len(l1.dt) and np.allclose(l0.dt, l1.dt, rtol=1e-13, atol=0)
    assert np.allclose(s0, s1, rtol=0, atol=1e-12)
    assert np.abs(s0[2:-2, 2:-2, 1]).max() > 1e-3  # the pulse moved


def test_shallow_water_module_equals_oracle_restatement(oracle_lib):
    c = ctl.dam_break_control(20, limiter=1, bc=3, time_final=0.05)
    q = ic.circular_dam(20, 20)
    l0, s0 = _run(c, q, ctl.EQ_SHALLOW_WATER, (), 0)
    l1, s1 = _run(c, q, ctl.EQ_SHALLOW_WATER_GENERIC, (ctl.GRAV_REFERENCE,), 0)
    assert np.array_equal(l0.dt, l1.dt) and np.array_equal(s0, s1)
