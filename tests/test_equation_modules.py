"""Equation modules on the oracle (CPU): every module's closed-form eigenvalues agree with LAPACK
dgeev on its Jacobian (the reference's calculateEigenSolution), for one, three and four
equations; the shallow-water Jacobian through the module interface reproduces the oracle's own
restatement; a tracer carried at a constant concentration stays at it; and the module/size
pairing is enforced."""
import dataclasses

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


def _n_control(m, n, **kw):
    c = ctl.dam_break_control(m, **kw)
    return dataclasses.replace(c, number_of_equations=n)


def pulse_n(m, n, w=0.2, base=0.0):
    x, y = np.meshgrid(*ic.cell_centres(m, m))
    q = np.zeros((m + 4, m + 4, n))
    q[..., 0] = base + np.exp(-((x - 0.1) ** 2 + (y + 0.2) ** 2) / (w * w))
    return q


def tracer_state(m, alpha=0.3):
    """dam break with hu, hv = 0 and a tracer hc = alpha * h (concentration alpha everywhere)"""
    q3 = ic.circular_dam(m, m)
    q = np.zeros((m + 4, m + 4, 4))
    q[..., :3] = q3
    q[..., 3] = alpha * q3[..., 0]
    return q


@pytest.mark.parametrize("module,n,prm,base", [
    (ctl.EQ_ADVECTION, 1, (1.0, -0.5), 0.0),
    (ctl.EQ_BURGERS, 1, (), 0.5),
    (ctl.EQ_SHALLOW_WATER_TRACER, 4, (ctl.GRAV_REFERENCE,), None),
])
def test_closed_form_matches_dgeev_for_n_equations(oracle_lib, module, n, prm, base):
    from oracle import oracle
    if not oracle.load_lapack():
        pytest.skip("no LAPACK for dgeev mode")
    c = _n_control(24, n, limiter=4, bc=2, time_final=0.05)
    q = tracer_state(24) if base is None else pulse_n(24, n, base=base)
    l0, s0 = _run(c, q, module, prm, 0)
    l1, s1 = _run(c, q, module, prm, 1)
    assert l0.status == 0 and l1.status == 0 and len(l0.dt) > 3
    assert len(l0.dt) == len(l1.dt) and np.allclose(l0.dt, l1.dt, rtol=1e-13, atol=0)
    assert np.allclose(s0, s1, rtol=0, atol=1e-11)
    assert not np.array_equal(s0, q)


def test_tracer_concentration_stays_constant(oracle_lib):
    """With hc = alpha h everywhere, the tracer row's flux is alpha times the mass flux
    (J(q).q row 4 = hu hc / h), so every HLL wave and correction carries hc = alpha h along:
    the concentration hc / h stays alpha to rounding."""
    c = _n_control(40, 4, limiter=1, bc=1, time_final=0.1)
    q = tracer_state(40, alpha=0.3)
    log, s = _run(c, q, ctl.EQ_SHALLOW_WATER_TRACER, (ctl.GRAV_REFERENCE,), 0)
    assert log.status == 0 and log.accepted > 10
    conc = s[2:-2, 2:-2, 3] / s[2:-2, 2:-2, 0]
    assert np.abs(conc - 0.3).max() < 1e-12
    assert np.abs(s[2:-2, 2:-2, 1]).max() > 1e-2  # the dam broke


def test_advection_conserves_and_moves_the_pulse(oracle_lib):
    """One-equation advection with velocity (a, b): the pulse's centre of mass moves by
    (a, b) * t (to the scheme's accuracy), and the sum over the grid is conserved while the
    pulse stays inside (up to the HLL epsilon drift of order dt/dx * 1e-10 per step)."""
    m, a, b, t = 64, 1.0, -0.5, 0.2
    c = _n_control(m, 1, limiter=4, bc=2, time_final=t)
    q = pulse_n(m, 1, w=0.1)
    log, s = _run(c, q, ctl.EQ_ADVECTION, (a, b), 0)
    assert log.status == 0
    x, y = (a_[2:-2, 2:-2] for a_ in np.meshgrid(*ic.cell_centres(m, m)))
    w0, w1 = q[2:-2, 2:-2, 0], s[2:-2, 2:-2, 0]
    assert abs(w1.sum() - w0.sum()) / w0.sum() < 1e-8
    cx0, cy0 = (x * w0).sum() / w0.sum(), (y * w0).sum() / w0.sum()
    cx1, cy1 = (x * w1).sum() / w1.sum(), (y * w1).sum() / w1.sum()
    assert abs((cx1 - cx0) - a * t) < 0.02 and abs((cy1 - cy0) - b * t) < 0.02


def test_module_size_pairing(oracle_lib):
    from oracle.oracle import Oracle
    o = Oracle(_n_control(8, 1, time_final=0.01))
    with pytest.raises(ValueError):
        o.set_equation(ctl.EQ_ACOUSTICS, 1.0, 1.0)   # three equations, not one
    assert o.run().status != 0                      # no module chosen yet: refused
    o.set_equation(ctl.EQ_ADVECTION, 1.0, 0.0)
    o.close()
    o = Oracle(ctl.dam_break_control(8, time_final=0.01))
    with pytest.raises(ValueError):
        o.set_equation(ctl.EQ_SHALLOW_WATER_TRACER, 9.81)
    o.close()
