"""The FP64 eta sweep's two shapes (include/paraclaws_b200.h: pcl_set_sweep_shape) against the
oracle: column windows and 16-column bands each reproduce the oracle's state, dt sequence, CFL
and accept/reject flags bit for bit, on grids whose sizes are not multiples of the band width,
chunk height or window width, for every limiter, the unlimited correction, first order, the three
boundary codes and a domain whose capacities are not exactly 1.  The automatic choice follows
the equation module and g (windows only where the shared-reciprocal quotient is out of range)
and changes nothing either."""
import dataclasses

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu

CASES = [
    # name, (mx, my), control overrides, time_final
    ("minmod_wall", (37, 23), dict(limiter_function=1, bc=1), 0.08),
    ("mc_zero_gradient_tall", (5, 70), dict(limiter_function=4, bc=2), 0.06),
    ("superbee_const_gradient", (129, 257), dict(limiter_function=2, bc=3), 0.03),
    ("vanleer_wall_wide", (300, 64), dict(limiter_function=3, bc=1), 0.03),
    ("unlimited", (64, 61), dict(use_limtiter=False, bc=2), 0.05),
    ("first_order_wall", (50, 33), dict(add_higher_order_flux_correction=False, bc=1), 0.05),
    ("nonunit_capacity", (45, 290), dict(limiter_function=1, bc=1, xi_min=0.1, xi_max=0.83, eta_min=-0.37,
                                         eta_max=1.9), 0.02),
]


def _control(grid, over, tf):
    mx, my = grid
    over = dict(over)
    bc = over.pop("bc")
    c = ctl.dam_break_control(mx, limiter=over.pop("limiter_function", 1), bc=bc, time_final=tf)
    return dataclasses.replace(c, m_eta=my, **over)


def _run(c, q, shape):
    s = Solver(c)
    s.set_sweep_shape(shape)
    s.upload(q)
    s.update_rank_boundaries()
    st = s.advance()
    out = s.download(), s.step_log(), st
    s.close()
    return out


@pytest.mark.parametrize("shape", [_lib.PCL_SHAPE_WINDOW, _lib.PCL_SHAPE_BAND, _lib.PCL_SHAPE_AUTO])
@pytest.mark.parametrize("name,grid,over,tf", CASES)
def test_shape_matches_oracle(pcl, oracle_lib, shape, name, grid, over, tf):
    from oracle.oracle import Oracle
    c = _control(grid, over, tf)
    q = ic.circular_dam(c.m_xi, c.m_eta)
    q[..., 1] = 0.2 * np.sin(np.arange(q.shape[1]))[None, :]  # momenta in both directions
    q[..., 2] = -0.3 * np.cos(np.arange(q.shape[0]))[:, None]
    a, lg, st = _run(c, q, shape)
    o = Oracle(c)
    o.set_state(q)
    o.update_rank_boundaries()
    lo = o.run()
    b = o.state()
    o.close()
    assert lo.status == 0 and st.status == 0 and st.accepted >= 5
    assert np.array_equal(lg.dt, lo.dt) and np.array_equal(lg.ierr, lo.ierr) and np.array_equal(lg.cfl, lo.cfl)
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ, max {np.abs(a - b).max():.3e}"


def test_shapes_agree_on_a_large_grid(pcl):
    """1536 x 2100: 97 bands of 35 chunks of 60 rows each on a 148-SM part (the chunk seams and
    the history rows carried across them are exercised): both forced shapes give the same bits
    over 12 accepted steps."""
    c = dataclasses.replace(ctl.dam_break_control(1536, limiter=1, bc=1, time_final=1e9), m_eta=2100)
    q = ic.gaussian_bumps(1536, 2100, seed=3)
    cu = ctl.CustomSettings(max_accepted_steps=12)
    outs = []
    for shape in (_lib.PCL_SHAPE_WINDOW, _lib.PCL_SHAPE_BAND):
        s = Solver(c, cu)
        s.set_sweep_shape(shape)
        s.upload(q)
        s.update_rank_boundaries()
        st = s.advance()
        assert st.status == 0 and st.accepted == 12
        outs.append((s.download(), s.step_log().dt))
        s.close()
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][0].view(np.int64), outs[1][0].view(np.int64))


def test_shape_argument_checked(pcl):
    s = Solver(ctl.dam_break_control(16, time_final=0.01))
    with pytest.raises(_lib.PclError):
        s.set_sweep_shape(3)
    s.set_sweep_shape(_lib.PCL_SHAPE_AUTO)
    s.close()
