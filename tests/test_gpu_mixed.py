"""The precision form (FP32 flux/limiter arithmetic, FP64 state, FP64 dt and sums) against the
FP64 path, which is itself bit-identical to the oracle.

Tolerance: the L1 error of h relative to the FP64 result, sum|h - h64| / sum|h64|, at most 1e-5
(the precision form's stated bound); momenta are compared on the same relative L1 scale of
sum|h64|.  Both runs take the same number of accepted steps; their dt sequences may differ in
the last bits because the wave speeds are rounded to FP32."""
import dataclasses

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu

L1_TOL = 1e-5


def _run(c, cu, q, precision, tile_rows=None):
    s = Solver(c, cu, precision=precision)
    if tile_rows:
        s.set_tile_rows(tile_rows)
    s.upload(q)
    s.update_rank_boundaries()
    st = s.advance()
    out = s.download()
    sums = s.conservation_sums()
    lg = s.step_log()
    s.close()
    return st, out, sums, lg


def _errors(a, b):
    ia, ib = a[2:-2, 2:-2], b[2:-2, 2:-2]
    scale = np.abs(ib[..., 0]).sum()
    l1 = [np.abs(ia[..., k] - ib[..., k]).sum() / scale for k in range(3)]
    linf = [np.abs(ia[..., k] - ib[..., k]).max() for k in range(3)]
    return l1, linf


CASES = [
    # name, grid (mx, my), limiter, bc, ic, steps
    ("dam200_mc_bc2", (200, 200), 4, 2, "dam", 300),
    ("bumps_257x131_minmod_wall", (257, 131), 1, 1, "bumps", 150),
    ("bumps_5x70_superbee_bc3", (5, 70), 2, 3, "bumps", 60),
    ("dam_300x124_vanleer_bc2", (300, 124), 3, 2, "dam", 120),
    ("bumps_500_minmod_bc2", (500, 500), 1, 2, "bumps", 200),
]


@pytest.mark.parametrize("name,grid,lim,bc,kind,steps", CASES)
def test_mixed_within_l1_of_fp64(pcl, name, grid, lim, bc, kind, steps):
    mx, my = grid
    c = dataclasses.replace(ctl.dam_break_control(mx, limiter=lim, bc=bc, time_final=100.0), m_eta=my)
    cu = ctl.CustomSettings(max_accepted_steps=steps)
    q = ic.circular_dam(mx, my) if kind == "dam" else ic.gaussian_bumps(mx, my, seed=4)
    st64, q64, s64, l64 = _run(c, cu, q, ctl.PRECISION_FP64)
    stm, qm, sm, lm = _run(c, cu, q, ctl.PRECISION_MIXED)
    assert st64.accepted == stm.accepted == steps
    assert np.array_equal(l64.ierr, lm.ierr)
    assert np.allclose(lm.dt, l64.dt, rtol=1e-5, atol=0)
    l1, linf = _errors(qm, q64)
    assert l1[0] <= L1_TOL, (l1, linf)
    assert l1[1] <= L1_TOL and l1[2] <= L1_TOL, (l1, linf)
    assert abs(sm[0] - s64[0]) / abs(s64[0]) < 1e-6  # mass (FP64 sums) within 1e-6 of the FP64 run


@pytest.mark.parametrize("over", [dict(use_limtiter=False), dict(add_higher_order_flux_correction=False)])
def test_mixed_unlimited_and_first_order(pcl, over):
    c = dataclasses.replace(ctl.dam_break_control(150, limiter=1, time_final=100.0), **over)
    cu = ctl.CustomSettings(max_accepted_steps=100)
    q = ic.circular_dam(150, 150)
    _, q64, _, _ = _run(c, cu, q, ctl.PRECISION_FP64)
    _, qm, _, _ = _run(c, cu, q, ctl.PRECISION_MIXED)
    l1, _ = _errors(qm, q64)
    assert max(l1) <= L1_TOL, l1


def test_mixed_tiling_does_not_change_results(pcl):
    """Per-cell arithmetic is independent of the work-item shape: bit-identical results."""
    c = dataclasses.replace(ctl.dam_break_control(333, limiter=4, time_final=100.0), m_eta=210)
    cu = ctl.CustomSettings(max_accepted_steps=40)
    q = ic.gaussian_bumps(333, 210, seed=9)
    ref = None
    for rows in (4, 17, 64, 256):
        _, qm, _, lg = _run(c, cu, q, ctl.PRECISION_MIXED, tile_rows=rows)
        if ref is None:
            ref = (qm, lg.dt)
        else:
            assert np.array_equal(qm, ref[0]) and np.array_equal(lg.dt, ref[1])


def test_mixed_mass_drift_matches_fp64(pcl):
    """With reflective walls the reference scheme is not exactly conservative: the eta sweep
    reads the pre-step ghost rows beside the x-swept interior (ghosts are filled once per step,
    main.f90:246), so the wall interfaces carry a small mass flux.  The mixed form must drift by
    the same amount as the FP64 path."""
    c = ctl.dam_break_control(256, limiter=4, bc=1, time_final=100.0)
    cu = ctl.CustomSettings(max_accepted_steps=300)
    q = ic.circular_dam(256, 256)
    m0 = q[2:-2, 2:-2, 0].sum()
    _, _, s64, _ = _run(c, cu, q, ctl.PRECISION_FP64)
    _, _, sm, _ = _run(c, cu, q, ctl.PRECISION_MIXED)
    drift64 = (s64[0] - m0) / m0
    driftm = (sm[0] - m0) / m0
    assert abs(drift64) < 1e-3
    assert abs(driftm - drift64) < 1e-7, (drift64, driftm)


def test_mixed_reports_bad_state(pcl):
    from paraclaws_b200._lib import PclError, PCL_ERR_NAN
    c = ctl.dam_break_control(64)
    s = Solver(c, precision=ctl.PRECISION_MIXED)
    q = ic.circular_dam(64, 64)
    q[30, 40, 1] = np.nan
    s.upload(q)
    s.update_rank_boundaries()
    with pytest.raises(PclError) as e:
        s.advance()
    assert e.value.code == PCL_ERR_NAN


@pytest.mark.parametrize("mx,my,lim,bc,tile", [
    (125, 129, 1, 1, 64),     # last strip and last row segment one cell wide: the finisher's sides
    (260, 97, 4, 3, 32),
    (64, 40, 2, 2, 16),
])
def test_single_launch_device_loop_equals_host_driven_steps(pcl, mx, my, lim, bc, tile):
    """The device loop runs each mixed attempt as one launch (edge CTAs fill their ghost cells,
    the last CTA runs the time control and the remaining ghost sides); the host-driven loop runs
    the sweeps, the time control and the ghost fill as separate kernels.  Same bits, same dt
    sequence."""
    from paraclaws_b200.solver import run_host_loop
    c = dataclasses.replace(ctl.dam_break_control(mx, limiter=lim, bc=bc, time_final=100.0), m_eta=my)
    cu = ctl.CustomSettings(max_accepted_steps=40)
    q = ic.gaussian_bumps(mx, my, seed=6)
    out = []
    for device_loop in (True, False):
        s = Solver(c, cu, precision=ctl.PRECISION_MIXED)
        s.set_tile_rows(tile)
        s.upload(q)
        s.update_rank_boundaries()
        if device_loop:
            s.advance()
            lg = s.step_log()
        else:
            lg = run_host_loop(s)
        out.append((s.download(), lg.dt, lg.ierr))
        s.close()
    assert len(out[0][1]) == len(out[1][1]) > 30
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][2], out[1][2])
    assert np.array_equal(out[0][0].view(np.int64), out[1][0].view(np.int64))
