"""Benchmark workloads at their full sizes.  The plain-large workload (4096^2, 16 seeded
Gaussian bumps, minmod, BC 2, CFL 0.9): the FP64 path against the oracle for its first attempted
steps, bit for bit, and size-independent properties over the benchmark's 500 steps.  The
512-grid batch: sampled instances against the same grids run alone.  Smaller grids are covered
against the oracle in test_gpu_parity_fp64.py; these tests check that nothing changes with size
(launch shapes, row striding, reductions over ~20k CTAs, the batch's builds and item heights)."""
import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu

M = 4096


def _control():
    # the benchmark's workload: dam-break settings with minmod and zero-gradient boundaries
    return ctl.dam_break_control(M, limiter=1, bc=2, time_final=1.0e9)


@pytest.fixture(scope="module")
def bumps():
    return ic.gaussian_bumps(M, M, seed=0)


def _solver(q, precision=ctl.PRECISION_FP64):
    s = Solver(_control(), ctl.CustomSettings(max_accepted_steps=0), precision=precision)
    s.upload(q)
    s.update_rank_boundaries()
    return s


def test_first_attempts_match_oracle(pcl, oracle_lib, bumps):
    """Two attempted steps of the 4096^2 workload (16.8 M cells each) equal the oracle's: state,
    dt sequence, CFL numbers and accept flags."""
    from oracle.oracle import Oracle
    s = _solver(bumps)
    st = s.advance(max_attempts=2)
    o = Oracle(_control(), ctl.CustomSettings(max_accepted_steps=0))
    o.set_state(bumps)
    o.update_rank_boundaries()
    log_o = o.run(max_attempts=2)
    assert st.status == 0 and log_o.status == 0
    lg = s.step_log()
    assert np.array_equal(lg.dt, log_o.dt)
    assert np.array_equal(lg.ierr, log_o.ierr)
    assert np.array_equal(lg.cfl, log_o.cfl)
    assert np.array_equal(s.download(), o.state())
    s.close()


def test_benchmark_run_is_deterministic(pcl, bumps):
    """500 attempted steps twice from the same state give the same bits and the same step log:
    the wave-speed reductions (atomic max over all CTAs) and the device time control do not
    depend on the order in which CTAs finish."""
    runs = []
    for _ in range(2):
        s = _solver(bumps)
        st = s.advance(max_attempts=500)
        assert st.status == 0
        runs.append((s.download(), s.step_log()))
        s.close()
    (qa, la), (qb, lb) = runs
    assert np.array_equal(la.dt, lb.dt) and np.array_equal(la.ierr, lb.ierr)
    assert np.array_equal(qa, qb)


def test_precision_form_within_tolerance_at_full_size(pcl, bumps):
    """The precision form on the same workload: after 100 steps its L1(h) error relative to the
    FP64 path is below the 1e-5 bound the precision form is held to, and both runs took the same
    number of accepted steps."""
    out = {}
    for prec in (ctl.PRECISION_FP64, ctl.PRECISION_MIXED):
        s = _solver(bumps, precision=prec)
        st = s.advance(max_attempts=100)
        assert st.status == 0
        out[prec] = (s.download()[2:-2, 2:-2, 0], st.accepted)
        s.close()
    (h64, a64), (hm, am) = out[ctl.PRECISION_FP64], out[ctl.PRECISION_MIXED]
    assert a64 == am
    l1 = np.abs(hm - h64).sum() / np.abs(h64).sum()
    assert l1 <= 1e-5, l1


def test_full_batch_instances_match_alone(pcl):
    """The batching form's benchmark batch (512 dam breaks, sides log-uniform 64 ... 1024, 95 M
    cells, one persistent launch per step) for 32 steps: sampled instances, the largest among
    them, end bit-identical to the same grid advanced alone for the same attempts."""
    from paraclaws_b200.batch import Batch
    sides = ic.log_uniform_sides(512, 64, 1024, 32, seed=2)
    b = Batch(512, precision=ctl.PRECISION_MIXED)
    settings = []
    for k, m in enumerate(sides):
        p = ic.seeded_dam_params(k, offset=0.25)
        cu = ctl.CustomSettings(precision_mode=ctl.PRECISION_MIXED, dam_radius=p.radius, dam_h_in=p.h_in,
                                dam_h_out=p.h_out, dam_x0=p.x0, dam_y0=p.y0)
        c = ctl.dam_break_control(m, limiter=1, time_final=1.0e9)
        settings.append((c, cu))
        b.add(c, None, cu)
    b.step(32)
    for k in sorted({0, 255, 511, int(np.argmax(sides))}):
        c, cu = settings[k]
        s = Solver(c, cu, precision=ctl.PRECISION_MIXED)
        s.initial_condition()
        s.update_rank_boundaries()
        st = s.advance(max_attempts=32)
        assert st.status == 0
        assert np.array_equal(b.step_log(k).dt, s.step_log().dt)
        assert np.array_equal(b.download(k), s.download())
        s.close()
    b.close()
