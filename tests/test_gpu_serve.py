"""Serving form: requests arriving over time are admitted into the running batch as memory and
slots allow, overlap on the device, and each result equals the same solve run alone (bit for
bit, which is within any tolerance)."""
import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.serve import SolveServer, poisson_requests
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _alone(r, precision):
    s = Solver(r.control, r.custom, precision=precision)
    s.initial_condition()
    s.update_rank_boundaries()
    s.advance()
    q = s.download()
    st = s.stats()
    s.close()
    return q, st


@pytest.mark.parametrize("precision", [ctl.PRECISION_FP64, ctl.PRECISION_MIXED])
def test_served_results_equal_solo_runs(pcl, precision):
    reqs = poisson_requests(10, rate=200.0, seed=5, side_lo=64, side_hi=256, t_end=(0.02, 0.08),
                            precision=precision)
    srv = SolveServer(precision=precision, budget_bytes=2e9, max_slots=8, steps_per_tick=8, keep_states=True)
    rep = srv.run(reqs, max_wall=120.0)
    srv.close()
    assert len(rep.results) == len(reqs)
    assert rep.peak_active >= 2  # requests overlapped on the device
    for res in rep.results:
        assert res.status == 0
        q, st = _alone(reqs[res.rid], precision)
        assert res.accepted == st.accepted
        assert np.array_equal(res.state, q)
    s = rep.summary()
    assert s["p50_s"] <= s["p99_s"] and s["throughput_cell_updates_per_s"] > 0


def test_memory_budget_limits_admission(pcl):
    reqs = poisson_requests(6, rate=1000.0, seed=9, side_lo=256, side_hi=256, t_end=(0.02, 0.03))
    one = SolveServer().footprint(reqs[0])
    srv = SolveServer(budget_bytes=2.5 * one, max_slots=8, steps_per_tick=8)
    rep = srv.run(reqs, max_wall=120.0)
    srv.close()
    assert len(rep.results) == 6
    assert rep.peak_active <= 2 and rep.peak_bytes <= 2.5 * one
    assert max(r.queued for r in rep.results) > 0.0  # later arrivals waited for memory


def test_device_initial_condition_matches_host_generator(pcl):
    c = ctl.dam_break_control(96, limiter=1)
    c.m_eta = 80
    cu = ctl.CustomSettings(dam_radius=0.37, dam_h_in=3.1, dam_h_out=1.0, dam_x0=0.11, dam_y0=-0.2)
    s = Solver(c, cu)
    s.initial_condition()
    dev = s.download()
    s.close()
    host = ic.circular_dam(96, 80, 0.37, 3.1, 1.0, 0.11, -0.2)
    assert np.array_equal(dev, host)
