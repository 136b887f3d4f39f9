"""Snapshots from the device loop: pcl_advance_to_snapshot stops where main.f90:256-268 writes
data, and pcl_write_snapshot produces writeData's files (utility/MOD_IO.f90:397-460) with the
states of the oracle at the same attempts."""
import os

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver, format_e26_16, run_device_loop_with_snapshots

pytestmark = pytest.mark.gpu


def _text(q, per_cell):
    """Expected file body: one record per padded cell, j outer, i inner."""
    nj, ni = q.shape[:2]
    lines = []
    for j in range(nj):
        for i in range(ni):
            vals = q[j, i] if per_cell is None else [0.0] * per_cell
            lines.append("".join(format_e26_16(v) for v in vals))
    return "\n".join(lines) + "\n"


def test_snapshots_match_oracle(pcl, oracle_lib, tmp_path):
    from oracle.oracle import Oracle
    c = ctl.dam_break_control(24, limiter=4, bc=2, time_final=0.06)
    c.number_of_snapshots = 3
    q0 = ic.circular_dam(24, 24)
    s = Solver(c)
    s.upload(q0)
    s.update_rank_boundaries()
    times = run_device_loop_with_snapshots(s, str(tmp_path))
    lg = s.step_log()
    s.close()
    assert times[0] == 0.0 and times[-1] == 0.06 and len(times) == 4
    dirs = sorted(os.listdir(tmp_path), key=float)
    assert dirs == ["%.10f" % t for t in times]
    # attempts after which each snapshot was taken: where the logged snapshot index grows
    snap_idx = np.concatenate([[1], lg.snap])
    marks = [0] + [k + 1 for k in range(len(lg.snap)) if snap_idx[k + 1] > snap_idx[k]]
    assert len(marks) == len(times)
    o = Oracle(c)
    o.set_state(q0)
    o.update_rank_boundaries()
    done = 0
    for t, k in zip(times, marks):
        if k > done:
            o.run(max_attempts=k - done)
            done = k
        sub = tmp_path / ("%.10f" % t) / "rank_0"
        assert (sub / "qout.dat").read_text() == _text(o.state(), None), t
        assert (sub / "aout.dat").read_text() == _text(o.state(), c.number_of_auxiliary_vars), t
    assert abs(o.time_state()["time"] - 0.06) == 0.0
    o.close()


def test_snapshot_of_unwritable_directory_fails_cleanly(pcl, tmp_path):
    c = ctl.dam_break_control(16)
    s = Solver(c)
    s.initial_condition()
    blocker = tmp_path / "file"
    blocker.write_text("x")
    from paraclaws_b200 import _lib
    with pytest.raises(_lib.PclError):
        s.write_snapshot(str(blocker / "out"), wait=True)
    s.close()
