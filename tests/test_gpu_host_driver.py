"""The C++ host program (main.f90 above the C ABI) reading control.in/custom.in, in both the
host-driven and the device-resident loop, against the oracle."""
import subprocess

import numpy as np
import pytest

from paraclaws_b200 import build as B
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("device_loop", [False, True])
def test_host_program_matches_oracle(pcl, oracle_lib, tmp_path, device_loop):
    from oracle.oracle import Oracle
    c = ctl.dam_break_control(60, limiter=4, bc=2, time_final=0.05)
    cu = ctl.CustomSettings(dam_radius=0.4, dam_h_in=2.5)
    ctl.write_control(tmp_path / "control.in", c)
    ctl.write_custom(tmp_path / "custom.in", cu)
    exe = B.HOST_BIN if B.HOST_BIN.exists() else B.build_host_driver()
    args = [str(exe)] + (["--device-loop"] if device_loop else [])
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "PROGRAM FINISHED SUCCESSFULLY" in r.stdout
    q = np.fromfile(tmp_path / "output" / "final_state.bin", dtype=np.float64).reshape(64, 64, 3)
    steps = np.genfromtxt(tmp_path / "output" / "steps.csv", delimiter=",", names=True)
    o = Oracle(c, cu)
    q0 = ic.circular_dam(60, 60, radius=0.4, h_in=2.5)
    o.set_state(q0)
    o.update_rank_boundaries()
    log = o.run()
    assert np.array_equal(np.atleast_1d(steps["dt"]), log.dt)
    assert np.array_equal(np.atleast_1d(steps["ierr"]).astype(int), log.ierr)
    assert np.array_equal(q, o.state())


def test_host_program_snapshots_same_in_both_loops(pcl, tmp_path):
    """--snapshots writes writeData's files at t0 and every snapshot time; the host-driven loop
    and the device loop (paused at snapshot times) write identical files."""
    c = ctl.dam_break_control(28, limiter=1, bc=3, time_final=0.04)
    c.number_of_snapshots = 4
    exe = B.HOST_BIN if B.HOST_BIN.exists() else B.build_host_driver()
    trees = []
    for mode in ([], ["--device-loop"]):
        d = tmp_path / ("dev" if mode else "host")
        d.mkdir()
        ctl.write_control(d / "control.in", c)
        ctl.write_custom(d / "custom.in", ctl.CustomSettings())
        r = subprocess.run([str(exe), "--snapshots"] + mode, cwd=d, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        snaps = sorted((p for p in (d / "output").iterdir() if p.is_dir()), key=lambda p: float(p.name))
        trees.append({p.name: ((p / "rank_0" / "qout.dat").read_text(), (p / "rank_0" / "aout.dat").read_text())
                      for p in snaps})
    assert list(trees[0]) == ["%.10f" % t for t in (0.0, 0.01, 0.02, 0.03, 0.04)]
    assert trees[0] == trees[1]
    body = trees[0]["0.0400000000"][0].splitlines()
    assert len(body) == 32 * 32 and all(len(line) == 78 for line in body)
