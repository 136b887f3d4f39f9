"""Bounded device waits that run out: the status reaches the host as PCL_ERR_TIMEOUT, the attempt
is void (the current solution and the time control stay as they were), and the context or batch
is usable again afterwards, with results bit-identical to runs that never timed out.

The waits are made to run out from the host (include/paraclaws_b200.h: pcl_batch_inject_stall,
pcl_inject_copy_stall) with short bounds: an FP64 batch's eta items wait for one xi item more
than the step has; the mixed kernel's row ring waits for a bulk copy that is never issued.  Both
are waits for a flag that nothing sets, ended by their bound: nothing faults or hangs.
"""
import ctypes as C
import time

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.batch import Batch
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.int64), np.asarray(b).view(np.int64))


def _instance(m, seed, steps):
    p = ic.seeded_dam_params(seed, offset=0.25)
    c = ctl.dam_break_control(m, limiter=1, bc=1, time_final=1.0e9)
    cu = ctl.CustomSettings(dam_radius=p.radius, dam_h_in=p.h_in, dam_h_out=p.h_out, dam_x0=p.x0, dam_y0=p.y0,
                            max_accepted_steps=steps)
    return c, cu


def _alone(c, cu, precision=ctl.PRECISION_FP64):
    s = Solver(c, cu, precision=precision)
    s.initial_condition()
    s.update_rank_boundaries()
    s.advance()
    out = s.download()
    s.close()
    return out


def _run_batch_to_end(b, limit=400):
    for _ in range(limit):
        b.step(4)
        done, _ = b.poll()
        if (done[done >= 0] == 1).all():
            return
    raise AssertionError("batch did not finish")


def test_fp64_batch_wait_runs_out_and_recovers(pcl):
    L = _lib.load()
    steps = 12
    specs = [(96, 1), (160, 2), (64, 3)]
    b = Batch(4, precision=ctl.PRECISION_FP64)
    cfg = [_instance(m, seed, steps) for m, seed in specs]
    slots = [b.add(c, None, cu) for c, cu in cfg]
    b.step(3)
    before = b.download(slots[1])
    st0 = b.stats(slots[1])
    assert st0.accepted >= 1 and st0.status == 0

    assert L.pcl_batch_inject_stall(b.h, slots[1], 1 << 12) == 0
    t0 = time.perf_counter()
    with pytest.raises(_lib.PclError) as e:
        b.step(1)
    assert e.value.code == _lib.PCL_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    done, status = b.poll()
    assert status[slots[1]] == _lib.PCL_ERR_TIMEOUT and done[slots[1]] == 1
    assert status[slots[0]] == 0 and status[slots[2]] == 0
    # the void attempt left the instance's solution and time control as they were
    assert _same_bits(b.download(slots[1]), before)
    st1 = b.stats(slots[1])
    assert st1.accepted == st0.accepted and st1.time == st0.time and st1.dt == st0.dt

    # recovery: switch the stall off, replace the instance, run everything to its step cap; every
    # instance equals the same grid solved alone, bit for bit
    assert L.pcl_batch_inject_stall(b.h, -1, 0) == 0
    b.remove(slots[1])
    slots[1] = b.add(cfg[1][0], None, cfg[1][1])
    _run_batch_to_end(b)
    for slot, (c, cu) in zip(slots, cfg):
        st = b.stats(slot)
        assert st.status == 0 and st.accepted == steps
        assert _same_bits(b.download(slot), _alone(c, cu)), f"slot {slot}"
    b.close()


def test_mixed_copy_wait_runs_out_and_recovers(pcl):
    L = _lib.load()
    m, steps = 200, 30
    c, cu = _instance(m, 4, steps)
    s = Solver(c, cu, precision=ctl.PRECISION_MIXED)
    s.initial_condition()
    s.update_rank_boundaries()
    q0 = s.download()
    s.advance(max_attempts=5)
    before = s.download()
    st0 = s.stats()

    assert L.pcl_inject_copy_stall(s.h, 37, 1 << 10) == 0
    t0 = time.perf_counter()
    with pytest.raises(_lib.PclError) as e:  # one host-driven attempt
        s.solve_dimensional_split()
    assert e.value.code == _lib.PCL_ERR_TIMEOUT
    with pytest.raises(_lib.PclError) as e:  # the device loop stops at once on the status
        s.advance(max_attempts=4)
    assert e.value.code == _lib.PCL_ERR_TIMEOUT
    assert time.perf_counter() - t0 < 10.0
    st1 = s.stats()
    assert st1.status == _lib.PCL_ERR_TIMEOUT
    assert st1.accepted == st0.accepted and st1.time == st0.time
    assert _same_bits(s.download(), before)

    # recovery on the same context: the normal build again, a restart from the initial state
    assert L.pcl_inject_copy_stall(s.h, -1, 0) == 0
    s.upload(q0)
    s.update_rank_boundaries()
    s.reset_time_control()
    st = s.advance()
    assert st.status == 0 and st.accepted == steps
    assert _same_bits(s.download(), _alone(c, cu, ctl.PRECISION_MIXED))
    s.close()


def test_injection_switches_check_their_arguments(pcl):
    L = _lib.load()
    b = Batch(2, precision=ctl.PRECISION_MIXED)
    assert L.pcl_batch_inject_stall(b.h, 0, 100) == _lib.PCL_ERR_BADARG  # FP64 batches only
    b.close()
    s = Solver(ctl.dam_break_control(32, time_final=0.01))
    assert L.pcl_inject_copy_stall(s.h, 3, 100) == _lib.PCL_ERR_BADARG  # mixed contexts only
    s.close()
