"""Batching form: one persistent launch per step advances many grids of uneven size, each with
its own dt.  Every instance must be bit-identical to the same grid advanced alone
(Solver.advance), for both precisions, whatever the schedule and whoever else is in the batch."""
import dataclasses

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.batch import Batch, Schedule, autotune
from paraclaws_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _instances(n, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        mx = int(rng.choice([20, 37, 64, 100, 131, 256, 300]))
        my = int(rng.choice([16, 33, 64, 97, 128, 260]))
        lim = int(rng.integers(1, 5))
        bc = int(rng.integers(1, 4))
        c = dataclasses.replace(ctl.dam_break_control(mx, limiter=lim, bc=bc, time_final=float(rng.uniform(0.01, 0.05))),
                                m_eta=my, initial_timestep=float(rng.choice([1e-10, 1e-4, 2e-3])))
        p = ic.seeded_dam_params(k, offset=0.25)
        q = ic.circular_dam(mx, my, p.radius, p.h_in, p.h_out, p.x0, p.y0)
        out.append((c, q))
    return out


def _alone(c, q, precision):
    s = Solver(c, precision=precision)
    s.upload(q)
    s.update_rank_boundaries()
    s.advance()
    r = s.download(), s.step_log()
    s.close()
    return r


@pytest.mark.parametrize("precision", [ctl.PRECISION_FP64, ctl.PRECISION_MIXED])
def test_batch_equals_alone(pcl, precision):
    inst = _instances(12, seed=precision)
    b = Batch(16, precision=precision)
    slots = [b.add(c, q) for c, q in inst]
    for _ in range(400):
        b.step(16)
        done, status = b.poll()
        assert np.all(status[slots] == 0)
        if np.all(done[slots] == 1):
            break
    for s, (c, q) in zip(slots, inst):
        qa, la = _alone(c, q, precision)
        lb = b.step_log(s)
        assert np.array_equal(lb.dt, la.dt)
        assert np.array_equal(lb.ierr, la.ierr)
        assert np.array_equal(b.download(s), qa)
    b.close()


@pytest.mark.parametrize("precision", [ctl.PRECISION_FP64, ctl.PRECISION_MIXED])
def test_schedule_does_not_change_results(pcl, precision):
    inst = _instances(5, seed=7)
    results = []
    scheds = ([Schedule(tile_rows=16), Schedule(tile_rows=128, blocks_per_sm=1), Schedule(tile_rows=0)]
              if precision == ctl.PRECISION_MIXED
              else [Schedule(x_rows=4, y_rows=16), Schedule(x_rows=16, y_rows=64, blocks_per_sm=1)])
    for sch in scheds:
        b = Batch(8, precision=precision)
        b.set_schedule(sch)
        slots = [b.add(c, q) for c, q in inst]
        b.step(40)
        results.append([b.download(s) for s in slots])
        b.close()
    for other in results[1:]:
        for a, c in zip(results[0], other):
            assert np.array_equal(a, c)


def test_descriptor_pool_and_global_descriptors_agree(pcl):
    """A mixed batch reads its item descriptors from the constant-memory pool (1024 entries);
    one with more slots than the pool holds reads them from global memory through another build
    of the kernel.  Both give the same bits, also while the first batch holds its pool range."""
    inst = _instances(6, seed=11)
    results = []
    pooled = Batch(8, precision=ctl.PRECISION_MIXED)
    unpooled = Batch(1100, precision=ctl.PRECISION_MIXED)
    for b in (pooled, unpooled):
        slots = [b.add(c, q) for c, q in inst]
        b.step(60)
        results.append([b.download(s) for s in slots])
    pooled.close()
    unpooled.close()
    for a, c in zip(results[0], results[1]):
        assert np.array_equal(a, c)


def test_add_and_remove_between_steps(pcl):
    """Membership changes between steps: a new instance starts from its own initial state and
    ends bit-identical to running alone, even though it joined mid-flight."""
    inst = _instances(4, seed=3)
    b = Batch(4, precision=ctl.PRECISION_MIXED)
    s0 = b.add(*inst[0])
    s1 = b.add(*inst[1])
    b.step(10)
    b.remove(s1)
    s2 = b.add(*inst[2])
    s3 = b.add(*inst[3])
    for _ in range(200):
        b.step(16)
        done, _ = b.poll()
        if all(done[s] == 1 for s in (s0, s2, s3)):
            break
    for s, k in ((s0, 0), (s2, 2), (s3, 3)):
        qa, _ = _alone(*inst[k], ctl.PRECISION_MIXED)
        assert np.array_equal(b.download(s), qa)
    b.close()


@pytest.mark.parametrize("first_mode", ["first_order", "unlimited", 1, 2, 3, 4])
def test_single_mode_builds_and_switch_to_mixed_modes(pcl, first_mode):
    """While every instance of a mixed batch has the same flux mode (first order, unlimited
    correction, or one limiter) the kernel built for that mode alone runs; adding an instance of
    another mode switches the batch to the build for any mix.  Every instance still ends
    bit-identical to running alone."""
    base = _instances(4, seed=5)
    same = []
    for c, q in base[:3]:
        if first_mode == "first_order":
            c = dataclasses.replace(c, add_higher_order_flux_correction=False)
        elif first_mode == "unlimited":
            c = dataclasses.replace(c, use_limtiter=False)
        else:
            c = dataclasses.replace(c, limiter_function=first_mode)
        same.append((c, q))
    c3, q3 = base[3]
    other = (dataclasses.replace(c3, limiter_function=1 if first_mode == 4 else 4), q3)
    b = Batch(4, precision=ctl.PRECISION_MIXED)
    slots = [b.add(c, q) for c, q in same]
    b.step(40)  # one captured chunk of the single-mode build plus single launches
    slots.append(b.add(*other))
    cases = same + [other]
    for _ in range(200):
        b.step(16)
        done, _ = b.poll()
        if all(done[s] == 1 for s in slots):
            break
    for s, (c, q) in zip(slots, cases):
        qa, la = _alone(c, q, ctl.PRECISION_MIXED)
        assert np.array_equal(b.step_log(s).dt, la.dt)
        assert np.array_equal(b.download(s), qa)
    b.close()


@pytest.mark.parametrize("precision,rows", [(ctl.PRECISION_MIXED, 16), (ctl.PRECISION_MIXED, 32),
                                            (ctl.PRECISION_MIXED, 0), (ctl.PRECISION_FP64, 16),
                                            (ctl.PRECISION_FP64, 32)])
def test_item_ghost_fill_matches_alone(pcl, precision, rows):
    """Edge items fill the ghost cells next to the cells they wrote; the finishing CTA fills a
    high side whose last strip (segment) is one column (row) wide.  Grids with m_xi one or two past
    a multiple of the strip width (124 columns mixed, 128 FP64) and m_eta one or two past a
    multiple of the item height (`rows`: mixed tile rows, FP64 eta strip rows), each side with its
    own boundary code, end bit-identical to running alone, ghost cells included."""
    shapes = [(125, 33), (249, 17), (129, 65), (257, 97), (248, 34), (126, 66)]
    codes = [(1, 3, 2, 3), (3, 1, 3, 2), (2, 2, 1, 1), (3, 3, 3, 3), (1, 2, 3, 1), (3, 2, 1, 3)]
    cases = []
    for k, ((mx, my), (b0, b1, b2, b3)) in enumerate(zip(shapes, codes)):
        c = dataclasses.replace(ctl.dam_break_control(mx, limiter=1 + k % 4, bc=1, time_final=0.03), m_eta=my,
                                bc_xi_lower=b0, bc_xi_upper=b1, bc_eta_lower=b2, bc_eta_upper=b3)
        p = ic.seeded_dam_params(k, offset=0.25)
        cases.append((c, ic.circular_dam(mx, my, p.radius, p.h_in, p.h_out, p.x0, p.y0)))
    b = Batch(8, precision=precision)
    b.set_schedule(Schedule(tile_rows=rows) if precision == ctl.PRECISION_MIXED else Schedule(x_rows=4, y_rows=rows))
    slots = [b.add(c, q) for c, q in cases]
    for _ in range(400):
        b.step(16)
        done, _ = b.poll()
        if all(done[s] == 1 for s in slots):
            break
    for s, (c, q) in zip(slots, cases):
        qa, la = _alone(c, q, precision)
        assert np.array_equal(b.step_log(s).dt, la.dt)
        assert np.array_equal(b.download(s), qa)
    b.close()


@pytest.mark.parametrize("precision", [ctl.PRECISION_MIXED, ctl.PRECISION_FP64])
def test_ghost_fill_by_finishing_cta_matches_alone(pcl, precision):
    """With many items per step (short items on one CTA per SM) the finishing CTA fills all ghost
    cells instead of the edge items; the grids still end bit-identical to running alone."""
    shapes = [(260, 260), (249, 257), (300, 201)]
    codes = [(1, 3, 2, 3), (3, 1, 3, 1), (2, 3, 1, 2)]
    cases = []
    for k, ((mx, my), (b0, b1, b2, b3)) in enumerate(zip(shapes, codes)):
        c = dataclasses.replace(ctl.dam_break_control(mx, limiter=1 + k, bc=1, time_final=0.01), m_eta=my,
                                bc_xi_lower=b0, bc_xi_upper=b1, bc_eta_lower=b2, bc_eta_upper=b3)
        p = ic.seeded_dam_params(k + 20, offset=0.25)
        cases.append((c, ic.circular_dam(mx, my, p.radius, p.h_in, p.h_out, p.x0, p.y0)))
    b = Batch(4, precision=precision)
    b.set_schedule(Schedule(tile_rows=4, blocks_per_sm=1) if precision == ctl.PRECISION_MIXED
                   else Schedule(x_rows=1, y_rows=4, blocks_per_sm=1))
    slots = [b.add(c, q) for c, q in cases]
    for _ in range(400):
        b.step(16)
        done, _ = b.poll()
        if all(done[s] == 1 for s in slots):
            break
    for s, (c, q) in zip(slots, cases):
        qa, la = _alone(c, q, precision)
        assert np.array_equal(b.step_log(s).dt, la.dt)
        assert np.array_equal(b.download(s), qa)
    b.close()


def test_full_batch_is_reported(pcl):
    from paraclaws_b200._lib import PclError, PCL_ERR_FULL
    c, q = _instances(1)[0]
    b = Batch(1)
    b.add(c, q)
    with pytest.raises(PclError) as e:
        b.add(c, q)
    assert e.value.code == PCL_ERR_FULL
    b.close()


def test_autotuner_picks_a_schedule(pcl, tmp_path):
    inst = _instances(6, seed=11)
    b = Batch(8, precision=ctl.PRECISION_MIXED)
    for c, q in inst:
        c.time_final = 100.0
        b.add(c, q)
    best, timings = autotune(b, steps_per_trial=4, cache=tmp_path / "t.json")
    assert best in [Schedule(**__import__("json").loads(k)) for k in timings]
    assert (tmp_path / "t.json").exists()
    best2, _ = autotune(b, cache=tmp_path / "t.json")
    assert best2 == best
    b.close()


@pytest.mark.parametrize("schedule", [Schedule(x_rows=8, y_rows=64), Schedule(x_rows=1, y_rows=4, blocks_per_sm=1)])
def test_large_and_small_grids_match_alone(pcl, schedule):
    """FP64 grids of more than 512^2 cells beside small ones in the same launches.  m_xi = 519
    leaves the last 4-column eta band one cell wide (its ghost side falls to the finishing CTA);
    517 does not.  Both schedules (few long items with edge-item ghost fill, many short ones with
    the finishing CTA's) end bit-identical to each grid run alone, ghost cells included."""
    shapes = [(519, 520), (517, 513), (100, 64), (260, 33)]
    codes = [(1, 3, 2, 3), (3, 1, 3, 2), (2, 2, 1, 1), (1, 1, 1, 1)]
    cases = []
    for k, ((mx, my), (b0, b1, b2, b3)) in enumerate(zip(shapes, codes)):
        c = dataclasses.replace(ctl.dam_break_control(mx, limiter=1 + k % 4, bc=1, time_final=0.01), m_eta=my,
                                bc_xi_lower=b0, bc_xi_upper=b1, bc_eta_lower=b2, bc_eta_upper=b3)
        p = ic.seeded_dam_params(k + 40, offset=0.25)
        cases.append((c, ic.circular_dam(mx, my, p.radius, p.h_in, p.h_out, p.x0, p.y0)))
    b = Batch(4, precision=ctl.PRECISION_FP64)
    b.set_schedule(schedule)
    slots = [b.add(c, q) for c, q in cases]
    for _ in range(400):
        b.step(16)
        done, status = b.poll()
        assert all(status[s] == 0 for s in slots)
        if all(done[s] == 1 for s in slots):
            break
    for s, (c, q) in zip(slots, cases):
        qa, la = _alone(c, q, ctl.PRECISION_FP64)
        assert np.array_equal(b.step_log(s).dt, la.dt)
        assert np.array_equal(b.download(s), qa)
    b.close()
