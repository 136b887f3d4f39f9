"""Serving form: a continuous-batching request loop for dam-break solves.

Requests (each a complete solve: grid, settings, end time) arrive over time.  The server keeps
one ``Batch`` on the GPU.  Between steps it admits waiting requests in arrival order while a
slot is free and the device-memory footprint stays within the budget, builds their initial
state on the device, and retires finished requests (download, free).  In between, every
admitted request advances in the same persistent launches, so requests of different sizes that
arrived at different times overlap on the device.  A request's result is bit-identical to
solving it alone (the batch never changes a cell's arithmetic).

Reported per run: time-to-solution (arrival to result on the host) p50/p99, queueing delay,
throughput in cell-updates/s, and device memory in use.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Deque, Dict, List, Optional

import numpy as np

from ._lib import PCL_ERR_FULL, PCL_ERR_TIMEOUT
from .batch import Batch, autotune
from .control import ControlSettings, CustomSettings, PRECISION_FP64, dam_break_control
from . import ic


@dataclass
class Request:
    rid: int
    control: ControlSettings
    custom: CustomSettings
    arrival: float              # seconds after the start of the run
    state: Optional[np.ndarray] = None   # None: the dam break of `custom`, built on the device


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    accepted: int
    cells: int
    status: int
    state: Optional[np.ndarray] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def queued(self) -> float:
        return self.admitted - self.arrival


def poisson_requests(n: int, rate: float, seed: int, side_lo: int = 128, side_hi: int = 2048,
                     t_end: tuple = (0.1, 1.0), limiter: int = 1, precision: int = PRECISION_FP64) -> List[Request]:
    """n dam-break requests with Poisson arrivals (rate per second), grid side log-uniform in
    [side_lo, side_hi] (multiple of 32), end time U(t_end), a seeded dam (radius, height ratio,
    centre offset) and reflective walls."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps) - gaps[0]
    sides = ic.log_uniform_sides(n, side_lo, side_hi, 32, seed + 1)
    out = []
    for k in range(n):
        te = float(rng.uniform(*t_end))
        p = ic.seeded_dam_params(seed * 100003 + k, offset=0.25)
        c = dam_break_control(sides[k], limiter=limiter, bc=1, time_final=te)
        cu = CustomSettings(precision_mode=precision, dam_radius=p.radius, dam_h_in=p.h_in, dam_h_out=p.h_out,
                            dam_x0=p.x0, dam_y0=p.y0)
        out.append(Request(k, c, cu, float(arrivals[k])))
    return out


@dataclass
class ServeReport:
    results: List[Result]
    wall: float
    cell_updates: float
    peak_bytes: int
    peak_active: int
    steps: int
    not_arrived: int = 0     # requests whose arrival time lay beyond the wall-clock limit

    def percentile(self, q: float) -> float:
        lat = sorted(r.latency for r in self.results)
        if not lat:
            return float("nan")
        k = min(len(lat) - 1, max(0, int(math.ceil(q / 100.0 * len(lat))) - 1))
        return lat[k]

    def summary(self) -> dict:
        return {
            "requests": len(self.results),
            "p50_s": self.percentile(50),
            "p99_s": self.percentile(99),
            "mean_queue_s": float(np.mean([r.queued for r in self.results])) if self.results else float("nan"),
            "throughput_cell_updates_per_s": self.cell_updates / self.wall if self.wall > 0 else 0.0,
            "wall_s": self.wall,
            "peak_device_bytes": self.peak_bytes,
            "peak_active": self.peak_active,
            "steps": self.steps,
            "errors": sum(1 for r in self.results if r.status != 0),
            "timed_out": sum(1 for r in self.results if r.status == PCL_ERR_TIMEOUT),
            "not_arrived": self.not_arrived,
        }


class SolveServer:
    """Continuous batching of solves on one GPU within a device-memory budget."""

    def __init__(self, precision: int = PRECISION_FP64, budget_bytes: float = 120e9, max_slots: int = 1024,
                 steps_per_tick: int = 16, device: int = 0, keep_states: bool = False, tune: bool = False):
        self.batch = Batch(max_slots, precision=precision, device=device)
        self.precision = precision
        self.budget = float(budget_bytes)
        self.steps_per_tick = int(steps_per_tick)
        self.keep_states = keep_states
        self.tune = tune
        self.in_use = 0
        self.active: Dict[int, tuple] = {}   # slot -> (request, admitted, bytes)

    def close(self) -> None:
        self.batch.close()

    def footprint(self, r: Request) -> int:
        return Batch.instance_bytes(r.control, r.custom, self.precision)

    def _admit(self, r: Request, now: float) -> bool:
        need = self.footprint(r)
        if self.in_use + need > self.budget or len(self.active) >= self.batch.max_instances:
            return False
        slot = self.batch.add(r.control, r.state, r.custom)
        self.active[slot] = (r, now, need)
        self.in_use += need
        return True

    def run(self, requests: List[Request], clock=time.perf_counter, max_wall: float = 600.0) -> ServeReport:
        """Serve `requests` in real time: request k becomes visible `arrival` seconds after start."""
        pending = sorted(requests, key=lambda r: r.arrival)
        arrived: Deque[Request] = deque()
        results: List[Result] = []
        t0 = clock()
        cell_updates = 0.0
        peak_bytes = peak_active = steps = 0
        tuned = not self.tune
        i = 0
        while (i < len(pending) or arrived or self.active) and clock() - t0 < max_wall:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                arrived.append(pending[i])
                i += 1
            # admit in arrival order while memory and slots allow (no overtaking).  A request larger
            # than the whole budget could never be admitted and would hold up every request behind
            # it: it is answered at once with PCL_ERR_FULL.
            while arrived:
                r = arrived[0]
                if self.footprint(r) > self.budget:
                    arrived.popleft()
                    t = clock() - t0
                    results.append(Result(r.rid, r.arrival, t, t, 0, r.control.m_xi * r.control.m_eta, PCL_ERR_FULL))
                    continue
                if not self._admit(r, clock() - t0):
                    break
                arrived.popleft()
            peak_bytes = max(peak_bytes, self.in_use)
            peak_active = max(peak_active, len(self.active))
            if not self.active:
                if i < len(pending):
                    time.sleep(max(0.0, min(pending[i].arrival - (clock() - t0), 0.05)))
                continue
            if not tuned and len(self.active) >= 4:
                autotune(self.batch, steps_per_trial=4)
                tuned = True
            self.batch.step(self.steps_per_tick)
            steps += self.steps_per_tick
            done, status = self.batch.poll()
            for slot in [s for s in list(self.active) if done[s] == 1]:
                r, adm, need = self.active.pop(slot)
                st = self.batch.stats(slot)
                state = self.batch.download(slot) if self.keep_states else None
                cells = r.control.m_xi * r.control.m_eta
                cell_updates += float(cells) * st.accepted
                results.append(Result(r.rid, r.arrival, adm, clock() - t0, st.accepted, cells, int(status[slot]), state))
                self.batch.remove(slot)
                self.in_use -= need
        wall = clock() - t0
        # max_wall ran out: every request still in flight or waiting is answered with a timeout, its
        # latency the time it had waited so far (a lower bound), so percentiles and the error count
        # include the requests that took longest.  Requests that had not arrived yet are left out.
        for slot in list(self.active):
            r, adm, need = self.active.pop(slot)
            st = self.batch.stats(slot)
            results.append(Result(r.rid, r.arrival, adm, wall, st.accepted, r.control.m_xi * r.control.m_eta,
                                  PCL_ERR_TIMEOUT))
            self.batch.remove(slot)
            self.in_use -= need
        while arrived:
            r = arrived.popleft()
            results.append(Result(r.rid, r.arrival, wall, wall, 0, r.control.m_xi * r.control.m_eta, PCL_ERR_TIMEOUT))
        return ServeReport(sorted(results, key=lambda r: r.rid), wall, cell_updates, peak_bytes, peak_active, steps,
                           not_arrived=len(pending) - i)
