"""Host-side mirror of the reference driver for the wave-propagation step.

``Solver`` owns one device context (one grid) and exposes the reference's routine boundary
(update_rank_boundaries, solve_dimensional_split, the time_control methods), so a host loop
reads like main.f90:193-283 (``run_host_loop``), and the device-resident whole-loop path
(``advance``).  All numerics run in libparaclaws_b200.so; there is no Python compute path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _lib
from .control import ControlSettings, CustomSettings, GRAV_REFERENCE, PRECISION_FP64


def to_c_control(control: ControlSettings, custom: Optional[CustomSettings] = None,
                 precision: Optional[int] = None) -> _lib.SolverControl:
    L = _lib.load()
    c = _lib.SolverControl()
    L.pcl_default_control(C.byref(c))
    c.num_equations = control.number_of_equations
    c.num_dimensions = control.number_of_dimensions
    c.num_ghost = control.number_of_ghost_cells
    c.num_aux = control.number_of_auxiliary_vars
    c.num_waves = control.number_of_waves
    c.t_start = float(control.time_start)
    c.t_final = float(control.time_final)
    c.number_of_snapshots = control.number_of_snapshots
    c.dt_initial = float(control.initial_timestep)
    c.adaptive_timestepping = int(bool(control.adaptive_timestepping))
    c.cfl_limit = float(control.CFL_limit)
    c.dt_min = float(control.min_allowed_dt)
    c.dt_max = float(control.max_allowed_dt)
    c.dt_max_growth_ratio = float(control.dt_max_growth_ratio)
    c.dt_min_shrink_ratio = float(control.dt_min_shrink_ratio)
    c.higher_order_flux_correction = int(bool(control.add_higher_order_flux_correction))
    c.use_limiter = int(bool(control.use_limtiter))
    c.limiter_method = control.limiter_function
    c.m_xi, c.m_eta = control.m_xi, control.m_eta
    c.xi_min, c.xi_max = float(control.xi_min), float(control.xi_max)
    c.eta_min, c.eta_max = float(control.eta_min), float(control.eta_max)
    c.bc_xi_lower, c.bc_xi_upper = control.bc_xi_lower, control.bc_xi_upper
    c.bc_eta_lower, c.bc_eta_upper = control.bc_eta_lower, control.bc_eta_upper
    cu = custom if custom is not None else CustomSettings()
    c.max_accepted_steps = int(cu.max_accepted_steps)
    c.precision_mode = int(cu.precision_mode if precision is None else precision)
    c.grav = float(cu.grav)
    c.initial_condition = int(cu.initial_condition)
    c.dam_radius, c.dam_h_in, c.dam_h_out = float(cu.dam_radius), float(cu.dam_h_in), float(cu.dam_h_out)
    c.dam_x0, c.dam_y0 = float(cu.dam_x0), float(cu.dam_y0)
    return c


@dataclass
class Stats:
    attempts: int
    accepted: int
    rejected: int
    launches: int
    time: float
    dt: float
    dt_previous: float
    cfl: float
    snapshot_index: int
    done: bool
    status: int
    last_ierr: int

    @classmethod
    def from_c(cls, s: _lib.RunStats) -> "Stats":
        return cls(s.attempts, s.accepted, s.rejected, s.launches, s.time, s.dt, s.dt_previous, s.cfl,
                   s.snapshot_index, bool(s.done), s.status, s.last_ierr)


@dataclass
class StepLog:
    dt: np.ndarray
    cfl: np.ndarray
    time: np.ndarray
    dt_next: np.ndarray
    ierr: np.ndarray
    snap: np.ndarray


class Solver:
    """One grid on one GPU behind the C ABI."""

    def __init__(self, control: ControlSettings, custom: Optional[CustomSettings] = None,
                 device: int = 0, precision: Optional[int] = None):
        self.L = _lib.load()
        self.control = control
        self.custom = custom if custom is not None else CustomSettings()
        self.c = to_c_control(control, self.custom, precision)
        h = C.c_void_p()
        _lib.check(self.L.pcl_create(C.byref(self.c), int(device), C.byref(h)), "pcl_create")
        self.h = h
        self.shape = (control.m_eta + 4, control.m_xi + 4, int(control.number_of_equations))

    # -- lifecycle --
    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.pcl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state --
    def upload(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        if q.shape != self.shape:
            raise ValueError(f"state shape {q.shape} != {self.shape}")
        _lib.check(self.L.pcl_upload_state(self.h, q.ctypes.data), "pcl_upload_state")

    def download(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        _lib.check(self.L.pcl_download_state(self.h, out.ctypes.data), "pcl_download_state")
        return out

    def initial_condition(self) -> None:
        """The dam-break state of the custom settings, built on the device."""
        _lib.check(self.L.pcl_initial_condition(self.h), "pcl_initial_condition")

    # -- reference routine boundary --
    def update_rank_boundaries(self) -> None:
        _lib.check(self.L.pcl_update_rank_boundaries(self.h), "pcl_update_rank_boundaries")

    def solve_dimensional_split(self) -> int:
        ierr = C.c_int()
        _lib.check(self.L.pcl_solve_dimensional_split(self.h, C.byref(ierr)), "pcl_solve_dimensional_split")
        return ierr.value

    def restore_solution(self) -> None:
        _lib.check(self.L.pcl_restore_solution(self.h), "pcl_restore_solution")

    def integrate_source_term(self) -> None:
        _lib.check(self.L.pcl_integrate_source_term(self.h), "pcl_integrate_source_term")

    def update_time(self, step_valid: bool) -> None:
        _lib.check(self.L.pcl_update_time(self.h, int(bool(step_valid))), "pcl_update_time")

    def reset_cfl(self) -> None:
        _lib.check(self.L.pcl_reset_cfl(self.h), "pcl_reset_cfl")

    def advance_snapshot_index(self) -> None:
        _lib.check(self.L.pcl_advance_snapshot_index(self.h), "pcl_advance_snapshot_index")

    def set_dt(self, dt: float) -> None:
        _lib.check(self.L.pcl_set_dt(self.h, float(dt)), "pcl_set_dt")

    def _get_d(self, fn) -> float:
        v = C.c_double()
        _lib.check(fn(self.h, C.byref(v)), fn.__name__)
        return v.value

    @property
    def time(self) -> float:
        return self._get_d(self.L.pcl_get_time)

    @property
    def dt(self) -> float:
        return self._get_d(self.L.pcl_get_dt)

    @property
    def previous_dt(self) -> float:
        return self._get_d(self.L.pcl_get_previous_dt)

    @property
    def cfl(self) -> float:
        return self._get_d(self.L.pcl_get_cfl)

    @property
    def snapshot_index(self) -> int:
        v = C.c_int()
        _lib.check(self.L.pcl_get_snapshot_index(self.h, C.byref(v)), "pcl_get_snapshot_index")
        return v.value

    def snapshot_time(self, idx: int) -> float:
        v = C.c_double()
        _lib.check(self.L.pcl_get_snapshot_time(self.h, int(idx), C.byref(v)), "pcl_get_snapshot_time")
        return v.value

    # -- whole loop on the device --
    def advance(self, max_attempts: int = 0) -> Stats:
        s = _lib.RunStats()
        _lib.check(self.L.pcl_advance(self.h, int(max_attempts), C.byref(s)), "pcl_advance")
        return Stats.from_c(s)

    def set_user_bc(self, fn_address: Optional[int], user: Optional[int] = None) -> None:
        """Install a pcl_user_bc_fn (its address, e.g. from a ctypes CDLL) for sides coded 1;
        None restores the built-in wall."""
        _lib.check(self.L.pcl_set_user_bc(self.h, fn_address, user), "pcl_set_user_bc")

    def set_equation(self, module: int, params=()) -> None:
        """Equation module (PCL_EQ_* of include/paraclaws_b200.h) and its parameters."""
        arr = (C.c_double * max(len(params), 1))(*[float(p) for p in params])
        _lib.check(self.L.pcl_set_equation(self.h, int(module), arr if params else None, len(params)),
                   "pcl_set_equation")

    def set_sweep_shape(self, eta_shape: int) -> None:
        """Shape of the FP64 eta sweep (_lib.PCL_SHAPE_*): a schedule, the results stay the same."""
        _lib.check(self.L.pcl_set_sweep_shape(self.h, int(eta_shape)), "pcl_set_sweep_shape")

    def sweep_shape(self) -> int:
        """The eta-sweep shape the FP64 path runs for this grid (_lib.PCL_SHAPE_WINDOW or _BAND)."""
        v = C.c_int()
        _lib.check(self.L.pcl_get_sweep_shape(self.h, C.byref(v)), "pcl_get_sweep_shape")
        return v.value

    def set_source_hook(self, fn_address: Optional[int], user: Optional[int] = None) -> None:
        """Install a pcl_source_fn (integrate_source_term with a non-zero phi); None: phi = 0."""
        _lib.check(self.L.pcl_set_source_hook(self.h, fn_address, user), "pcl_set_source_hook")

    def advance_to_snapshot(self) -> Stats:
        """The device loop up to the next snapshot time (or the end); see write_snapshot."""
        s = _lib.RunStats()
        _lib.check(self.L.pcl_advance_to_snapshot(self.h, C.byref(s)), "pcl_advance_to_snapshot")
        return Stats.from_c(s)

    def write_snapshot(self, output_dir: str, wait: bool = True) -> None:
        """writeData of the current state under output_dir (reference text format)."""
        _lib.check(self.L.pcl_write_snapshot(self.h, str(output_dir).encode(), int(bool(wait))), "pcl_write_snapshot")

    def snapshot_wait(self) -> None:
        _lib.check(self.L.pcl_snapshot_wait(self.h), "pcl_snapshot_wait")

    def stats(self) -> Stats:
        s = _lib.RunStats()
        _lib.check(self.L.pcl_get_stats(self.h, C.byref(s)), "pcl_get_stats")
        return Stats.from_c(s)

    def io_bytes(self) -> dict:
        h2d, d2h = C.c_longlong(), C.c_longlong()
        _lib.check(self.L.pcl_get_io_bytes(self.h, C.byref(h2d), C.byref(d2h)), "pcl_get_io_bytes")
        return {"h2d": h2d.value, "d2h": d2h.value}

    def conservation_sums(self) -> np.ndarray:
        out = (C.c_double * 3)()
        _lib.check(self.L.pcl_conservation_sums(self.h, out), "pcl_conservation_sums")
        return np.array(list(out))

    def set_mesh_metrics(self, kappa: np.ndarray, lr_xi: np.ndarray, lr_eta: np.ndarray) -> None:
        """Per-cell capacity and face length ratios of a mapped grid, shaped (m_eta+4, m_xi+4)
        (the reference's column-major arrays); see paraclaws_b200.mesh."""
        shape = self.shape[:2]
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (kappa, lr_xi, lr_eta)]
        for a in arrs:
            if a.shape != shape:
                raise ValueError(f"metric shape {a.shape} != {shape}")
        _lib.check(self.L.pcl_set_mesh_metrics(self.h, *(a.ctypes.data for a in arrs)), "pcl_set_mesh_metrics")

    def set_tile_rows(self, rows: int) -> None:
        _lib.check(self.L.pcl_set_tile_rows(self.h, int(rows)), "pcl_set_tile_rows")

    def reset_time_control(self) -> None:
        _lib.check(self.L.pcl_reset_time_control(self.h), "pcl_reset_time_control")

    def profile_kernels(self, reps: int = 10) -> list:
        out = (C.c_double * 8)()
        n = C.c_int()
        _lib.check(self.L.pcl_profile_kernels(self.h, int(reps), out, C.byref(n)), "pcl_profile_kernels")
        return [out[k] for k in range(n.value)]

    def synchronize(self) -> None:
        _lib.check(self.L.pcl_synchronize(self.h), "pcl_synchronize")

    def step_log(self) -> StepLog:
        n = C.c_longlong()
        _lib.check(self.L.pcl_get_step_log(self.h, None, 0, C.byref(n)), "pcl_get_step_log")
        recs = (_lib.StepRecord * max(n.value, 1))()
        _lib.check(self.L.pcl_get_step_log(self.h, recs, n.value, C.byref(n)), "pcl_get_step_log")
        k = n.value
        arr = np.frombuffer(recs, dtype=np.dtype([("dt", "f8"), ("cfl", "f8"), ("time", "f8"),
                                                  ("dt_next", "f8"), ("ierr", "i4"), ("snap", "i4")]),
                            count=k)
        return StepLog(arr["dt"].copy(), arr["cfl"].copy(), arr["time"].copy(), arr["dt_next"].copy(),
                       arr["ierr"].copy(), arr["snap"].copy())

    @property
    def stream(self) -> int:
        return self.L.pcl_get_stream(self.h) or 0

    @property
    def device_bytes(self) -> int:
        return int(self.L.pcl_device_bytes(self.h))


def format_e26_16(value: float) -> str:
    """A value in the E26.16 field of the reference's snapshot format."""
    L = _lib.load()
    buf = C.create_string_buffer(27)
    _lib.check(L.pcl_format_e26_16(float(value), buf), "pcl_format_e26_16")
    return buf.value.decode()


def run_device_loop_with_snapshots(s: Solver, output_dir: str) -> list:
    """main.f90:178-283 on the device with writeData at t0 and at every snapshot time; the
    formatting of one snapshot overlaps the steps to the next.  Returns the snapshot times."""
    times = [s.time]
    s.write_snapshot(output_dir, wait=False)
    while True:
        st = s.advance_to_snapshot()
        if st.time >= s.control.time_final or st.done or st.status != 0:
            if st.status == 0 and st.time >= s.control.time_final:
                s.write_snapshot(output_dir, wait=False)
                times.append(st.time)
            break
        s.write_snapshot(output_dir, wait=False)
        times.append(st.time)
    s.snapshot_wait()
    return times


def run_host_loop(s: Solver, max_attempts: int = 0) -> StepLog:
    """main.f90:193-283 driven from the host, one C-ABI call per reference routine."""
    rows = []
    max_acc = int(s.custom.max_accepted_steps)
    accepted = 0
    nsnap = max(int(s.control.number_of_snapshots), 1)
    snaps = [s.snapshot_time(k) for k in range(1, nsnap + 1)]
    st = s.stats()
    while st.time < s.control.time_final:
        if max_acc > 0 and accepted >= max_acc:
            break
        if max_attempts > 0 and len(rows) >= max_attempts:
            break
        dt_used = st.dt
        ierr = s.solve_dimensional_split()
        if ierr < 0:
            s.update_time(False)
            st = s.stats()
            s.restore_solution()
            s.reset_cfl()
        else:
            s.integrate_source_term()
            s.update_rank_boundaries()
            s.update_time(True)
            st = s.stats()
            idx = st.snapshot_index
            if idx <= nsnap and st.time >= snaps[idx - 1]:
                s.advance_snapshot_index()
                st.snapshot_index = idx + 1
            s.reset_cfl()
            accepted += 1
        rows.append((dt_used, st.cfl, st.time, st.dt, ierr, st.snapshot_index))
    a = np.array(rows, dtype=np.float64).reshape(-1, 6)
    return StepLog(a[:, 0], a[:, 1], a[:, 2], a[:, 3], a[:, 4].astype(np.int32), a[:, 5].astype(np.int32))
