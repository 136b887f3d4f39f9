"""ctypes front end of the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker or as the timed CPU stand-in for the reference.  parity unpinned:
the Fortran reference cannot be built in this image; see oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

ORC_OK = 0
ORC_ERR_NAN = -1
ORC_ERR_NEG_DEPTH = -2
ORC_ERR_BADARG = -5
ORC_ERR_FATAL_DT = -7
ORC_ERR_LAPACK = -8


class OrcParams(C.Structure):
    _fields_ = [
        ("m_xi", C.c_int), ("m_eta", C.c_int), ("num_ghost", C.c_int), ("higher_order", C.c_int),
        ("use_limiter", C.c_int), ("limiter_method", C.c_int), ("bc_xi_lower", C.c_int),
        ("bc_xi_upper", C.c_int), ("bc_eta_lower", C.c_int), ("bc_eta_upper", C.c_int),
        ("n_snapshots", C.c_int), ("adaptive", C.c_int), ("eigen_mode", C.c_int), ("num_equations", C.c_int),
        ("xi_min", C.c_double), ("xi_max", C.c_double), ("eta_min", C.c_double), ("eta_max", C.c_double),
        ("grav", C.c_double), ("t_start", C.c_double), ("t_final", C.c_double), ("dt_initial", C.c_double),
        ("cfl_limit", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double), ("growth", C.c_double),
        ("shrink", C.c_double), ("max_accepted", C.c_longlong),
    ]


def build() -> Path:
    """Compile liboracle.so with oracle/Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        P = C.POINTER
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.orc_load_lapack.argtypes = [C.c_char_p]
        L.orc_create.argtypes = [P(OrcParams)]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_status.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_state.argtypes = [C.c_void_p, dp]
        L.orc_get_state.argtypes = [C.c_void_p, dp]
        L.orc_get_mesh.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
        L.orc_set_mesh.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_set_friction.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_equation.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.orc_module_num_equations.argtypes = [C.c_int]
        L.orc_update_rank_boundaries.argtypes = [C.c_void_p]
        L.orc_solve_dimensional_split.argtypes = [C.c_void_p, P(C.c_int)]
        L.orc_sweep.argtypes = [C.c_void_p, C.c_int, P(C.c_double)]
        L.orc_update_time.argtypes = [C.c_void_p, C.c_int]
        L.orc_reset_cfl.argtypes = [C.c_void_p]
        L.orc_set_dt.argtypes = [C.c_void_p, C.c_double]
        L.orc_set_time_state.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int]
        L.orc_get_time_state.argtypes = [C.c_void_p, dp, ip]
        L.orc_run.argtypes = [C.c_void_p, C.c_longlong, dp, ip, C.c_longlong, P(C.c_longlong), P(C.c_longlong)]
        L.orc_hll_interface.argtypes = [C.c_int, dp, dp, C.c_double, C.c_int, dp, dp]
        L.orc_limiter_phi.argtypes = [C.c_int, C.c_double]
        L.orc_limiter_phi.restype = C.c_double
        _lib = L
    return _lib


def lapack_path() -> Optional[str]:
    """scipy's bundled OpenBLAS (exports scipy_dgeev_ / scipy_dgemv_)."""
    try:
        import scipy
    except ImportError:
        return None
    d = Path(scipy.__file__).resolve().parent.parent / "scipy.libs"
    for p in sorted(d.glob("libscipy_openblas*.so")):
        return str(p)
    return None


def load_lapack() -> bool:
    p = lapack_path()
    return p is not None and lib().orc_load_lapack(p.encode()) == ORC_OK


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def params_from(control, custom=None, eigen_mode: int = 0) -> OrcParams:
    """OrcParams from paraclaws_b200.control.ControlSettings (+ CustomSettings)."""
    from paraclaws_b200.control import GRAV_REFERENCE
    p = OrcParams()
    p.m_xi, p.m_eta = control.m_xi, control.m_eta
    p.num_ghost = control.number_of_ghost_cells
    p.higher_order = int(bool(control.add_higher_order_flux_correction))
    p.use_limiter = int(bool(control.use_limtiter))
    p.limiter_method = control.limiter_function
    p.bc_xi_lower, p.bc_xi_upper = control.bc_xi_lower, control.bc_xi_upper
    p.bc_eta_lower, p.bc_eta_upper = control.bc_eta_lower, control.bc_eta_upper
    p.n_snapshots = control.number_of_snapshots
    p.adaptive = int(bool(control.adaptive_timestepping))
    p.eigen_mode = eigen_mode
    p.num_equations = int(control.number_of_equations)
    p.xi_min, p.xi_max = float(control.xi_min), float(control.xi_max)
    p.eta_min, p.eta_max = float(control.eta_min), float(control.eta_max)
    p.grav = float(custom.grav) if custom is not None else GRAV_REFERENCE
    p.t_start, p.t_final = float(control.time_start), float(control.time_final)
    p.dt_initial = float(control.initial_timestep)
    p.cfl_limit = float(control.CFL_limit)
    p.dt_min, p.dt_max = float(control.min_allowed_dt), float(control.max_allowed_dt)
    p.growth, p.shrink = float(control.dt_max_growth_ratio), float(control.dt_min_shrink_ratio)
    p.max_accepted = int(custom.max_accepted_steps) if custom is not None else 0
    return p


@dataclass
class RunLog:
    dt: np.ndarray        # dt used by each attempted step
    cfl: np.ndarray       # CFL of the attempt
    time: np.ndarray      # time after the attempt
    dt_next: np.ndarray   # dt after the attempt
    ierr: np.ndarray      # 1 accepted / -1 rejected
    snap: np.ndarray      # snapshot index after the attempt
    accepted: int
    status: int


class Oracle:
    """One oracle context (one grid)."""

    def __init__(self, control, custom=None, eigen_mode: int = 0):
        L = lib()
        if eigen_mode == 1 and not load_lapack():
            raise RuntimeError("LAPACK (scipy OpenBLAS) not available for eigen_mode=1")
        self.p = params_from(control, custom, eigen_mode)
        self.h = L.orc_create(C.byref(self.p))
        if not self.h:
            raise ValueError("oracle rejected the settings")
        self.shape = (control.m_eta + 4, control.m_xi + 4, int(control.number_of_equations))

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    __del__ = close

    def set_state(self, q: np.ndarray) -> None:
        q = np.ascontiguousarray(q, dtype=np.float64)
        assert q.shape == self.shape
        lib().orc_set_state(self.h, q)

    def state(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        lib().orc_get_state(self.h, out)
        return out

    def mesh(self):
        n = self.shape[:2]
        arrs = [np.empty(n, dtype=np.float64) for _ in range(5)]
        lib().orc_get_mesh(self.h, *arrs)
        return dict(zip(["xi", "eta", "kappa", "lr_xi", "lr_eta"], arrs))

    def set_friction(self, c: float) -> None:
        """source_function phi = (0, -c hu, -c hv) (0: the dam break's phi = 0)."""
        lib().orc_set_friction(self.h, float(c))

    def set_equation(self, module: int, p0: float = 0.0, p1: float = 0.0) -> None:
        """Equation module (ORC_EQ_* of oracle.h: the same ids as the library's PCL_EQ_*), whose
        num_equations must be the context's."""
        if lib().orc_set_equation(self.h, int(module), float(p0), float(p1)) != 0:
            raise ValueError(f"equation module {module} does not fit this context")

    def set_mesh(self, kappa, lr_xi, lr_eta) -> None:
        """Metrics of a mapped grid (arrays shaped like mesh()['kappa'])."""
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (kappa, lr_xi, lr_eta)]
        for a in arrs:
            if a.shape != self.shape[:2]:
                raise ValueError(f"metric shape {a.shape} != {self.shape[:2]}")
        lib().orc_set_mesh(self.h, *arrs)

    def status(self) -> int:
        return lib().orc_status(self.h)

    def update_rank_boundaries(self) -> int:
        return lib().orc_update_rank_boundaries(self.h)

    def sweep(self, ixy: int):
        cfl = C.c_double()
        st = lib().orc_sweep(self.h, ixy, C.byref(cfl))
        return st, cfl.value

    def solve_dimensional_split(self):
        ierr = C.c_int()
        st = lib().orc_solve_dimensional_split(self.h, C.byref(ierr))
        return st, ierr.value

    def update_time(self, valid: bool) -> int:
        return lib().orc_update_time(self.h, int(bool(valid)))

    def reset_cfl(self) -> None:
        lib().orc_reset_cfl(self.h)

    def set_dt(self, dt: float) -> None:
        lib().orc_set_dt(self.h, float(dt))

    def set_time_state(self, time: float, dt: float, cfl: float, snapshot_index: int = 1) -> None:
        lib().orc_set_time_state(self.h, float(time), float(dt), float(cfl), int(snapshot_index))

    def time_state(self) -> dict:
        d = np.zeros(8, dtype=np.float64)
        i = np.zeros(4, dtype=np.int32)
        lib().orc_get_time_state(self.h, d, i)
        return dict(time=d[0], dt=d[1], dt_previous=d[2], cfl=d[3], cfl_previous=d[4],
                    time_final=d[5], next_snapshot=d[6], snapshot_index=int(i[0]),
                    snapshot_exception=int(i[1]), n_snapshots=int(i[2]))

    def run(self, max_attempts: int = 0, log_cap: int = 1 << 16) -> RunLog:
        """main.f90:193-283 until time_final (or the accepted-step cap, or max_attempts)."""
        ld = np.zeros(log_cap * 4, dtype=np.float64)
        li = np.zeros(log_cap * 2, dtype=np.int32)
        na = C.c_longlong()
        nacc = C.c_longlong()
        st = lib().orc_run(self.h, int(max_attempts), ld, li, int(log_cap), C.byref(na), C.byref(nacc))
        n = min(na.value, log_cap)
        ld = ld[: n * 4].reshape(n, 4)
        li = li[: n * 2].reshape(n, 2)
        return RunLog(dt=ld[:, 0].copy(), cfl=ld[:, 1].copy(), time=ld[:, 2].copy(),
                      dt_next=ld[:, 3].copy(), ierr=li[:, 0].copy(), snap=li[:, 1].copy(),
                      accepted=nacc.value, status=st)


def hll_interface(ixy: int, qL, qR, grav: float, eigen_mode: int = 0):
    lam = np.zeros(2, dtype=np.float64)
    w = np.zeros(6, dtype=np.float64)
    st = lib().orc_hll_interface(ixy, np.ascontiguousarray(qL, dtype=np.float64),
                                 np.ascontiguousarray(qR, dtype=np.float64), grav, eigen_mode, lam, w)
    return st, lam, w.reshape(2, 3)


def limiter_phi(method: int, r: float) -> float:
    return lib().orc_limiter_phi(method, float(r))
