"""ctypes binding of libparaclaws_b200.so (include/paraclaws_b200.h).

The library is built in-tree (paraclaws_b200/build.py).  There is no fallback: if the shared
library cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

from . import build as _build

HEADER = Path(__file__).resolve().parent.parent / "include" / "paraclaws_b200.h"

PCL_OK = 0
PCL_ERR_NAN = -1
PCL_ERR_NEG_DEPTH = -2
PCL_ERR_TIMEOUT = -3
PCL_SHAPE_AUTO, PCL_SHAPE_WINDOW, PCL_SHAPE_BAND = 0, 1, 2  # pcl_set_sweep_shape
PCL_ERR_OOM = -4
PCL_ERR_BADARG = -5
PCL_ERR_CUDA = -6
PCL_ERR_FATAL_DT = -7
PCL_ERR_IO = -8
PCL_ERR_FULL = -9


class SolverControl(C.Structure):
    _fields_ = [
        ("num_equations", C.c_int), ("num_dimensions", C.c_int), ("num_ghost", C.c_int),
        ("num_aux", C.c_int), ("num_waves", C.c_int), ("number_of_snapshots", C.c_int),
        ("adaptive_timestepping", C.c_int), ("higher_order_flux_correction", C.c_int),
        ("use_limiter", C.c_int), ("limiter_method", C.c_int), ("m_xi", C.c_int), ("m_eta", C.c_int),
        ("bc_xi_lower", C.c_int), ("bc_xi_upper", C.c_int), ("bc_eta_lower", C.c_int),
        ("bc_eta_upper", C.c_int), ("precision_mode", C.c_int), ("initial_condition", C.c_int),
        ("t_start", C.c_double), ("t_final", C.c_double), ("dt_initial", C.c_double),
        ("cfl_limit", C.c_double), ("dt_min", C.c_double), ("dt_max", C.c_double),
        ("dt_max_growth_ratio", C.c_double), ("dt_min_shrink_ratio", C.c_double),
        ("xi_min", C.c_double), ("xi_max", C.c_double), ("eta_min", C.c_double), ("eta_max", C.c_double),
        ("grav", C.c_double), ("dam_radius", C.c_double), ("dam_h_in", C.c_double),
        ("dam_h_out", C.c_double), ("dam_x0", C.c_double), ("dam_y0", C.c_double),
        ("max_accepted_steps", C.c_longlong),
    ]


class RunStats(C.Structure):
    _fields_ = [
        ("attempts", C.c_longlong), ("accepted", C.c_longlong), ("rejected", C.c_longlong),
        ("launches", C.c_longlong), ("time", C.c_double), ("dt", C.c_double), ("dt_previous", C.c_double), ("cfl", C.c_double),
        ("snapshot_index", C.c_int), ("done", C.c_int), ("status", C.c_int), ("last_ierr", C.c_int),
    ]


class StepRecord(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("cfl", C.c_double), ("time", C.c_double), ("dt_next", C.c_double),
        ("ierr", C.c_int), ("snapshot_index", C.c_int),
    ]


class PclError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {status_string(code)} ({code})")


_lib = None


def lib_path() -> Path:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the shared library (building it first when sources are newer and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if build_if_missing:
        try:
            if _build.needs_build():
                _build.build()
        except RuntimeError:
            if not path.exists():
                raise
    if not path.exists():
        raise RuntimeError(f"{path} is not built; run paraclaws_b200/build.py")
    L = C.CDLL(str(path))
    P = C.POINTER
    vp = C.c_void_p
    L.pcl_default_control.argtypes = [P(SolverControl)]
    L.pcl_default_control.restype = None
    L.pcl_read_solver_control.argtypes = [C.c_char_p, C.c_char_p, P(SolverControl)]
    L.pcl_create.argtypes = [P(SolverControl), C.c_int, P(vp)]
    L.pcl_destroy.argtypes = [vp]
    for name in ("pcl_upload_state", "pcl_download_state"):
        getattr(L, name).argtypes = [vp, vp]
    for name in ("pcl_update_rank_boundaries", "pcl_restore_solution", "pcl_integrate_source_term", "pcl_initial_condition",
                 "pcl_reset_cfl", "pcl_advance_snapshot_index", "pcl_synchronize"):
        getattr(L, name).argtypes = [vp]
    L.pcl_solve_dimensional_split.argtypes = [vp, P(C.c_int)]
    L.pcl_set_mesh_metrics.argtypes = [vp, vp, vp, vp]
    L.pcl_advance_to_snapshot.argtypes = [vp, P(RunStats)]
    L.pcl_write_snapshot.argtypes = [vp, C.c_char_p, C.c_int]
    L.pcl_snapshot_wait.argtypes = [vp]
    L.pcl_format_e26_16.argtypes = [C.c_double, C.c_char_p]
    L.pcl_set_user_bc.argtypes = [vp, vp, vp]
    L.pcl_set_source_hook.argtypes = [vp, vp, vp]
    L.pcl_set_equation.argtypes = [vp, C.c_int, vp, C.c_int]
    L.pcl_set_sweep_shape.argtypes = [vp, C.c_int]
    L.pcl_get_sweep_shape.argtypes = [vp, P(C.c_int)]
    L.pcl_compute_mesh_metrics.argtypes = [P(SolverControl), vp, vp, vp, vp, vp]
    L.pcl_update_time.argtypes = [vp, C.c_int]
    L.pcl_set_dt.argtypes = [vp, C.c_double]
    for name in ("pcl_get_time", "pcl_get_dt", "pcl_get_previous_dt", "pcl_get_cfl"):
        getattr(L, name).argtypes = [vp, P(C.c_double)]
    L.pcl_get_snapshot_index.argtypes = [vp, P(C.c_int)]
    L.pcl_get_snapshot_time.argtypes = [vp, C.c_int, P(C.c_double)]
    L.pcl_advance.argtypes = [vp, C.c_longlong, P(RunStats)]
    L.pcl_get_stats.argtypes = [vp, P(RunStats)]
    L.pcl_reset_time_control.argtypes = [vp]
    L.pcl_profile_kernels.argtypes = [vp, C.c_int, P(C.c_double), P(C.c_int)]
    L.pcl_get_step_log.argtypes = [vp, P(StepRecord), C.c_longlong, P(C.c_longlong)]
    L.pcl_get_stream.argtypes = [vp]
    L.pcl_get_stream.restype = vp
    L.pcl_state_doubles.argtypes = [vp]
    L.pcl_state_doubles.restype = C.c_longlong
    L.pcl_device_bytes.argtypes = [vp]
    L.pcl_device_bytes.restype = C.c_longlong
    L.pcl_get_io_bytes.argtypes = [vp, P(C.c_longlong), P(C.c_longlong)]
    L.pcl_conservation_sums.argtypes = [vp, P(C.c_double)]
    L.pcl_batch_create.argtypes = [C.c_int, C.c_int, C.c_int, P(vp)]
    L.pcl_batch_destroy.argtypes = [vp]
    L.pcl_batch_instance_bytes.argtypes = [P(SolverControl)]
    L.pcl_batch_instance_bytes.restype = C.c_longlong
    L.pcl_batch_add.argtypes = [vp, P(SolverControl), vp, P(C.c_int)]
    L.pcl_batch_remove.argtypes = [vp, C.c_int]
    L.pcl_batch_step.argtypes = [vp, C.c_int]
    L.pcl_batch_poll.argtypes = [vp, P(C.c_int), P(C.c_int)]
    L.pcl_batch_stats.argtypes = [vp, C.c_int, P(RunStats)]
    L.pcl_batch_download.argtypes = [vp, C.c_int, vp]
    L.pcl_batch_get_step_log.argtypes = [vp, C.c_int, P(StepRecord), C.c_longlong, P(C.c_longlong)]
    L.pcl_batch_set_schedule.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int]
    L.pcl_batch_info.argtypes = [vp, P(C.c_int), P(C.c_int), P(C.c_longlong), P(C.c_longlong)]
    L.pcl_batch_get_stream.argtypes = [vp]
    L.pcl_batch_get_stream.restype = vp
    L.pcl_set_tile_rows.argtypes = [vp, C.c_int]
    L.pcl_solve_dimensional_split_noalloc.argtypes = [P(SolverControl), C.c_int, vp, vp, vp, C.c_longlong,
                                                      C.c_double, P(C.c_double), P(C.c_int)]
    L.pcl_check_quotients.argtypes = [vp, vp, C.c_longlong, P(C.c_longlong), P(C.c_longlong)]
    L.pcl_check_quotients_random.argtypes = [C.c_longlong, C.c_ulonglong, P(C.c_longlong), P(C.c_longlong)]
    L.pcl_check_flux_paths.argtypes = [C.c_longlong, C.c_ulonglong, C.c_double, P(C.c_longlong),
                                       P(C.c_longlong), P(C.c_longlong)]
    L.pcl_batch_inject_stall.argtypes = [vp, C.c_int, C.c_uint]
    L.pcl_inject_copy_stall.argtypes = [vp, C.c_int, C.c_uint]
    L.pcl_host_alloc.argtypes = [P(vp), C.c_longlong]
    L.pcl_host_free.argtypes = [vp]
    L.pcl_status_string.argtypes = [C.c_int]
    L.pcl_status_string.restype = C.c_char_p
    _lib = L
    return L


def status_string(code: int) -> str:
    try:
        return load(build_if_missing=False).pcl_status_string(int(code)).decode()
    except Exception:  # library unavailable while formatting an error
        return "status"


def check(code: int, where: str) -> int:
    if code < 0:
        raise PclError(code, where)
    return code


# pcl_map_fn: void (*)(double xi, double eta, double* x, double* y, void* user)
MapFn = C.CFUNCTYPE(None, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)


def declared_functions() -> list:
    """Names of the functions include/paraclaws_b200.h declares."""
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*?[\s\*]+(pcl_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))
