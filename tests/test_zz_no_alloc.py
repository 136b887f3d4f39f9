"""pcl_solve_dimensional_split_noalloc: the one-step entry point for callers that cannot
allocate device memory (their memory belongs to another allocator, or they must not pay the
synchronisation of cudaMalloc/cudaFree).  It keeps all scratch in a static array of the library
and must give the same results as the regular entry point, pcl_solve_dimensional_split, which
allocates its scratch in pcl_create.  The FP64 path is bit-exact, so the tolerance is zero, as
in the other FP64 parity tests.

This file sorts last so that a run stopping at its first failure has run everything else."""
import ctypes as C

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver, to_c_control

pytestmark = pytest.mark.gpu


def _regular_step(c, q):
    """Ghost fill and one attempted step through the regular context entry points."""
    s = Solver(c)
    s.upload(q)
    s.update_rank_boundaries()
    filled = s.download()
    ierr = s.solve_dimensional_split()
    cfl = s.cfl
    out = s.download()
    s.close()
    return filled, ierr, cfl, out


def _planes(q, ld):
    """(m_eta+4, m_xi+4, 3) reference-layout state -> 3 planes of rows with leading dimension ld."""
    nj, ni, _ = q.shape
    p = np.zeros((3, nj, ld), dtype=np.float64)
    p[:, :, :ni] = np.moveaxis(q, 2, 0)
    return p


def _noalloc_step(c, filled, ld, dt, out_fill=0.0, stream=None):
    import torch
    L = _lib.load()
    d_in = torch.from_numpy(_planes(filled, ld)).cuda()
    d_out = torch.full_like(d_in, out_fill)
    torch.cuda.synchronize()
    sc = to_c_control(c)
    cfl = C.c_double()
    ierr = C.c_int()
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = L.pcl_solve_dimensional_split_noalloc(C.byref(sc), 0, handle, C.c_void_p(d_in.data_ptr()),
                                               C.c_void_p(d_out.data_ptr()), ld, dt, C.byref(cfl), C.byref(ierr))
    torch.cuda.synchronize()
    out = d_out.cpu().numpy()
    ni = filled.shape[1]
    return rc, ierr.value, cfl.value, np.ascontiguousarray(np.moveaxis(out[:, :, :ni], 0, 2)), out


def _case_a():
    c = ctl.dam_break_control(100, limiter=4, bc=2)
    c.m_eta = 80
    c.initial_timestep = 2e-3
    q = ic.gaussian_bumps(100, 80, seed=11)
    q[..., 1] = 0.2 * np.sin(np.arange(104))[None, :]
    q[..., 2] = -0.1 * np.cos(np.arange(84))[:, None]
    return c, q, 111


def _case_b():
    c = ctl.dam_break_control(128, limiter=1, bc=1)
    c.m_eta = 64
    c.initial_timestep = 1e-3
    q = ic.circular_dam(128, 64, radius=0.45, h_in=3.0)
    return c, q, 132


def test_noalloc_matches_regular_step_twice_in_a_row(pcl):
    results = []
    for case in (_case_a, _case_b, _case_a):
        c, q, ld = case()
        filled, ierr, cfl, out = _regular_step(c, q)
        rc, ierr_n, cfl_n, out_n, _ = _noalloc_step(c, filled, ld, c.initial_timestep)
        assert rc == 0
        assert ierr_n == ierr == 1
        assert cfl_n == cfl
        assert np.array_equal(out_n, out)
        results.append(out_n)
    # the repeated first case is unaffected by what the previous call left in the scratch
    assert np.array_equal(results[0], results[2])


def test_noalloc_on_a_caller_stream_keeps_the_current_device(pcl):
    """The stream argument: a caller's own (non-default) stream; the call leaves the caller's
    current device as it found it."""
    import torch
    for case in (_case_b, _case_a):
        c, q, ld = case()
        filled, ierr, cfl, out = _regular_step(c, q)
        before = torch.cuda.current_device()
        st = torch.cuda.Stream()
        rc, ierr_n, cfl_n, out_n, _ = _noalloc_step(c, filled, ld, c.initial_timestep, stream=st)
        assert torch.cuda.current_device() == before
        assert rc == 0 and ierr_n == ierr == 1 and cfl_n == cfl
        assert np.array_equal(out_n, out)


def test_noalloc_rejected_attempt_leaves_output(pcl):
    c, q, ld = _case_a()
    c.initial_timestep = 0.05  # CFL far above CFL_target / shrink: rejected after the xi sweep
    filled, ierr, cfl, _ = _regular_step(c, q)
    rc, ierr_n, cfl_n, _, raw = _noalloc_step(c, filled, ld, c.initial_timestep, out_fill=-7.0)
    assert rc == 0 and ierr_n == ierr == -1 and cfl_n == cfl
    assert np.all(raw == -7.0)


def test_noalloc_rejects_grids_beyond_its_scratch(pcl):
    import torch
    L = _lib.load()
    c = ctl.dam_break_control(129)
    sc = to_c_control(c)
    ierr = C.c_int()
    buf_in = torch.zeros(3 * 133 * 133, dtype=torch.float64, device="cuda")
    buf_out = torch.zeros_like(buf_in)
    rc = L.pcl_solve_dimensional_split_noalloc(C.byref(sc), 0, None, C.c_void_p(buf_in.data_ptr()),
                                               C.c_void_p(buf_out.data_ptr()), 133, 1e-3, None, C.byref(ierr))
    assert rc == _lib.PCL_ERR_BADARG
    assert torch.count_nonzero(buf_out).item() == 0
