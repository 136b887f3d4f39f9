"""Device hooks: the user boundary condition (BC code 1) and the source term.  Host code enqueues
its own device kernels, in host-driven calls and inside the device loop's CUDA graphs.  A user
wall written against the hook's view reproduces the built-in wall bit for bit, and a user
friction source reproduces the oracle's integrate_source_term with the same phi bit for bit."""
import ctypes as C
import dataclasses
import subprocess

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import build as B
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic
from paraclaws_b200.solver import Solver, run_host_loop

pytestmark = pytest.mark.gpu

USER_BC_SRC = r'''
#include <cuda_runtime.h>
#include "paraclaws_b200.h"

// reflective wall: mirror the two nearest interior cells, normal momentum negated
__global__ void wall(pcl_bc_view v, int sides, int force) {
  if (!force && *v.attempt_accepted != 1) return;
  const int n = v.m_xi > v.m_eta ? v.m_xi : v.m_eta;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int side = tid / (2 * n), rem = tid % (2 * n), layer = rem / n, idx = 1 + rem % n;
  if (side >= 4 || !(sides & (1 << side))) return;
  double* b = v.state + (long long)(*v.current_buffer) * v.buffer_stride;
  const long long P = v.pitch;
  if (side < 2) {
    const int j = idx;
    if (j > v.m_eta) return;
    const int i = side == 0 ? -1 + layer : v.m_xi + 1 + layer;
    const int im = side == 0 ? 1 - i : 2 * v.m_xi + 1 - i;
    for (int me = 0; me < 3; ++me) {
      double* p = b + me * v.plane_stride + (j + 1) * P;
      p[i + 1] = me == 1 ? -p[im + 1] : p[im + 1];
    }
  } else {
    const int i = idx;
    if (i > v.m_xi) return;
    const int j = side == 2 ? -1 + layer : v.m_eta + 1 + layer;
    const int jm = side == 2 ? 1 - j : 2 * v.m_eta + 1 - j;
    for (int me = 0; me < 3; ++me) {
      double* p = b + me * v.plane_stride + (i + 1);
      p[(j + 1) * P] = me == 2 ? -p[(jm + 1) * P] : p[(jm + 1) * P];
    }
  }
}

// inflow at xi low: h = 3, hu = 0.5 h, hv = 0 in both ghost columns
__global__ void inflow(pcl_bc_view v, int force) {
  if (!force && *v.attempt_accepted != 1) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + t / 2, i = -1 + t % 2;
  if (j > v.m_eta) return;
  double* b = v.state + (long long)(*v.current_buffer) * v.buffer_stride + (j + 1) * (long long)v.pitch + (i + 1);
  b[0] = 3.0;
  b[v.plane_stride] = 1.5;
  b[2 * v.plane_stride] = 0.0;
}

extern "C" int user_wall(const pcl_bc_view* v, int sides, int force, void* stream, void* user) {
  const int n = v->m_xi > v->m_eta ? v->m_xi : v->m_eta;
  wall<<<(8 * n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*v, sides, force);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
extern "C" int user_inflow(const pcl_bc_view* v, int sides, int force, void* stream, void* user) {
  if (sides != 1) return 1;  // only xi low is coded 1 in the test
  inflow<<<(2 * v->m_eta + 127) / 128, 128, 0, (cudaStream_t)stream>>>(*v, force);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
extern "C" int user_fails(const pcl_bc_view*, int, int, void*, void*) { return 7; }

// source_function phi = (0, -c hu, -c hv), forward Euler q_p += phi_p dt on the interior
__global__ void friction(pcl_device_view v, int force, double c) {
  if (!force && *v.attempt_accepted != 1) return;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= v.m_xi * v.m_eta) return;
  const int i = 1 + t % v.m_xi, j = 1 + t / v.m_xi;
  const double dt = *v.step_dt;
  double* b = v.state + (long long)(*v.current_buffer) * v.buffer_stride + (j + 1) * (long long)v.pitch + (i + 1);
  const double phi[3] = {0.0, -c * b[v.plane_stride], -c * b[2 * v.plane_stride]};
  for (int me = 0; me < 3; ++me) b[me * v.plane_stride] = b[me * v.plane_stride] + phi[me] * dt;
}
extern "C" int user_friction(const pcl_device_view* v, int force, void* stream, void* user) {
  const double c = *static_cast<const double*>(user);
  const int n = v->m_xi * v->m_eta;
  friction<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*v, force, c);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
'''


@pytest.fixture(scope="module")
def userlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("userbc")
    src = d / "user_bc.cu"
    src.write_text(USER_BC_SRC)
    so = d / "libuserbc.so"
    cmd = [B.nvcc(), "-shared", "-Xcompiler", "-fPIC", *B.ARCH, "--fmad=false", "-I", str(B.ROOT / "include"), str(src),
           "-o", str(so)]
    subprocess.run(cmd, check=True, capture_output=True)
    return C.CDLL(str(so))


def _addr(lib, name):
    return C.cast(getattr(lib, name), C.c_void_p).value


@pytest.mark.parametrize("device_loop", [False, True])
def test_user_wall_equals_builtin_wall(pcl, userlib, device_loop):
    c = dataclasses.replace(ctl.dam_break_control(48, limiter=4, bc=1, time_final=0.05), m_eta=40)
    q = ic.gaussian_bumps(48, 40, seed=3)
    q[..., 1] = 0.2
    out = []
    for hook in (None, _addr(userlib, "user_wall")):
        s = Solver(c)
        if hook:
            s.set_user_bc(hook)
        s.upload(q)
        s.update_rank_boundaries()
        if device_loop:
            s.advance()
            dts = s.step_log().dt
        else:
            dts = run_host_loop(s).dt
        out.append((s.download(), dts, s.stats().accepted))
        s.close()
    assert out[0][2] == out[1][2] > 5
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])


def test_user_inflow_fills_its_side(pcl, userlib):
    c = ctl.dam_break_control(32, limiter=1, bc=2, time_final=0.03)
    c.bc_xi_lower = 1
    s = Solver(c)
    s.set_user_bc(_addr(userlib, "user_inflow"))
    s.upload(ic.lake_at_rest(32, 32))
    s.update_rank_boundaries()
    q = s.download()
    assert np.all(q[2:-2, 0:2, 0] == 3.0) and np.all(q[2:-2, 0:2, 1] == 1.5)
    st = s.advance()
    assert st.status == 0 and st.accepted > 3
    q = s.download()
    assert np.all(q[2:-2, 0:2, 0] == 3.0) and np.all(q[2:-2, 0:2, 2] == 0.0)
    assert q[2:-2, 2, 1].mean() > 0.1  # the inflow pushes water into the grid
    s.close()


def test_failing_hook_is_reported(pcl, userlib):
    c = ctl.dam_break_control(16, bc=1)
    s = Solver(c)
    s.set_user_bc(_addr(userlib, "user_fails"))
    s.initial_condition()
    with pytest.raises(_lib.PclError) as e:
        s.update_rank_boundaries()
    assert "device hook" in str(e.value)
    s.set_user_bc(None)
    s.update_rank_boundaries()
    s.close()


@pytest.mark.parametrize("device_loop", [False, True])
def test_friction_source_matches_oracle(pcl, oracle_lib, userlib, device_loop):
    from oracle.oracle import Oracle
    c = ctl.dam_break_control(40, limiter=1, bc=2, time_final=0.05)
    q = ic.circular_dam(40, 40)
    coeff = C.c_double(3.5)
    s = Solver(c)
    s.set_source_hook(_addr(userlib, "user_friction"), C.addressof(coeff))
    s.upload(q)
    s.update_rank_boundaries()
    if device_loop:
        s.advance()
        dts = s.step_log().dt
    else:
        dts = run_host_loop(s).dt
    o = Oracle(c)
    o.set_friction(3.5)
    o.set_state(q)
    o.update_rank_boundaries()
    lo = o.run()
    assert np.array_equal(dts, lo.dt)
    a, b = s.download(), o.state()
    s.close()
    o.close()
    assert np.array_equal(a, b)
    # the source acted: momentum differs from the frictionless run
    s = Solver(c)
    s.upload(q)
    s.update_rank_boundaries()
    s.advance()
    assert not np.array_equal(s.download(), a)
    s.close()
