"""Equation modules on the FP64 path: the generic sweeps run the reference's step for a module's
N x N Jacobian (flux J(q).q in dgemv order, HLL on the largest |eigenvalue|), with the state
sized by control.in's num_equations.  The dam-break module through the generic path (N = 3)
equals the specialised kernels bit for bit; linear acoustics (N = 3), advection and Burgers
(N = 1) and shallow water with a tracer (N = 4) equal the oracle running its own restatement of
the same module bit for bit, over limiters and boundary codes."""
import dataclasses

import numpy as np
import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic, mesh
from paraclaws_b200.solver import Solver, run_host_loop

pytestmark = pytest.mark.gpu


def pulse(mx, my, w=0.15):
    x, y = np.meshgrid(*ic.cell_centres(mx, my))
    q = np.zeros((my + 4, mx + 4, 3))
    q[..., 0] = np.exp(-((x - 0.1) ** 2 + (y + 0.05) ** 2) / (w * w))
    return q


@pytest.mark.parametrize("device_loop", [False, True])
def test_generic_shallow_water_equals_specialised(pcl, device_loop):
    c = dataclasses.replace(ctl.dam_break_control(70, limiter=4, bc=2, time_final=0.08), m_eta=54)
    q = ic.gaussian_bumps(70, 54, seed=2)
    out = []
    for module in (ctl.EQ_SHALLOW_WATER, ctl.EQ_SHALLOW_WATER_GENERIC):
        s = Solver(c)
        s.set_equation(module)
        s.upload(q)
        s.update_rank_boundaries()
        if device_loop:
            s.advance()
            dt = s.step_log().dt
        else:
            dt = run_host_loop(s).dt
        out.append((s.download(), dt))
        s.close()
    assert len(out[0][1]) > 10 and np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][0], out[1][0])


@pytest.mark.parametrize("lim,bc", [(1, 2), (4, 1), (2, 3), (3, 2)])
def test_acoustics_matches_oracle(pcl, oracle_lib, lim, bc):
    from oracle.oracle import Oracle
    c = dataclasses.replace(ctl.dam_break_control(48, limiter=lim, bc=bc, time_final=0.3), m_eta=40)
    q = pulse(48, 40)
    s = Solver(c)
    s.set_equation(ctl.EQ_ACOUSTICS, (2.0, 0.5))
    s.upload(q)
    s.update_rank_boundaries()
    st = s.advance()
    o = Oracle(c)
    o.set_equation(ctl.EQ_ACOUSTICS, 2.0, 0.5)
    o.set_state(q)
    o.update_rank_boundaries()
    lo = o.run()
    assert st.status == 0 and lo.status == 0 and st.accepted > 10
    assert np.array_equal(s.step_log().dt, lo.dt)
    a, b = s.download(), o.state()
    s.close()
    o.close()
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ"
    assert np.abs(a[2:-2, 2:-2, 1]).max() > 1e-3  # the pulse radiated


def test_equation_module_rejections(pcl):
    c = ctl.dam_break_control(16)
    s = Solver(c, precision=ctl.PRECISION_MIXED)
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0, 1.0))
    s.close()
    s = Solver(c)
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0,))        # needs K and rho
    with pytest.raises(_lib.PclError):
        s.set_equation(7)
    s.set_mesh_metrics(*mesh.metrics(c, mesh.stretch(2.0, 2.0)))
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0, 1.0))    # mapped grids take the shallow-water module
    s.close()


def _n_control(mx, my, n, **kw):
    return dataclasses.replace(ctl.dam_break_control(mx, **kw), m_eta=my, number_of_equations=n)


def _n_state(mx, my, n, module):
    x, y = np.meshgrid(*ic.cell_centres(mx, my))
    q = np.zeros((my + 4, mx + 4, n))
    if module == ctl.EQ_SHALLOW_WATER_TRACER:
        q[..., :3] = ic.gaussian_bumps(mx, my, seed=4)
        q[..., 1] = 0.2 * np.sin(3 * y)
        q[..., 3] = np.where(x > 0.1, 0.5, 0.1) * q[..., 0]  # a tracer front
    else:
        q[..., 0] = (0.3 if module == ctl.EQ_BURGERS else 0.0) + np.exp(-((x - 0.1) ** 2 + (y + 0.05) ** 2) / 0.04)
        if module == ctl.EQ_BURGERS:
            q[..., 0] -= 0.6 * np.exp(-((x + 0.3) ** 2 + (y - 0.2) ** 2) / 0.02)  # both signs of the speed
    return q


N_CASES = [
    (ctl.EQ_ADVECTION, 1, (1.0, -0.6), 1, 2), (ctl.EQ_ADVECTION, 1, (-0.4, 0.8), 4, 3),
    (ctl.EQ_ADVECTION, 1, (0.7, 0.7), 0, 1), (ctl.EQ_BURGERS, 1, (), 2, 2), (ctl.EQ_BURGERS, 1, (), 3, 1),
    (ctl.EQ_SHALLOW_WATER_TRACER, 4, (ctl.GRAV_REFERENCE,), 1, 1),
    (ctl.EQ_SHALLOW_WATER_TRACER, 4, (ctl.GRAV_REFERENCE,), 4, 2),
    (ctl.EQ_SHALLOW_WATER_TRACER, 4, (2.5,), 3, 3),
]


@pytest.mark.parametrize("module,n,prm,lim,bc", N_CASES)
@pytest.mark.parametrize("device_loop", [False, True])
def test_n_equation_modules_match_oracle(pcl, oracle_lib, module, n, prm, lim, bc, device_loop):
    """num_equations = 1 and 4 through the generic path, bit-exact against the oracle (state,
    dt sequence, accept/reject flags).  lim = 0: unlimited second-order correction."""
    from oracle.oracle import Oracle
    over = dict(use_limtiter=False) if lim == 0 else {}
    c = dataclasses.replace(_n_control(45, 37, n, limiter=max(lim, 1), bc=bc, time_final=0.12), **over)
    q = _n_state(45, 37, n, module)
    s = Solver(c)
    s.set_equation(module, prm)
    s.upload(q)
    s.update_rank_boundaries()
    if device_loop:
        st = s.advance()
        lg = s.step_log()
    else:
        lg = run_host_loop(s)
        st = s.stats()
    o = Oracle(c)
    o.set_equation(module, *(list(prm) + [0.0, 0.0])[:2])
    o.set_state(q)
    o.update_rank_boundaries()
    lo = o.run()
    assert st.status == 0 and lo.status == 0 and lo.accepted > 5
    assert np.array_equal(lg.dt, lo.dt) and np.array_equal(lg.ierr, lo.ierr)
    a, b = s.download(), o.state()
    s.close()
    o.close()
    assert a.shape == (41, 49, n)
    assert np.array_equal(a, b), f"{np.count_nonzero(a != b)} values differ"
    assert not np.array_equal(a, q)


@pytest.mark.parametrize("bc", [1, 2])
def test_shallow_water_as_n3_generic_equals_specialised_mixed_grid(pcl, bc):
    """N = 3 through the generic sweeps (the dam-break Jacobian as a module) equals the
    specialised kernels on a grid whose capacities are not all 1 (the table-metric build)."""
    c = dataclasses.replace(ctl.dam_break_control(61, limiter=1, bc=bc, time_final=0.05), m_eta=47)
    q = ic.gaussian_bumps(61, 47, seed=9)
    out = []
    for module in (ctl.EQ_SHALLOW_WATER, ctl.EQ_SHALLOW_WATER_GENERIC):
        s = Solver(c)
        s.set_equation(module)
        s.upload(q)
        s.update_rank_boundaries()
        s.advance()
        out.append((s.download(), s.step_log().dt))
        s.close()
    assert np.array_equal(out[0][1], out[1][1]) and np.array_equal(out[0][0], out[1][0])


def test_num_waves_above_two_run_the_two_wave_step(pcl):
    """HLL makes two waves; the reference's further waves stay zero, so num_waves = 3 gives the
    two-wave results, and num_waves = 1 is refused."""
    base = ctl.dam_break_control(40, limiter=4, bc=1, time_final=0.05)
    q = ic.circular_dam(40, 40)
    out = []
    for nw in (2, 3):
        s = Solver(dataclasses.replace(base, number_of_waves=nw))
        s.upload(q)
        s.update_rank_boundaries()
        s.advance()
        out.append(s.download())
        s.close()
    assert np.array_equal(out[0], out[1])
    with pytest.raises(_lib.PclError):
        Solver(dataclasses.replace(base, number_of_waves=1))


def test_n_equation_context_rules(pcl):
    c1 = _n_control(16, 16, 1, time_final=0.01)
    s = Solver(c1)
    with pytest.raises(_lib.PclError):
        s.advance()                                     # no module for one equation yet
    with pytest.raises(_lib.PclError):
        s.set_equation(ctl.EQ_ACOUSTICS, (1.0, 1.0))    # a three-equation module
    with pytest.raises(_lib.PclError):
        s.initial_condition()                           # the dam break needs h, hu, hv
    s.set_equation(ctl.EQ_ADVECTION, (1.0, 0.0))
    q = np.zeros((20, 20, 1))
    q[..., 0] = 1.0
    s.upload(q)
    s.update_rank_boundaries()
    st = s.advance()
    assert st.status == 0 and s.download().shape == (20, 20, 1)
    s.close()
    with pytest.raises(_lib.PclError):
        Solver(_n_control(16, 16, 4), precision=ctl.PRECISION_MIXED)   # mixed: three equations
    with pytest.raises(_lib.PclError):
        Solver(_n_control(16, 16, 5))                                  # no module has five


@pytest.mark.parametrize("module,n,prm", [(ctl.EQ_ADVECTION, 1, (1.0, -0.6)), (ctl.EQ_BURGERS, 1, ()),
                                          (ctl.EQ_ACOUSTICS, 3, (2.0, 0.5)),
                                          (ctl.EQ_SHALLOW_WATER_TRACER, 4, (ctl.GRAV_REFERENCE,))])
def test_generic_eta_shapes_agree(pcl, module, n, prm):
    """The generic path's eta sweep in bands (the default) and in column windows
    (pcl_set_sweep_shape) gives the same bits, on a grid whose sizes are multiples of neither the
    band width nor the chunk height nor the window width."""
    from paraclaws_b200 import _lib
    outs = []
    for shape in (_lib.PCL_SHAPE_BAND, _lib.PCL_SHAPE_WINDOW):
        c = _n_control(133, 271, n, limiter=1, bc=1, time_final=0.05)
        s = Solver(c)
        s.set_equation(module, prm)
        s.set_sweep_shape(shape)
        assert s.sweep_shape() == shape
        s.upload(_n_state(133, 271, n, module))
        s.update_rank_boundaries()
        st = s.advance()
        assert st.status == 0 and st.accepted > 5
        outs.append((s.download(), s.step_log().dt))
        s.close()
    assert np.array_equal(outs[0][1], outs[1][1])
    assert np.array_equal(outs[0][0].view(np.int64), outs[1][0].view(np.int64))
