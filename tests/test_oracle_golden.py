"""The CPU oracle against the golden fixtures (tests/golden) and hand-derived known answers.

The fixtures come from tests/golden/make_golden.py: control.in written by the reference's own
input generator, and a separate Python transliteration of the reference loops calling LAPACK
dgeev / BLAS dgemv.  In eigen_mode 1 the oracle makes the same library calls and must agree
bit for bit; in the closed-form mode (the FP64 parity definition of the CUDA path) the wave
speeds differ from dgeev's by a few ulps and everything else follows.
"""
import dataclasses
import json
import math
from pathlib import Path

import numpy as np
import pytest

from paraclaws_b200 import control as ctl
from paraclaws_b200 import ic

GOLD = Path(__file__).resolve().parent / "golden"
G = ctl.GRAV_REFERENCE


def _hex(v):
    return [float.fromhex(x) for x in v]


# --------------------------------------------------------------------------------------------
# control.in
# --------------------------------------------------------------------------------------------
@pytest.mark.parametrize("tag", ["default", "dam_break_example"])
def test_control_writer_matches_reference_generator(tmp_path, tag):
    meta = json.loads((GOLD / f"control_{tag}.json").read_text())
    assert meta["field_order"] == ctl.ControlSettings.FIELD_ORDER
    c = ctl.ControlSettings(**meta["defaults"])
    out = tmp_path / "control.in"
    ctl.write_control(out, c)
    assert out.read_bytes() == (GOLD / f"control_{tag}.in").read_bytes()
    if tag == "default":
        assert dataclasses.asdict(ctl.ControlSettings()) == meta["defaults"]


@pytest.mark.parametrize("tag", ["default", "dam_break_example"])
def test_control_reader_python_and_c(tag):
    import ctypes as C

    from paraclaws_b200 import _lib
    meta = json.loads((GOLD / f"control_{tag}.json").read_text())
    c = ctl.read_control(GOLD / f"control_{tag}.in")
    for k, v in meta["defaults"].items():
        assert getattr(c, k) == v, k
    L = _lib.load()
    sc = _lib.SolverControl()
    assert L.pcl_read_solver_control(str(GOLD / f"control_{tag}.in").encode(), None, C.byref(sc)) == 0
    d = meta["defaults"]
    assert (sc.m_xi, sc.m_eta, sc.limiter_method) == (d["m_xi"], d["m_eta"], d["limiter_function"])
    assert sc.cfl_limit == d["CFL_limit"] and sc.dt_max == d["max_allowed_dt"] and sc.dt_initial == d["initial_timestep"]
    assert sc.adaptive_timestepping == int(d["adaptive_timestepping"])
    assert sc.higher_order_flux_correction == int(d["add_higher_order_flux_correction"])
    assert (sc.bc_xi_lower, sc.bc_eta_upper) == (d["bc_xi_lower"], d["bc_eta_upper"])
    assert sc.grav == G


def test_fortran_list_directed_values(tmp_path):
    p = tmp_path / "control.in"
    vals = ctl.ControlSettings().values()
    lines = [str(v) for v in vals]
    lines[9] = "T"              # logical without periods
    lines[15] = ".TRUE. extra"  # trailing text after the value
    lines[8] = "1.0d-10"        # Fortran d exponent
    lines[20] = "-1, 2"         # comma separator: first value only
    p.write_text("\n".join(lines) + "\n")
    c = ctl.read_control(p)
    assert c.adaptive_timestepping is True and c.add_higher_order_flux_correction is True
    assert c.initial_timestep == 1e-10 and c.xi_min == -1.0


def test_custom_roundtrip(tmp_path):
    cu = ctl.CustomSettings(max_accepted_steps=500, precision_mode=1, dam_radius=0.3)
    ctl.write_custom(tmp_path / "custom.in", cu)
    assert ctl.read_custom(tmp_path / "custom.in") == cu


# --------------------------------------------------------------------------------------------
# single-interface HLL
# --------------------------------------------------------------------------------------------
def _kats():
    return json.loads((GOLD / "hll_kat.json").read_text())


def test_hll_dgeev_mode_matches_golden(oracle_lib):
    if not oracle_lib.load_lapack():
        pytest.skip("no LAPACK")
    for row in _kats():
        st, lam, W = oracle_lib.hll_interface(row["ixy"], _hex(row["qL"]), _hex(row["qR"]), G, eigen_mode=1)
        assert st == 0
        assert list(lam) == _hex(row["lambda"])
        assert list(W[0]) == _hex(row["W1"]) and list(W[1]) == _hex(row["W2"])


def test_hll_closed_form_within_ulps_of_dgeev(oracle_lib):
    """Closed-form |u|+sqrt(g h) vs LAPACK dgeev: wave speeds agree to a few ulps."""
    differ = 0
    for row in _kats():
        st, lam, W = oracle_lib.hll_interface(row["ixy"], _hex(row["qL"]), _hex(row["qR"]), G, eigen_mode=0)
        ref = _hex(row["lambda"])
        assert st == 0
        ulp = math.ulp(abs(ref[1]))
        assert abs(lam[1] - ref[1]) <= 4 * ulp
        differ += lam[1] != ref[1]
        w = np.concatenate([W[0], W[1]])
        wr = np.array(_hex(row["W1"]) + _hex(row["W2"]))
        assert np.allclose(w, wr, rtol=1e-9, atol=1e-12)
    assert differ < len(_kats())  # most interfaces agree exactly


def test_hll_equal_states_eps_quirk(oracle_lib):
    """Equal states give W2 = -W1 = q*eps/(2 s2 - eps) != 0 because of the eps in the HLL
    denominator (SMOD_approximate_Riemann_solvers.f90:214)."""
    q = [1.0, 0.0, 0.0]
    st, lam, W = oracle_lib.hll_interface(1, q, q, G, eigen_mode=0)
    s2 = math.sqrt(G)
    assert lam[1] == s2 and lam[0] == -s2
    qs = ((0.0 - s2 * 1.0) + (-s2) * 1.0) / ((1e-10 + -s2) - s2)
    assert W[0][0] == qs - 1.0 and W[1][0] == 1.0 - qs
    # q* - 1 cancels down to ~1e-11, so only ~5 significant digits survive
    assert W[0][0] > 0 and abs(W[0][0] / (1e-10 / (2 * s2)) - 1) < 1e-4


def test_flux_is_jacobian_times_state(oracle_lib):
    """The HLL 'flux' is J(q).q: the momentum flux is hu^2/h + g h^2 (pressure term doubled)."""
    qL = [2.0, 0.0, 0.0]
    qR = [1.0, 0.0, 0.0]
    st, lam, W = oracle_lib.hll_interface(1, qL, qR, G, eigen_mode=0)
    s2 = lam[1]
    # momentum component of q*: (fR - fL - s2*0 + s1*0)/den with fR - fL = g*(1 - 4)
    den = (1e-10 + -s2) - s2
    assert W[1][1] == 0.0 - (G * 1.0 * 1.0 - G * 2.0 * 2.0) / den


# --------------------------------------------------------------------------------------------
# limiter functions (by code; the reference's comments swap 2 and 3)
# --------------------------------------------------------------------------------------------
@pytest.mark.parametrize("method,r,expect", [
    (1, -1.0, 0.0), (1, 0.5, 0.5), (1, 2.0, 1.0),
    (2, -0.5, 0.0), (2, 0.25, 0.5), (2, 0.75, 1.0), (2, 1.5, 1.5), (2, 3.0, 2.0),
    (3, -2.0, 0.0), (3, 1.0, 1.0), (3, 3.0, 1.5),
    (4, -1.0, 0.0), (4, 0.2, 0.4), (4, 1.0, 1.0), (4, 2.0, 1.5), (4, 5.0, 2.0),
])
def test_limiter_phi(oracle_lib, method, r, expect):
    assert oracle_lib.limiter_phi(method, r) == expect


# --------------------------------------------------------------------------------------------
# time control (time_control/MOD_time_control.f90:153-243)
# --------------------------------------------------------------------------------------------
def _tc(adaptive=True, **over):
    c = dataclasses.replace(ctl.dam_break_control(8, time_final=1.0), adaptive_timestepping=adaptive,
                            number_of_snapshots=10, **over)
    from oracle.oracle import Oracle
    return Oracle(c)


@pytest.mark.parametrize("cfl,dt,expect", [
    (0.45, 1e-3, 1e-3 * 1.2),            # growth clamp: 0.9/0.45 = 2 >= 1.2
    (0.9005, 1e-3, 1e-3),                 # 1 % dead band
    (1.5, 1e-3, 1e-3 * (0.9 / 1.5)),      # shrink, no lower clamp on the factor
    (0.0, 1e-3, 1e-3),                    # CFL = 0: factor 1
    (0.01, 9e-3, 1e-2),                   # dt_max clamp
])
def test_update_time_accepted(oracle_lib, cfl, dt, expect):
    o = _tc()
    o.set_time_state(0.0, dt, cfl, 1)
    assert o.update_time(True) == 0
    t = o.time_state()
    assert t["dt"] == expect and t["time"] == 0.0 + expect and t["dt_previous"] == dt


def test_update_time_snapshot_alignment(oracle_lib):
    o = _tc()
    o.set_time_state(0.099, 5e-3, 0.9, 1)   # next snapshot at 0.1
    o.update_time(True)
    t = o.time_state()
    assert t["dt"] == 0.1 - 0.099 and t["time"] == 0.099 + (0.1 - 0.099) and t["snapshot_exception"] == 1


def test_update_time_rejected_and_fatal(oracle_lib):
    o = _tc()
    o.set_time_state(0.3, 4e-3, 2.5, 1)
    assert o.update_time(False) == 0
    t = o.time_state()
    assert t["dt"] == 0.25 * 4e-3 and t["time"] == 0.3
    o.set_time_state(0.3, 1e-10, 2.5, 1)
    o.update_time(False)
    assert o.time_state()["dt"] == 1e-10  # dt_min clamp
    f = _tc(adaptive=False)
    f.set_time_state(0.0, 1e-3, 2.5, 1)
    assert f.update_time(False) == oracle_lib.ORC_ERR_FATAL_DT


def test_snapshot_times():
    o = _tc()
    t = o.time_state()
    assert t["next_snapshot"] == 0.0 + 1 * (1.0 / 10)


# --------------------------------------------------------------------------------------------
# whole runs against the transliteration
# --------------------------------------------------------------------------------------------
CASES = ["mc_bc2", "minmod_bc3", "superbee_bc2", "vanleer_bc3", "reject_mc_bc2"]
SETTINGS = {"mc_bc2": (8, 6, 4, 2, 1e-3), "minmod_bc3": (7, 9, 1, 3, 1e-3), "superbee_bc2": (6, 6, 2, 2, 1e-3),
            "vanleer_bc3": (9, 5, 3, 3, 1e-3), "reject_mc_bc2": (8, 8, 4, 2, 0.2)}


def _tiny(name, eigen_mode):
    from oracle.oracle import Oracle
    mx, my, lim, bc, dt0 = SETTINGS[name]
    c = dataclasses.replace(ctl.dam_break_control(mx, limiter=lim, bc=bc), m_eta=my, initial_timestep=dt0)
    o = Oracle(c, eigen_mode=eigen_mode)
    gold = np.load(GOLD / "tiny_runs.npz")
    o.set_state(gold[f"{name}_ic"])
    o.update_rank_boundaries()
    log = o.run(max_attempts=len(gold[f"{name}_dt"]))
    return o, log, gold


@pytest.mark.parametrize("name", CASES)
def test_tiny_run_dgeev_mode_bit_exact(oracle_lib, name):
    if not oracle_lib.load_lapack():
        pytest.skip("no LAPACK")
    o, log, gold = _tiny(name, 1)
    assert np.array_equal(log.dt, gold[f"{name}_dt"])
    assert np.array_equal(log.ierr, gold[f"{name}_ierr"])
    assert np.array_equal(o.state(), gold[f"{name}_state"])


@pytest.mark.parametrize("name", CASES)
def test_tiny_run_closed_form_close(oracle_lib, name):
    o, log, gold = _tiny(name, 0)
    assert np.array_equal(log.ierr, gold[f"{name}_ierr"])
    assert np.allclose(log.dt, gold[f"{name}_dt"], rtol=1e-12, atol=0)
    assert np.allclose(o.state(), gold[f"{name}_state"], rtol=1e-11, atol=1e-13)


def test_lake_at_rest_drift(oracle_lib):
    """h = 1, u = v = 0: the eps of the HLL denominator lifts h by (dt/dxi + dt/deta)*eps per
    step, exactly as the reference does; a textbook HLL would keep h = 1."""
    from oracle.oracle import Oracle
    m = 16
    c = dataclasses.replace(ctl.dam_break_control(m, limiter=1), initial_timestep=1e-3)
    o = Oracle(c)
    o.set_state(ic.lake_at_rest(m, m))
    o.update_rank_boundaries()
    st, ierr = o.solve_dimensional_split()
    assert ierr == 1
    q = o.state()[2:-2, 2:-2]
    d = 2.0 / m
    expect = (1e-3 / d + 1e-3 / d) * 1e-10
    assert np.all(q[..., 1] == 0.0)
    # The eta sweep reads the pre-step ghost rows (h = 1) next to the x-swept interior
    # (h = 1 + dt/dxi*eps): ghosts are filled once per accepted step (main.f90:246), so the
    # rows beside the top and bottom walls pick up a tiny, antisymmetric hv.
    hv = q[..., 2]
    assert np.all(hv[2:-2] == 0.0)
    assert np.all(hv[0] < 0.0) and np.all(hv[-1] > 0.0) and np.all(np.abs(hv) < 1e-12)
    rel = (q[2:-2, :, 0] - 1.0) / expect
    assert np.all(np.abs(rel - 1.0) < 1e-3)


def test_dgeev_vs_closed_form_dam_break(oracle_lib):
    """The two eigen modes on the 64^2 dam break: same accept/reject sequence, dt within
    1e-13 relative, states within 1e-10 (the gap the reference's LAPACK choice leaves)."""
    if not oracle_lib.load_lapack():
        pytest.skip("no LAPACK")
    from oracle.oracle import Oracle
    c = ctl.dam_break_control(64, limiter=4, time_final=0.1)
    q = ic.circular_dam(64, 64)
    res = []
    for mode in (0, 1):
        o = Oracle(c, eigen_mode=mode)
        o.set_state(q)
        o.update_rank_boundaries()
        res.append((o.run(), o.state()))
    (l0, s0), (l1, s1) = res
    assert np.array_equal(l0.ierr, l1.ierr)
    assert np.allclose(l0.dt, l1.dt, rtol=1e-13, atol=0)
    assert np.allclose(s0, s1, rtol=1e-10, atol=1e-12)


def test_error_status(oracle_lib):
    from oracle.oracle import Oracle
    c = ctl.dam_break_control(16)
    for val, code in ((np.nan, oracle_lib.ORC_ERR_NAN), (-0.5, oracle_lib.ORC_ERR_NEG_DEPTH)):
        o = Oracle(c)
        q = ic.circular_dam(16, 16)
        q[8, 8, 0] = val
        o.set_state(q)
        o.update_rank_boundaries()
        st, _ = o.solve_dimensional_split()
        assert st == code


# --------------------------------------------------------------------------------------------
# mesh metrics and initial conditions
# --------------------------------------------------------------------------------------------
def test_mesh_metrics_uniform(oracle_lib):
    from oracle.oracle import Oracle
    o = Oracle(ctl.dam_break_control(200))
    m = o.mesh()
    assert np.all(np.abs(m["kappa"] - 1.0) < 1e-12)
    assert len(np.unique(m["kappa"])) > 1       # capacity is 1 only up to rounding
    assert np.all(m["lr_xi"] == m["lr_xi"][:, :1])   # length ratio along xi depends on j only
    assert np.all(m["lr_eta"] == m["lr_eta"][:1, :])


def test_circular_dam_ic_matches_reference_expression():
    q = ic.circular_dam(200, 200)
    x, y = ic.cell_centres(200, 200)
    inside = 0
    for j in range(len(y)):
        for i in range(len(x)):
            r = math.sqrt(x[i] * x[i] + y[j] * y[j])
            assert q[j, i, 0] == (2.0 if r < 0.5 else 1.0)
            inside += r < 0.5
    assert inside == int((q[..., 0] == 2.0).sum()) > 0
    assert np.all(q[..., 1:] == 0.0)


def test_seeded_generators_are_deterministic():
    a = ic.gaussian_bumps(64, 64, seed=0)
    b = ic.gaussian_bumps(64, 64, seed=0)
    assert np.array_equal(a, b) and not np.array_equal(a, ic.gaussian_bumps(64, 64, seed=1))
    assert 1.0 <= a[..., 0].min() and a[..., 0].max() < 1.0 + 16 * 1.0
    p = ic.seeded_dam_params(5, offset=0.25)
    assert 0.2 <= p.radius <= 0.6 and 1.5 <= p.h_in <= 5.0 and abs(p.x0) <= 0.25
    sides = ic.log_uniform_sides(512, 64, 1024, 32, seed=2)
    assert all(s % 32 == 0 and 64 <= s <= 1024 for s in sides)
