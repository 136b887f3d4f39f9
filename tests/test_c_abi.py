"""The C ABI without a GPU: the library loads, exports every function include/paraclaws_b200.h
declares, its structs have the layout the ctypes binding assumes, and the host-only entry
points (defaults, control.in reader, status strings) work."""
import ctypes as C
import subprocess
from pathlib import Path

import pytest

from paraclaws_b200 import _lib
from paraclaws_b200 import control as ctl

ROOT = Path(__file__).resolve().parent.parent


def test_exports_every_declared_function(pcl):
    names = _lib.declared_functions()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.lib_path())], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    for n in names:
        assert hasattr(pcl, n)


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "paraclaws_b200.h"\n'
        "int main(void){printf(\"%zu %zu %zu %zu %zu\\n\", sizeof(pcl_solver_control), "
        "offsetof(pcl_solver_control, t_start), offsetof(pcl_solver_control, max_accepted_steps), "
        "sizeof(pcl_run_stats), sizeof(pcl_step_record)); return 0;}\n")
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert got == [C.sizeof(_lib.SolverControl), _lib.SolverControl.t_start.offset,
                   _lib.SolverControl.max_accepted_steps.offset, C.sizeof(_lib.RunStats), C.sizeof(_lib.StepRecord)]


def test_default_control_matches_reference_defaults(pcl):
    sc = _lib.SolverControl()
    pcl.pcl_default_control(C.byref(sc))
    d = ctl.ControlSettings()
    assert (sc.num_equations, sc.num_ghost, sc.num_aux, sc.num_waves) == (3, 2, 10, 2)
    assert sc.t_final == d.time_final and sc.number_of_snapshots == d.number_of_snapshots
    assert sc.dt_initial == d.initial_timestep and sc.cfl_limit == d.CFL_limit
    assert sc.dt_max == d.max_allowed_dt and sc.dt_min == d.min_allowed_dt
    assert sc.dt_max_growth_ratio == d.dt_max_growth_ratio and sc.dt_min_shrink_ratio == d.dt_min_shrink_ratio
    assert sc.m_xi == d.m_xi and sc.limiter_method == d.limiter_function
    assert sc.grav == ctl.GRAV_REFERENCE == float(__import__("numpy").float32(9.81))


def test_read_control_with_custom(pcl, tmp_path):
    c = ctl.dam_break_control(4096, limiter=1)
    cu = ctl.CustomSettings(max_accepted_steps=500, precision_mode=1, dam_radius=0.3, dam_x0=0.1)
    ctl.write_control(tmp_path / "control.in", c)
    ctl.write_custom(tmp_path / "custom.in", cu)
    sc = _lib.SolverControl()
    r = pcl.pcl_read_solver_control(str(tmp_path / "control.in").encode(), str(tmp_path / "custom.in").encode(),
                                    C.byref(sc))
    assert r == 0
    assert (sc.m_xi, sc.limiter_method, sc.higher_order_flux_correction, sc.cfl_limit) == (4096, 1, 1, 0.9)
    assert (sc.max_accepted_steps, sc.precision_mode, sc.dam_radius, sc.dam_x0) == (500, 1, 0.3, 0.1)
    assert pcl.pcl_read_solver_control(str(tmp_path / "missing.in").encode(), None, C.byref(sc)) == _lib.PCL_ERR_IO


def test_status_strings(pcl):
    for code in range(0, -10, -1):
        s = pcl.pcl_status_string(code).decode()
        assert s and s != "unknown status"
    assert pcl.pcl_status_string(-99).decode() == "unknown status"


def test_fortran_e26_16_field(pcl):
    """The snapshot format's E26.16 field (utility/MOD_IO.f90:441, format(50e26.16)):
    right-justified 0.<16 digits>E+ee, the exponent letter dropped beyond two digits."""
    from paraclaws_b200.solver import format_e26_16
    cases = {
        2.0: "   0.2000000000000000E+01",
        1.0: "   0.1000000000000000E+01",
        0.0: "   0.0000000000000000E+00",
        -1.5e-5: "  -0.1500000000000000E-04",
        9.8100004196166992: "   0.9810000419616699E+01",
        0.1: "   0.1000000000000000E+00",
        123456.789: "   0.1234567890000000E+06",
        1e-100: "   0.1000000000000000E-99",     # 0.1 x 10^-99: still two digits
        1e-101: "   0.1000000000000000-100",
        -2.5e120: "  -0.2500000000000000+121",
        0.9999999999999999: "   0.9999999999999999E+00",
        0.3: "   0.3000000000000000E+00",    # 0.29999999999999998889...: rounds up at 16 digits
    }
    for v, want in cases.items():
        got = format_e26_16(v)
        assert len(got) == 26 and got == " " + want, (v, got, want)
