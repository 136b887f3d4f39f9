"""The Fortran side of the drop-in boundary (paraclaws_b200/fortran/*.f90) stays in step with the C
ABI it binds (include/paraclaws_b200.h).  No Fortran compiler exists in this image, so this
checks the sources as text:
  * every bind(C) interface names a declared function, with the same number of arguments and a
    matching kind for each (by value / by reference, int / long long / double / char / struct);
  * the bind(C) derived types list the C structs' fields in the same order with the same kinds;
  * the overrides call only interfaces the module declares, and keep the dummy-argument lists of
    the reference procedures they replace (solver/MOD_solve.f90:23,295,338;
    domain/MOD_domain.f90:192 for update_rank_boundaries).
"""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "paraclaws_b200.h"
FDIR = ROOT / "paraclaws_b200" / "fortran"


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    protos = {}
    for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_ \*]*?)\b(pcl_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        if ret.startswith("typedef"):
            continue
        params = [] if args in ("", "void") else [" ".join(a.split()) for a in args.split(",")]
        protos[name] = (ret, params)
    return protos


def c_kind(param: str) -> str:
    """A C parameter's kind in the terms the Fortran side can express."""
    p = param.replace("const ", "")
    stars = p.count("*")
    base = p.replace("*", " ").split()[0] if p.split() else ""
    if base == "unsigned" and stars == 0:
        return "int"
    if stars == 0:
        return {"int": "int", "double": "double", "long": "long long"}.get(base, base)
    if stars == 2:
        return "ptr&"
    if base in ("int", "double", "char", "pcl_solver_control", "pcl_run_stats"):
        return base + "&"
    return "ptr"   # an opaque handle or any other pointer, passed as type(c_ptr), value


def f_interfaces(path: Path):
    text = path.read_text()
    out = {}
    for m in re.finditer(r"^\s*([a-z]+\([a-z_]+\))\s+function\s+(pcl_[a-z0-9_]+)\s*\(([^)]*)\)\s*bind\(C\)(.*?)end function",
                         text, flags=re.S | re.M | re.I):
        ret, name, args, body = m.group(1), m.group(2), m.group(3), m.group(4)
        names = [a.strip() for a in args.split(",") if a.strip()]
        decls = {}
        for line in body.splitlines():
            line = line.strip()
            if "::" not in line or line.startswith("import"):
                continue
            lhs, rhs = line.split("::")
            for v in rhs.split(","):
                decls[v.strip()] = lhs.replace(" ", "").lower()
        out[name] = (ret.lower(), [(a, decls.get(a)) for a in names])
    return out


def f_kind(decl: str) -> str:
    by_value = ",value" in decl
    if decl.startswith("type(c_ptr)"):
        return "ptr" if by_value else "ptr&"
    if decl.startswith("integer(c_int)"):
        return "int" if by_value else "int&"
    if decl.startswith("integer(c_long_long)"):
        return "long long" if by_value else "long long&"
    if decl.startswith("real(c_double)"):
        return "double" if by_value else "double&"
    if decl.startswith("character(kind=c_char)"):
        return "char&"
    m = re.match(r"type\((pcl_[a-z_]+)\)", decl)
    if m:
        return m.group(1) + "&"
    raise AssertionError(f"unknown Fortran declaration {decl}")


def test_every_interface_matches_the_header():
    protos = c_prototypes()
    ifaces = f_interfaces(FDIR / "MOD_paraclaws_b200.f90")
    assert len(ifaces) >= 30
    ret_map = {"integer(c_int)": "int", "integer(c_long_long)": "long long", "type(c_ptr)": "ptr"}
    for name, (ret, args) in ifaces.items():
        assert name in protos, f"{name} is not declared in {HEADER.name}"
        cret, cparams = protos[name]
        cret_k = "ptr" if "*" in cret else ("long long" if "long long" in cret else cret.split()[-1])
        assert ret_map[ret] == cret_k, f"{name}: returns {ret}, C returns {cret}"
        assert len(args) == len(cparams), f"{name}: {len(args)} arguments, C has {len(cparams)}"
        for (arg, decl), cp in zip(args, cparams):
            assert decl is not None, f"{name}: argument {arg} is not declared"
            assert f_kind(decl) == c_kind(cp), f"{name}({arg}): Fortran {decl} vs C {cp}"


def _c_struct_fields(name):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (name, name), text, flags=re.S).group(1)
    fields = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        m = re.match(r"(long long|int|double)\s+(.*)", decl)
        kind = {"long long": "long long", "int": "int", "double": "double"}[m.group(1)]
        fields += [(v.strip(), kind) for v in m.group(2).split(",")]
    return fields


def _f_type_fields(name):
    text = (FDIR / "MOD_paraclaws_b200.f90").read_text()
    body = re.search(r"type, bind\(C\) :: %s\n(.*?)end type" % name, text, flags=re.S).group(1)
    kinds = {"integer(c_int)": "int", "integer(c_long_long)": "long long", "real(c_double)": "double"}
    fields = []
    for line in body.splitlines():
        if "::" in line:
            lhs, rhs = line.split("::")
            fields += [(v.strip(), kinds[lhs.strip()]) for v in rhs.split(",")]
    return fields


@pytest.mark.parametrize("name", ["pcl_solver_control", "pcl_run_stats"])
def test_bound_types_match_the_c_structs(name):
    assert _f_type_fields(name) == _c_struct_fields(name)


def _procedures(path):
    text = path.read_text()
    return {m.group(2): [a.strip() for a in m.group(3).split(",")]
            for m in re.finditer(r"^\s*(module\s+)?subroutine\s+([a-z_]+)\s*\(([^)]*)\)", text, flags=re.M)}


def test_overrides_keep_the_reference_interfaces_and_call_only_bound_functions():
    ifaces = f_interfaces(FDIR / "MOD_paraclaws_b200.f90")
    expected = {
        "MOD_solve.f90": {
            "solve_dimensional_split": ["decomposition", "t_ctrl", "work", "mesh", "solution", "ierr"],
            "integrate_source_term": ["decomposition", "t_ctrl", "mesh", "solution"],
            "execute_post": ["decomposition", "mesh", "solution"],
        },
        "SMOD_boundary_conditions.f90": {
            "update_rank_boundaries": ["decomposition", "mesh", "solution"],
        },
    }
    for fname, procs in expected.items():
        path = FDIR / fname
        got = _procedures(path)
        for proc, args in procs.items():
            assert got.get(proc) == args, f"{fname}: {proc}({got.get(proc)}) vs the reference's {args}"
        calls = set(re.findall(r"\b(pcl_[a-z0-9_]+)\s*\(", path.read_text()))
        calls.discard("pcl_check")
        assert calls, fname
        missing = sorted(c for c in calls if c not in ifaces)
        assert not missing, f"{fname} calls {missing}, which MOD_paraclaws_b200 does not bind"
    text = (FDIR / "MOD_solve.f90").read_text()
    assert re.search(r"^module MOD_solve\b", text, flags=re.M)
    text = (FDIR / "SMOD_boundary_conditions.f90").read_text()
    assert re.search(r"^submodule\(MOD_domain\) SMOD_boundary_conditions\b", text, flags=re.M)
