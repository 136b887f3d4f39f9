"""control.in / custom.in: the reference's run-time input files.

``ControlSettings`` mirrors the reference's ``control_settings.py:21-140`` (same fields, same
defaults, same positional ``FIELD_ORDER``) and ``write_control`` reproduces
``write_input.py:25-34`` byte for byte (one value per line, Python ``str`` formatting,
Fortran logicals as ``.true.``/``.false.``).  ``read_control`` restates the list-directed
reads of ``utility/MOD_IO.f90:55-94``: the first value of each record, in order, with Fortran
logical and ``d``-exponent syntax accepted.

``custom.in`` is written but never read by the reference (its ``FIELD_ORDER`` is empty,
``custom_settings.py:16-22``); this library uses it, positionally as well, for the settings the
reference has no slot for (``CustomSettings``).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable, List

# g as the reference sets it: the default-real literal 9.81 assigned to a double
# (examples/2D_dam_break/cartesian/SMOD_setup.f90:21) -> float32(9.81) widened.
GRAV_REFERENCE = 9.8100004196166992


@dataclass
class ControlSettings:
    """The 28 positional values of control.in (control_settings.py:21-140)."""

    number_of_equations: int = 3
    number_of_dimensions: int = 2
    number_of_ghost_cells: int = 2
    number_of_auxiliary_vars: int = 10
    number_of_waves: int = 2
    time_start: float = 0
    time_final: float = 0.5
    number_of_snapshots: int = 5
    initial_timestep: float = 1e-10
    adaptive_timestepping: bool = True
    CFL_limit: float = 0.1
    min_allowed_dt: float = 1e-10
    max_allowed_dt: float = 5e-5
    dt_max_growth_ratio: float = 1.2
    dt_min_shrink_ratio: float = 0.5
    add_higher_order_flux_correction: bool = False
    use_limtiter: bool = True  # sic: the reference's field name (control_settings.py:82)
    limiter_function: int = 1
    m_xi: int = 21
    m_eta: int = 21
    xi_min: float = -1
    xi_max: float = 1
    eta_min: float = -1
    eta_max: float = 1
    bc_xi_lower: int = 2
    bc_xi_upper: int = 2
    bc_eta_lower: int = 2
    bc_eta_upper: int = 2

    FIELD_ORDER = [
        "number_of_equations", "number_of_dimensions", "number_of_ghost_cells",
        "number_of_auxiliary_vars", "number_of_waves", "time_start", "time_final",
        "number_of_snapshots", "initial_timestep", "adaptive_timestepping", "CFL_limit",
        "min_allowed_dt", "max_allowed_dt", "dt_max_growth_ratio", "dt_min_shrink_ratio",
        "add_higher_order_flux_correction", "use_limtiter", "limiter_function", "m_xi", "m_eta",
        "xi_min", "xi_max", "eta_min", "eta_max", "bc_xi_lower", "bc_xi_upper", "bc_eta_lower",
        "bc_eta_upper",
    ]

    def values(self) -> list:
        return [getattr(self, f) for f in self.FIELD_ORDER]


# kinds of the control.in records as read_solver_control declares them (MOD_IO.f90:36-53)
_CONTROL_KINDS = {
    "number_of_equations": int, "number_of_dimensions": int, "number_of_ghost_cells": int,
    "number_of_auxiliary_vars": int, "number_of_waves": int, "time_start": float,
    "time_final": float, "number_of_snapshots": int, "initial_timestep": float,
    "adaptive_timestepping": bool, "CFL_limit": float, "min_allowed_dt": float,
    "max_allowed_dt": float, "dt_max_growth_ratio": float, "dt_min_shrink_ratio": float,
    "add_higher_order_flux_correction": bool, "use_limtiter": bool, "limiter_function": int,
    "m_xi": int, "m_eta": int, "xi_min": float, "xi_max": float, "eta_min": float,
    "eta_max": float, "bc_xi_lower": int, "bc_xi_upper": int, "bc_eta_lower": int,
    "bc_eta_upper": int,
}

# initial-condition kinds of custom.in
IC_FILE = 0          # raw float64 state in the reference layout, file initial_state.bin
IC_CIRCULAR_DAM = 1  # examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:34-46

# equation modules (include/paraclaws_b200.h PCL_EQ_*)
EQ_SHALLOW_WATER = 0
EQ_SHALLOW_WATER_GENERIC = 1
EQ_ACOUSTICS = 2
EQ_ADVECTION = 3              # one equation, params (a, b)
EQ_BURGERS = 4                # one equation, no params
EQ_SHALLOW_WATER_TRACER = 5   # four equations (h, hu, hv, hc), params (g)
EQ_NUM_EQUATIONS = {EQ_SHALLOW_WATER: 3, EQ_SHALLOW_WATER_GENERIC: 3, EQ_ACOUSTICS: 3, EQ_ADVECTION: 1,
                    EQ_BURGERS: 1, EQ_SHALLOW_WATER_TRACER: 4}

PRECISION_FP64 = 0
PRECISION_MIXED = 1


@dataclass
class CustomSettings:
    """custom.in as this library reads it (positional, one value per line, like control.in)."""

    max_accepted_steps: int = 0          # 0: run to time_final only
    precision_mode: int = PRECISION_FP64
    grav: float = GRAV_REFERENCE
    initial_condition: int = IC_CIRCULAR_DAM
    dam_radius: float = 0.5
    dam_h_in: float = 2.0
    dam_h_out: float = 1.0
    dam_x0: float = 0.0
    dam_y0: float = 0.0

    FIELD_ORDER = [
        "max_accepted_steps", "precision_mode", "grav", "initial_condition", "dam_radius",
        "dam_h_in", "dam_h_out", "dam_x0", "dam_y0",
    ]

    def values(self) -> list:
        return [getattr(self, f) for f in self.FIELD_ORDER]


_CUSTOM_KINDS = {
    "max_accepted_steps": int, "precision_mode": int, "grav": float, "initial_condition": int,
    "dam_radius": float, "dam_h_in": float, "dam_h_out": float, "dam_x0": float, "dam_y0": float,
}


def format_val(val):
    """write_input.py:25-28: Fortran logicals for bools, Python str for everything else."""
    if isinstance(val, bool):
        return ".true." if val else ".false."
    return val


def write_values(path: Path | str, values: Iterable) -> None:
    """write_input.py:31-34."""
    with Path(path).open("w", encoding="utf-8") as f:
        for val in values:
            f.write(f"{format_val(val)}\n")


def write_control(path: Path | str, control: ControlSettings) -> None:
    write_values(path, control.values())


def write_custom(path: Path | str, custom: CustomSettings) -> None:
    write_values(path, custom.values())


def _first_token(record: str) -> str:
    """First value of a list-directed record: separators are blanks and commas; '/' ends it."""
    rec = record.strip()
    for i, ch in enumerate(rec):
        if ch in " \t,/":
            return rec[:i]
    return rec


def parse_fortran_value(token: str, kind):
    """One list-directed item of the given kind."""
    t = token.strip()
    if not t:
        raise ValueError("empty record")
    if kind is bool:
        u = t.upper()
        if u.startswith("."):
            u = u[1:]
        if u.startswith("T"):
            return True
        if u.startswith("F"):
            return False
        raise ValueError(f"not a Fortran logical: {token!r}")
    if kind is int:
        return int(t)
    return float(t.replace("d", "e").replace("D", "e"))


def _read_positional(path: Path | str, kinds: dict, order: List[str]) -> dict:
    records = Path(path).read_text(encoding="utf-8").splitlines()
    records = [r for r in records if r.strip() != ""]
    if len(records) < len(order):
        raise ValueError(f"{path}: {len(records)} records, expected {len(order)}")
    return {name: parse_fortran_value(_first_token(records[k]), kinds[name])
            for k, name in enumerate(order)}


def read_control(path: Path | str) -> ControlSettings:
    """read_solver_control (utility/MOD_IO.f90:25-109) for the control.in part."""
    vals = _read_positional(path, _CONTROL_KINDS, ControlSettings.FIELD_ORDER)
    return ControlSettings(**vals)


def read_custom(path: Path | str) -> CustomSettings:
    vals = _read_positional(path, _CUSTOM_KINDS, CustomSettings.FIELD_ORDER)
    return CustomSettings(**vals)


def validate(control: ControlSettings) -> None:
    """Reject settings outside what the step supports: 1 .. 4 equations (the equation modules'
    sizes; 3 for the shallow-water modules), at least the two waves HLL makes (further waves stay
    zero in the reference and change nothing)."""
    if not 1 <= control.number_of_equations <= 4 or control.number_of_waves < 2:
        raise ValueError("num_equations must be 1 .. 4 and num_waves at least 2 (HLL makes two waves)")
    if control.number_of_ghost_cells != 2:
        raise ValueError("the second-order correction needs exactly 2 ghost layers")
    if control.m_xi < 2 or control.m_eta < 2:
        raise ValueError("grids need at least 2 cells per direction")
    for bc in (control.bc_xi_lower, control.bc_xi_upper, control.bc_eta_lower, control.bc_eta_upper):
        if bc not in (1, 2, 3):
            raise ValueError(f"boundary condition {bc} is not 1 (wall), 2 or 3")
    if (control.add_higher_order_flux_correction and control.use_limtiter
            and control.limiter_function not in (1, 2, 3, 4)):
        raise ValueError("invalid limiter choice")  # MOD_flux_correction.f90:110-111
    if control.min_allowed_dt > control.max_allowed_dt:
        raise ValueError("Invalid timestep bounds")  # MOD_time_control.f90:114-119


def dam_break_control(m: int, limiter: int = 4, bc: int = 2, time_final: float = 0.5,
                      cfl: float = 0.9, **over) -> ControlSettings:
    """Control settings of the dam-break workloads: CFL 0.9, dt_max 1e-2 (the example's value,
    examples/2D_dam_break/cartesian/control_settings.py:68), second order with a limiter."""
    c = ControlSettings(
        time_final=time_final, CFL_limit=cfl, max_allowed_dt=1e-2,
        add_higher_order_flux_correction=True, use_limtiter=True, limiter_function=limiter,
        m_xi=m, m_eta=m, bc_xi_lower=bc, bc_xi_upper=bc, bc_eta_lower=bc, bc_eta_upper=bc)
    return dataclasses.replace(c, **over)
