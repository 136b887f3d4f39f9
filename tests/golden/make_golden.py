"""Generate the golden fixtures in this directory (run once, in the container that has the
reference checked out; the fixtures are committed and the tests never read the reference).

    python tests/golden/make_golden.py <path of the reference checkout>

1. control.in / custom.in written by the reference's own input generator (write_input.py with
   control_settings.py of the project root and of examples/2D_dam_break/cartesian).
2. Single-interface HLL known answers from transliteration.py (LAPACK dgeev + BLAS dgemv
   through scipy, the library calls of the reference).
3. Tiny full runs of the main loop from transliteration.py (dt sequence, accept flags, final
   state) for several limiter / boundary settings, including rejected steps.
"""
from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))

import transliteration as T  # noqa: E402

GRAV = 9.8100004196166992  # float32(9.81) widened, as the reference's default-real literal


def _load(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.path.insert(0, str(path.parent))
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.path.pop(0)
    return mod


def reference_inputs(ref: Path) -> None:
    for tag, d in (("default", ref), ("dam_break_example", ref / "examples" / "2D_dam_break" / "cartesian")):
        for mod in ("control_settings", "custom_settings", "write_input"):
            sys.modules.pop(mod, None)
        cs = _load(d / "control_settings.py", "control_settings")
        cu = _load(d / "custom_settings.py", "custom_settings")
        wi = _load(d / "write_input.py", "write_input")
        wi.write_input_files(cu.CustomSettings(), cs.ControlSettings(), HERE / f"custom_{tag}.in",
                             HERE / f"control_{tag}.in")
        meta = {"field_order": list(cs.ControlSettings.FIELD_ORDER),
                "defaults": {k: getattr(cs.ControlSettings(), k) for k in cs.ControlSettings.FIELD_ORDER}}
        (HERE / f"control_{tag}.json").write_text(json.dumps(meta, indent=1) + "\n")


def hll_kats() -> None:
    rng = np.random.Generator(np.random.PCG64(2024))
    rows = []
    for k in range(64):
        ixy = 1 + (k % 2)
        qL = [float(rng.uniform(0.3, 3.0)), float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))]
        if k % 8 == 0:
            qR = list(qL)  # equal states: only the eps term of the HLL denominator acts
        else:
            qR = [float(rng.uniform(0.3, 3.0)), float(rng.uniform(-2, 2)), float(rng.uniform(-2, 2))]
        lam, W1, W2 = T.hll(ixy, qL, qR, GRAV)
        rows.append({"ixy": ixy, "qL": [x.hex() for x in qL], "qR": [x.hex() for x in qR],
                     "lambda": [float(x).hex() for x in lam], "W1": [x.hex() for x in W1],
                     "W2": [x.hex() for x in W2]})
    (HERE / "hll_kat.json").write_text(json.dumps(rows, indent=0) + "\n")


TINY_CASES = [
    # name, m_xi, m_eta, limiter, bc, dt0, attempts
    ("mc_bc2", 8, 6, 4, 2, 1e-3, 12),
    ("minmod_bc3", 7, 9, 1, 3, 1e-3, 12),
    ("superbee_bc2", 6, 6, 2, 2, 1e-3, 8),
    ("vanleer_bc3", 9, 5, 3, 3, 1e-3, 8),
    ("reject_mc_bc2", 8, 8, 4, 2, 0.2, 10),
]


def tiny_params(m_xi, m_eta, limiter, bc, dt0):
    return dict(m_xi=m_xi, m_eta=m_eta, xi_min=-1.0, xi_max=1.0, eta_min=-1.0, eta_max=1.0, grav=GRAV,
                t_start=0.0, t_final=0.5, n_snapshots=5, dt_initial=dt0, cfl=0.9, dt_min=1e-10, dt_max=1e-2,
                growth=1.2, shrink=0.5, higher_order=True, use_limiter=True, limiter=limiter, bc=bc)


def tiny_ic(m_xi, m_eta, bc):
    """Circular dam for zero-gradient walls; a smooth mound for the extrapolating BC 3, whose
    linear extrapolation across the dam edge of a 7-cell grid would drive a ghost depth
    negative (the reference then aborts on complex eigenvalues)."""
    from paraclaws_b200 import ic
    if bc == 3:
        x, y = ic.cell_centres(m_xi, m_eta)
        q = ic.empty_state(m_xi, m_eta)
        q[..., 0] = 1.0 + 0.2 * np.exp(-(y[:, None] ** 2 + x[None, :] ** 2) / 0.5)
    else:
        q = ic.circular_dam(m_xi, m_eta)
    q[..., 1] = 0.05 * np.cos(np.arange(m_xi + 4))[None, :]
    q[..., 2] = 0.03 * np.sin(np.arange(m_eta + 4))[:, None]
    return q


def tiny_runs() -> None:
    out = {}
    for name, mx, my, lim, bc, dt0, att in TINY_CASES:
        s = T.Solver(tiny_params(mx, my, lim, bc, dt0))
        s.set_state(tiny_ic(mx, my, bc))
        s.bc()
        log = s.run(att)
        out[f"{name}_dt"] = np.array([r[0] for r in log])
        out[f"{name}_ierr"] = np.array([r[1] for r in log], dtype=np.int32)
        out[f"{name}_state"] = s.state()
        out[f"{name}_ic"] = tiny_ic(mx, my, bc)
    np.savez_compressed(HERE / "tiny_runs.npz", **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    ref = Path(sys.argv[1])
    reference_inputs(ref)
    hll_kats()
    tiny_runs()
    print("golden fixtures written to", HERE)
