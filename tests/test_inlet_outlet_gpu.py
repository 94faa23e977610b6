"""Velocity inlet and pressure outlet on the GPU (pylbm's Problem.inlet / Problem.outlet,
core.py:67-78,116-117,130-148) against pylbm's own float64 results: the Schaefer-Turek
channel of karman.py:21-42 at 4 nodes per diameter (solid cylinder, parabolic inlet, outlet)
with the momentum-exchange drag after every step, and a BGK channel from a random state.
Tolerances are pylbm's cross-backend ones (tests/test_equivalence.py:21)."""

from __future__ import annotations

import numpy as np
import pytest

from golden_io import load
from oracle import lbm_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {"f32": 3e-6, "f16": 1e-4, "bf16": 6e-4}


def _problem(d):
    from pylbm_b200.problem import Problem

    p = d["params"]
    return Problem(tuple(p["shape"]), tau=p["tau"], collision=p["collision"],
                   periodic=tuple(p["periodic"]), u_lid=p["u_lid"], force=tuple(p["force"]),
                   solid=d.get("solid"), inlet=d["inlet"], outlet=bool(d["outlet"]))


@pytest.mark.parametrize("variant", ["fused", "fused-plain", "fused-fp16"])
@pytest.mark.parametrize("name", ["inout_karman_trt", "inout_channel_bgk"])
def test_inlet_outlet_against_pylbm(name, variant):
    from pylbm_b200.backend import VARIANTS

    d = load(name)
    p = _problem(d)
    s = VARIANTS[variant](p)
    s.set_populations(d["f0"])
    steps = int(d["steps"])
    if p.solid is not None:
        force = s.advance_with_force(steps).cpu().numpy()
        scale = np.abs(d["force_hist"]).max()
        tol = 1e-4 if s.storage == "f32" else 2e-2
        assert np.abs(force - d["force_hist"]).max() < tol * scale
    else:
        s.step(steps)
    err = np.abs(s.populations() - d["f"]).max()
    bar = TOL[s.storage]
    if s.storage == "f16":
        # the cylinder's start-up transient: fp16 storage rounding alone (the float64 oracle
        # with h = f - w rounded to fp16 after every step) is ~3.7e-4 from pylbm here
        bar = max(bar, 1.5 * _rounded_storage_error(d, np.float16))
    assert err < bar, err


def _rounded_storage_error(d, dtype) -> float:
    case = O.Case.from_problem(_problem(d))
    w = np.array(O.D2Q9.w).reshape(9, 1, 1)
    src = O.solid_sources(case) if case.solid is not None else None
    f = (d["f0"] - w).astype(dtype).astype(np.float64) + w
    for _ in range(int(d["steps"])):
        f = O.step(f, case, np, src)
        f = (f - w).astype(dtype).astype(np.float64) + w
    return float(np.abs(f - d["f"]).max())


def test_inlet_outlet_long_run_against_oracle():
    """500 steps of a channel with a cylinder, parabolic inlet and outlet (tau = 0.6, TRT,
    from rest), fp32 shifted storage, against the float64 oracle (pinned bit for bit to pylbm
    on these boundaries). pylbm's own 4-nodes-per-diameter Schaefer-Turek lattice (tau = 0.506)
    is not used here: it diverges in float64 too after a few hundred steps."""
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.problem import Problem

    nx, ny = 120, 40
    yy, xx = np.mgrid[0:ny, 0:nx]
    solid = (xx - 30.0) ** 2 + (yy - 20.5) ** 2 <= 25.0
    y = np.arange(ny) + 0.5
    inlet = 4.0 * 0.06 * y * (ny - y) / ny**2
    p = Problem((nx, ny), tau=0.6, collision="trt", solid=solid, inlet=inlet, outlet=True)
    case = O.Case.from_problem(p)
    f0 = p.initial_populations()
    ref = O.run(case, f0, 500)
    s = VARIANTS["fused"](p)
    s.set_populations(f0)
    s.step(500)
    assert np.isfinite(ref).all()
    assert np.abs(s.populations() - ref).max() < TOL["f32"]
