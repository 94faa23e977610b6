"""The checkers of the adjoint, on the CPU: the oracle's float64 drag objective reproduces
pylbm's own central finite difference (fixture dJdg, made by running pylbm's NumPy solver),
its torch path gives the same J, and torch autograd through it agrees with central
differences (so it can serve as the gradient reference of the GPU adjoint)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm_oracle as O
from tests.golden_io import load


def _fixture_case(g: float) -> tuple:
    d = load("dJdg")
    p = d["params"]
    case = O.Case(tuple(p["shape"]), p["tau"], "bgk", tuple(p["periodic"]), 0.0, (g, 0.0),
                  solid=d["solid"])
    return case, d


def test_oracle_objective_reproduces_pylbm_fd():
    case, d = _fixture_case(1e-6)
    p = d["params"]
    f0 = O.equilibrium(O.D2Q9, np.ones(case.array_shape), np.zeros((2,) + case.array_shape))
    J = O.drag_objective(case, f0, p["T"], p["t0"])
    assert J == pytest.approx(float(d["J"]), rel=1e-12)
    eps = p["eps"]
    jp = O.drag_objective(_fixture_case(p["g"] + eps)[0], f0, p["T"], p["t0"])
    jm = O.drag_objective(_fixture_case(p["g"] - eps)[0], f0, p["T"], p["t0"])
    assert (jp - jm) / (2 * eps) == pytest.approx(float(d["dJdg"]), rel=1e-9)


def test_oracle_torch_autograd_matches_fd():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    nx, ny, T, t0 = 16, 10, 40, 30
    yy, xx = np.mgrid[0:ny, 0:nx]
    solid = (xx - 5.0) ** 2 + (yy - 4.5) ** 2 <= 2.2 ** 2
    F = 1e-4 * rng.standard_normal((2, ny, nx))
    f0 = O.equilibrium(O.D2Q9, np.ones((ny, nx)), np.zeros((2, ny, nx)))

    def J_np(field):
        c = O.Case((nx, ny), 0.6, "bgk", (True, False), 0.0, (1e-4, 0.0), solid=solid,
                   force_field=field)
        return O.drag_objective(c, f0, T, t0)

    Ft = torch.tensor(F, dtype=torch.float64, requires_grad=True)
    ct = O.Case((nx, ny), 0.6, "bgk", (True, False), 0.0, (1e-4, 0.0), solid=solid,
                force_field=Ft)
    Jt = O.drag_objective(ct, torch.tensor(f0), T, t0, xp=torch, checkpoint=7)
    assert Jt.item() == pytest.approx(J_np(F), rel=1e-12)
    Jt.backward()
    g = Ft.grad.numpy()
    v = rng.standard_normal(F.shape)
    eps = 1e-6
    fd = (J_np(F + eps * v) - J_np(F - eps * v)) / (2 * eps)
    assert float((g * v).sum()) == pytest.approx(fd, rel=1e-7)
