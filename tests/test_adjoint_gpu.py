"""The GPU adjoint of the drag objective: its dJ/dF agrees with (1) pylbm's own central finite
difference with respect to the uniform force (fixture dJdg: sum over nodes of dJ/dF_x),
(2) central finite differences of the float64 oracle along random directions on a 128 x 64
channel over T = 2000 steps (the 128 x 64 version of the 1024 x 256 case), and (3) torch
autograd through the float64 oracle (the differentiable restatement of pylbm's torch-eager
roll solver). Bar: relative error <= 1e-4."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm_oracle as O
from tests.golden_io import load

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _problem(shape, tau, g, solid):
    from pylbm_b200.problem import Problem

    return Problem(shape, tau=tau, periodic=(True, False), force=(g, 0.0), solid=solid)


def test_gradient_matches_pylbm_fd_of_uniform_force():
    from pylbm_b200.adjoint import DragAdjoint

    d = load("dJdg")
    p = d["params"]
    prob = _problem(tuple(p["shape"]), p["tau"], p["g"], d["solid"])
    adj = DragAdjoint(prob, p["T"], p["t0"], checkpoint=20)
    F = torch.zeros((2,) + prob.array_shape, dtype=torch.float32, device="cuda")
    J = adj.objective(F)
    assert J == pytest.approx(float(d["J"]), rel=2e-5)
    g = adj.gradient()
    dJdg = float(g[0].sum().item())
    assert dJdg == pytest.approx(float(d["dJdg"]), rel=1e-4)
    assert float(g[:, prob.solid].abs().max().item()) == 0.0  # solid nodes carry no gradient


def _channel(nx=128, ny=64, seed=1):
    from pylbm_b200 import workloads as W

    solid, F = W.cylinder_channel(nx=nx, ny=ny, xc=25.0, yc=32.25, diameter=10.0,
                                  sigma=1e-7, seed=seed)
    return solid, F.astype(np.float32)


def test_gradient_matches_float64_fd_128x64():
    from pylbm_b200.adjoint import DragAdjoint

    T, t0, tau, g = 2000, 1500, 0.56, 1e-6
    solid, F = _channel()
    prob = _problem((128, 64), tau, g, solid)
    adj = DragAdjoint(prob, T, t0, checkpoint=45)
    J = adj.objective(torch.as_tensor(F, device="cuda"))
    grad = adj.gradient().cpu().numpy()
    f0 = prob.initial_populations()

    def J64(field):
        c = O.Case((128, 64), tau, "bgk", (True, False), 0.0, (g, 0.0), solid=solid,
                   force_field=field)
        return O.drag_objective(c, f0, T, t0)

    F64 = F.astype(np.float64)
    assert J == pytest.approx(J64(F64), rel=1e-4)
    rng = np.random.default_rng(2)
    for k in range(2):
        v = rng.standard_normal(F.shape) * ~solid  # directions over fluid nodes
        eps = 1e-7
        fd = (J64(F64 + eps * v) - J64(F64 - eps * v)) / (2 * eps)
        ad = float((grad * v).sum())
        assert ad == pytest.approx(fd, rel=1e-4), (k, ad, fd)


def test_gradient_matches_torch_autograd_oracle():
    from pylbm_b200.adjoint import DragAdjoint

    T, t0, tau, g = 300, 200, 0.56, 1e-5
    solid, F = _channel(nx=64, ny=32, seed=3)
    solid = np.zeros((32, 64), bool)
    yy, xx = np.mgrid[0:32, 0:64]
    solid[(xx - 14.0) ** 2 + (yy - 16.25) ** 2 <= 5.0 ** 2] = True
    F = (1e-5 * np.random.default_rng(4).standard_normal((2, 32, 64))).astype(np.float32)
    prob = _problem((64, 32), tau, g, solid)
    adj = DragAdjoint(prob, T, t0, checkpoint=17)
    adj.objective(torch.as_tensor(F, device="cuda"))
    grad = adj.gradient().cpu().numpy()
    Ft = torch.tensor(F.astype(np.float64), requires_grad=True)
    case = O.Case((64, 32), tau, "bgk", (True, False), 0.0, (g, 0.0), solid=solid,
                  force_field=Ft)
    J = O.drag_objective(case, torch.tensor(prob.initial_populations()), T, t0, xp=torch,
                         checkpoint=25)
    J.backward()
    ref = Ft.grad.numpy()
    scale = np.abs(ref).max()
    assert np.abs(grad - ref).max() < 1e-4 * scale
    assert np.linalg.norm(grad - ref) < 1e-4 * np.linalg.norm(ref)


def test_autograd_function_backward_is_the_adjoint():
    from pylbm_b200.adjoint import DragAdjoint, drag_objective

    d = load("dJdg")
    p = d["params"]
    prob = _problem(tuple(p["shape"]), p["tau"], p["g"], d["solid"])
    adj = DragAdjoint(prob, 120, 80, checkpoint=16)
    F = torch.zeros((2,) + prob.array_shape, dtype=torch.float32, device="cuda",
                    requires_grad=True)
    J = drag_objective(F, adj)
    J.backward()
    ref = adj.gradient().float()
    assert torch.equal(F.grad, ref)
    assert np.isfinite(J.item())
