"""Physical validation drivers on the B200 backend, reading velocities on the device.

Restatements of pylbm's shear-wave decay (validation/shear_wave.py:10-45) and body-force
Poiseuille channel (validation/poiseuille.py:10-62) for this backend: the same problems,
measurements and stopping rules, with the velocity field taken from ``lbm_macroscopic``
(fp32, on the device) so that a check copies a profile, not the float64 state
(pylbm's drivers call ``Solver.macroscopic``, base.py:79-82, which decodes the whole state on
the host).
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .problem import Problem


def _solver(p: Problem, variant: str) -> Any:
    from .backend import VARIANTS

    return VARIANTS[variant](p)


def run_shear_wave(tau: float, n: int = 64, amplitude: float = 0.01, steps: int | None = None,
                   samples: int = 20, collision: str = "bgk", variant: str = "fused") -> dict:
    """Decay of u_x = A sin(2 pi y / n) in a periodic n x n box: a least-squares fit of the
    log of the mode amplitude gives the measured viscosity, against (tau - 1/2) / 3."""
    import torch

    k = 2 * np.pi / n
    y = np.arange(n)
    u0 = np.zeros((2, n, n))
    u0[0] = amplitude * np.sin(k * y)[:, None]
    p = Problem((n, n), tau=tau, collision=collision, periodic=(True, True), init_u=u0)
    nu_th = p.nu
    if steps is None:  # decay to ~exp(-2)
        steps = int(2.0 / (nu_th * k * k))
    s = _solver(p, variant)
    chunk = max(s.step_multiple, steps // samples)
    chunk -= chunk % s.step_multiple
    mode = torch.as_tensor(np.sin(k * y), dtype=torch.float64, device=s.dev)
    ts, amps = [], []
    for _ in range(samples + 1):
        _, u = s.macroscopic_device()
        prof = u[0].double().mean(dim=1)
        ts.append(s.steps_done)
        amps.append(2.0 / n * float(prof @ mode))
        s.step(chunk)
    ts_a, amps_a = np.array(ts, float), np.array(amps)
    slope = np.polyfit(ts_a, np.log(np.abs(amps_a)), 1)[0]
    nu_meas = -slope / (k * k)
    return {"tau": tau, "n": n, "variant": variant, "nu_theory": nu_th,
            "nu_measured": float(nu_meas), "rel_error": float(abs(nu_meas - nu_th) / nu_th)}


def poiseuille_analytic(h: int, force: float, nu: float) -> np.ndarray:
    """u_x at the node centres y_j = j + 1/2 for walls at y = 0 and y = h (rho = 1)."""
    y = np.arange(h) + 0.5
    return force / (2.0 * nu) * y * (h - y)


def run_poiseuille(h: int, tau: float = 0.8, u_max: float = 0.02, collision: str = "bgk",
                   nx: int = 8, variant: str = "fused", tol: float = 1e-9,
                   max_steps: int = 2_000_000) -> dict:
    """Body-force channel between walls at y = 0 and y = h, run to steady state; relative L2 /
    Linf errors of the x-averaged velocity profile against the parabola."""
    nu = (tau - 0.5) / 3.0
    force = 8.0 * nu * u_max / h**2
    p = Problem((nx, h), tau=tau, collision=collision, periodic=(True, False),
                force=(force, 0.0))
    s = _solver(p, variant)
    ref = poiseuille_analytic(h, force, nu)
    check = max(s.step_multiple * 50, int(0.5 * h * h / nu))
    check += check % s.step_multiple
    old = np.zeros(h)
    best, stale = np.inf, 0
    prof = old
    while s.steps_done < max_steps:
        s.step(check)
        _, u = s.macroscopic_device()
        # the device velocity is the physical one (sum c f - F/2) / rho, as pylbm's
        prof = u[0].double().mean(dim=1).cpu().numpy()
        change = float(np.abs(prof - old).max()) / u_max
        old = prof
        if change < tol:
            break
        if change < 0.5 * best:  # stop at the round-off floor
            best, stale = change, 0
        else:
            stale += 1
        if stale >= 5 and best < 1e-4:
            break
    err = prof - ref
    return {"h": h, "tau": tau, "collision": collision, "variant": variant,
            "steps": s.steps_done, "L2": float(np.sqrt(np.sum(err**2) / np.sum(ref**2))),
            "Linf": float(np.abs(err).max() / ref.max())}


def poiseuille_convergence(hs: tuple[int, ...] = (8, 16, 32, 64), **kw: Any) -> dict:
    """Errors for several channel widths plus the fitted order of convergence."""
    runs = [run_poiseuille(h, **kw) for h in hs]
    errs = np.array([r["L2"] for r in runs])
    order = float(-np.polyfit(np.log(hs), np.log(errs), 1)[0]) if (errs > 0).all() else None
    return {"runs": runs, "order": order}
