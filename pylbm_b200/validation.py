"""Physical validation drivers on the B200 backend, reading velocities on the device.

Restatements of pylbm's shear-wave decay (validation/shear_wave.py:10-45), body-force
Poiseuille channel (validation/poiseuille.py:10-62) and Schaefer-Turek Karman street
(validation/karman.py:21-130) for this backend: the same problems, measurements and stopping
rules, with the velocity field taken from ``lbm_macroscopic`` (fp32, on the device) so that a
check copies a profile, not the float64 state (pylbm's drivers call ``Solver.macroscopic``,
base.py:79-82, which decodes the whole state on the host), and the cylinder force from the
step kernel's own FP64 momentum-exchange sum.
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


# Schaefer & Turek (1996) benchmark 2D-2 reference intervals (karman.py:17)
KARMAN_REFERENCE = {"St": (0.2950, 0.3050), "cd_max": (3.2200, 3.2400), "cl_max": (0.9900, 1.0100)}


def schafer_turek_problem(d: int = 20, u_mean: float = 0.05, collision: str = "trt") -> Problem:
    """The lattice of benchmark 2D-2 with ``d`` nodes per cylinder diameter, as pylbm builds it
    (karman.py:21-42): channel 2.2 x 0.41, cylinder of diameter 0.1 at (0.2, 0.2) as solid
    nodes, parabolic velocity inlet with maximum 1.5 u_mean, pressure outlet, Re = 100, and a
    small transverse kick behind the cylinder to start the shedding."""
    dx = 0.1 / d
    nx, ny = round(2.2 / dx), round(0.41 / dx)
    xc, yc = (np.arange(nx) + 0.5) * dx, (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(xc, yc)
    solid = (X - 0.2) ** 2 + (Y - 0.2) ** 2 <= 0.05**2
    yy = np.arange(ny) + 0.5
    inlet = 4.0 * (1.5 * u_mean) * yy * (ny - yy) / ny**2
    nu = u_mean * d / 100.0
    init_u = np.zeros((2, ny, nx))
    init_u[0] = inlet[:, None]
    init_u[0][solid] = 0.0
    init_u[1] = 0.05 * u_mean * np.exp(-((X - 0.3) ** 2 + (Y - 0.2) ** 2) / 0.05**2)
    return Problem((nx, ny), tau=3.0 * nu + 0.5, collision=collision, periodic=(False, False),
                   solid=solid, inlet=inlet, outlet=True, init_u=init_u)


def run_karman(d: int = 40, u_mean: float = 0.05, periods: float = 20.0,
               t_transient: float = 60.0, collision: str = "trt", variant: str = "fused",
               sample_every: int = 10) -> dict:
    """Benchmark 2D-2 on the device: the momentum-exchange force on the cylinder comes from the
    step kernel itself (FP64, every step) instead of a host-side sum over the state every
    ``sample_every`` steps (karman.py:85-107); the statistics are pylbm's (lift spectrum with
    a Hann window, zero padding and a parabolic peak for St; maxima of c_D, c_L)."""
    import torch

    p = schafer_turek_problem(d, u_mean, collision)
    s = _solver(p, variant)
    t_conv = d / u_mean  # steps per convective unit
    n_trans = int(t_transient * t_conv)
    n_meas = int(periods * t_conv)
    n_meas -= n_meas % sample_every
    s.step(n_trans)
    forces = s.advance_with_force(n_meas).cpu().numpy()[sample_every - 1::sample_every]
    scale = 2.0 / (1.0 * u_mean**2 * d)
    cd, cl = forces[:, 0] * scale, forces[:, 1] * scale
    sig = cl - cl.mean()
    nfft = 16 * len(sig)
    spec = np.abs(np.fft.rfft(sig * np.hanning(len(sig)), nfft))
    k = float(np.argmax(spec[1:]) + 1)
    ki = int(k)
    if 1 <= ki < len(spec) - 1:
        a, b, g = spec[ki - 1], spec[ki], spec[ki + 1]
        k = ki + 0.5 * (a - g) / (a - 2 * b + g)
    st = k / (nfft * sample_every) * d / u_mean
    _, u = s.macroscopic_device()  # vorticity on the device, in units of u_mean / d
    ux, uy = u[0].double(), u[1].double()
    vort = torch.gradient(uy, dim=1)[0] - torch.gradient(ux, dim=0)[0]
    vort[torch.as_tensor(p.solid, device=vort.device)] = float("nan")
    return {"d": d, "u_mean": u_mean, "tau": p.tau, "collision": collision, "variant": variant,
            "shape": list(p.shape), "steps": s.steps_done, "St": float(st),
            "cd_max": float(cd.max()), "cl_max": float(cl.max()), "cd_mean": float(cd.mean()),
            "reference": KARMAN_REFERENCE, "vorticity": (vort * d / u_mean).cpu().numpy()}
