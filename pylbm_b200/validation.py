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


# ----------------------------------------------------------------------------- Ghia cavity
# Table II, Re = 400, x = 0.9063 breaks the monotonic run of its neighbours and is a known
# misprint of the 1982 tables; pylbm leaves it out of its error norms (validation/ghia.py:17)
GHIA_SKIP = {("v", 400, 0.9063)}


def ghia_data_path() -> Any:
    """pylbm's tabulation of Ghia, Ghia & Shin (1982), read where pylbm is installed
    (pylbm/validation/data/ghia1982.json); not copied into this package."""
    import importlib.util
    from pathlib import Path

    spec = importlib.util.find_spec("pylbm")
    if spec is None or spec.origin is None:
        raise FileNotFoundError("the Ghia tables are read from an installed pylbm; none found")
    return Path(spec.origin).parent / "validation" / "data" / "ghia1982.json"


def ghia_reference(re: int, path: Any = None) -> dict:
    """Centreline velocities of the 1982 tables for Re in {100, 400, 1000}: u(y) on x = 1/2
    and v(x) on y = 1/2, in units of the lid speed and the cavity side."""
    import json
    from pathlib import Path

    t = json.loads(Path(path or ghia_data_path()).read_text())
    key = str(int(re))
    return {"y": np.asarray(t["u_vertical"]["y"], float),
            "u": np.asarray(t["u_vertical"][key], float),
            "x": np.asarray(t["v_horizontal"]["x"], float),
            "v": np.asarray(t["v_horizontal"][key], float)}


def cavity_centrelines(ux: np.ndarray, uy: np.ndarray, u_lid: float) -> dict:
    """u / U on the vertical and v / U on the horizontal centreline of (ny, nx) fields, at the
    node centres (i + 1/2) / n of a half-way bounce-back cavity (the mean of the two middle
    nodes for even n), with the wall values appended at 0 and 1 (u = U on the lid)."""
    ny, nx = ux.shape

    def centre(a: np.ndarray, axis: int) -> np.ndarray:
        n = a.shape[axis]
        lo, hi = (n - 1) // 2, n // 2
        return 0.5 * (np.take(a, lo, axis=axis) + np.take(a, hi, axis=axis))

    y = np.r_[0.0, (np.arange(ny) + 0.5) / ny, 1.0]
    x = np.r_[0.0, (np.arange(nx) + 0.5) / nx, 1.0]
    return {"y": y, "u": np.r_[0.0, centre(ux, 1) / u_lid, 1.0],
            "x": x, "v": np.r_[0.0, centre(uy, 0) / u_lid, 0.0]}


def ghia_errors(prof: dict, re: int, ref: dict) -> dict:
    """RMS and maximum deviation from the tables at their interior points (linear
    interpolation of the profiles), per component and combined; units of the lid speed."""
    out = {}
    for comp, axis in (("u", "y"), ("v", "x")):
        pts = ref[axis]
        keep = (pts > 0.0) & (pts < 1.0)
        keep &= np.array([(comp, int(re), round(float(p), 4)) not in GHIA_SKIP for p in pts])
        dev = np.interp(pts[keep], prof[axis], prof[comp]) - ref[comp][keep]
        out[f"{comp}_L2"] = float(np.sqrt(np.mean(dev * dev)))
        out[f"{comp}_Linf"] = float(np.abs(dev).max())
    out["L2"] = float(np.sqrt(0.5 * (out["u_L2"] ** 2 + out["v_L2"] ** 2)))
    out["Linf"] = max(out["u_Linf"], out["v_Linf"])
    return out


def run_ghia(re: int, n: int = 128, u_lid: float = 0.1, collision: str = "bgk",
             variant: str = "fused", tol: float = 1e-5, max_steps: int = 1_000_000,
             check_every: int | None = None, data_path: Any = None) -> dict:
    """The lid-driven cavity at Reynolds number ``re`` run to a steady state on this backend
    and compared with Ghia et al. (1982), as pylbm's validation/ghia.py:96-132 does: every
    ``check_every`` steps (default max(1000, 4 n)) the RMS change of the velocity field over
    the lid speed is compared with ``tol``; a non-finite field stops the run; 16-bit storages,
    whose round-off floor lies above ``tol``, stop once the change has not improved for ten
    checks and is within 50 tol ("plateau"). The velocity comes from the device (fp32
    ``lbm_macroscopic``), so a check copies two fields, not the float64 state."""
    import torch

    ref = ghia_reference(re, data_path)
    p = Problem.cavity(n, re=re, u_lid=u_lid, collision=collision)
    s = _solver(p, variant)
    every = check_every or max(1000, 4 * n)
    every -= every % s.step_multiple
    u_old = s.macroscopic_device()[1].double()
    converged: Any = False
    best, stale, change = float("inf"), 0, float("nan")
    while s.steps_done < max_steps:
        s.step(every)
        u = s.macroscopic_device()[1].double()
        if not bool(torch.isfinite(u).all()):
            break
        change = float(torch.sqrt(torch.mean((u - u_old) ** 2))) / u_lid
        u_old = u
        if change < tol:
            converged = True
            break
        if change < 0.9 * best:
            best, stale = change, 0
        else:
            stale += 1
        if stale >= 10 and best < 50 * tol:
            converged = "plateau"
            break
    uh = u_old.cpu().numpy()
    prof = cavity_centrelines(uh[0], uh[1], u_lid)
    return {"re": re, "n": n, "variant": variant, "collision": collision, "tau": p.tau,
            "steps": s.steps_done, "converged": converged, "last_change": change,
            "errors": ghia_errors(prof, re, ref),
            "profile": {k: v.tolist() for k, v in prof.items()}}
