"""Generate the golden fixtures in this folder by running pylbm itself.

    [PYLBM_SRC=/path/to/pylbm/src] python tests/golden/make_golden.py

pylbm (the reference implementation) is imported read-only from ``PYLBM_SRC`` or, without it,
from the offline install ``baseline/_ref`` (``baseline/install_ref.py``). It is needed only to
(re)generate the fixtures; the parity tests read the committed ``.npz`` files. Every fixture stores the problem parameters (JSON), the initial state when it is not
the rest equilibrium, the step count and pylbm's float64 NumPy result:

* ``eq_*``      pylbm's own equivalence cases (tests/test_equivalence.py:9-20), 100 steps,
                plus random-field periodic cases;
* ``config1``   D2Q9 BGK lid-driven cavity 128x128, U = 0.1, Re = 100, 1000 steps;
* ``solid_*``   forced channel with a solid disc: state after the run and the
                momentum-exchange force after every step (karman.py:45-53,88-96);
* ``tags_*``    the streaming index map: pylbm's core.stream applied to integer tags with the
                lid off, and to zeros with the lid on (the construction of
                torch_backend.py:80-101);
* ``dJdg``      central finite difference, on pylbm's NumPy solver, of the mean x drag over
                steps t0..T with respect to the uniform body force g_x (small channel + disc);
* ``inout_*``   velocity inlet and pressure outlet (core.py:67-78,116-117,130-148): pylbm's
                Schaefer-Turek channel at 4 nodes per diameter (karman.py:21-42) with the drag
                after every step, and a BGK channel from a random state.
"""

from __future__ import annotations

import dataclasses
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.dont_write_bytecode = True
sys.path.insert(0, str(HERE.parents[1]))
from baseline import import_pylbm  # noqa: E402

import_pylbm()  # PYLBM_SRC or the offline install baseline/_ref

from pylbm import core  # noqa: E402
from pylbm.backends.numpy_backend import NumpySolver  # noqa: E402
from pylbm.lattice import equilibrium  # noqa: E402
from pylbm.problem import Problem  # noqa: E402
from pylbm.validation.karman import _force_masks  # noqa: E402


def params_of(p: Problem) -> dict:
    return {"shape": list(p.shape), "tau": p.tau, "collision": p.collision,
            "periodic": list(p.periodic), "u_lid": p.u_lid, "force": list(p.force),
            "magic": p.magic, "s_e": p.s_e, "s_eps": p.s_eps}


def save(name: str, **arrays) -> None:
    np.savez_compressed(HERE / f"{name}.npz", **arrays)
    print(f"wrote {name}.npz", {k: getattr(v, "shape", v) for k, v in arrays.items()
                                if k != "params"})


def random_state(p: Problem, seed: int, amp: float = 0.05) -> np.ndarray:
    rng = np.random.default_rng(seed)
    shp = p.array_shape
    rho = 1.0 + 0.01 * rng.standard_normal(shp)
    u = amp * (rng.random((p.dim,) + shp) - 0.5)
    return equilibrium(p.lattice, rho, u)


def equivalence_cases() -> None:
    cases = {
        "eq_cavity2d_bgk": Problem((40, 28), tau=0.7, u_lid=0.1),
        "eq_cavity2d_trt": Problem((40, 28), tau=0.7, u_lid=0.1, collision="trt"),
        "eq_cavity2d_mrt": Problem((40, 28), tau=0.7, u_lid=0.1, collision="mrt"),
        "eq_channel2d_force": Problem((40, 28), tau=0.7, periodic=(True, False),
                                      force=(1e-5, 2e-6)),
        "eq_periodic2d_mrt_force": Problem((32, 24), tau=0.6, periodic=(True, True),
                                           force=(1e-5, -3e-6), collision="mrt"),
        "eq_cavity3d_bgk": Problem((20, 14, 12), tau=0.7, u_lid=0.1),
        "eq_periodic3d_trt": Problem((16, 12, 10), tau=0.7, periodic=(True, True, False),
                                     force=(1e-5, 1e-6, 0.0), collision="trt"),
    }
    for name, p in cases.items():
        s = NumpySolver(p)
        s.step(100)
        save(name, params=json.dumps(params_of(p)), steps=100, f=s.populations())
    # random initial fields on periodic boxes (the config-2 / config-3 kind of input)
    rnd = {
        "eq_random2d_bgk": (Problem((32, 20), tau=0.6, periodic=(True, True)), 11),
        "eq_random2d_trt": (Problem((32, 20), tau=0.6, periodic=(True, True),
                                    collision="trt"), 12),
        "eq_random2d_mrt_lid": (Problem((24, 20), tau=0.8, u_lid=0.07, collision="mrt"), 13),
        "eq_random3d_trt": (Problem((12, 10, 8), tau=0.55, periodic=(True, True, True),
                                    collision="trt"), 14),
        "eq_random3d_bgk_lid": (Problem((12, 10, 8), tau=0.8, u_lid=0.05,
                                        periodic=(True, False, False)), 15),
    }
    for name, (p, seed) in rnd.items():
        f0 = random_state(p, seed)
        s = NumpySolver(p)
        s.set_populations(f0)
        s.step(60)
        save(name, params=json.dumps(params_of(p)), steps=60, f0=f0, f=s.populations())


def config1() -> None:
    p = Problem.cavity(128, re=100, u_lid=0.1)
    s = NumpySolver(p)
    s.step(1000)
    rho, u = s.macroscopic()
    save("config1", params=json.dumps(params_of(p)), steps=1000, f=s.populations(),
         rho=rho, u=u)


def disc(nx: int, ny: int, xc: float, yc: float, r: float) -> np.ndarray:
    yy, xx = np.mgrid[0:ny, 0:nx]
    return (xx - xc) ** 2 + (yy - yc) ** 2 <= r * r


def solid_cases() -> None:
    cases = {
        "solid_channel_bgk": (Problem((48, 24), tau=0.6, periodic=(True, False),
                                      force=(1e-5, 0.0)), disc(48, 24, 12.0, 12.5, 4.0), 80),
        "solid_cavity_trt": (Problem((32, 30), tau=0.7, u_lid=0.08, collision="trt"),
                             disc(32, 30, 15.5, 14.0, 5.0), 80),
        "solid_periodic_mrt": (Problem((30, 26), tau=0.65, periodic=(True, True),
                                       force=(2e-5, -1e-5), collision="mrt"),
                               disc(30, 26, 10.0, 13.0, 3.5), 80),
    }
    for name, (p, solid, steps) in cases.items():
        p = dataclasses.replace(p, solid=solid)
        masks, c = _force_masks(p)
        mk = np.stack(masks).astype(float)
        s = NumpySolver(p)
        hist = []
        for _ in range(steps):
            s.step(1)
            per_dir = (s.populations() * mk).sum(axis=(1, 2))
            hist.append(2.0 * (per_dir[:, None] * c).sum(0))
        save(name, params=json.dumps(params_of(p)), steps=steps, solid=solid,
             f=s.populations(), force_hist=np.array(hist))


def inout_cases() -> None:
    from pylbm.validation.karman import schafer_turek_problem

    p = schafer_turek_problem(d=4, u_mean=0.05, collision="trt")
    masks, c = _force_masks(p)
    mk = np.stack(masks).astype(float)
    s = NumpySolver(p)
    f0 = s.populations()
    hist = []
    for _ in range(60):
        s.step(1)
        per_dir = (s.populations() * mk).sum(axis=(1, 2))
        hist.append(2.0 * (per_dir[:, None] * c).sum(0))
    save("inout_karman_trt", params=json.dumps(params_of(p)), steps=60, solid=p.solid,
         inlet=p.inlet, outlet=True, f0=f0, f=s.populations(), force_hist=np.array(hist))
    nx, ny = 40, 12
    yy = np.arange(ny) + 0.5
    inlet = 4.0 * 0.06 * yy * (ny - yy) / ny**2
    p = Problem((nx, ny), tau=0.62, periodic=(False, False), inlet=inlet, outlet=True)
    f0 = random_state(p, 21, amp=0.03)
    s = NumpySolver(p)
    s.set_populations(f0)
    s.step(50)
    save("inout_channel_bgk", params=json.dumps(params_of(p)), steps=50, inlet=inlet,
         outlet=True, f0=f0, f=s.populations())


def tag_maps() -> None:
    cases = {
        "tags_cavity2d": Problem((7, 5), u_lid=0.1),
        "tags_channel2d_solid": dataclasses.replace(
            Problem((9, 6), periodic=(True, False), u_lid=0.1), solid=disc(9, 6, 4, 2.5, 1.2)),
        "tags_periodic2d": Problem((6, 5), periodic=(True, True)),
        "tags_cavity3d": Problem((5, 4, 3), u_lid=0.1),
        "tags_mixed3d": Problem((4, 5, 3), periodic=(True, False, False), u_lid=0.2),
        "tags_mixed3d_b": Problem((4, 3, 5), periodic=(False, True, True)),
    }
    ops = core.Ops(np)
    for name, p in cases.items():
        shp = (p.lattice.q,) + p.array_shape
        still = dataclasses.replace(p, u_lid=0.0)
        src = core.stream(np.arange(np.prod(shp), dtype=np.float64).reshape(shp),
                          core.make_geometry(still, np.asarray), ops)
        src = np.stack(src).astype(np.int64)
        lid = np.stack(core.stream(np.zeros(shp), core.make_geometry(p, np.asarray), ops))
        extra = {"solid": p.solid} if p.solid is not None else {}
        save(name, params=json.dumps(params_of(p)), src=src, lid=lid, **extra)


def drag_fd() -> None:
    """dJ/dg_x of the small adjoint case by central differences on pylbm's NumPy solver."""
    nx, ny, T, t0 = 64, 32, 400, 300
    solid = disc(nx, ny, 16.0, 16.5, 5.0)

    def J(g: float) -> float:
        p = Problem((nx, ny), tau=0.56, periodic=(True, False), force=(g, 0.0))
        p = dataclasses.replace(p, solid=solid)
        masks, c = _force_masks(p)
        mk = np.stack(masks).astype(float)
        s = NumpySolver(p)
        acc, cnt = 0.0, 0
        for t in range(1, T + 1):
            s.step(1)
            if t >= t0:
                per_dir = (s.populations() * mk).sum(axis=(1, 2))
                acc += 2.0 * float((per_dir * c[:, 0]).sum())
                cnt += 1
        return acc / cnt

    g, eps = 1e-6, 1e-8
    jp, jm, j0 = J(g + eps), J(g - eps), J(g)
    save("dJdg", params=json.dumps({"shape": [nx, ny], "tau": 0.56, "periodic": [True, False],
                                    "g": g, "T": T, "t0": t0, "eps": eps}),
         solid=solid, J=j0, dJdg=(jp - jm) / (2 * eps))


if __name__ == "__main__":
    equivalence_cases()
    config1()
    solid_cases()
    tag_maps()
    drag_fd()
    inout_cases()
