"""The b200 backend through pylbm's own entry points, with pylbm's own Problem objects.

pylbm itself is imported read-only from its offline install (``baseline/_ref``) or
``PYLBM_SRC``; the tests are skipped when neither is present. After ``register()``:

* ``pylbm.backends.status()`` lists every b200 variant as available, and ``get`` returns
  subclasses of pylbm's ``Solver`` (backends/__init__.py:53-90, base.py:18-96);
* ``pylbm.backends.make`` builds every variant for pylbm's equivalence cases
  (tests/test_equivalence.py:9-21 -- the same problems, as recorded in this repository's
  ``eq_*`` fixtures) and the result after 100 steps matches pylbm's NumPy float64 solver at
  pylbm's tolerances (TOL, tests/test_equivalence.py:21);
* AA equals AB as in pylbm's check (tests/test_equivalence.py:55-62);
* ``pylbm.validation.make_solver``, the CLI ``pylbm run`` (cli.py:26-66) and the benchmark
  engine's ``measure`` (benchmark.py:183-236) run on ``--backend b200`` unchanged.
"""

from __future__ import annotations

import numpy as np
import pytest

from golden_io import load, names

pytestmark = pytest.mark.gpu

TOL = {"f32": 3e-6, "f16": 1e-4, "bf16": 6e-4}  # pylbm's tests/test_equivalence.py:21
# pylbm's own equivalence cases (the other eq_* fixtures are random-field cases)
PYLBM_CASES = ("eq_cavity2d_bgk", "eq_cavity2d_trt", "eq_cavity2d_mrt", "eq_channel2d_force",
               "eq_periodic2d_mrt_force", "eq_cavity3d_bgk", "eq_periodic3d_trt")


@pytest.fixture(scope="module")
def pylbm():
    from baseline import import_pylbm

    try:
        mod = import_pylbm()
    except ImportError as e:
        pytest.skip(str(e))
    from pylbm_b200.backend import register

    register()
    return mod


def pylbm_problem(pylbm, name: str):  # noqa: ANN001, ANN201
    from pylbm.problem import Problem

    prm = load(name)["params"]
    return Problem(tuple(prm["shape"]), tau=prm["tau"], collision=prm["collision"],
                   periodic=tuple(prm["periodic"]), u_lid=prm["u_lid"],
                   force=tuple(prm["force"]), magic=prm["magic"], s_e=prm["s_e"],
                   s_eps=prm["s_eps"])


def test_registry_lists_b200_as_pylbm_solvers(pylbm):
    import pylbm.backends as B

    st = {(b, v): (ok, why) for b, v, ok, why in B.status() if b == "b200"}
    assert set(st) == {("b200", v) for v in ("fused", "fused-aa", "fused-fp16", "fused-bf16",
                                              "fused-aa-fp16", "fused-aa-bf16", "fused-plain")}
    assert all(ok for ok, _ in st.values()), st
    for _, v in st:
        cls = B.get("b200", v)
        assert issubclass(cls, B.Solver)
        assert cls.step is B.Solver.step and cls.macroscopic is B.Solver.macroscopic
    assert ("b200", "fused") in B.available()


@pytest.mark.parametrize("variant", ["fused", "fused-aa", "fused-fp16", "fused-bf16",
                                     "fused-aa-fp16", "fused-aa-bf16", "fused-plain"])
@pytest.mark.parametrize("case", PYLBM_CASES)
def test_pylbm_equivalence_cases(pylbm, variant, case):
    import pylbm.backends as B

    assert case in names("eq_")
    p = pylbm_problem(pylbm, case)
    ok, why = B.get("b200", variant).supports(p)
    if not ok:
        pytest.skip(why)
    ref = B.make("numpy", "roll", p)
    ref.step(100)
    s = B.make("b200", variant, p)
    assert isinstance(s, B.Solver)
    s.step(100)
    f = s.populations()
    assert f.shape == ref.populations().shape
    assert np.abs(f - ref.populations()).max() < TOL[s.storage]
    # pylbm's macroscopic on the b200 state equals pylbm's on its own state, within TOL
    rho, u = s.macroscopic()
    rho_r, u_r = ref.macroscopic()
    assert np.abs(rho - rho_r).max() < 10 * TOL[s.storage]
    assert np.abs(u - u_r).max() < 10 * TOL[s.storage]


@pytest.mark.parametrize("storage,tol", [("", 1e-6), ("-fp16", TOL["f16"])])
def test_aa_equals_ab_through_pylbm(pylbm, storage, tol):
    """pylbm's AA-vs-AB check (1e-6 for fp32). In 16-bit storage the two patterns round the
    lid term at different places (AB adds it to the pulled, already rounded value; AA's odd
    step stores p - t rounded and the next pull adds t back), so they agree to the storage
    tolerance rather than bit for bit."""
    import pylbm.backends as B
    from pylbm.problem import Problem

    p = Problem((64, 40), tau=0.6, u_lid=0.1, collision="trt")
    a, b = B.make("b200", "fused" + storage, p), B.make("b200", "fused-aa" + storage, p)
    a.step(60)
    b.step(60)
    assert np.abs(a.populations() - b.populations()).max() < tol


def test_make_solver_and_unsupported(pylbm):
    import pylbm.backends as B
    from pylbm.problem import Problem
    from pylbm.validation import make_solver

    s = make_solver(Problem.cavity(48, re=100), "b200", "fused")
    s.step(10)
    assert np.isfinite(s.populations()).all()
    solid = np.zeros((20, 30), dtype=bool)
    solid[8:12, 10:14] = True
    p = Problem((30, 20), tau=0.7, periodic=(True, False), solid=solid)
    with pytest.raises(B.Unsupported):  # pylbm's own exception class
        B.make("b200", "fused-aa", p)


def test_cli_run_on_b200(pylbm, capsys):
    from pylbm.cli import main

    main(["run", "cavity", "--n", "64", "--steps", "200", "--backend", "b200",
          "--variant", "fused"])
    out = capsys.readouterr().out
    assert "b200/fused" in out and "MLUPS" in out
    main(["run", "cavity3d", "--n", "24", "--steps", "40", "--backend", "b200",
          "--variant", "fused-aa-fp16", "--collision", "trt"])
    assert "b200/fused-aa-fp16" in capsys.readouterr().out


def test_benchmark_engine_measures_b200(pylbm):
    from pylbm.benchmark import Plan, measure

    plan = Plan(name="t", sizes_2d=[256], sizes_3d=[], slow_2d=[], compile_2d=[], slow_3d=[],
                compile_3d=[], collision_size=256, repeats=2, min_time=0.05, copy_mib=64)
    lines: list = []
    rec = measure("b200", "fused", 2, 512, plan, copy_bw=6000.0, log=lines.append)
    assert rec is not None, lines
    assert rec["backend"] == "b200" and rec["value"] > 0 and rec["bytes_per_unit"] == 72
    rec = measure("b200", "fused-aa-fp16", 3, 64, plan, copy_bw=6000.0, log=lines.append)
    assert rec is not None and rec["bytes_per_unit"] == 76
