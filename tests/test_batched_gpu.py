"""Batched uneven lattices on the GPU: every lattice of a batch evolves exactly as it does
in its own single-lattice solver (same row code and arithmetic), graph replay equals plain
launches, results stay within pylbm's tolerances of the float64 oracle, and the autotuner
leaves the state untouched."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = {"f32": 3e-6, "f16": 1e-4, "bf16": 6e-4}


def _problems(collision, count=6, seed=3):
    from pylbm_b200 import workloads as W

    return W.cavity_batch_problems(count=count, lo=16, hi=96, seed=seed, collision=collision)


@pytest.mark.parametrize("variant", ["fused", "fused-fp16", "fused-bf16", "fused-plain"])
@pytest.mark.parametrize("collision", ["mrt", "bgk", "trt"])
def test_batch_matches_single_lattice_solvers(variant, collision):
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.batched import BatchedSolver
    from pylbm_b200.problem import Problem

    probs = _problems(collision)
    probs.append(Problem((40, 24), tau=0.7, collision=collision, periodic=(True, True)))
    rng = np.random.default_rng(1)
    b = BatchedSolver(probs, variant)
    f0 = []
    for i, p in enumerate(probs):  # random states so every lattice moves
        from pylbm_b200.lattice import equilibrium

        f = equilibrium(p.lattice, 1 + 0.01 * rng.standard_normal(p.array_shape),
                        0.04 * (rng.random((2,) + p.array_shape) - 0.5))
        f0.append(f)
        b.set_populations(i, f)
    b.step(25)
    for i, p in enumerate(probs):
        s = VARIANTS[variant](p)
        s.set_populations(f0[i])
        s.step(25)
        assert np.array_equal(b.populations(i), s.populations()), i
    b.close()


def test_graph_replay_equals_plain_launches():
    from pylbm_b200.batched import BatchedSolver

    probs = _problems("mrt", count=9, seed=5)
    g = BatchedSolver(probs, "fused-fp16")
    k = BatchedSolver(probs, "fused-fp16")
    g.step(31, graph=True)
    g.step(31, graph=True)  # the cached graph, replayed
    k.step(62, graph=False)
    for i in range(len(probs)):
        assert np.array_equal(g.populations(i), k.populations(i))
    g.close()
    k.close()


@pytest.mark.parametrize("variant", ["fused", "fused-fp16"])
def test_batch_against_float64_oracle(variant):
    from pylbm_b200.batched import BatchedSolver

    probs = _problems("mrt", count=4, seed=7)
    b = BatchedSolver(probs, variant)
    b.step(120)
    for i, p in enumerate(probs):
        case = O.Case(p.shape, p.tau, p.collision, p.periodic, p.u_lid)
        ref = O.run(case, p.initial_populations(), 120)
        assert np.abs(b.populations(i) - ref).max() < TOL[b.storage], i
        rho, u = O.macroscopic(ref, case)
        uv = b.velocity(i).double().cpu().numpy()
        assert np.abs(uv - np.stack(u)).max() < (1e-6 if b.storage == "f32" else 2e-3) * p.u_lid
    b.close()


def test_autotune_preserves_state_and_caches(tmp_path):
    from pylbm_b200.autotune import autotune_batch
    from pylbm_b200.batched import BatchedSolver

    probs = _problems("mrt", count=8, seed=9)
    b = BatchedSolver(probs, "fused-fp16")
    b.step(10)
    before = [b.populations(i) for i in range(len(probs))]
    r = autotune_batch(b, steps=4, reps=1, path=tmp_path / "tune.json")
    assert not r["cached"] and tuple(r["launch"]) == b.launch
    assert all(np.array_equal(before[i], b.populations(i)) for i in range(len(probs)))
    assert b.steps_done == 10
    r2 = autotune_batch(b, path=tmp_path / "tune.json")
    assert r2["cached"] and r2["launch"] == r["launch"]
    b.step(10)
    assert all(np.isfinite(b.populations(i)).all() for i in range(len(probs)))
    b.close()


def test_batch_rejects_ragged_rows():
    from pylbm_b200._lib import LbmError
    from pylbm_b200.batched import BatchedSolver
    from pylbm_b200.problem import Problem

    with pytest.raises(LbmError):
        BatchedSolver([Problem((36, 20), u_lid=0.05, collision="mrt")], "fused-fp16")
