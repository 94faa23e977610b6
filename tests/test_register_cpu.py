"""Registration into pylbm's backend registry, without a GPU: the b200 entries resolve
through pylbm's lazy ``get`` to subclasses of pylbm's ``Solver``, never crash ``status()``,
and report themselves unavailable (no CUDA device) instead of raising. Skipped when pylbm is
not installed (``baseline/_ref`` or ``PYLBM_SRC``)."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.fixture(scope="module")
def B():  # noqa: N802
    from baseline import import_pylbm

    try:
        import_pylbm()
    except ImportError as e:
        pytest.skip(str(e))
    import pylbm.backends as backends

    from pylbm_b200.backend import register

    added = register()
    assert len(added) == 7
    return backends


def test_entries_resolve_to_pylbm_solvers(B):
    for b, v in B.entries():
        if b != "b200":
            continue
        cls = B.get(b, v)
        assert issubclass(cls, B.Solver)
        assert cls.backend == "b200" and cls.variant == v
        assert cls.step is B.Solver.step
        assert cls.bytes_per_node.fget is not None


def test_status_never_crashes_and_reports_unavailable(B):
    import torch

    st = [s for s in B.status() if s[0] == "b200"]
    assert len(st) == 7
    if not torch.cuda.is_available():
        assert all(not ok and why for _, _, ok, why in st)
        from pylbm.problem import Problem

        with pytest.raises(B.Unsupported):
            B.make("b200", "fused", Problem.cavity(16, re=10))


def test_supports_with_pylbm_problems(B):
    from pylbm.problem import Problem

    cls = B.get("b200", "fused-aa")
    assert cls.supports(Problem.cavity(32, re=100))[0]
    solid = np.zeros((8, 8), dtype=bool)
    ok, why = cls.supports(Problem((8, 8), solid=solid))
    assert not ok and "two-buffer" in why
    assert B.get("b200", "fused").supports(Problem((8, 8), solid=solid))[0]
