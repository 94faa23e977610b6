"""The Ghia, Ghia & Shin (1982) lid-driven cavity on the b200 backend (pylbm's
validation/ghia.py:96-132 driver restated with device velocities). The tables are read from
pylbm's installed data file; skipped when pylbm is not installed. Bars: pylbm's own test
(tests/test_reference.py:34-38: Re = 100 on 48^2 converges with L-inf < 0.03) on every
storage, and tighter ones on a finer grid."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _pylbm():
    from baseline import import_pylbm

    try:
        import_pylbm()
    except ImportError as e:
        pytest.skip(str(e))


@pytest.mark.parametrize("variant", ["fused", "fused-aa", "fused-fp16", "fused-plain"])
def test_ghia_re100_48(variant):
    from pylbm_b200.validation import run_ghia

    r = run_ghia(100, 48, variant=variant, tol=1e-6 if "fp16" not in variant else 1e-5)
    print(f"\nGhia Re=100 48^2 {variant}: {r['steps']} steps, {r['converged']}, "
          f"Linf {r['errors']['Linf']:.4f}, L2 {r['errors']['L2']:.4f}")
    assert r["converged"]
    assert r["errors"]["Linf"] < 0.03


# pylbm's recorded runs of the same driver (results/validation.json, "ghia"): Re, n,
# variant, collision, its L-inf error
RECORDED = [(100, 128, "fused", "bgk", 0.00587), (100, 64, "fused", "bgk", 0.00603),
            (400, 256, "fused", "bgk", 0.0047), (1000, 256, "fused", "bgk", 0.00805),
            (1000, 256, "fused", "trt", 0.00742), (1000, 256, "fused", "mrt", 0.00823),
            (1000, 256, "fused-aa", "bgk", 0.00805), (100, 128, "fused-fp16", "bgk", 0.00504),
            (1000, 256, "fused-aa-fp16", "bgk", 0.01288)]


@pytest.mark.parametrize("re,n,variant,collision,linf", RECORDED)
def test_ghia_matches_pylbms_recorded_runs(re, n, variant, collision, linf):
    from pylbm_b200.validation import run_ghia

    r = run_ghia(re, n, collision=collision, variant=variant)
    print(f"\nGhia Re={re} {n}^2 {variant} {collision}: {r['steps']} steps, {r['converged']}, "
          f"Linf {r['errors']['Linf']:.5f} (pylbm {linf}), L2 {r['errors']['L2']:.5f}")
    assert r["converged"]
    assert r["errors"]["Linf"] <= 1.25 * linf + 0.002
