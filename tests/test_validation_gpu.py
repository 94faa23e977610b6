"""pylbm's physical validation (tests/test_validation.py:9-19) on the B200 backend: the
shear-wave viscosity within 2 % for tau = 0.6, 1.0, 1.4; the body-force Poiseuille channel
second order for BGK and exact for TRT (here to the fp32 round-off floor instead of pylbm's
float64 1e-9)."""

from __future__ import annotations

import pytest

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["fused", "fused-aa", "fused-fp16"])
@pytest.mark.parametrize("tau", [0.6, 1.0, 1.4])
def test_shear_wave_viscosity(tau, variant):
    from pylbm_b200.validation import run_shear_wave

    r = run_shear_wave(tau, n=32, variant=variant)
    assert r["rel_error"] < 0.02, r


@pytest.mark.parametrize("variant", ["fused", "fused-aa"])
def test_poiseuille_bgk_second_order_and_trt_exact(variant):
    from pylbm_b200.validation import poiseuille_convergence, run_poiseuille

    c = poiseuille_convergence((8, 16), collision="bgk", variant=variant)
    assert 1.9 < c["order"] < 2.1, c
    r = run_poiseuille(12, collision="trt", variant=variant)
    assert r["L2"] < 2e-5, r


def test_karman_benchmark_2d2():
    """Schaefer-Turek 2D-2 at 40 nodes per diameter (pylbm's own recorded run of this lattice,
    results/validation.json: St 0.2996, cd_max 3.312, cl_max 1.005): St and the lift maximum
    within the benchmark's intervals; the drag maximum at least the benchmark's lower bound and
    within the ~2 % excess of this resolution."""
    from pylbm_b200.validation import KARMAN_REFERENCE, run_karman

    r = run_karman(d=40)
    print({k: r[k] for k in ("St", "cd_max", "cl_max", "cd_mean", "steps")})
    lo, hi = KARMAN_REFERENCE["St"]
    assert lo <= r["St"] <= hi, r["St"]
    lo, hi = KARMAN_REFERENCE["cl_max"]
    assert lo - 0.01 <= r["cl_max"] <= hi + 0.01, r["cl_max"]
    assert KARMAN_REFERENCE["cd_max"][0] <= r["cd_max"] <= 3.35, r["cd_max"]
