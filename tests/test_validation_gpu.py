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
