"""The validation drivers' problems, checked without a GPU: the restated Schaefer-Turek 2D-2
lattice (karman.py:21-42) reproduces pylbm's own at 4 nodes per diameter (the fixture made by
running pylbm: shape, relaxation time, solid cylinder, inlet profile and initial state), and
the Poiseuille parabola is pylbm's (poiseuille.py:10-14)."""

from __future__ import annotations

import numpy as np
import pytest

from golden_io import load


def test_schafer_turek_lattice_matches_pylbm():
    from pylbm_b200.validation import schafer_turek_problem

    d = load("inout_karman_trt")
    p = schafer_turek_problem(d=4, u_mean=0.05, collision="trt")
    assert list(p.shape) == d["params"]["shape"]
    assert p.tau == d["params"]["tau"] and p.collision == d["params"]["collision"]
    assert np.array_equal(p.solid, d["solid"])
    assert np.array_equal(p.inlet, d["inlet"]) and p.outlet
    assert np.array_equal(p.initial_populations(), d["f0"])


def test_poiseuille_parabola():
    from pylbm_b200.validation import poiseuille_analytic

    h, force, nu = 12, 1e-6, 0.1
    u = poiseuille_analytic(h, force, nu)
    y = np.arange(h) + 0.5
    assert np.allclose(u, force / (2 * nu) * y * (h - y))
    assert np.allclose(u, u[::-1])  # symmetric about the channel centre


def test_ghia_measurement_equals_pylbms():
    """The centreline profiles and error norms of the Ghia driver equal pylbm's
    (validation/ghia.py:39-80) on arbitrary fields, odd and even sizes, every Re."""
    from baseline import import_pylbm

    try:
        import_pylbm()
    except ImportError as e:
        pytest.skip(str(e))
    from pylbm.validation import ghia as G

    from pylbm_b200 import validation as V

    rng = np.random.default_rng(3)
    for shape in ((48, 48), (49, 47), (129, 128)):
        ux, uy = rng.random(shape) * 0.1, rng.random(shape) * 0.1
        for re in (100, 400, 1000):
            mine = V.ghia_errors(V.cavity_centrelines(ux, uy, 0.1), re, V.ghia_reference(re))
            theirs = G.errors(G.centerlines(ux, uy, 0.1), re)
            assert mine.keys() == theirs.keys()
            for k in theirs:
                assert mine[k] == pytest.approx(theirs[k], rel=1e-14, abs=1e-15)
