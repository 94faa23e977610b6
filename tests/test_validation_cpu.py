"""The validation drivers' problems, checked without a GPU: the restated Schaefer-Turek 2D-2
lattice (karman.py:21-42) reproduces pylbm's own at 4 nodes per diameter (the fixture made by
running pylbm: shape, relaxation time, solid cylinder, inlet profile and initial state), and
the Poiseuille parabola is pylbm's (poiseuille.py:10-14)."""

from __future__ import annotations

import numpy as np

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
