"""The D3Q19 MRT collision of the oracle (no pylbm counterpart: pylbm's MRT is D2Q9 only, so
this row is pinned by algebra, not by fixtures): the moment basis is orthogonal with the row
norms published by d'Humieres et al. (2002); with every rate equal to 1/tau the collision is
BGK, with and without a body force; mass and momentum are conserved; the rate of each moment
follows the convention of the CUDA library (lattice.cuh mrt_rate_slot)."""

from __future__ import annotations

import numpy as np

from oracle import lbm_oracle as O

# d'Humieres et al. (2002), squared norms of (rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx,
# 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz)
PUBLISHED_NORMS = (19, 2394, 252, 10, 40, 10, 40, 10, 40, 36, 72, 12, 24, 4, 4, 4, 8, 8, 8)


def _state(shape, seed):
    rng = np.random.default_rng(seed)
    arr = shape[::-1]
    return O.equilibrium(O.D3Q19, 1 + 0.01 * rng.standard_normal(arr),
                         0.03 * rng.standard_normal((3,) + arr)) + 1e-4 * rng.standard_normal(
        (19,) + arr)


def test_basis_is_orthogonal_with_the_published_norms():
    M = np.array(O.MRT3_M, dtype=np.int64)
    G = M @ M.T
    assert np.array_equal(G, np.diag(np.diag(G)))
    assert tuple(np.diag(G)) == PUBLISHED_NORMS
    assert O.MRT3_NORM == tuple(float(v) for v in PUBLISHED_NORMS)


def test_equal_rates_give_bgk():
    f = _state((6, 5, 4), 1)
    for force in ((0.0, 0.0, 0.0), (1e-5, -2e-6, 3e-6)):
        mrt = O.Case((6, 5, 4), 0.8, "mrt", (True,) * 3, force=force)
        bgk = O.Case((6, 5, 4), 0.8, "bgk", (True,) * 3, force=force)
        mrt.mrt_rates = lambda: (1.0 / 0.8,) * 19
        a = O.collide(list(f), mrt)
        b = O.collide(list(f), bgk)
        assert np.abs(a - b).max() < 1e-15


def test_mass_and_momentum_are_conserved():
    case = O.Case((8, 6, 5), 0.7, "mrt", (True,) * 3)
    f = _state((8, 6, 5), 2)
    c = np.array(O.D3Q19.c, dtype=np.float64)
    def mom(x):  # noqa: ANN001, ANN202
        return c.T @ x.reshape(19, -1).sum(axis=1)

    m0, j0 = f.sum(), mom(f)
    g = O.run(case, f, 20)
    assert abs(g.sum() - m0) < 1e-11 * abs(m0)
    assert np.abs(mom(g) - j0).max() < 1e-12


def test_rate_convention():
    case = O.Case((4, 4, 4), 0.7, "mrt", (True,) * 3, s_e=1.3, s_eps=1.5)
    s = case.mrt_rates()
    s_nu, s_q = 1.0 / 0.7, O.magic_rate(1.0 / 0.7)
    assert [s[k] for k in (0, 3, 5, 7)] == [0.0] * 4
    assert s[1] == 1.3 and [s[k] for k in (2, 10, 12)] == [1.5] * 3
    assert [s[k] for k in (4, 6, 8, 16, 17, 18)] == [s_q] * 6
    assert [s[k] for k in (9, 11, 13, 14, 15)] == [s_nu] * 5
