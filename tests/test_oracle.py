"""The oracle reproduces pylbm's float64 results (fixtures made by running pylbm)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import lbm_oracle as O
from tests.golden_io import case_of, initial, load, names


@pytest.mark.parametrize("name", names("eq_") + ["config1"])
def test_oracle_matches_pylbm(name):
    d = load(name)
    case = case_of(d)
    f = O.run(case, initial(d, case), int(d["steps"]))
    # same operations in the same order: bitwise
    assert np.array_equal(f, d["f"])


def test_oracle_macroscopic_matches_pylbm():
    d = load("config1")
    case = case_of(d)
    rho, u = O.macroscopic(d["f"], case)
    assert np.array_equal(rho, d["rho"])
    assert np.array_equal(np.stack(u), d["u"])


@pytest.mark.parametrize("name", names("solid_"))
def test_oracle_solids_and_momentum_exchange(name):
    d = load(name)
    case = case_of(d)
    f = initial(d, case)
    masks = O.force_masks(case)
    src = O.solid_sources(case)
    hist = []
    for _ in range(int(d["steps"])):
        f = O.step(f, case, np, src)
        hist.append(O.momentum_exchange(f, case, masks))
    assert np.array_equal(f, d["f"])
    np.testing.assert_allclose(np.array(hist), d["force_hist"], rtol=1e-13, atol=1e-18)


@pytest.mark.parametrize("name", names("inout_"))
def test_oracle_inlet_outlet(name):
    """Velocity inlet and pressure outlet (core.py:67-78,116-117,130-148) reproduce pylbm bit
    for bit, with a solid disc and the momentum-exchange force where the fixture has them."""
    d = load(name)
    case = case_of(d)
    f = initial(d, case)
    masks = O.force_masks(case) if case.solid is not None else None
    src = O.solid_sources(case) if case.solid is not None else None
    hist = []
    for _ in range(int(d["steps"])):
        f = O.step(f, case, np, src)
        if masks is not None:
            hist.append(O.momentum_exchange(f, case, masks))
    assert np.array_equal(f, d["f"])
    if "force_hist" in d:
        np.testing.assert_allclose(np.array(hist), d["force_hist"], rtol=1e-13, atol=1e-18)


@pytest.mark.parametrize("name", names("tags_"))
def test_oracle_stream_index_map(name):
    d = load(name)
    case = case_of(d)
    lat = case.lat
    shp = (lat.q,) + case.array_shape
    still = O.Case(case.shape, case.tau, case.collision, case.periodic, 0.0, case.force,
                   solid=case.solid)
    src = np.stack(O.stream(np.arange(np.prod(shp), dtype=np.float64).reshape(shp), still))
    assert np.array_equal(src.astype(np.int64), d["src"])
    lid = np.stack(O.stream(np.zeros(shp), case))
    assert np.array_equal(lid, d["lid"])


def test_force_field_reduces_to_uniform_force():
    """A force field of zeros plus the uniform force gives pylbm's uniform-force result."""
    d = load("eq_channel2d_force")
    case = case_of(d)
    zero = np.zeros((case.dim,) + case.array_shape)
    ff = O.Case(case.shape, case.tau, case.collision, case.periodic, case.u_lid, case.force,
                force_field=zero)
    f = O.run(ff, initial(d, case), int(d["steps"]))
    np.testing.assert_allclose(f, d["f"], rtol=0, atol=1e-15)


def test_lattice_tables():
    for lat in (O.D2Q9, O.D3Q19):
        c = np.array(lat.c, float)
        w = np.array(lat.w)
        assert np.isclose(w.sum(), 1.0)
        assert np.allclose((w[:, None] * c).sum(0), 0.0)
        assert np.allclose(np.einsum("i,ia,ib->ab", w, c, c), np.eye(lat.d) / 3.0)
        assert all((c[list(lat.opp)] == -c).all(axis=1))
    M = np.array(O.MRT_M, float)
    assert np.allclose(M @ M.T, np.diag(O.MRT_NORM))
