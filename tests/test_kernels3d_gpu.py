"""D3Q19 kernel families on the GPU: the register row kernel (default for the pull) and the
TMA-staged kernel (LBM_FLAG_STAGED) must both permute stored values exactly like pylbm's
streaming (checked through the oracle's stream, which is pinned to pylbm's index maps) and
agree with the one-node-per-thread kernel after full steps."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import lbm_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHAPES = [((24, 5, 4), (True, True, True)), ((16, 6, 5), (False, False, False)),
          ((40, 3, 4), (True, False, True)), ((264, 2, 3), (False, True, False)),
          ((520, 3, 2), (True, True, True)), ((256, 4, 3), (True, False, False)),
          # fully periodic rows of 64..512 nodes: 16-bit staged steps use the row-staged kernel
          ((128, 5, 4), (True, True, True)), ((256, 3, 2), (True, True, True))]
STORAGES = {"f32s": 3, "f16": 1, "bf16": 2}


def _smooth_state(p, u0=0.05):
    """Equilibrium of a periodic Taylor-Green-like velocity field on the box itself."""
    from pylbm_b200.lattice import D3Q19, equilibrium

    nz, ny, nx = p.array_shape
    z, y, x = np.meshgrid(*(2 * np.pi * np.arange(n) / n for n in (nz, ny, nx)), indexing="ij")
    u = np.stack([u0 * np.sin(x) * np.cos(y) * np.cos(z), -u0 * np.cos(x) * np.sin(y) * np.cos(z),
                  0.3 * u0 * np.sin(z) * np.cos(x)])
    return equilibrium(D3Q19, 1.0 + 0.01 * np.cos(x + 2 * y), u)


def _values(shape, storage, seed):
    rng = np.random.default_rng(seed)
    vals = rng.uniform(-1.0, 1.0, shape)
    dt = {"f32s": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[storage]
    t = torch.as_tensor(vals, dtype=torch.float32).to(dt)
    return t.to(torch.float64).numpy(), t


@pytest.mark.parametrize("flags", [0, 2], ids=["register", "staged"])
@pytest.mark.parametrize("storage", list(STORAGES))
@pytest.mark.parametrize("shape,per", SHAPES)
def test_d3q19_pull_permutation_bit_exact(flags, storage, shape, per):
    from pylbm_b200 import _lib
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    p = Problem(shape, periodic=per)
    shp = (19,) + p.array_shape
    vals, t = _values(shp, storage, seed=sum(shape))
    d = make_desc(p, STORAGES[storage])
    d.collision = _lib.STREAM_ONLY
    d.flags = flags
    src = t.reshape(-1).cuda()
    dst = torch.empty_like(src)
    _lib.call("lbm_launch", ctypes.byref(d), src.data_ptr(), dst.data_ptr(), 0, 0)
    got = dst.to(torch.float64).cpu().numpy().reshape(shp)
    case = O.Case(p.shape, p.tau, p.collision, p.periodic, 0.0, p.force)
    assert np.array_equal(got, np.stack(O.stream(vals, case)))
    assert _lib.device_error(clear=True) == 0


@pytest.mark.parametrize("flags", [0, 2], ids=["register", "staged"])
@pytest.mark.parametrize("storage", list(STORAGES))
@pytest.mark.parametrize("shape,per", SHAPES)
def test_d3q19_aa_pair_permutation_bit_exact(flags, storage, shape, per):
    """One AA pair (odd step in place, then even step) of stream-only steps on the swapped
    layout equals two pulls of the oracle's stream, value for value."""
    from pylbm_b200 import _lib
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    p = Problem(shape, periodic=per)
    shp = (19,) + p.array_shape
    vals, t = _values(shp, storage, seed=sum(shape) + 7)
    d = make_desc(p, STORAGES[storage])
    d.collision = _lib.STREAM_ONLY
    d.flags = flags
    opp = p.lattice.opp
    buf = t[opp].reshape(-1).contiguous().cuda()
    _lib.call("lbm_advance", ctypes.byref(d), buf.data_ptr(), buf.data_ptr(), 1, 2, 0)
    got = buf.to(torch.float64).cpu().numpy().reshape(shp)[opp]
    case = O.Case(p.shape, p.tau, p.collision, p.periodic, 0.0, p.force)
    assert np.array_equal(got, np.stack(O.stream(np.stack(O.stream(vals, case)), case)))
    assert _lib.device_error(clear=True) == 0


@pytest.mark.parametrize("flags", [0, 2], ids=["register", "staged"])
@pytest.mark.parametrize("variant", ["fused", "fused-fp16", "fused-aa", "fused-aa-bf16"])
@pytest.mark.parametrize("coll,extra", [("trt", {"periodic": (True, True, True)}),
                                        ("bgk", {"u_lid": 0.06}),
                                        ("trt", {"periodic": (True, False, False),
                                                 "force": (1e-5, 0.0, -2e-5)})])
def test_d3q19_kernels_match_generic(flags, variant, coll, extra):
    from pylbm_b200 import _lib
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.problem import Problem

    p = Problem((264, 10, 9), tau=0.57, collision=coll, **extra)
    f0 = _smooth_state(p)
    a = VARIANTS[variant](p)
    g = VARIANTS[variant](p)
    a.desc.flags = flags
    g.desc.flags = _lib.FLAG_GENERIC
    for s in (a, g):
        s.set_populations(f0)
        s.step(12)
    if a.storage == "f32":
        diff = np.abs(a.populations() - g.populations()).max()
        assert diff < 1e-6, diff
    else:  # 16-bit: the same explicitly rounded collision, bit for bit
        assert np.array_equal(a.populations(), g.populations())


@pytest.mark.parametrize("variant", ["fused-fp16", "fused-bf16"])
@pytest.mark.parametrize("coll,force", [("trt", None), ("bgk", (1e-5, -2e-6, 3e-6))])
@pytest.mark.parametrize("nx", [64, 128, 512])
def test_d3q19_row_staged_kernel_matches_generic(variant, coll, force, nx):
    """The row-staged 16-bit kernel (whole periodic rows, two nodes per thread, packed
    collisions) gives the generic kernel's result bit for bit."""
    from pylbm_b200 import _lib
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.problem import Problem

    p = Problem((nx, 12, 10), tau=0.58, collision=coll, periodic=(True, True, True),
                force=force)
    f0 = _smooth_state(p)
    a, g = VARIANTS[variant](p), VARIANTS[variant](p)
    a.desc.flags = _lib.FLAG_STAGED
    g.desc.flags = _lib.FLAG_GENERIC
    for s in (a, g):
        s.set_populations(f0)
        s.step(12)
    assert _lib.device_error() == 0
    assert np.array_equal(a.populations(), g.populations())


@pytest.mark.parametrize("variant", ["fused", "fused-fp16", "fused-aa", "fused-aa-bf16"])
@pytest.mark.parametrize("shape,extra", [
    # rows shorter than a warp share it in power-of-two segments: whole periodic rows (fp16
    # 16 lanes, fp32 32), walls on every axis (8 / 16 lanes; a warp holds rows next to a wall
    # and rows that are not), partial segments (5 of 8 / 10 of 16 lanes) with a force
    ((128, 12, 9), {"collision": "trt", "periodic": (True, True, True)}),
    ((64, 12, 9), {"collision": "bgk", "u_lid": 0.06}),
    ((40, 12, 9), {"collision": "trt", "periodic": (True, False, False),
                   "force": (1e-5, 0.0, -2e-5)}),
    ((8, 20, 9), {"collision": "bgk", "periodic": (True, True, False), "u_lid": 0.05}),
])
def test_d3q19_short_rows_match_generic(variant, shape, extra):
    """The register row kernels on rows of fewer than 32 lanes give the generic kernel's
    result (bit for bit in 16-bit storage)."""
    from pylbm_b200 import _lib
    from pylbm_b200.backend import VARIANTS
    from pylbm_b200.problem import Problem

    p = Problem(shape, tau=0.57, **extra)
    f0 = _smooth_state(p)
    a, g = VARIANTS[variant](p), VARIANTS[variant](p)
    g.desc.flags = _lib.FLAG_GENERIC
    for s in (a, g):
        s.set_populations(f0)
        s.step(12)
    assert _lib.device_error() == 0
    if a.storage == "f32":
        diff = np.abs(a.populations() - g.populations()).max()
        assert diff < 1e-6, diff
    else:
        assert np.array_equal(a.populations(), g.populations())
