"""C ABI checks that need no GPU: the library loads, exports every declared symbol, its
compiled lattice tables match pylbm's, and argument validation rejects bad descriptors."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import lbm_oracle as O
from pylbm_b200 import _lib
from pylbm_b200.backend import make_desc, solid_bits
from pylbm_b200.problem import Problem

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        names += re.findall(r"^\s*(?:int|const char\*|double|void)\s+\*?(lbm_\w+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = declared_symbols()
    assert "lbm_launch" in names and "lbm_advance" in names
    for n in names:
        assert hasattr(lib, n), n
    assert lib.lbm_abi_version() == 2


@pytest.mark.parametrize("lat,ref", [(_lib.D2Q9, O.D2Q9), (_lib.D3Q19, O.D3Q19)])
def test_compiled_lattice_tables_match_pylbm(lat, ref):
    info = _lib.lattice_info(lat)
    assert info["q"] == ref.q and info["d"] == ref.d
    assert np.array_equal(info["c"], np.array(ref.c))
    assert np.array_equal(info["w"], np.array(ref.w))
    assert np.array_equal(info["opp"], np.array(ref.opp))


def _validate(d) -> int:
    return _lib.load().lbm_validate(ctypes.byref(d))


def test_validate_accepts_pylbm_problems():
    for p in (Problem.cavity(128, re=100), Problem((64, 32), periodic=(True, True), collision="trt"),
              Problem((16, 12, 10), collision="trt", periodic=(True, True, False), force=(1e-5, 0, 0)),
              Problem((32, 24), collision="mrt", u_lid=0.1)):
        for st in range(4):
            assert _validate(make_desc(p, st)) == 0


@pytest.mark.parametrize("field,value,code", [
    ("lattice", 7, -2), ("collision", 5, -3), ("storage", 9, -4), ("nx", 0, -6),
    ("nz", 3, -6), ("r0", 2.5, -8), ("r0", float("nan"), -8), ("fx", float("inf"), -8),
    ("ny", 70000, -6),
])
def test_validate_rejects(field, value, code):
    d = make_desc(Problem((64, 32), periodic=(True, True)), _lib.STORE_F32)
    setattr(d, field, value)
    assert _validate(d) == code
    assert _lib.error_string(code) != "unknown error"


def test_validate_mrt_3d_lid_periodic_and_index_limit():
    assert _validate(make_desc(Problem((8, 8, 8), collision="mrt"), 0)) == 0  # D3Q19 MRT
    d = make_desc(Problem((8, 8, 8), collision="trt"), 0)
    d.collision = _lib.MRT  # the TRT descriptor leaves r2, r3 at zero: not MRT rates
    assert _validate(d) == -8
    d = make_desc(Problem((8, 8), periodic=(True, False), u_lid=0.1), 0)
    d.periodic_mask = 3
    assert _validate(d) == -9
    d = make_desc(Problem((8, 8), periodic=(True, True)), 0)
    d.nx, d.ny = 1 << 15, 1 << 13  # 9 * 2^28 >= 2^31
    assert _validate(d) == -7
    d = make_desc(Problem((8, 8), periodic=(True, True)), 0)
    d.mx_force = 8  # momentum exchange without solids
    assert _validate(d) == -15


def test_launch_rejects_bad_buffers_without_touching_the_gpu():
    lib = _lib.load()
    d = make_desc(Problem((64, 32), periodic=(True, True)), _lib.STORE_F32)
    assert lib.lbm_launch(ctypes.byref(d), None, None, 0, 0) == -1
    assert lib.lbm_launch(ctypes.byref(d), 64, 64, 0, 0) == -11     # AB aliasing
    assert lib.lbm_launch(ctypes.byref(d), 64, 128, 1, 0) == -11    # AA needs src == dst
    assert lib.lbm_launch(ctypes.byref(d), 66, 128, 0, 0) == -10    # misaligned fp32
    assert lib.lbm_launch(ctypes.byref(d), 64, 128, 7, 0) == -5     # pattern
    assert lib.lbm_advance(ctypes.byref(d), 64, 64, 1, 3, 0) == -12  # odd AA count
    assert lib.lbm_advance(ctypes.byref(d), 64, 128, 0, -1, 0) == -12
    d.solid_bits = 64
    assert lib.lbm_launch(ctypes.byref(d), 64, 64, 1, 0) == -15     # AA with solids


def test_inlet_outlet_validation_without_touching_the_gpu():
    """Inlet / outlet (pylbm's Problem.inlet / outlet) need D2Q9, walls on x and the AB pull."""
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    lib = _lib.load()
    d = make_desc(Problem((64, 32)), _lib.STORE_F32)
    d.outlet = 1
    assert lib.lbm_validate(ctypes.byref(d)) == 0
    d.inlet_u = 256
    assert lib.lbm_validate(ctypes.byref(d)) == 0
    assert lib.lbm_launch(ctypes.byref(d), 64, 64, 1, 0) == -17     # AA with open boundaries
    d.inlet_u = 258
    assert lib.lbm_validate(ctypes.byref(d)) == -10                 # misaligned profile
    d.inlet_u = 256
    d.outlet = 2
    assert lib.lbm_validate(ctypes.byref(d)) == -15
    d.outlet = 1
    d.periodic_mask = 1                                             # periodic x
    assert lib.lbm_validate(ctypes.byref(d)) == -17
    d3 = make_desc(Problem((16, 8, 8)), _lib.STORE_F32)
    d3.outlet = 1
    assert lib.lbm_validate(ctypes.byref(d3)) == -17
    assert "inlet" in lib.lbm_error_string(-17).decode()


def test_backend_supports_inlet_outlet_on_two_buffer_d2q9():
    import numpy as np

    from pylbm_b200 import backend as B
    from pylbm_b200.problem import Problem

    p = Problem((40, 12), inlet=np.full(12, 0.05), outlet=True)
    assert B.B200Fused.supports(p)[0] and B.B200FusedFP16.supports(p)[0]
    assert not B.VARIANTS["fused-aa"].supports(p)[0]
    assert not B.B200Fused.supports(Problem((40, 12), periodic=(True, False), outlet=True))[0]


def test_solid_bit_packing():
    rng = np.random.default_rng(0)
    m = rng.random((7, 13)) < 0.3
    bits = solid_bits(m)
    flat = m.reshape(-1)
    for n in range(flat.size):
        assert bool((bits[n >> 5] >> (n & 31)) & 1) == flat[n]
