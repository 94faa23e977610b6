"""ctypes binding of the C ABI in ``include/pylbm_b200.h``.

The shared library is built in-tree (``python -m pylbm_b200.build``) into
``pylbm_b200/_lib/libpylbm_b200.so``. There is no fallback: if the library is missing every
solver reports itself unavailable and any attempt to step raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libpylbm_b200.so"

# constants mirrored from include/pylbm_b200.h
D2Q9, D3Q19 = 0, 1
BGK, TRT, MRT, STREAM_ONLY = 0, 1, 2, 3
STORE_F32, STORE_F16, STORE_BF16, STORE_F32_SHIFTED = 0, 1, 2, 3
PATTERN_AB, PATTERN_AA_ODD, PATTERN_AA_EVEN = 0, 1, 2
LAYOUT_NATURAL, LAYOUT_AA_SWAPPED = 0, 1
E_TIMEOUT = -13
FLAG_GENERIC = 1
FLAG_STAGED = 2


class LbmDesc(ctypes.Structure):
    _fields_ = [
        ("lattice", ctypes.c_int32),
        ("collision", ctypes.c_int32),
        ("storage", ctypes.c_int32),
        ("periodic_mask", ctypes.c_int32),
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("ulid", ctypes.c_float),
        ("fx", ctypes.c_float),
        ("fy", ctypes.c_float),
        ("fz", ctypes.c_float),
        ("r0", ctypes.c_float),
        ("r1", ctypes.c_float),
        ("r2", ctypes.c_float),
        ("r3", ctypes.c_float),
        ("solid_bits", ctypes.c_void_p),
        ("force_field", ctypes.c_void_p),
        ("mx_force", ctypes.c_void_p),
        ("mx_stride", ctypes.c_int64),
        ("flags", ctypes.c_int32),
        ("outlet", ctypes.c_int32),
        ("inlet_u", ctypes.c_void_p),
    ]


class LbmError(RuntimeError):
    """A non-zero status from the library (code < 0: invalid argument; > 0: CUDA error)."""

    def __init__(self, code: int, what: str) -> None:
        self.code = code
        super().__init__(f"{what}: {error_string(code)} (code {code})")


_LIB: ctypes.CDLL | None = None
_LOAD_ERROR = ""

_vp, _i, _u64, _d = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(LbmDesc)
_SIGNATURES = {
    "lbm_abi_version": ([], _i),
    "lbm_error_string": ([_i], ctypes.c_char_p),
    "lbm_lattice_info": ([_i, _vp, _vp, _vp, _vp, _vp], _i),
    "lbm_validate": ([_d], _i),
    "lbm_launch": ([_d, _vp, _vp, _i, _u64], _i),
    "lbm_advance": ([_d, _vp, _vp, _i, _i, _u64], _i),
    "lbm_moments_f64": ([_d, _vp, _i, _vp, _u64], _i),
    "lbm_moments_f64_noalloc": ([_d, _vp, _i, _vp, _u64], _i),
    "lbm_macroscopic": ([_d, _vp, _i, _vp, _vp, _u64], _i),
    "lbm_encode_f64": ([_d, _vp, _vp, _i, _u64], _i),
    "lbm_decode_f64": ([_d, _vp, _i, _vp, _u64], _i),
    "lbm_batch_create": ([_d, _i, _vp], _i),
    "lbm_batch_destroy": ([_vp], _i),
    "lbm_batch_info": ([_vp, _vp, _vp, _vp], _i),
    "lbm_batch_offsets": ([_vp, _vp], _i),
    "lbm_batch_set_launch": ([_vp, _i, _i], _i),
    "lbm_batch_get_launch": ([_vp, _vp, _vp], _i),
    "lbm_batch_step": ([_vp, _vp, _vp, _i, _u64], _i),
    "lbm_batch_graph_launch": ([_vp, _vp, _vp, _i, _u64], _i),
    "lbm_forward_record": ([_d, _vp, _vp, _vp, _u64], _i),
    "lbm_adjoint_step": ([_d, _vp, _vp, _vp, _vp, ctypes.c_double, _u64], _i),
    "lbm_set_staged_config": ([_i, _i, _i, _i, _i], _i),
    "lbm_get_staged_config": ([_i, _i, _vp, _vp, _vp], _i),
    "lbm_device_error": ([_i], _i),
    "lbm_selftest_wait_timeout": ([_d, _vp, _u64, _u64], _i),
}


def load() -> ctypes.CDLL:
    """The loaded library (raises if it was not built)."""
    global _LIB, _LOAD_ERROR
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        _LOAD_ERROR = f"{LIB_PATH.name} not built (run python -m pylbm_b200.build)"
        raise RuntimeError(_LOAD_ERROR)
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if lib.lbm_abi_version() != 2:
        raise RuntimeError("libpylbm_b200 ABI version mismatch")
    _LIB = lib
    return lib


def available() -> tuple[bool, str]:
    try:
        load()
        return True, ""
    except Exception as e:  # library missing or unloadable
        return False, str(e)


def error_string(code: int) -> str:
    try:
        return load().lbm_error_string(code).decode()
    except Exception:
        return "unknown error"


def check(code: int, what: str) -> None:
    if code != 0:
        raise LbmError(code, what)


def call(name: str, *args) -> None:  # noqa: ANN002
    """Call an int-returning entry point and raise LbmError on a non-zero status."""
    check(getattr(load(), name)(*args), name)


def staged_config(lattice: int, elem_bytes: int) -> tuple[int, int, int]:
    """(width, stages, warps) of the TMA-staged kernels."""
    w, s, k = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    call("lbm_get_staged_config", lattice, elem_bytes, ctypes.byref(w), ctypes.byref(s),
         ctypes.byref(k))
    return w.value, s.value, k.value


def set_staged_config(lattice: int, elem_bytes: int, width: int, stages: int,
                      warps: int) -> None:
    call("lbm_set_staged_config", lattice, elem_bytes, width, stages, warps)


def device_error(clear: bool = True) -> int:
    """0, or E_TIMEOUT when a kernel's bounded wait gave up (synchronises the device)."""
    return load().lbm_device_error(int(clear))


def lattice_info(lattice: int) -> dict:
    """The lattice tables compiled into the kernels."""
    import numpy as np

    q, d = ctypes.c_int(), ctypes.c_int()
    c = (ctypes.c_int * 57)()
    w = (ctypes.c_double * 19)()
    opp = (ctypes.c_int * 19)()
    call("lbm_lattice_info", lattice, ctypes.byref(q), ctypes.byref(d), c, w, opp)
    n = q.value
    return {"q": n, "d": d.value,
            "c": np.array(c[: 3 * n]).reshape(n, 3)[:, : d.value],
            "w": np.array(w[:n]), "opp": np.array(opp[:n])}
