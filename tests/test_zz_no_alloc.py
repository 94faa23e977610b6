"""lbm_moments_f64_noalloc, the allocation-free FP64 moment sums, through the C ABI.

Callers that cannot let a library allocate device memory (their own pool owns it all, or a
long loop must not risk an allocation stall or failure) use this entry point instead of
lbm_moments_f64, which takes stream-ordered scratch on every call. It must give the same
sums: two calls in a row, on two different states, each compared with the allocating entry
point within the moment tests' tolerance (rtol 1e-12) and with an independent float64 sum of
the decoded state; in both buffer layouts. It must also allocate nothing: across its calls
the high-water mark of the device's stream-ordered memory pool does not rise above what was
already in use, while the allocating entry point, as a control, raises it. The file is
collected last so that a run stopping at the first failure has already run every other test;
it also passes alone.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7  # cuda.h CUmemPool_attribute
CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8


class _Pool:
    """The current stream-ordered memory pool of device 0, read through the driver API."""

    def __init__(self) -> None:
        self.cu = ctypes.CDLL("libcuda.so.1")
        dev = ctypes.c_int()
        assert self.cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()) == 0
        self.pool = ctypes.c_void_p()
        assert self.cu.cuDeviceGetMemPool(ctypes.byref(self.pool), dev) == 0

    def _get(self, attr: int) -> int:
        v = ctypes.c_uint64()
        assert self.cu.cuMemPoolGetAttribute(self.pool, attr, ctypes.byref(v)) == 0
        return v.value

    def used_high(self) -> int:
        return self._get(CU_MEMPOOL_ATTR_USED_MEM_HIGH)

    def used_now(self) -> int:
        return self._get(CU_MEMPOOL_ATTR_USED_MEM_CURRENT)

    def reset_high(self) -> None:
        zero = ctypes.c_uint64(0)  # the only value this attribute accepts
        assert self.cu.cuMemPoolSetAttribute(self.pool, CU_MEMPOOL_ATTR_USED_MEM_HIGH,
                                             ctypes.byref(zero)) == 0


def _state(p, storage_id, seed):
    """A seeded stored state (f - w_i of magnitude ~1e-2) made on the device."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    h = (torch.rand(p.lattice.q * p.n_nodes, device="cuda", generator=g) - 0.5) * 0.02
    dt = {3: torch.float32, 1: torch.float16, 2: torch.bfloat16}[storage_id]
    return h.to(dt)


def _decoded_sums(lib, d, p, buf, layout, stream):
    """float64 mass and momentum of the decoded canonical state, summed by torch."""
    f = torch.empty(p.lattice.q * p.n_nodes, dtype=torch.float64, device="cuda")
    assert lib.lbm_decode_f64(ctypes.byref(d), buf.data_ptr(), layout, f.data_ptr(),
                              stream) == 0
    f = f.view(p.lattice.q, -1).sum(dim=1)
    c = torch.as_tensor(np.asarray(p.lattice.c, dtype=np.float64), device="cuda")
    return torch.cat([f.sum().view(1), (f[:, None] * c).sum(0)]).cpu().numpy()


@pytest.mark.parametrize("lattice_shape,storage_id,layout", [
    ((512, 384), 3, 0), ((48, 40, 36), 1, 0), ((4096, 4096), 2, 0), ((96, 80), 3, 1),
    ((40, 36, 32), 2, 1)])
def test_noalloc_moments_match_allocating_entry_point(lattice_shape, storage_id, layout):
    from pylbm_b200 import _lib
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    lib = _lib.load()
    per = (True,) * len(lattice_shape)
    p = Problem(lattice_shape, periodic=per, collision="trt")
    d = make_desc(p, storage_id)
    stream = torch.cuda.current_stream().cuda_stream
    for seed in (1, 2):  # two calls in a row: the second sees the first call's leftovers
        buf = _state(p, storage_id, seed)
        want = torch.empty(p.dim + 1, dtype=torch.float64, device="cuda")
        got = torch.full((p.dim + 1,), float("nan"), dtype=torch.float64, device="cuda")
        assert lib.lbm_moments_f64(ctypes.byref(d), buf.data_ptr(), layout, want.data_ptr(),
                                   stream) == 0
        assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), buf.data_ptr(), layout,
                                           got.data_ptr(), stream) == 0
        torch.cuda.synchronize()
        g = got.cpu().numpy()
        np.testing.assert_allclose(g, want.cpu().numpy(), rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(g, _decoded_sums(lib, d, p, buf, layout, stream),
                                   rtol=1e-10, atol=1e-7)


def test_noalloc_allocates_nothing():
    from pylbm_b200 import _lib
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    lib = _lib.load()
    p = Problem((2048, 1024), periodic=(True, True))
    d = make_desc(p, 3)
    buf = _state(p, 3, 5)
    out = torch.empty(3, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    pool = _Pool()
    # the first call on the device does the one-time address look-up; then count from zero
    assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), buf.data_ptr(), 0, out.data_ptr(),
                                       stream) == 0
    torch.cuda.synchronize()
    base = pool.used_now()  # memory of the pool others hold (normally none)
    pool.reset_high()
    for _ in range(2):
        assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), buf.data_ptr(), 0,
                                           out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert pool.used_high() <= base
    # control: the allocating entry point does show up in the same counter
    assert lib.lbm_moments_f64(ctypes.byref(d), buf.data_ptr(), 0, out.data_ptr(), stream) == 0
    torch.cuda.synchronize()
    assert pool.used_high() > base


def test_noalloc_rejects_bad_arguments():
    from pylbm_b200 import _lib
    from pylbm_b200.backend import make_desc
    from pylbm_b200.problem import Problem

    lib = _lib.load()
    d = make_desc(Problem((64, 32), periodic=(True, True)), 3)
    out = torch.empty(3, dtype=torch.float64, device="cuda")
    assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), None, 0, out.data_ptr(), 0) == -1
    buf = torch.zeros(9 * 64 * 32, dtype=torch.float32, device="cuda")
    assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), buf.data_ptr(), 5, out.data_ptr(),
                                       0) == -15
