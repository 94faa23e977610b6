"""lbm_moments_f64_noalloc, the allocation-free FP64 moment sums, through the C ABI.

Callers that cannot let a library allocate device memory (their own pool owns it all, or a
long loop must not risk an allocation stall or failure) use this entry point instead of
lbm_moments_f64, which takes stream-ordered scratch on every call. It must give the same
sums: two calls in a row, on two different states, each compared with the allocating entry
point within the moment tests' tolerance (rtol 1e-12). The file is collected last so that a
run stopping at the first failure has already run every other test; it also passes alone.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _state(p, storage_id, seed):
    """A seeded stored state (f - w_i of magnitude ~1e-2) made on the device."""
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    h = (torch.rand(p.lattice.q * p.n_nodes, device="cuda", generator=g) - 0.5) * 0.02
    dt = {3: torch.float32, 1: torch.float16, 2: torch.bfloat16}[storage_id]
    return h.to(dt)


@pytest.mark.parametrize("lattice_shape,storage_id", [((512, 384), 3), ((48, 40, 36), 1),
                                                      ((4096, 4096), 2)])
def test_noalloc_moments_match_allocating_entry_point(lattice_shape, storage_id):
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
        assert lib.lbm_moments_f64(ctypes.byref(d), buf.data_ptr(), 0, want.data_ptr(),
                                   stream) == 0
        assert lib.lbm_moments_f64_noalloc(ctypes.byref(d), buf.data_ptr(), 0, got.data_ptr(),
                                           stream) == 0
        torch.cuda.synchronize()
        np.testing.assert_allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=1e-12,
                                   atol=1e-9)


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
