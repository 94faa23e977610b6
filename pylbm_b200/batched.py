"""Many independent D2Q9 lattices of uneven sizes advanced together.

``BatchedSolver`` holds every lattice's populations back to back in one pair of torch CUDA
buffers; one kernel launch advances all lattices by one time step (``lbm_batch_step``), and
``step(n)`` replays n such launches from one captured CUDA graph (``lbm_batch_graph_launch``).
The launch shape is chosen by :func:`pylbm_b200.autotune.autotune_batch`. pylbm has no
counterpart (one solver per lattice); per lattice the update is exactly the single-lattice
fused step, so each lattice's state can be exchanged with pylbm's canonical float64 layout.
"""

from __future__ import annotations

import ctypes
from typing import Any, Sequence

import numpy as np

from . import _lib
from .backend import VARIANTS, Unsupported, _stream, cuda_ok, make_desc

try:
    import torch
except Exception:  # pragma: no cover
    torch = None  # type: ignore[assignment]


class BatchedSolver:
    """A batch of D2Q9 box problems sharing collision operator and storage format.

    ``variant`` names the storage as pylbm's fused variants do ("fused" = fp32 with shifted
    arithmetic, "fused-fp16", "fused-bf16", "fused-plain"). Every lattice's nx must be a
    multiple of 4 (fp32) or 8 (16-bit) elements."""

    def __init__(self, problems: Sequence[Any], variant: str = "fused-fp16",
                 device: Any = None) -> None:
        ok, why = cuda_ok()
        if not ok:
            raise Unsupported(f"batched lattices unavailable: {why}")
        cls = VARIANTS[variant]
        if cls.aa:
            raise Unsupported("batched lattices use the two-buffer pull")
        self.problems = list(problems)
        if not self.problems:
            raise ValueError("empty batch")
        for p in self.problems:
            ok, why = cls.supports(p)
            if not ok or p.dim != 2 or getattr(p, "solid", None) is not None or p.has_force:
                raise Unsupported(f"batched lattices need D2Q9 boxes without forces: {why}")
        self.variant = variant
        self.storage = cls.storage
        self.itemsize = cls.itemsize
        self.dev = torch.device(device or "cuda")
        sid = cls.storage_id()
        n = len(self.problems)
        self.descs = (_lib.LbmDesc * n)(*[make_desc(p, sid) for p in self.problems])
        self.handle = ctypes.c_void_p()
        _lib.call("lbm_batch_create", self.descs, n, ctypes.byref(self.handle))
        elems, nodes, items = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int()
        _lib.call("lbm_batch_info", self.handle, ctypes.byref(elems), ctypes.byref(nodes),
                  ctypes.byref(items))
        self.elements, self.nodes, self.items = elems.value, nodes.value, items.value
        offs = (ctypes.c_int64 * n)()
        _lib.call("lbm_batch_offsets", self.handle, offs)
        self.offsets = list(offs)
        dtype = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[self.storage]
        self.A = torch.empty(self.elements, dtype=dtype, device=self.dev)
        self.B = torch.empty_like(self.A)
        self.steps_done = 0
        for i, p in enumerate(self.problems):
            self.set_populations(i, p.initial_populations())

    # ------------------------------------------------------------------ state
    def _slice_ptr(self, t: Any, i: int) -> int:
        return t.data_ptr() + self.offsets[i] * t.element_size()

    def set_populations(self, i: int, f: np.ndarray) -> None:
        """Load lattice i's canonical float64 post-collision state (9, ny, nx)."""
        p = self.problems[i]
        f = np.ascontiguousarray(np.asarray(f, dtype=np.float64))
        if f.shape != (9,) + tuple(p.array_shape):
            raise ValueError(f"lattice {i}: populations must have shape {(9,) + tuple(p.array_shape)}")
        t = torch.from_numpy(f).to(self.dev)
        _lib.call("lbm_encode_f64", ctypes.byref(self.descs[i]), t.data_ptr(),
                  self._slice_ptr(self.A, i), _lib.LAYOUT_NATURAL, _stream())
        torch.cuda.current_stream().synchronize()

    def populations(self, i: int) -> np.ndarray:
        p = self.problems[i]
        out = torch.empty(9 * p.n_nodes, dtype=torch.float64, device=self.dev)
        _lib.call("lbm_decode_f64", ctypes.byref(self.descs[i]), self._slice_ptr(self.A, i),
                  _lib.LAYOUT_NATURAL, out.data_ptr(), _stream())
        return out.cpu().numpy().reshape((9,) + tuple(p.array_shape))

    def velocity(self, i: int) -> Any:
        """Physical velocity (2, ny, nx) of lattice i as a float32 device tensor."""
        p = self.problems[i]
        rho = torch.empty(p.n_nodes, dtype=torch.float32, device=self.dev)
        u = torch.empty(2 * p.n_nodes, dtype=torch.float32, device=self.dev)
        _lib.call("lbm_macroscopic", ctypes.byref(self.descs[i]), self._slice_ptr(self.A, i),
                  _lib.LAYOUT_NATURAL, rho.data_ptr(), u.data_ptr(), _stream())
        return u.view((2,) + tuple(p.array_shape))

    # ------------------------------------------------------------------ stepping
    @property
    def launch(self) -> tuple[int, int]:
        blk, bps = ctypes.c_int(), ctypes.c_int()
        _lib.call("lbm_batch_get_launch", self.handle, ctypes.byref(blk), ctypes.byref(bps))
        return blk.value, bps.value

    def set_launch(self, block: int, blocks_per_sm: int) -> None:
        _lib.call("lbm_batch_set_launch", self.handle, int(block), int(blocks_per_sm))

    def step(self, n: int = 1, graph: bool = True) -> None:
        """Advance every lattice n steps: one launch per step, replayed from a CUDA graph."""
        if n <= 0:
            return
        fn = "lbm_batch_graph_launch" if graph else "lbm_batch_step"
        _lib.call(fn, self.handle, self.A.data_ptr(), self.B.data_ptr(), int(n), _stream())
        if n % 2:
            self.A, self.B = self.B, self.A
        self.steps_done += n

    def synchronize(self) -> None:
        torch.cuda.synchronize(self.dev)

    @property
    def bytes_per_node(self) -> int:
        return 2 * 9 * self.itemsize

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.load().lbm_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self) -> None:  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass
