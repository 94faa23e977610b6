"""Gradient of a momentum-exchange drag objective with respect to a per-node force field.

The objective is J(F) = mean_{t = t0 .. T} Fx(f_t): the x momentum-exchange force on the solid
obstacles (pylbm's karman.py:45-53,88-96) averaged over the states after t0 .. T steps of the
D2Q9 BGK fused step driven by a uniform Guo force plus the control field F (2, ny, nx).

``DragAdjoint`` evaluates J with a checkpointed forward pass (state saved every ``checkpoint``
steps, default 45 ~ sqrt(2000); the force history is summed in FP64 on the GPU) and dJ/dF with
the hand-written adjoint kernel: for each segment, from the last one back, the forward steps
are recomputed from the segment's checkpoint recording rho and u (``lbm_forward_record``),
then the reverse steps run in reverse order (``lbm_adjoint_step``), accumulating dJ/dF in
FP64. ``drag_objective(F, adj)`` wraps both in a ``torch.autograd.Function``.
"""

from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from . import _lib
from .backend import B200Fused, Unsupported, _stream

try:
    import torch
except Exception:  # pragma: no cover
    torch = None  # type: ignore[assignment]


class DragAdjoint:
    """J and dJ/dF for one problem (D2Q9 BGK box with solids; the uniform force is
    ``problem.force``, the control field is passed to :meth:`objective`)."""

    def __init__(self, problem: Any, steps: int, t0: int, checkpoint: int = 45,
                 f0: np.ndarray | None = None) -> None:
        if problem.dim != 2 or problem.collision != "bgk":
            raise Unsupported("the adjoint is implemented for D2Q9 BGK")
        if getattr(problem, "solid", None) is None:
            raise Unsupported("the drag objective needs solid obstacles")
        if not 0 < t0 <= steps:
            raise ValueError("need 0 < t0 <= steps")
        self.problem = problem
        self.T, self.t0, self.K = int(steps), int(t0), int(checkpoint)
        self.solver = B200Fused(problem, force_field=np.zeros((2,) + tuple(problem.array_shape),
                                                              np.float32))
        self.dev = self.solver.dev
        self.N = problem.n_nodes
        self.f0 = problem.initial_populations() if f0 is None else np.asarray(f0, np.float64)
        self.count = self.T - self.t0 + 1
        self._checkpoints: list = []
        self.history = None
        self.J = None

    # ------------------------------------------------------------------ forward
    def objective(self, F: Any) -> float:
        """J for control field F (2, ny, nx); keeps the checkpoints for :meth:`gradient`."""
        s = self.solver
        s.set_force_field(F)
        s.set_populations(self.f0)
        s.steps_done = 0
        self._checkpoints = []
        hist = torch.zeros((self.T, 2), dtype=torch.float64, device=self.dev)
        t = 0
        while t < self.T:
            if t % self.K == 0:
                self._checkpoints.append(s.A.clone())
            n = min(self.K - t % self.K, self.T - t)
            if t + n >= self.t0:  # the chunk reaches the averaging window
                k = max(0, self.t0 - 1 - t)
                if k:
                    s.step(k)
                hist[t + k:t + n] = s.advance_with_force(n - k)
            else:
                s.step(n)
            t += n
        self.history = hist
        self.J = float(hist[self.t0 - 1:self.T, 0].sum().item()) / self.count
        return self.J

    # ------------------------------------------------------------------ reverse
    def gradient(self) -> Any:
        """dJ/dF (2, ny, nx) as a float64 device tensor (needs a prior :meth:`objective`)."""
        if not self._checkpoints:
            raise RuntimeError("call objective() first")
        s, N, K = self.solver, self.N, self.K
        desc = ctypes.byref(s.desc)
        grad = torch.zeros(2 * N, dtype=torch.float64, device=self.dev)
        mu_in = torch.empty(9 * N, dtype=torch.float32, device=self.dev)
        mu_out = torch.empty_like(mu_in)
        ru = torch.empty((K, 3 * N), dtype=torch.float32, device=self.dev)
        a = torch.empty_like(s.A)
        b = torch.empty_like(s.A)
        stream = _stream()
        first = True
        for seg in reversed(range(len(self._checkpoints))):
            t_start = seg * K
            t_end = min(t_start + K, self.T)
            a.copy_(self._checkpoints[seg])
            for k in range(t_end - t_start):  # recompute f_{t+1} from f_t, record rho, u
                _lib.call("lbm_forward_record", desc, a.data_ptr(), b.data_ptr(),
                          ru[k].data_ptr(), stream)
                a, b = b, a
            for t in reversed(range(t_start, t_end)):
                w = 1.0 / self.count if self.t0 <= t + 1 <= self.T else 0.0
                _lib.call("lbm_adjoint_step", desc, ru[t - t_start].data_ptr(),
                          None if first else mu_in.data_ptr(), mu_out.data_ptr(),
                          grad.data_ptr(), w, stream)
                first = False
                mu_in, mu_out = mu_out, mu_in
        return grad.view((2,) + tuple(self.problem.array_shape))

    # ------------------------------------------------------------------ timing helpers
    def forward_step(self, n: int = 1) -> None:
        """n plain forward steps (the unit the adjoint cost is compared with)."""
        self.solver.step(n)

    def reverse_step(self, n: int = 1) -> None:
        """n recompute + adjoint step pairs on scratch buffers (timing only). Pairs replay
        from a CUDA graph of 32, as the forward steps of a launch-bound lattice do, so the two
        are timed alike."""
        s, N = self.solver, self.N
        if not hasattr(self, "_scratch"):
            self._scratch = (torch.zeros(9 * N, device=self.dev), torch.zeros(9 * N, device=self.dev),
                             torch.zeros(3 * N, device=self.dev),
                             torch.zeros(2 * N, dtype=torch.float64, device=self.dev),
                             torch.empty_like(s.A), s.A.clone())
            self._pairs(2)  # kernel set-up outside any capture
            self._rev_graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self._rev_graph):
                self._pairs(32)
        for _ in range(n // 32):
            self._rev_graph.replay()
        self._pairs(n % 32)

    def _pairs(self, n: int) -> None:
        """n (even) recompute + adjoint step pairs on the scratch buffers, in place."""
        desc = ctypes.byref(self.solver.desc)
        mi, mo, ru, g, b, a = self._scratch
        for _ in range(n):
            _lib.call("lbm_forward_record", desc, a.data_ptr(), b.data_ptr(), ru.data_ptr(),
                      _stream())
            a, b = b, a
            _lib.call("lbm_adjoint_step", desc, ru.data_ptr(), mi.data_ptr(), mo.data_ptr(),
                      g.data_ptr(), 1.0, _stream())
            mi, mo = mo, mi
        if n % 2:  # keep the buffer roles of an even count for the captured graph
            self._scratch = (mi, mo, ru, g, b, a)


class _DragObjective(torch.autograd.Function if torch is not None else object):
    @staticmethod
    def forward(ctx: Any, F: Any, adj: DragAdjoint) -> Any:  # noqa: D102
        J = adj.objective(F.detach())
        ctx.adj = adj
        ctx.dtype = F.dtype
        return torch.tensor(J, dtype=torch.float64, device=F.device)

    @staticmethod
    def backward(ctx: Any, gJ: Any) -> Any:  # noqa: D102
        g = ctx.adj.gradient()
        return (gJ * g).to(ctx.dtype), None


def drag_objective(F: Any, adj: DragAdjoint) -> Any:
    """J(F) as a differentiable torch scalar (float64); backward runs the adjoint."""
    return _DragObjective.apply(F, adj)
