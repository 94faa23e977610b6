"""pylbm backend ``b200``: the fused stream-collide step on the CUDA library.

Drop-in for pylbm's fused backends (``--variant fused`` / ``fused-aa``): the classes here honour
pylbm's Solver contract (backends/base.py:18-96) and FusedSolver's buffer conventions
(backends/_fused.py:42-136):

* the canonical state exchanged by ``set_populations`` / ``populations`` is the float64
  post-collision SoA array ``(q, *array_shape)``;
* buffers are flat torch CUDA tensors of ``q * N`` stored values, ``A`` and ``B`` ping-ponging
  for the two-buffer pull, a single ``A`` for the AA pattern (population i in slot opp(i)
  between step pairs), 16-bit storages holding f - w_i;
* every launch goes through the C ABI (``lbm_launch`` / ``lbm_advance``) on torch's current
  stream.

``register()`` adds the variants to pylbm's registry when pylbm is installed, so
``pylbm.backends.get("b200", "fused")`` and ``pylbm run cavity --backend b200`` work
unchanged. The module also runs without pylbm (its own ``Problem`` mirror).
"""

from __future__ import annotations

import ctypes
import sys
import types
from typing import Any, ClassVar

import numpy as np

from . import _lib
from .lattice import runtime_rates

try:
    import torch
except Exception:  # pragma: no cover - torch is a hard dependency of the GPU path
    torch = None  # type: ignore[assignment]

try:  # pylbm's own exception when pylbm is installed, so callers catch the same class
    from pylbm.backends.base import Unsupported  # type: ignore[import-not-found]
except Exception:  # pragma: no cover - stand-alone use

    class Unsupported(Exception):  # type: ignore[no-redef]
        """Raised when a backend/variant cannot run a given problem."""


_TORCH_DTYPES = {"f32": "float32", "f16": "float16", "bf16": "bfloat16"}


def cuda_ok() -> tuple[bool, str]:
    if torch is None:
        return False, "torch not installed"
    if not torch.cuda.is_available():
        return False, "no CUDA device"
    return _lib.available()


def solid_bits(solid: np.ndarray) -> np.ndarray:
    """Pack a bool node mask (array layout) into 32-bit words: bit n & 31 of word n >> 5."""
    flat = np.ascontiguousarray(np.asarray(solid, dtype=bool).reshape(-1))
    nwords = (flat.size + 31) // 32
    padded = np.zeros(nwords * 32, dtype=bool)
    padded[: flat.size] = flat
    return np.packbits(padded, bitorder="little").view("<u4").astype(np.uint32)


def make_desc(problem: Any, storage_id: int) -> _lib.LbmDesc:
    """C descriptor of a box problem: pylbm's #define header and scalar_args
    (cupy_backend.py:51-70, _fused.py:129-136) as one struct."""
    lat = problem.lattice
    shp = tuple(problem.shape) + (1,) * (3 - problem.dim)
    force = tuple(problem.force) + (0.0,) * (3 - problem.dim)
    r = runtime_rates(problem)
    d = _lib.LbmDesc()
    d.lattice = _lib.D2Q9 if lat.name == "D2Q9" else _lib.D3Q19
    d.collision = {"bgk": _lib.BGK, "trt": _lib.TRT, "mrt": _lib.MRT}[problem.collision]
    d.storage = storage_id
    d.periodic_mask = sum(1 << a for a, p in enumerate(problem.periodic) if p)
    d.nx, d.ny, d.nz = shp
    d.ulid = float(problem.u_lid)
    d.fx, d.fy, d.fz = force
    d.r0, d.r1, d.r2, d.r3 = r
    return d


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


class B200Fused:
    """Fused pull (two-buffer) stream-collide on the B200 library, fp32 storage with shifted
    (f - w) arithmetic."""

    backend: ClassVar[str] = "b200"
    variant: ClassVar[str] = "fused"
    description: ClassVar[str] = ("hand-written CUDA for sm_100a via a C ABI (ctypes), fused, "
                                  "two buffers, fp32 with shifted arithmetic")
    storage: ClassVar[str] = "f32"
    shifted: ClassVar[bool] = True
    aa: ClassVar[bool] = False
    itemsize: ClassVar[int] = 4
    step_multiple: ClassVar[int] = 1
    equivalent: ClassVar[bool] = True
    lattices: ClassVar[tuple] = ("D2Q9", "D3Q19")
    collisions: ClassVar[tuple] = ("bgk", "trt", "mrt")

    # ------------------------------------------------------------------ capabilities
    @classmethod
    def available(cls) -> tuple[bool, str]:
        return cuda_ok()

    @classmethod
    def supports(cls, problem: Any) -> tuple[bool, str]:
        if getattr(problem, "inlet", None) is not None or getattr(problem, "outlet", False):
            if cls.aa:
                return False, "inlet / outlet need the two-buffer variant (fused, fused-fp16, ...)"
            if problem.dim != 2 or problem.periodic[0]:
                return False, "inlet / outlet are defined for D2Q9 with walls on the x axis"
            if problem.shape[0] < 3:
                return False, "inlet / outlet need nx >= 3"
        if getattr(problem, "solid", None) is not None and cls.aa:
            return False, "solid obstacles need the two-buffer variant (fused, fused-fp16, ...)"
        if problem.lattice.name not in cls.lattices:
            return False, f"{problem.lattice.name} not implemented"
        if problem.collision not in cls.collisions:
            return False, f"{problem.collision} not implemented"
        if problem.lattice.q * problem.n_nodes >= 2**31:
            return False, "int32 indexing limit"
        if problem.dim == 2 and problem.shape[1] > 65535 or (
                problem.dim == 3 and max(problem.shape[1:]) > 65535):
            return False, "ny / nz above 65535"
        return True, ""

    @classmethod
    def storage_id(cls) -> int:
        if cls.storage == "f16":
            return _lib.STORE_F16
        if cls.storage == "bf16":
            return _lib.STORE_BF16
        return _lib.STORE_F32_SHIFTED if cls.shifted else _lib.STORE_F32

    # ------------------------------------------------------------------ construction
    def __init__(self, problem: Any, device: Any = None, force_field: Any = None) -> None:
        ok, why = self.supports(problem)
        if not ok:
            raise Unsupported(f"{self.backend}/{self.variant}: {why}")
        ok, why = self.available()
        if not ok:
            raise Unsupported(f"{self.backend}/{self.variant} unavailable: {why}")
        self.problem = problem
        self.steps_done = 0
        self.dev = torch.device(device or "cuda")
        self.q = problem.lattice.q
        self.N = problem.n_nodes
        self.tdtype = getattr(torch, _TORCH_DTYPES[self.storage])
        self.desc = make_desc(problem, self.storage_id())
        self._keep: list = []  # device tensors the descriptor points at
        if getattr(problem, "solid", None) is not None:
            bits = torch.as_tensor(solid_bits(problem.solid).view(np.int32), device=self.dev)
            self._keep.append(bits)
            self.solid_mask = bits
            self.desc.solid_bits = bits.data_ptr()
        if getattr(problem, "inlet", None) is not None:  # u_x(y) on the left wall
            uin = torch.as_tensor(np.asarray(problem.inlet, dtype=np.float32).reshape(-1),
                                  device=self.dev).contiguous()
            if uin.numel() != problem.shape[1]:
                raise ValueError(f"inlet must hold ny = {problem.shape[1]} values")
            self._keep.append(uin)
            self.desc.inlet_u = uin.data_ptr()
        self.desc.outlet = int(bool(getattr(problem, "outlet", False)))
        if force_field is not None:
            self.set_force_field(force_field)
        _lib.call("lbm_validate", ctypes.byref(self.desc))
        self.A = torch.empty(self.q * self.N, device=self.dev, dtype=self.tdtype)
        self.B = None if self.aa else torch.empty_like(self.A)
        self.set_populations(problem.initial_populations())

    def set_force_field(self, field: Any) -> None:
        """Per-node Guo force added to the uniform force: (d, *array_shape) float32."""
        t = torch.as_tensor(field, dtype=torch.float32, device=self.dev).contiguous()
        if tuple(t.shape) != (self.problem.dim,) + tuple(self.problem.array_shape):
            raise ValueError(f"force field must have shape (d, *array_shape), got {tuple(t.shape)}")
        self.force_field = t
        self._keep.append(t)
        self.desc.force_field = t.data_ptr()

    # ------------------------------------------------------------------ state
    @property
    def layout(self) -> int:
        return _lib.LAYOUT_AA_SWAPPED if self.aa else _lib.LAYOUT_NATURAL

    def set_populations(self, f: Any) -> None:
        """Load a canonical float64 post-collision state (q, *array_shape): a numpy array, or
        a torch tensor (already on the device: no host copy)."""
        want = (self.q,) + tuple(self.problem.array_shape)
        if torch.is_tensor(f):
            t = f.to(device=self.dev, dtype=torch.float64).contiguous()
        else:
            f = np.asarray(f, dtype=np.float64)
            t = None
        if tuple(f.shape) != want:
            raise ValueError(f"populations must have shape {want}, got {tuple(f.shape)}")
        if t is None:
            t = torch.from_numpy(np.ascontiguousarray(f)).to(self.dev)
        _lib.call("lbm_encode_f64", ctypes.byref(self.desc), t.data_ptr(), self.A.data_ptr(),
                  self.layout, _stream())
        torch.cuda.current_stream().synchronize()

    def populations(self) -> np.ndarray:
        """The canonical float64 post-collision state (q, *array_shape)."""
        out = torch.empty(self.q * self.N, dtype=torch.float64, device=self.dev)
        _lib.call("lbm_decode_f64", ctypes.byref(self.desc), self.A.data_ptr(), self.layout,
                  out.data_ptr(), _stream())
        return out.cpu().numpy().reshape((self.q,) + tuple(self.problem.array_shape))

    @property
    def state(self) -> Any:
        """The current stored buffer (flat torch tensor, storage format, ``layout``)."""
        return self.A

    def memory_bytes(self) -> int:
        return (1 if self.aa else 2) * self.q * self.N * self.itemsize

    # ------------------------------------------------------------------ stepping
    def step(self, n: int = 1) -> None:
        """Advance n time steps (a multiple of ``step_multiple``)."""
        if n % self.step_multiple:
            raise ValueError(f"{self.name} advances in multiples of {self.step_multiple} steps")
        self._advance(n)
        self.steps_done += n

    # Lattices below GRAPH_MAX_NODES are launch-bound (a 128^2 step moves ~2.4 us of data,
    # less than a host launch costs): their steps replay from a CUDA graph of GRAPH_CHUNK
    # launches, captured once per descriptor and buffer orientation.
    use_graphs: ClassVar[bool] = True
    GRAPH_MAX_NODES: ClassVar[int] = 1 << 20
    GRAPH_CHUNK: ClassVar[int] = 64  # even: A and B end where they started

    def _advance(self, n: int) -> None:
        if self.use_graphs and self.N < self.GRAPH_MAX_NODES and n >= self.GRAPH_CHUNK:
            g = self._graph()
            for _ in range(n // self.GRAPH_CHUNK):
                g.replay()
            n %= self.GRAPH_CHUNK
        if n == 0:
            return
        b = self.A if self.aa else self.B
        _lib.call("lbm_advance", ctypes.byref(self.desc), self.A.data_ptr(), b.data_ptr(),
                  int(self.aa), int(n), _stream())
        if not self.aa and n % 2:
            self.A, self.B = self.B, self.A

    def _graph(self) -> Any:
        key = (bytes(self.desc), self.A.data_ptr())
        graphs = self.__dict__.setdefault("_graphs", {})
        g = graphs.get(key)
        if g is not None:
            return g
        # one-time kernel set-up (attributes, occupancy queries) outside the capture, on copies
        sa = self.A.clone()
        sb = sa if self.aa else torch.empty_like(sa)
        _lib.call("lbm_advance", ctypes.byref(self.desc), sa.data_ptr(), sb.data_ptr(),
                  int(self.aa), 2, _stream())
        torch.cuda.current_stream().synchronize()
        del sa, sb
        g = torch.cuda.CUDAGraph()
        b = self.A if self.aa else self.B
        with torch.cuda.graph(g):
            _lib.call("lbm_advance", ctypes.byref(self.desc), self.A.data_ptr(), b.data_ptr(),
                      int(self.aa), self.GRAPH_CHUNK, _stream())
        if len(graphs) >= 4:
            graphs.clear()
        graphs[key] = g
        return g

    def launch(self, pattern: int) -> None:
        """One kernel launch of the given pattern (pylbm's FusedSolver._launch)."""
        if pattern == _lib.PATTERN_AB:
            _lib.call("lbm_launch", ctypes.byref(self.desc), self.A.data_ptr(),
                      self.B.data_ptr(), pattern, _stream())
            self.A, self.B = self.B, self.A
        else:
            _lib.call("lbm_launch", ctypes.byref(self.desc), self.A.data_ptr(),
                      self.A.data_ptr(), pattern, _stream())

    def advance_with_force(self, n: int) -> Any:
        """Advance n steps (two-buffer, solids required) and return the momentum-exchange
        force on the solids after every step: float64 device tensor (n, d)."""
        if self.aa or getattr(self.problem, "solid", None) is None:
            raise ValueError("the momentum-exchange force needs solids and the two-buffer variant")
        out = torch.zeros((n, self.problem.dim), dtype=torch.float64, device=self.dev)
        d = _lib.LbmDesc.from_buffer_copy(self.desc)
        d.mx_force = out.data_ptr()
        d.mx_stride = self.problem.dim
        _lib.call("lbm_advance", ctypes.byref(d), self.A.data_ptr(), self.B.data_ptr(), 0,
                  int(n), _stream())
        if n % 2:
            self.A, self.B = self.B, self.A
        self.steps_done += n
        return out

    def synchronize(self) -> None:
        torch.cuda.synchronize(self.dev)

    # ------------------------------------------------------------------ observables
    def moments_f64(self) -> np.ndarray:
        """FP64 global sums on the device: [mass, momentum_x, momentum_y(, momentum_z)]."""
        out = torch.empty(self.problem.dim + 1, dtype=torch.float64, device=self.dev)
        _lib.call("lbm_moments_f64", ctypes.byref(self.desc), self.A.data_ptr(), self.layout,
                  out.data_ptr(), _stream())
        return out.cpu().numpy()

    def macroscopic_device(self) -> tuple[Any, Any]:
        """(rho[N], u[d, N]) as float32 device tensors (array layout shapes)."""
        rho = torch.empty(self.N, dtype=torch.float32, device=self.dev)
        u = torch.empty(self.problem.dim * self.N, dtype=torch.float32, device=self.dev)
        _lib.call("lbm_macroscopic", ctypes.byref(self.desc), self.A.data_ptr(), self.layout,
                  rho.data_ptr(), u.data_ptr(), _stream())
        shp = tuple(self.problem.array_shape)
        return rho.view(shp), u.view((self.problem.dim,) + shp)

    def macroscopic(self) -> tuple[np.ndarray, np.ndarray]:
        """(rho, u) as float64 numpy arrays from the canonical state, with pylbm's formula
        u = (sum c f* - F/2) / rho (core.py:255-266, base.py:79-82)."""
        f = self.populations()
        p = self.problem
        c = p.lattice.c
        rho = f[0]
        for i in range(1, self.q):
            rho = rho + f[i]
        force = [np.full(p.array_shape, v) for v in p.force]
        if getattr(self, "force_field", None) is not None:
            ff = self.force_field.double().cpu().numpy()
            force = [force[a] + ff[a] for a in range(p.dim)]
        forced = p.has_force or getattr(self, "force_field", None) is not None
        u = []
        for a in range(p.dim):
            j = None
            for i in range(self.q):
                if c[i, a] == 0:
                    continue
                term = f[i] if c[i, a] == 1 else -f[i]
                j = term if j is None else j + term
            if forced:
                j = j + 0.5 * force[a]
            u.append(j / rho)
        if forced:
            u = [(u[a] * rho - force[a]) / rho for a in range(p.dim)]
        return np.asarray(rho), np.stack(u)

    # ------------------------------------------------------------------ misc
    @property
    def name(self) -> str:
        return f"{self.backend}/{self.variant}"

    @property
    def bytes_per_node(self) -> int:
        """Minimal traffic per lattice update: read q + write q stored values."""
        return 2 * self.q * self.itemsize


class B200FusedAA(B200Fused):
    variant = "fused-aa"
    description = "hand-written CUDA for sm_100a, AA-pattern in-place streaming, fp32 shifted"
    aa = True
    step_multiple = 2


class B200FusedFP16(B200Fused):
    variant = "fused-fp16"
    description = "hand-written CUDA for sm_100a, fp16 storage of f - w_i, fp32 arithmetic"
    storage = "f16"
    itemsize = 2


class B200FusedBF16(B200Fused):
    variant = "fused-bf16"
    description = "hand-written CUDA for sm_100a, bf16 storage of f - w_i, fp32 arithmetic"
    storage = "bf16"
    itemsize = 2


class B200FusedAAFP16(B200FusedAA):
    variant = "fused-aa-fp16"
    description = "hand-written CUDA for sm_100a, AA pattern + fp16 storage of f - w_i"
    storage = "f16"
    itemsize = 2


class B200FusedAABF16(B200FusedAA):
    variant = "fused-aa-bf16"
    description = "hand-written CUDA for sm_100a, AA pattern + bf16 storage of f - w_i"
    storage = "bf16"
    itemsize = 2


class B200FusedPlain(B200Fused):
    variant = "fused-plain"
    description = ("hand-written CUDA for sm_100a, fp32 storage of f with unshifted arithmetic "
                   "(pylbm's own fp32 scheme)")
    shifted = False


VARIANTS: dict[str, type] = {c.variant: c for c in (
    B200Fused, B200FusedAA, B200FusedFP16, B200FusedBF16, B200FusedAAFP16, B200FusedAABF16,
    B200FusedPlain)}


def pylbm_classes(solver_base: Any) -> dict[str, type]:
    """The variants as subclasses of pylbm's abstract ``Solver`` (backends/base.py:18-96):
    isinstance checks against pylbm's base hold, and ``step`` / ``macroscopic`` are pylbm's
    own (base.py:68-82) rather than this module's equivalents, so the two cannot drift."""
    out = {}
    for v, cls in VARIANTS.items():
        ns = {"__module__": "pylbm.backends.b200_backend", "__doc__": cls.__doc__,
              "step": solver_base.step, "macroscopic": solver_base.macroscopic}
        out[v] = types.new_class(cls.__name__, (cls, solver_base),
                                 exec_body=lambda d, ns=ns: d.update(ns))
    return out


def register(backends: Any = None) -> list[tuple[str, str]]:
    """Add the ``b200`` variants to pylbm's backend registry (backends/__init__.py:16-34).

    pylbm resolves an entry by importing ``pylbm.backends.<module>`` lazily
    (backends/__init__.py:53-63); a module of that name holding the :func:`pylbm_classes` is
    installed in ``sys.modules``, so the lookup finds it without touching pylbm's files."""
    if backends is None:
        import pylbm.backends as backends  # type: ignore[import-not-found,no-redef]
    global Unsupported
    if not issubclass(Unsupported, backends.Unsupported):
        # this module was imported before pylbm was importable: from now on raise a class
        # that pylbm's callers catch as theirs and stand-alone callers as this module's
        Unsupported = type("Unsupported", (backends.Unsupported, Unsupported),
                           {"__module__": __name__, "__doc__": Unsupported.__doc__})
    mod = types.ModuleType(f"{backends.__name__}.b200_backend",
                           "pylbm backend b200: pylbm_b200's fused solvers as pylbm Solvers")
    added = []
    for v, cls in pylbm_classes(backends.Solver).items():
        setattr(mod, cls.__name__, cls)
        backends._ENTRIES[("b200", v)] = f"b200_backend:{cls.__name__}"
        added.append(("b200", v))
    sys.modules[mod.__name__] = mod
    if hasattr(backends, "COLORS"):
        backends.COLORS.setdefault("b200", "#76b900")
    return added
