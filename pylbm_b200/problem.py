"""Problem descriptions for users of the b200 backend who do not have pylbm installed.

The solver classes read a problem through attributes only:

    shape, tau, collision, periodic, u_lid, force, magic, s_e, s_eps,
    solid, inlet, outlet, dim, lattice, array_shape, n_nodes, has_force,
    initial_populations()

pylbm's own ``pylbm.problem.Problem`` (problem.py:15-126) carries the same attributes, so in
the drop-in case (pylbm installed, ``register()`` called) pylbm's objects go to the solvers
unchanged and this module is not involved. ``Box`` below is the stand-alone descriptor; its
field names are pylbm's so that code written against either runs with both.
"""

from __future__ import annotations

from typing import Any

import numpy as np

from .lattice import LATTICES, Lattice, equilibrium

COLLISIONS = ("bgk", "trt", "mrt")
_LATTICE_OF_DIM = {2: "D2Q9", 3: "D3Q19"}


def _axes(value: Any, dim: int, what: str, cast: type) -> tuple:
    """A per-axis tuple from a scalar or a sequence of length ``dim``."""
    if value is None:
        value = cast()
    if np.isscalar(value):
        return (cast(value),) * dim
    out = tuple(cast(v) for v in value)
    if len(out) != dim:
        raise ValueError(f"{what} needs one entry per axis ({dim}), got {len(out)}")
    return out


class Box:
    """A rectangular lattice: ``shape`` = (nx, ny) or (nx, ny, nz), x fastest in memory.

    Every axis is either periodic or closed by half-way bounce-back walls. ``u_lid`` moves the
    wall at the high end of the last axis in +x; ``force`` is a uniform body force (Guo);
    ``solid`` marks stationary obstacle nodes and ``inlet`` / ``outlet`` open the x walls
    (velocity profile u_x(y) on the left, rho = 1 on the right), both in array layout
    (slowest axis first). ``init_rho`` / ``init_u`` give the initial equilibrium fields.
    """

    def __init__(self, shape: Any, *, tau: float = 0.6, collision: str = "bgk",
                 periodic: Any = False, u_lid: float = 0.0, force: Any = 0.0,
                 magic: float = 3.0 / 16.0, s_e: float = 1.64, s_eps: float = 1.54,
                 solid: Any = None, inlet: Any = None, outlet: bool = False,
                 init_rho: Any = None, init_u: Any = None) -> None:
        shape = tuple(int(n) for n in shape)
        if len(shape) not in _LATTICE_OF_DIM:
            raise ValueError(f"a box has 2 or 3 axes, got shape {shape}")
        if min(shape) < 1:
            raise ValueError(f"every axis needs at least one node, got shape {shape}")
        dim = len(shape)
        self.shape = shape
        self.tau = float(tau)
        self.collision = str(collision).lower()
        self.periodic = _axes(periodic, dim, "periodic", bool)
        self.u_lid = float(u_lid)
        self.force = _axes(force, dim, "force", float)
        self.magic = float(magic)
        self.s_e = float(s_e)
        self.s_eps = float(s_eps)
        self.solid = None if solid is None else np.asarray(solid, dtype=bool)
        self.inlet = None if inlet is None else np.asarray(inlet, dtype=np.float64)
        self.outlet = bool(outlet)
        self.init_rho = init_rho
        self.init_u = init_u
        problems = self._problems()
        if problems:
            raise ValueError("; ".join(problems))

    def _problems(self) -> list[str]:
        """Every reason this box cannot be simulated (empty when it can)."""
        out = []
        if self.collision not in COLLISIONS:
            out.append(f"collision must be one of {COLLISIONS}, got {self.collision!r}")
        if not self.tau > 0.5:
            out.append(f"tau must exceed 1/2 (positive viscosity), got {self.tau}")
        if self.u_lid != 0.0 and self.periodic[-1]:
            out.append("a moving lid is a wall: the last axis cannot be periodic")
        if self.solid is not None and self.solid.shape != self.array_shape:
            out.append(f"solid must have the array shape {self.array_shape}, "
                       f"got {self.solid.shape}")
        if self.inlet is not None and self.inlet.shape != (self.array_shape[-2],):
            out.append(f"inlet holds u_x for each of the {self.array_shape[-2]} rows, "
                       f"got shape {self.inlet.shape}")
        return out

    # ------------------------------------------------------------------ derived
    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def lattice(self) -> Lattice:
        return LATTICES[_LATTICE_OF_DIM[self.dim]]

    @property
    def array_shape(self) -> tuple:
        """Array axes, slowest first: (ny, nx) or (nz, ny, nx)."""
        return self.shape[::-1]

    @property
    def n_nodes(self) -> int:
        n = 1
        for s in self.shape:
            n *= s
        return n

    @property
    def nu(self) -> float:
        """Kinematic viscosity c_s^2 (tau - 1/2), c_s^2 = 1/3."""
        return (self.tau - 0.5) / 3.0

    @property
    def has_force(self) -> bool:
        return any(self.force)

    def initial_populations(self) -> np.ndarray:
        """float64 (q, *array_shape) equilibrium of the initial fields (rho = 1, u = 0 unless
        ``init_rho`` / ``init_u`` are given)."""
        rho = (np.ones(self.array_shape) if self.init_rho is None
               else np.broadcast_to(np.asarray(self.init_rho, dtype=np.float64),
                                    self.array_shape))
        u = (np.zeros((self.dim,) + self.array_shape) if self.init_u is None
             else np.asarray(self.init_u, dtype=np.float64))
        return equilibrium(self.lattice, rho, u)

    def __repr__(self) -> str:
        return (f"Box(shape={self.shape}, tau={self.tau}, collision={self.collision!r}, "
                f"periodic={self.periodic}, u_lid={self.u_lid}, force={self.force})")

    @staticmethod
    def cavity(n: Any, re: float | None = None, u_lid: float = 0.1, tau: float | None = None,
               collision: str = "bgk", dim: int = 2) -> Box:
        """The module-level :func:`cavity`, reachable as ``Problem.cavity`` as in pylbm."""
        return cavity(n, re=re, u_lid=u_lid, tau=tau, collision=collision, dim=dim)


def cavity(n: Any, re: float | None = None, u_lid: float = 0.1, tau: float | None = None,
           collision: str = "bgk", dim: int = 2) -> Box:
    """Lid-driven cavity of edge ``n`` (or shape ``n``), walls on every axis. The relaxation
    time comes from ``tau`` or from the Reynolds number Re = u_lid n / nu of the first axis."""
    shape = tuple(n) if isinstance(n, (tuple, list)) else (int(n),) * dim
    if tau is None:
        if re is None:
            raise ValueError("a cavity needs either re or tau")
        nu = u_lid * shape[0] / re
        tau = 0.5 + 3.0 * nu
    return Box(shape, tau=tau, collision=collision, u_lid=u_lid)


# pylbm's name for the same descriptor: code written against pylbm.problem.Problem runs here
Problem = Box
