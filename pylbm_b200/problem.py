"""A stand-alone ``Problem`` with the fields and behaviour of pylbm's (problem.py:15-126).

The solver classes accept either this class or pylbm's own ``Problem`` (they only read the
attributes below), so the backend works with or without pylbm installed.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .lattice import D2Q9, D3Q19, Lattice, equilibrium, magic_rate

COLLISIONS = ("bgk", "trt", "mrt")


@dataclass
class Problem:
    """A lattice-Boltzmann problem on a rectangular box: ``shape`` is (nx, ny) or
    (nx, ny, nz); each axis is periodic or bounded by half-way bounce-back walls; the top wall
    of the last axis moves with ``u_lid`` in +x; ``force`` is a uniform Guo body force;
    ``solid`` marks stationary obstacle nodes (array layout)."""

    shape: tuple
    tau: float = 0.6
    collision: str = "bgk"
    periodic: tuple | None = None
    u_lid: float = 0.0
    force: tuple | None = None
    magic: float = 3.0 / 16.0
    s_e: float = 1.64
    s_eps: float = 1.54
    solid: np.ndarray | None = None
    inlet: np.ndarray | None = None
    outlet: bool = False
    init_rho: np.ndarray | None = None
    init_u: np.ndarray | None = None
    meta: dict = field(default_factory=dict)

    def __post_init__(self) -> None:
        # same validation and messages as pylbm's problem.py:44-61
        self.shape = tuple(int(s) for s in self.shape)
        if self.dim not in (2, 3):
            raise ValueError("shape must be 2D or 3D")
        if self.periodic is None:
            self.periodic = (False,) * self.dim
        self.periodic = tuple(bool(p) for p in self.periodic)
        if self.force is None:
            self.force = (0.0,) * self.dim
        self.force = tuple(float(v) for v in self.force)
        if self.collision not in COLLISIONS:
            raise ValueError(f"collision must be one of {COLLISIONS}")
        if self.collision == "mrt" and self.dim != 2:
            raise ValueError("MRT is implemented for D2Q9 only")
        if self.u_lid and self.periodic[-1]:
            raise ValueError("a moving lid needs a wall on the last axis")
        if not 0.5 < self.tau:
            raise ValueError("tau must be > 0.5")

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def lattice(self) -> Lattice:
        return D2Q9 if self.dim == 2 else D3Q19

    @property
    def array_shape(self) -> tuple:
        return tuple(reversed(self.shape))

    @property
    def n_nodes(self) -> int:
        return int(np.prod(self.shape))

    @property
    def nu(self) -> float:
        return (self.tau - 0.5) / 3.0

    @property
    def has_force(self) -> bool:
        return any(v != 0.0 for v in self.force)

    def is_box(self) -> bool:
        return self.solid is None and self.inlet is None and not self.outlet

    def trt_rates(self) -> tuple[float, float]:
        s_plus = 1.0 / self.tau
        return s_plus, magic_rate(s_plus, self.magic)

    def initial_populations(self) -> np.ndarray:
        shp = self.array_shape
        rho = np.ones(shp) if self.init_rho is None else np.asarray(self.init_rho, float)
        u = np.zeros((self.dim,) + shp) if self.init_u is None else np.asarray(self.init_u,
                                                                                float)
        return equilibrium(self.lattice, rho, u)

    @staticmethod
    def cavity(n, re=None, u_lid=0.1, tau=None, collision="bgk", dim=2) -> Problem:  # noqa: ANN001
        """Lid-driven cavity; give ``re`` (Re = u_lid n / nu) or ``tau`` (problem.py:117-126)."""
        shape = (n,) * dim if isinstance(n, int) else tuple(n)
        if tau is None:
            if re is None:
                raise ValueError("give re or tau")
            tau = 3.0 * u_lid * shape[0] / re + 0.5
        return Problem(shape, tau=tau, collision=collision, u_lid=u_lid)
