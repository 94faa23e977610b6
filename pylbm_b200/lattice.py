"""Lattice tables and relaxation-rate helpers of the host side.

The tables are pylbm's (lattice.py:49-67, 71-88): the kernels hard-code the same velocity
orders, so population i here, in the CUDA library and in pylbm are the same population. The
library's own compiled tables are available through ``_lib.lattice_info`` and are checked
against these.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Lattice:
    name: str
    d: int
    c: np.ndarray  # (q, d) int
    w: np.ndarray  # (q,)
    opp: np.ndarray  # (q,)

    @property
    def q(self) -> int:
        return len(self.w)


def _lattice(name: str, c: list, w: list) -> Lattice:
    ca = np.array(c, dtype=np.int64)
    opp = np.array([int(np.flatnonzero((ca == -ci).all(axis=1))[0]) for ci in ca])
    return Lattice(name, ca.shape[1], ca, np.array(w, dtype=np.float64), opp)


D2Q9 = _lattice("D2Q9",
                [[0, 0], [1, 0], [0, 1], [-1, 0], [0, -1], [1, 1], [-1, 1], [-1, -1], [1, -1]],
                [4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
D3Q19 = _lattice("D3Q19",
                 [[0, 0, 0], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1],
                  [0, 0, -1], [1, 1, 0], [-1, -1, 0], [1, -1, 0], [-1, 1, 0], [1, 0, 1],
                  [-1, 0, -1], [1, 0, -1], [-1, 0, 1], [0, 1, 1], [0, -1, -1], [0, 1, -1],
                  [0, -1, 1]],
                 [1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
LATTICES = {"D2Q9": D2Q9, "D3Q19": D3Q19}


def magic_rate(s_nu: float, magic: float = 3.0 / 16.0) -> float:
    """TRT odd rate s- with Lambda = (1/s+ - 1/2)(1/s- - 1/2) = magic (lattice.py:90-97)."""
    return 1.0 / (0.5 + magic / (1.0 / s_nu - 0.5))


def equilibrium(lat: Lattice, rho: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Second-order equilibrium f_i^eq(rho, u); u has shape (d, ...) (lattice.py:112-119)."""
    usq = sum(u[a] ** 2 for a in range(lat.d))
    out = np.empty((lat.q,) + np.shape(rho), dtype=np.float64)
    for i in range(lat.q):
        cu = sum(lat.c[i, a] * u[a] for a in range(lat.d))
        out[i] = lat.w[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return out


def runtime_rates(problem) -> tuple[float, float, float, float]:  # noqa: ANN001
    """(r0, r1, r2, r3) of the C descriptor, pylbm's codegen.runtime_rates (codegen.py:437-445):
    BGK (1/tau, 0, 0, 0); TRT (s+, s-, 0, 0); MRT (s_nu, s_e, s_eps, s_q)."""
    s_nu = 1.0 / problem.tau
    if problem.collision == "bgk":
        return s_nu, 0.0, 0.0, 0.0
    if problem.collision == "trt":
        return s_nu, magic_rate(s_nu, problem.magic), 0.0, 0.0
    # MRT always uses Lambda = 3/16 for the energy-flux rate (problem.py:102-106)
    return s_nu, float(problem.s_e), float(problem.s_eps), magic_rate(s_nu, 3.0 / 16.0)
