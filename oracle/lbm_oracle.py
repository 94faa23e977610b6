"""Float64 oracle of pylbm's lattice-Boltzmann step -- test infrastructure, never shipped.

A restatement of pylbm's readable array-level algorithm, written for this repository:

* ``stream``        pull streaming with periodic wrap, stationary solids and box walls with
                    Ladd's moving-lid term, later axes overriding earlier ones at corners
                    (pylbm core.py:88-127; solid sources core.py:56-66,101-105);
* ``collide``       moments with Guo's half force, equilibria, Guo source, BGK / TRT / MRT
                    relaxation (core.py:151-247; rates problem.py:94-106, lattice.py:90-109);
* ``macroscopic``   rho and the physical velocity (sum c f* - F/2) / rho (core.py:255-266);
* ``momentum_exchange``  the momentum-exchange force on the solids, 2 sum_i c_i sum f*_i over
                    fluid nodes whose neighbour x + c_i is solid (karman.py:45-53,88-96).

The operations are evaluated in the same order as pylbm's, so with a uniform force and no
force field the results are bitwise those of pylbm's NumPy backend; this is checked against
fixtures produced by pylbm itself (tests/golden). The one extension is ``force_field``: a
per-node force (d, *array_shape) added to the uniform force wherever pylbm uses
``p.force[a]`` (core.py:166-167,192-199,264-265). With ``xp=torch`` the same code runs on
float64 tensors and is differentiable (the autograd oracle of the adjoint).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np

# ----------------------------------------------------------------------------- lattices
# Velocity orders and weights of pylbm's lattice.py:49-67 (tables that must be identical).


@dataclass(frozen=True)
class Lat:
    name: str
    c: tuple  # q tuples of d ints
    w: tuple  # q floats

    @property
    def q(self) -> int:
        return len(self.w)

    @property
    def d(self) -> int:
        return len(self.c[0])

    @property
    def opp(self) -> tuple:
        return tuple(self.c.index(tuple(-v for v in ci)) for ci in self.c)


D2Q9 = Lat("D2Q9",
           ((0, 0), (1, 0), (0, 1), (-1, 0), (0, -1), (1, 1), (-1, 1), (-1, -1), (1, -1)),
           (4 / 9,) + (1 / 9,) * 4 + (1 / 36,) * 4)
D3Q19 = Lat("D3Q19",
            ((0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
             (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1),
             (1, 0, -1), (-1, 0, 1), (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)),
            (1 / 3,) + (1 / 18,) * 6 + (1 / 36,) * 12)

# Lallemand-Luo moment basis, rows (rho, e, eps, jx, qx, jy, qy, pxx, pxy) (lattice.py:71-87)
MRT_M = ((1, 1, 1, 1, 1, 1, 1, 1, 1),
         (-4, -1, -1, -1, -1, 2, 2, 2, 2),
         (4, -2, -2, -2, -2, 1, 1, 1, 1),
         (0, 1, 0, -1, 0, 1, -1, -1, 1),
         (0, -2, 0, 2, 0, 1, -1, -1, 1),
         (0, 0, 1, 0, -1, 1, 1, -1, -1),
         (0, 0, -2, 0, 2, 1, 1, -1, -1),
         (0, 1, -1, 1, -1, 0, 0, 0, 0),
         (0, 0, 0, 0, 0, 1, -1, 1, -1))
MRT_NORM = tuple(float(sum(v * v for v in row)) for row in MRT_M)


def _d3q19_mrt_rows() -> tuple:
    """Orthogonal D3Q19 moment basis of d'Humieres et al. (2002, Phil. Trans. R. Soc. A 360,
    437-451) as polynomials of c, evaluated on the D3Q19 velocities below: rows (rho, e, eps,
    jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz). pylbm has no
    D3Q19 MRT; this extends its D2Q9 form (core.py:228-246) to 3D."""
    def rows(c: tuple) -> tuple:
        x, y, z = c
        c2 = x * x + y * y + z * z
        return (1, 19 * c2 - 30, (21 * c2 * c2 - 53 * c2 + 24) // 2,
                x, (5 * c2 - 9) * x, y, (5 * c2 - 9) * y, z, (5 * c2 - 9) * z,
                3 * x * x - c2, (3 * c2 - 5) * (3 * x * x - c2),
                y * y - z * z, (3 * c2 - 5) * (y * y - z * z),
                x * y, y * z, x * z,
                (y * y - z * z) * x, (z * z - x * x) * y, (x * x - y * y) * z)
    cols = [rows(c) for c in D3Q19.c]
    return tuple(tuple(col[k] for col in cols) for k in range(19))


MRT3_M = _d3q19_mrt_rows()
MRT3_NORM = tuple(float(sum(v * v for v in row)) for row in MRT3_M)


def magic_rate(s_nu: float, magic: float = 3.0 / 16.0) -> float:
    """Odd rate for TRT magic parameter Lambda (lattice.py:90-97)."""
    return 1.0 / (0.5 + magic / (1.0 / s_nu - 0.5))


# ----------------------------------------------------------------------------- case
@dataclass
class Case:
    """The fields of pylbm's Problem (problem.py:27-42) that the fused step uses."""

    shape: tuple
    tau: float = 0.6
    collision: str = "bgk"
    periodic: tuple | None = None
    u_lid: float = 0.0
    force: tuple | None = None
    magic: float = 3.0 / 16.0
    s_e: float = 1.64
    s_eps: float = 1.54
    solid: Any = None        # bool (ny, nx) / (nz, ny, nx)
    force_field: Any = None  # (d, *array_shape) float64, added to ``force``
    extra: dict = field(default_factory=dict)
    inlet: Any = None        # u_x(y) of the velocity inlet on the left wall, (ny,), 2D
    outlet: bool = False     # pressure outlet (rho = 1) on the right boundary, 2D

    def __post_init__(self) -> None:
        self.shape = tuple(int(s) for s in self.shape)
        if self.periodic is None:
            self.periodic = (False,) * self.dim
        self.periodic = tuple(bool(v) for v in self.periodic)
        if self.force is None:
            self.force = (0.0,) * self.dim
        self.force = tuple(float(v) for v in self.force)

    @classmethod
    def from_problem(cls, p: Any, force_field: Any = None) -> Case:
        return cls(p.shape, p.tau, p.collision, p.periodic, p.u_lid, p.force, p.magic,
                   p.s_e, p.s_eps, getattr(p, "solid", None), force_field,
                   inlet=getattr(p, "inlet", None), outlet=bool(getattr(p, "outlet", False)))

    @property
    def dim(self) -> int:
        return len(self.shape)

    @property
    def lat(self) -> Lat:
        return D2Q9 if self.dim == 2 else D3Q19

    @property
    def array_shape(self) -> tuple:
        return tuple(reversed(self.shape))

    @property
    def has_force(self) -> bool:
        return any(v != 0.0 for v in self.force) or self.force_field is not None

    def trt_rates(self) -> tuple:
        sp = 1.0 / self.tau
        return sp, magic_rate(sp, self.magic)

    def mrt_rates(self) -> tuple:
        s_nu = 1.0 / self.tau
        s_q = magic_rate(s_nu, 3.0 / 16.0)  # problem.py:102-106 always uses 3/16
        if self.dim == 2:
            return (0.0, self.s_e, self.s_eps, 0.0, s_q, 0.0, s_q, s_nu, s_nu)
        # D3Q19: e -> s_e; eps and the fourth-order pi moments -> s_eps; the energy fluxes q
        # and the third-order m moments -> s_q; the five shear moments -> 1/tau
        se, sp = self.s_e, self.s_eps
        return (0.0, se, sp, 0.0, s_q, 0.0, s_q, 0.0, s_q, s_nu, sp, s_nu, sp, s_nu, s_nu,
                s_nu, s_q, s_q, s_q)

    def mrt_basis(self) -> tuple:
        """(M, |M_k|^2) of the lattice's MRT."""
        return (MRT_M, MRT_NORM) if self.dim == 2 else (MRT3_M, MRT3_NORM)

    def force_component(self, a: int) -> Any:
        """Total force along axis a: a float, or an array when a force field is set."""
        if self.force_field is None:
            return self.force[a]
        return self.force_field[a] + self.force[a]


# ----------------------------------------------------------------------------- array api
class _Xp:
    def __init__(self, xp: Any) -> None:
        self.xp = xp
        self.torch = xp.__name__ == "torch"

    def roll(self, a: Any, shifts: tuple, axes: tuple) -> Any:
        if self.torch:
            return self.xp.roll(a, shifts=shifts, dims=axes)
        return np.roll(a, shifts, axis=axes)

    def copy(self, a: Any) -> Any:
        return a.clone() if self.torch else a.copy()

    def where(self, c: Any, a: Any, b: Any) -> Any:
        return self.xp.where(c, a, b)

    def stack(self, xs: list) -> Any:
        return self.xp.stack(xs)


def _face(dim: int, axis: int, side: int) -> tuple:
    idx: list = [slice(None)] * dim
    idx[dim - 1 - axis] = side
    return tuple(idx)


def solid_sources(case: Case, to_array: Any = np.asarray) -> list | None:
    """Per direction: the source node x - c_i is solid (np.roll wrap; core.py:56-66)."""
    if case.solid is None:
        return None
    lat = case.lat
    solid = np.asarray(case.solid, dtype=bool)
    axes = tuple(range(case.dim))
    out = []
    for i in range(lat.q):
        shifts = tuple(lat.c[i][a] for a in reversed(range(case.dim)))
        out.append(to_array(np.roll(solid, shifts, axis=axes)))
    return out


# ----------------------------------------------------------------------------- step
def stream(f: Any, case: Case, xp: Any = np, solid_src: list | None = None) -> list:
    """Pull streaming with half-way bounce-back (core.py:88-127); returns q arrays."""
    X = _Xp(xp)
    lat, d = case.lat, case.dim
    axes = tuple(range(d))
    out = []
    for i in range(lat.q):
        shifts = tuple(lat.c[i][a] for a in reversed(range(d)))
        out.append(X.roll(f[i], shifts, axes) if any(shifts) else X.copy(f[i]))
    if case.solid is not None:
        src = solid_src if solid_src is not None else solid_sources(
            case, (lambda a: xp.as_tensor(a, device=f.device)) if X.torch else np.asarray)
        opp = lat.opp
        for i in range(lat.q):
            if any(lat.c[i]):
                out[i] = X.where(src[i], f[opp[i]], out[i])
    opp = lat.opp
    for a in range(d):
        if case.periodic[a]:
            continue
        top = a == d - 1
        for i in range(lat.q):
            ca = lat.c[i][a]
            if ca == 1:  # the source lies behind the low wall
                fc = _face(d, a, 0)
                val = f[opp[i]][fc]
                if a == 0 and case.inlet is not None:  # moving-wall inlet (core.py:67-78,116-117)
                    val = val + 6.0 * lat.w[i] * lat.c[i][0] * _as(case.inlet, f, X)
                out[i][fc] = val
            elif ca == -1:  # the source lies behind the high wall
                fc = _face(d, a, -1)
                val = f[opp[i]][fc]
                if top and case.u_lid != 0.0 and lat.c[i][0] != 0:
                    val = val + 6.0 * lat.w[i] * lat.c[i][0] * case.u_lid
                out[i][fc] = val
    if case.outlet:
        _outlet(out, f, case)
    return out


def _as(a: Any, like: Any, X: Any) -> Any:
    """``a`` as an array of the backend of ``like`` (numpy or torch)."""
    if X.torch:
        return X.xp.as_tensor(np.asarray(a), dtype=like.dtype, device=like.device)
    return np.asarray(a, dtype=np.float64)


def _outlet(out: list, f: Any, case: Case) -> None:
    """Pressure outlet on the right boundary (core.py:130-148, D2Q9): the populations that
    enter from the right (c_x = -1) are the equilibrium at rho = 1 with the velocity of the
    neighbouring column, taken from the stored post-collision state."""
    lat = case.lat
    col = [f[i][..., -2] for i in range(lat.q)]
    rho = col[0]
    for i in range(1, lat.q):
        rho = rho + col[i]
    ux = (col[1] - col[3] + col[5] - col[6] - col[7] + col[8]) / rho
    uy = (col[2] - col[4] + col[5] + col[6] - col[7] - col[8]) / rho
    usq = ux * ux + uy * uy
    for i in range(lat.q):
        if lat.c[i][0] == -1:
            cu = lat.c[i][0] * ux + lat.c[i][1] * uy
            out[i][..., -1] = lat.w[i] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)


def moments(f: list, case: Case) -> tuple:
    """rho and u = (sum c f + F/2) / rho (core.py:151-169)."""
    lat = case.lat
    rho = f[0]
    for i in range(1, lat.q):
        rho = rho + f[i]
    u = []
    for a in range(case.dim):
        j = None
        for i in range(lat.q):
            ci = lat.c[i][a]
            if ci == 0:
                continue
            term = f[i] if ci == 1 else -f[i]
            j = term if j is None else j + term
        Fa = case.force_component(a)
        if _nonzero(Fa):
            j = j + 0.5 * Fa
        u.append(j / rho)
    return rho, u


def _nonzero(v: Any) -> bool:
    return not isinstance(v, float) or v != 0.0


def equilibria(rho: Any, u: list, case: Case) -> tuple:
    """(feq_i, c_i.u) lists (core.py:172-186)."""
    lat = case.lat
    usq = u[0] * u[0]
    for a in range(1, case.dim):
        usq = usq + u[a] * u[a]
    feq, cus = [], []
    for i in range(lat.q):
        cu: Any = 0.0
        for a in range(case.dim):
            if lat.c[i][a] != 0:
                cu = cu + lat.c[i][a] * u[a]
        cus.append(cu)
        feq.append(lat.w[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq))
    return feq, cus


def guo_source(u: list, cus: list, case: Case) -> list:
    """S_i = w_i [3 (c_i - u).F + 9 (c_i.u)(c_i.F)] (core.py:189-200)."""
    lat = case.lat
    F = [case.force_component(a) for a in range(case.dim)]
    uf: Any = 0.0
    for a in range(case.dim):
        if _nonzero(F[a]):
            uf = uf + u[a] * F[a]
    out = []
    for i in range(lat.q):
        if case.force_field is None:
            cf: Any = float(sum(lat.c[i][a] * F[a] for a in range(case.dim)))
        else:
            cf = 0.0
            for a in range(case.dim):
                if lat.c[i][a] != 0:
                    cf = cf + lat.c[i][a] * F[a]
        out.append(lat.w[i] * (3.0 * (cf - uf) + 9.0 * cus[i] * cf))
    return out


def collide(f: list, case: Case, xp: Any = np) -> Any:
    """BGK / TRT / MRT collision with Guo forcing (core.py:203-247)."""
    lat = case.lat
    rho, u = moments(f, case)
    feq, cus = equilibria(rho, u, case)
    src = guo_source(u, cus, case) if case.has_force else None
    out: list = []
    if case.collision == "bgk":
        om = 1.0 / case.tau
        for i in range(lat.q):
            v = f[i] - om * (f[i] - feq[i])
            if src is not None:
                v = v + (1.0 - 0.5 * om) * src[i]
            out.append(v)
    elif case.collision == "trt":
        sp, sm = case.trt_rates()
        opp = lat.opp
        for i in range(lat.q):
            o = opp[i]
            fp, fm = 0.5 * (f[i] + f[o]), 0.5 * (f[i] - f[o])
            ep, em = 0.5 * (feq[i] + feq[o]), 0.5 * (feq[i] - feq[o])
            v = f[i] - sp * (fp - ep) - sm * (fm - em)
            if src is not None:
                gp, gm = 0.5 * (src[i] + src[o]), 0.5 * (src[i] - src[o])
                v = v + (1.0 - 0.5 * sp) * gp + (1.0 - 0.5 * sm) * gm
            out.append(v)
    elif case.collision == "mrt":
        s = case.mrt_rates()
        basis, norm = case.mrt_basis()
        dm = []
        for k in range(lat.q):
            acc: Any = 0.0
            for i in range(lat.q):
                m = float(basis[k][i])
                if m != 0.0:
                    term = -s[k] * m * (f[i] - feq[i])
                    if src is not None:
                        term = term + (1.0 - 0.5 * s[k]) * m * src[i]
                    acc = acc + term
            dm.append(acc)
        for i in range(lat.q):
            v = f[i]
            for k in range(lat.q):
                m = float(basis[k][i])
                if m != 0.0:
                    v = v + (m / norm[k]) * dm[k]
            out.append(v)
    else:
        raise ValueError(case.collision)
    return _Xp(xp).stack(out)


def step(f: Any, case: Case, xp: Any = np, solid_src: list | None = None) -> Any:
    """One time step on the stored post-collision state (core.py:250-252)."""
    return collide(stream(f, case, xp, solid_src), case, xp)


def run(case: Case, f0: Any, steps: int, xp: Any = np) -> Any:
    f = f0
    src = solid_sources(case, (lambda a: xp.as_tensor(a, device=f0.device))
                        if xp.__name__ == "torch" else np.asarray)
    for _ in range(steps):
        f = step(f, case, xp, src)
    return f


def macroscopic(f: Any, case: Case) -> tuple:
    """(rho, [u_a]) with u = (sum c f* - F/2) / rho from the stored state (core.py:255-266)."""
    lat = case.lat
    rho, u = moments([f[i] for i in range(lat.q)], case)
    if case.has_force:
        u = [(u[a] * rho - case.force_component(a)) / rho for a in range(case.dim)]
    return rho, u


def equilibrium(lat: Lat, rho: np.ndarray, u: np.ndarray) -> np.ndarray:
    """Second-order equilibrium for rho and u (d, ...) (lattice.py:112-119)."""
    usq = sum(u[a] ** 2 for a in range(lat.d))
    out = np.empty((lat.q,) + rho.shape)
    for i in range(lat.q):
        cu = sum(lat.c[i][a] * u[a] for a in range(lat.d))
        out[i] = lat.w[i] * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return out


# ----------------------------------------------------------------------------- forces
def force_masks(case: Case) -> list:
    """Per direction: fluid nodes whose neighbour x + c_i is solid (karman.py:45-53)."""
    lat = case.lat
    solid = np.asarray(case.solid, dtype=bool)
    axes = tuple(range(case.dim))
    masks = []
    for i in range(lat.q):
        shifts = tuple(-lat.c[i][a] for a in reversed(range(case.dim)))
        masks.append(~solid & np.roll(solid, shifts, axis=axes))
    return masks


def momentum_exchange(f: Any, case: Case, masks: list | None = None, xp: Any = np) -> Any:
    """2 sum_i c_i sum_{x in mask_i} f*_i(x) (karman.py:88-96); returns (d,)."""
    lat = case.lat
    masks = masks if masks is not None else force_masks(case)
    if xp.__name__ == "torch":
        mk = xp.stack([xp.as_tensor(m, dtype=f.dtype, device=f.device) for m in masks])
        ct = xp.as_tensor(np.array(lat.c, dtype=np.float64), dtype=f.dtype, device=f.device)
        per_dir = (f * mk).reshape(lat.q, -1).sum(dim=1)
        return 2.0 * (per_dir[:, None] * ct).sum(0)
    mk = np.stack(masks).astype(np.float64)
    per_dir = (np.asarray(f) * mk).reshape(lat.q, -1).sum(axis=1)
    return 2.0 * (per_dir[:, None] * np.array(lat.c, dtype=np.float64)).sum(0)


def drag_objective(case: Case, f0: Any, steps: int, t0: int, xp: Any = np,
                   checkpoint: int = 0) -> Any:
    """J = mean over t = t0..steps of the x momentum-exchange force on the state after t
    steps. With torch and ``checkpoint`` > 0 the forward is segment-checkpointed."""
    masks = force_masks(case)
    src = solid_sources(case, (lambda a: xp.as_tensor(a, device=f0.device))
                        if xp.__name__ == "torch" else np.asarray)
    f = f0
    acc: Any = 0.0
    count = 0

    def seg(ff: Any, k: int) -> Any:
        for _ in range(k):
            ff = step(ff, case, xp, src)
        return ff

    t = 0
    while t < steps:
        k = 1 if t + 1 >= t0 else (min(checkpoint, t0 - 1 - t) if checkpoint else 1)
        if xp.__name__ == "torch" and checkpoint and k > 1:
            from torch.utils.checkpoint import checkpoint as ckpt

            f = ckpt(seg, f, k, use_reentrant=False)
        else:
            f = seg(f, k)
        t += k
        if t >= t0:
            acc = acc + momentum_exchange(f, case, masks, xp)[0]
            count += 1
    return acc / count
