"""Seeded synthetic inputs for the benchmark configurations (no datasets are involved).

* ``fourier_state``  D2Q9 periodic box: rho = 1 + 0.01 N(0,1) per node, u a sum of 8 random
                     Fourier modes with integer wavevectors and random phases scaled to
                     max|u| = 0.05, f = feq(rho, u). The same seed gives the same modes at any
                     resolution, so a 256^2 case is the 4096^2 field sampled on a coarser grid.
* ``taylor_green_3d``  D3Q19 periodic cube: u = U0 (sin kx cos ky cos kz, -cos kx sin ky cos kz, 0),
                     k = 2 pi / n, rho = 1.
* ``cavity_batch``   independent D2Q9 cavities: edges log-uniform in [lo, hi] per axis,
                     tau ~ U[0.51, 1.0], lid speed ~ U[0.05, 0.1].
* ``cylinder_channel``  D2Q9 channel (x periodic, walls in y) with a solid disc and a seeded
                     N(0, sigma^2) per-node control force.
"""

from __future__ import annotations

import numpy as np

from .lattice import D2Q9, D3Q19, equilibrium


def fourier_velocity(shape: tuple, seed: int, n_modes: int = 8, amp: float = 0.05,
                     kmax: int = 4) -> np.ndarray:
    """(2, ny, nx) velocity field: a sum of ``n_modes`` periodic Fourier modes."""
    nx, ny = shape
    rng = np.random.default_rng(seed)
    ks = []
    while len(ks) < n_modes:
        k = tuple(int(v) for v in rng.integers(-kmax, kmax + 1, size=2))
        if k != (0, 0):
            ks.append(k)
    amps = rng.standard_normal((n_modes, 2))
    phases = rng.uniform(0.0, 2.0 * np.pi, (n_modes, 2))
    x = np.arange(nx) / nx
    y = np.arange(ny) / ny
    u = np.zeros((2, ny, nx))
    for m, (kx, ky) in enumerate(ks):
        cx = 2.0 * np.pi * kx * x
        cy = 2.0 * np.pi * ky * y
        for a in range(2):
            # cos(cx + cy + phi) = cos(cx + phi) cos(cy) - sin(cx + phi) sin(cy): separable
            u[a] += amps[m, a] * (np.cos(cy)[:, None] * np.cos(cx + phases[m, a])[None, :]
                                  - np.sin(cy)[:, None] * np.sin(cx + phases[m, a])[None, :])
    umax = np.sqrt((u ** 2).sum(axis=0)).max()
    return u * (amp / umax)


def fourier_state(n: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(rho, u) of the D2Q9 single-lattice throughput case on an n x n periodic box."""
    rng = np.random.default_rng(seed + 1)
    rho = 1.0 + 0.01 * rng.standard_normal((n, n))
    return rho, fourier_velocity((n, n), seed)


def fourier_populations(n: int, seed: int = 0) -> np.ndarray:
    rho, u = fourier_state(n, seed)
    return equilibrium(D2Q9, rho, u)


def taylor_green_3d(n: int, u0: float = 0.05) -> tuple[np.ndarray, np.ndarray]:
    """(rho, u) of the analytic 3D Taylor-Green vortex, one wavelength per box edge."""
    k = 2.0 * np.pi / n
    c = np.arange(n)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    u = np.zeros((3, n, n, n))
    u[0] = u0 * np.sin(k * x) * np.cos(k * y) * np.cos(k * z)
    u[1] = -u0 * np.cos(k * x) * np.sin(k * y) * np.cos(k * z)
    return np.ones((n, n, n)), u


def taylor_green_3d_populations(n: int, u0: float = 0.05) -> np.ndarray:
    rho, u = taylor_green_3d(n, u0)
    return equilibrium(D3Q19, rho, u)


def cavity_batch(count: int = 64, lo: int = 128, hi: int = 1024, seed: int = 0,
                 multiple: int = 8) -> list[dict]:
    """Parameters of ``count`` independent lid-driven D2Q9 cavities: each edge drawn
    log-uniform in [lo, hi] and rounded to a multiple of ``multiple`` (rows of whole 16-byte
    vectors for 16-bit storage), tau ~ U[0.51, 1.0], lid speed ~ U[0.05, 0.1]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        edges = []
        for _ in range(2):
            e = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
            edges.append(int(min(hi, max(lo, multiple * round(e / multiple)))))
        out.append({"shape": tuple(edges), "tau": float(rng.uniform(0.51, 1.0)),
                    "u_lid": float(rng.uniform(0.05, 0.1))})
    return out


def cavity_batch_problems(count: int = 64, lo: int = 128, hi: int = 1024, seed: int = 0,
                          collision: str = "mrt") -> list:
    """The batch of :func:`cavity_batch` as Problems (MRT with pylbm's default rates)."""
    from .problem import Problem

    return [Problem(c["shape"], tau=c["tau"], u_lid=c["u_lid"], collision=collision)
            for c in cavity_batch(count, lo, hi, seed)]


def cylinder_channel(nx: int = 1024, ny: int = 256, xc: float = 200.0, yc: float = 129.0,
                     diameter: float = 40.0, sigma: float = 1e-7,
                     seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """(solid mask (ny, nx), control force field (2, ny, nx) ~ N(0, sigma^2))."""
    yy, xx = np.mgrid[0:ny, 0:nx]
    solid = (xx - xc) ** 2 + (yy - yc) ** 2 <= (0.5 * diameter) ** 2
    rng = np.random.default_rng(seed)
    field = sigma * rng.standard_normal((2, ny, nx))
    return solid, field


# ----------------------------------------------------------------------------- on the device
def equilibrium_device(lat, rho, u):  # noqa: ANN001, ANN201
    """:func:`pylbm_b200.lattice.equilibrium` on float64 torch tensors, same operation order
    (for multi-GB initial states, built where they are used)."""
    import torch

    usq = sum(u[a] ** 2 for a in range(lat.d))
    out = torch.empty((lat.q,) + tuple(rho.shape), dtype=torch.float64, device=rho.device)
    for i in range(lat.q):
        cu = sum(int(lat.c[i, a]) * u[a] for a in range(lat.d))
        out[i] = float(lat.w[i]) * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return out


def fourier_populations_device(n: int, seed: int = 0, device: str = "cuda"):  # noqa: ANN201
    """:func:`fourier_populations` as a float64 device tensor (fields from the same seeded
    host generator, equilibrium on the device)."""
    import torch

    rho, u = fourier_state(n, seed)
    return equilibrium_device(D2Q9, torch.as_tensor(rho, device=device),
                              torch.as_tensor(u, device=device))


def taylor_green_3d_populations_device(n: int, u0: float = 0.05,
                                       device: str = "cuda"):  # noqa: ANN201
    """:func:`taylor_green_3d_populations` built on the device (float64 tensor)."""
    import torch

    k = 2.0 * np.pi / n
    s = torch.sin(k * torch.arange(n, dtype=torch.float64, device=device))
    c = torch.cos(k * torch.arange(n, dtype=torch.float64, device=device))
    # array axes (z, y, x)
    ux = u0 * c[:, None, None] * c[None, :, None] * s[None, None, :]
    uy = -u0 * c[:, None, None] * s[None, :, None] * c[None, None, :]
    u = torch.stack([ux, uy, torch.zeros_like(ux)])
    return equilibrium_device(D3Q19, torch.ones((n, n, n), dtype=torch.float64, device=device), u)
