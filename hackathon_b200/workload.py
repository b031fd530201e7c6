"""Seeded synthetic problems for the compact Helmholtz solver (tests and benchmarks).

The reference defines its problems through source-level callbacks
(2D_Program/user_input.c, 3D_Program/user_input.c).  The benchmark configurations instead
use a problem class with a known solution: the unit square/cube, homogeneous Dirichlet
data, constant wavenumber k, and a source that is a sum of sine modes

    f = sum_m A_m sin(p_m pi x) sin(q_m pi y) [sin(r_m pi z)]

with complex amplitudes A_m ~ CN(0, 1) (real and imaginary parts N(0, 1/2)), optionally
plus i.i.d. CN(0, var) noise at every interior grid point.  The continuous solution is
u = sum_m A_m sin(..)/(k^2 - pi^2 (p^2 + q^2 [+ r^2])).

Random numbers come from splitmix64 (Steele, Lea & Flood 2014) turned into doubles in
[0,1) by the top 53 bits, and into normals by the Box-Muller transform.  Seeds follow
`seed = config_index * 1000 + rhs_index`.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_MASK = (1 << 64) - 1


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n successive splitmix64 outputs (uint64) from `seed`."""
    out = np.empty(n, dtype=np.uint64)
    s = seed & _MASK
    for t in range(n):
        s = (s + 0x9E3779B97F4A7C15) & _MASK
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        out[t] = z ^ (z >> 31)
    return out


def splitmix64_fast(seed: int, n: int) -> np.ndarray:
    """Vectorised splitmix64: identical output to `splitmix64` for large n."""
    with np.errstate(over="ignore"):
        idx = np.arange(1, n + 1, dtype=np.uint64)
        s = np.uint64(seed & _MASK) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = s
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniforms(seed: int, n: int) -> np.ndarray:
    """Doubles in [0, 1) from the top 53 bits of splitmix64."""
    u = splitmix64_fast(seed, n)
    return (u >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normals(seed: int, n: int) -> np.ndarray:
    """n standard normals by Box-Muller over pairs of uniforms."""
    m = (n + 1) // 2
    u = uniforms(seed, 2 * m)
    u1 = 1.0 - u[0::2]  # (0, 1]
    u2 = u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    z = np.empty(2 * m)
    z[0::2] = r * np.cos(2.0 * math.pi * u2)
    z[1::2] = r * np.sin(2.0 * math.pi * u2)
    return z[:n]


def complex_normals(seed: int, n: int, var: float = 1.0) -> np.ndarray:
    """CN(0, var): real and imaginary parts N(0, var/2)."""
    z = normals(seed, 2 * n) * math.sqrt(var / 2.0)
    return z[0::2] + 1j * z[1::2]


@dataclass
class SineModes:
    """Mode indices (1-based) and complex amplitudes of a sine-mode source."""

    p: np.ndarray
    q: np.ndarray
    r: np.ndarray | None
    amp: np.ndarray


def sine_modes(seed: int, n_modes: int, pmax: int, dim: int = 2) -> SineModes:
    u = uniforms(seed, dim * n_modes)
    idx = np.minimum((u * pmax).astype(np.int64), pmax - 1) + 1
    amp = complex_normals(seed ^ 0x5A5A5A5A, n_modes)
    p = idx[0::dim]
    q = idx[1::dim]
    r = idx[2::dim] if dim == 3 else None
    return SineModes(p=p, q=q, r=r, amp=amp)


def _sin_table(n: int, modes: np.ndarray) -> np.ndarray:
    """sin(p pi x_i) on the extended grid x_i = i/(n+1), i = 0..n+1, with the two end points
    set to exactly zero (homogeneous Dirichlet)."""
    x = np.arange(n + 2, dtype=np.float64) / (n + 1)
    t = np.sin(math.pi * np.outer(modes, x))
    t[:, 0] = 0.0
    t[:, -1] = 0.0
    return t


def source_2d(n: int, modes: SineModes, noise_seed: int | None = None, noise_var: float = 0.0,
              fast: bool = False) -> np.ndarray:
    """f on the (n+2)^2 extended grid, x fastest: array [n+2 (y), n+2 (x)] complex128.
    fast=True sums the modes with a matrix product (same values up to summation order)."""
    sx = _sin_table(n, modes.p)  # [m, n+2]
    sy = _sin_table(n, modes.q)
    if fast:
        f = (sy.T * modes.amp[None, :]) @ sx.astype(np.complex128)
    else:
        f = np.einsum("m,my,mx->yx", modes.amp, sy, sx)
    if noise_seed is not None and noise_var > 0.0:
        f[1:-1, 1:-1] += complex_normals(noise_seed, n * n, noise_var).reshape(n, n)
    f[0, :] = f[-1, :] = 0.0
    f[:, 0] = f[:, -1] = 0.0
    return np.ascontiguousarray(f)


def exact_2d(n: int, modes: SineModes, k: complex) -> np.ndarray:
    """Continuous solution sampled at the interior points: [n (y), n (x)]."""
    sx = _sin_table(n, modes.p)[:, 1:-1]
    sy = _sin_table(n, modes.q)[:, 1:-1]
    den = k * k - math.pi ** 2 * (modes.p.astype(np.float64) ** 2 + modes.q.astype(np.float64) ** 2)
    return np.einsum("m,my,mx->yx", modes.amp / den, sy, sx)


def source_3d(n: int, modes: SineModes) -> np.ndarray:
    """f on the (n+2)^3 extended grid: array [z, y, x] complex128."""
    sx = _sin_table(n, modes.p)
    sy = _sin_table(n, modes.q)
    sz = _sin_table(n, modes.r)
    f = np.einsum("m,mz,my,mx->zyx", modes.amp, sz, sy, sx, optimize=True)
    return np.ascontiguousarray(f)


def exact_3d(n: int, modes: SineModes, k: complex) -> np.ndarray:
    sx = _sin_table(n, modes.p)[:, 1:-1]
    sy = _sin_table(n, modes.q)[:, 1:-1]
    sz = _sin_table(n, modes.r)[:, 1:-1]
    pp = modes.p.astype(np.float64) ** 2 + modes.q.astype(np.float64) ** 2 + modes.r.astype(np.float64) ** 2
    den = k * k - math.pi ** 2 * pp
    return np.einsum("m,mz,my,mx->zyx", modes.amp / den, sz, sy, sx, optimize=True)


# ---- the benchmark configurations (sizes and distributions of the published configs) ----

@dataclass(frozen=True)
class Config2D:
    index: int
    n: int
    order: int
    k: float
    batch: int
    n_modes: int
    pmax: int
    noise_var: float = 0.0


CONFIG_README = Config2D(index=0, n=100, order=6, k=10.0, batch=1, n_modes=8, pmax=20)
CONFIG_2D_1023 = Config2D(index=1, n=1023, order=6, k=50.0, batch=64, n_modes=32, pmax=200, noise_var=1e-3)
CONFIG_2D_2047 = Config2D(index=3, n=2047, order=6, k=100.0, batch=16, n_modes=8, pmax=20)


def batch_sources_2d(cfg: Config2D, count: int | None = None) -> np.ndarray:
    """[count, n+2, n+2] extended-grid sources for RHS indices 0..count-1."""
    count = cfg.batch if count is None else count
    out = np.empty((count, cfg.n + 2, cfg.n + 2), dtype=np.complex128)
    for b in range(count):
        seed = cfg.index * 1000 + b
        m = sine_modes(seed, cfg.n_modes, cfg.pmax)
        out[b] = source_2d(cfg.n, m, noise_seed=seed + 0x1000000 if cfg.noise_var else None,
                           noise_var=cfg.noise_var)
    return out
