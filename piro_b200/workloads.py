"""Seeded synthetic inputs for the benchmark configurations.

No public dataset is involved: every field is generated from numpy
default_rng seeds with the shapes and distributions the configurations name.
Grid sizes are ghost-inclusive (the .ini `n` is size - 2) with unit spacing
h = 1, so the Laplacian norm is 1.
"""
from __future__ import annotations

import numpy as np


def gaussian_bump(n: int, sigma: float, centre: float, amplitude: float = 1.0) -> np.ndarray:
    """exp(-r^2 / (2 sigma^2)) on an n^3 grid, x fastest (index x + y*n + z*n*n)."""
    ax = np.arange(n, dtype=np.float64) - centre
    g = np.exp(-ax ** 2 / (2.0 * sigma ** 2))
    f = amplitude * g[:, None, None] * g[None, :, None] * g[None, None, :]
    return f.astype(np.float32).reshape(-1)


def zero_boundary(u: np.ndarray, nx: int, ny: int, nz: int) -> np.ndarray:
    v = u.reshape(nz, ny, nx).copy()
    v[0, :, :] = v[-1, :, :] = 0
    v[:, 0, :] = v[:, -1, :] = 0
    v[:, :, 0] = v[:, :, -1] = 0
    return v.reshape(-1)


def heat_fe_32(seed: int = 0):
    """Forward Euler heat, 32^3, constant alpha 0.01, dt = 0.2 h^2/(6 alpha),
    bump (sigma 4 cells, centre 15.5) + U[0, 1e-3) noise, zero boundary."""
    n = 32
    rng = np.random.default_rng(seed)
    u0 = gaussian_bump(n, 4.0, 15.5) + rng.uniform(0.0, 1e-3, n ** 3).astype(np.float32)
    u0 = zero_boundary(u0, n, n, n).astype(np.float32)
    alpha = np.full(n ** 3, 0.01, np.float32)
    dt = np.float32(0.2 / (6 * 0.01))
    return dict(n=(n, n, n), u0=u0, alpha=alpha, dt=dt, steps=100)


def smoothed_lognormal(n: int, sigma_log: float, filt: float, seed: int) -> np.ndarray:
    """alpha = exp(sigma_log * z), z ~ N(0,1) Gaussian-filtered over `filt`
    cells (periodic) and re-standardised."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    z = rng.standard_normal((n, n, n))
    z = gaussian_filter(z, sigma=filt, mode="wrap")
    z = (z - z.mean()) / z.std()
    return np.exp(sigma_log * z).astype(np.float32).reshape(-1)


def heat_be_128(seed: int = 2, n: int = 128):
    """Backward Euler, 128^3: alpha smoothed log-normal (sigma 1.5, filter 8,
    seed 2), dt = 50 h^2/(6 max alpha), c1-style bump scaled to the grid,
    homogeneous Dirichlet; 20 steps."""
    alpha = smoothed_lognormal(n, 1.5, 8.0, seed)
    dt = np.float32(50.0 / (6.0 * float(alpha.max())))
    rng = np.random.default_rng(0)
    s = n / 32.0
    u0 = gaussian_bump(n, 4.0 * s, (n - 1) / 2.0) + rng.uniform(0.0, 1e-3, n ** 3).astype(np.float32)
    u0 = zero_boundary(u0, n, n, n).astype(np.float32)
    return dict(n=(n, n, n), u0=u0, alpha=alpha, dt=dt, steps=20)


def spmv_256(seed: int = 1, n: int = 256):
    """Format sweep, 256^3: alpha log-normal (mu 0, sigma 1) per cell, seed 1;
    a random-phase sinusoid field."""
    rng = np.random.default_rng(seed)
    alpha = np.exp(rng.standard_normal(n ** 3)).astype(np.float32)
    k = rng.integers(1, 4, size=3)
    phi = rng.uniform(0, 2 * np.pi)
    ax = np.arange(n, dtype=np.float64)
    f = np.sin(2 * np.pi * (k[0] * ax[None, None, :] + k[1] * ax[None, :, None] + k[2] * ax[:, None, None]) / n + phi)
    u = f.astype(np.float32).reshape(-1)
    return dict(n=(n, n, n), u=u, alpha=alpha)


def advection(n: int, seed: int = 1):
    """Upwind advection (space scheme 1): velocity w = (1.0, 0.5, 0.25) passed
    as v = -w because the upwind gradient rows are a backward difference over
    2h (stencils.cpp:78-154); dt = 0.5 * 2h / |w|_1, i.e. CFL 0.5 in the
    reference's scaling.  Field: sin(2 pi (k . x) / n + phi), k and phi from
    default_rng(seed)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 4, size=3)
    phi = rng.uniform(0, 2 * np.pi)
    ax = np.arange(n, dtype=np.float64)
    f = np.sin(2 * np.pi * (k[0] * ax[None, None, :] + k[1] * ax[None, :, None] + k[2] * ax[:, None, None]) / n + phi)
    u0 = f.astype(np.float32).reshape(-1)
    w = np.array([1.0, 0.5, 0.25])
    N = n ** 3
    v = np.concatenate([np.full(N, -w[d], np.float32) for d in range(3)])
    dt = np.float32(0.5 * 2.0 / np.abs(w).sum())
    return dict(n=(n, n, n), u0=u0, v=v, dt=dt, steps=1000, gnorm=np.float32(2.0))


def batched(seed: int = 3, count: int = 512, lo: int = 16, hi: int = 96):
    """Batched heat problems: cube sides uniform in [lo, hi] (ghost-inclusive),
    alpha log-uniform in [1e-3, 1e-1], forward or backward Euler, all drawn
    from default_rng(seed); dt = 0.2 h^2/(6 alpha) (forward) or 50 times the
    explicit limit h^2/(6 alpha) (backward), h = 1.  Field: a centred Gaussian
    bump (sigma n/8) plus U[0, 1e-3) noise, zero boundary."""
    rng = np.random.default_rng(seed)
    n = rng.integers(lo, hi + 1, size=count).astype(np.int32)
    alpha = (10.0 ** rng.uniform(-3.0, -1.0, size=count)).astype(np.float32)
    scheme = rng.integers(0, 2, size=count).astype(np.int32)
    dt = np.where(scheme == 0, 0.2 / (6.0 * alpha), 50.0 / (6.0 * alpha)).astype(np.float32)
    fields = []
    for k in range(count):
        m = int(n[k])
        f = gaussian_bump(m, m / 8.0, (m - 1) / 2.0) + rng.uniform(0.0, 1e-3, m ** 3).astype(np.float32)
        fields.append(zero_boundary(f, m, m, m).astype(np.float32))
    return dict(n=n, alpha=alpha, dt=dt, scheme=scheme, fields=fields)


def pack_batch(fields, offsets, total):
    """Member fields into one array at the given offsets."""
    u = np.zeros(total, np.float32)
    for f, o in zip(fields, offsets):
        u[int(o):int(o) + f.size] = f
    return u
