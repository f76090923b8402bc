"""Seeded synthetic workloads of the solve configurations, and the FP64 direct solve that
checks their solutions.

Every generator returns row-major arrays with the boundary ring included.  The reference
publishes no datasets for this path; these are the configurations' stated distributions:

* Poisson, uniform source: -Lap u = f on the unit square, N x N interior nodes, h = 1/(N+1),
  homogeneous Dirichlet, f ~ U[-1, 1] i.i.d. from a seed.
* Poisson, modal source: f = sum of 32 modes sin(k pi x) sin(l pi y), k, l ~ U{1..64},
  amplitudes ~ N(0, 1), plus 1e-3 * U[-1, 1] noise.
* Convection-diffusion velocity from a stream function psi = sum of 8 modes with
  k, l <= 4 and N(0, 1) amplitudes, v = (d psi/dy, -d psi/dx) rescaled to max|v| = 1.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .core import Grid, Stencil


@dataclass
class PoissonProblem:
    n: int          # interior nodes per direction
    grid: Grid      # (n+2) x (n+2), ring included
    h: float
    stencil: Stencil  # S with v + 1*S v = -Lap_h v
    coeff: float = 1.0


def poisson_problem(n: int) -> PoissonProblem:
    h = 1.0 / (n + 1)
    return PoissonProblem(n, Grid.square(n + 2, h), h, Stencil.poisson_neg_laplacian(h, h))


def _embed(interior: np.ndarray) -> np.ndarray:
    n = interior.shape[0]
    full = np.zeros((n + 2, n + 2))
    full[1:-1, 1:-1] = interior
    return full.ravel()


def poisson_uniform_rhs(n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return _embed(rng.uniform(-1.0, 1.0, (n, n)))


def poisson_modes_rhs(n: int, seed: int, modes: int = 32, kmax: int = 64, noise: float = 1e-3) -> np.ndarray:
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    t = np.arange(1, n + 1) * h
    f = np.zeros((n, n))
    for _ in range(modes):
        k, l = rng.integers(1, kmax + 1, size=2)
        a = rng.normal()
        f += a * np.outer(np.sin(l * np.pi * t), np.sin(k * np.pi * t))  # rows = y, cols = x
    f += noise * rng.uniform(-1.0, 1.0, (n, n))
    return _embed(f)


def stream_velocity(n: int, seed: int, modes: int = 8, kmax: int = 4):
    """(vx, vy) on the (n+2)^2 grid from psi = sum a sin(k pi x) sin(l pi y), max|v| = 1."""
    rng = np.random.default_rng(seed)
    h = 1.0 / (n + 1)
    t = np.arange(0, n + 2) * h
    x, y = t[None, :], t[:, None]  # x varies along columns; separable, broadcast to the grid
    vx = np.zeros((n + 2, n + 2))
    vy = np.zeros((n + 2, n + 2))
    for _ in range(modes):
        k, l = rng.integers(1, kmax + 1, size=2)
        a = rng.normal()
        # psi = a sin(k pi x) sin(l pi y)
        vx += a * np.sin(k * np.pi * x) * (l * np.pi) * np.cos(l * np.pi * y)    # d psi / dy
        vy += -a * (k * np.pi) * np.cos(k * np.pi * x) * np.sin(l * np.pi * y)   # -d psi / dx
    m = np.sqrt(vx * vx + vy * vy).max()
    if m > 0:
        vx /= m
        vy /= m
    return vx.ravel(), vy.ravel()


def dst_poisson_solve(f_full: np.ndarray, n: int) -> np.ndarray:
    """Exact solution of the 5-point -Lap_h u = f with homogeneous Dirichlet data (DST-I)."""
    from scipy.fft import dstn, idstn

    h = 1.0 / (n + 1)
    f = f_full.reshape(n + 2, n + 2)[1:-1, 1:-1]
    j = np.arange(1, n + 1)
    s = np.sin(j * np.pi / (2 * (n + 1))) ** 2
    lam = (4.0 / (h * h)) * (s[:, None] + s[None, :])
    u = idstn(dstn(f, type=1, workers=-1) / lam, type=1, workers=-1)
    return _embed(u)


def neg_laplacian_residual(u_full: np.ndarray, f_full: np.ndarray, n: int) -> float:
    """||f + Lap_h u||_2 over the interior, in FP64 with numpy (the plain-operator check)."""
    h = 1.0 / (n + 1)
    u = u_full.reshape(n + 2, n + 2)
    f = f_full.reshape(n + 2, n + 2)
    lap = (u[:-2, 1:-1] + u[2:, 1:-1] + u[1:-1, :-2] + u[1:-1, 2:] - 4.0 * u[1:-1, 1:-1]) / (h * h)
    r = f[1:-1, 1:-1] + lap
    return float(np.sqrt(np.sum(r * r)))
