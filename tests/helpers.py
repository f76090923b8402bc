"""Shared test inputs, restating the reference tests' own generators."""
import math

import numpy as np


def gaussian_ic(n: int, h: float) -> np.ndarray:
    """crates/runtime/tests/solvers.rs:22-38: Gaussian centred at (0.5, 0.5), sigma 0.1."""
    sigma = 0.1
    inv_2s2 = 1.0 / (2.0 * sigma * sigma)
    data = np.zeros(n * n)
    for row in range(n):
        for col in range(n):
            x = col * h
            y = row * h
            dx = x - 0.5
            dy = y - 0.5
            r2 = math.fma(dx, dx, dy * dy) if hasattr(math, "fma") else dx * dx + dy * dy
            data[row * n + col] = math.exp(-r2 * inv_2s2)
    return data


def quadratic_field(n: int, h: float) -> np.ndarray:
    """x^2 + y^2 sampled on the grid (ops.rs:1235-1242)."""
    data = np.zeros(n * n)
    for row in range(n):
        for col in range(n):
            x = col * h
            y = row * h
            data[row * n + col] = x * x + y * y
    return data


def sin_sin_field(n: int, h: float) -> np.ndarray:
    """sin(pi x) sin(pi y) (crates/runtime/tests/analytical.rs:455-465)."""
    data = np.zeros(n * n)
    for row in range(n):
        for col in range(n):
            data[row * n + col] = math.sin(math.pi * col * h) * math.sin(math.pi * row * h)
    return data


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
