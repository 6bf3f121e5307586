"""Counter-based SplitMix64 random numbers for seeded synthetic inputs.

u(seed, stream, index) is a pure function of its counters, so any array of draws can be generated
in any order or in pieces and still be identical; the initial-velocity perturbations of the
benchmarks and tests use it (stream = component, index = cell).
"""
from __future__ import annotations

import numpy as np

SEED = 20261203
_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea and Flood 2014) on uint64 counters."""
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & _M
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & _M
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & _M
        return z ^ (z >> np.uint64(31))


def uniform(seed: int, stream: int, n: int, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    """n draws in [lo, hi) for counters (seed, stream, 0..n-1), float64."""
    idx = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed) ^ (np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)))
        bits = splitmix64(idx ^ key)
    u01 = (bits >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return lo + (hi - lo) * u01


def normal(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normal draws (Box-Muller on two uniform streams)."""
    u1 = uniform(seed, 2 * stream + 1000, n, 0.0, 1.0)
    u2 = uniform(seed, 2 * stream + 1001, n, 0.0, 1.0)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def perturbed_rest3(W: int, H: int, D: int, amplitude: float = 1e-4, seed: int = SEED, ux: float = 0.0) -> np.ndarray:
    """3D macro field (ux, uy, uz, rho) per cell: rho = 1, ux given, uy and uz seeded uniform noise
    of the given amplitude."""
    N = W * H * D
    m = np.zeros((N, 4), dtype=np.float32)
    m[:, 0] = ux
    m[:, 1] = amplitude * uniform(seed, 1, N)
    m[:, 2] = amplitude * uniform(seed, 2, N)
    m[:, 3] = 1.0
    return m.reshape(-1)


def perturbed_rest2(W: int, H: int, amplitude: float = 1e-4, seed: int = SEED) -> np.ndarray:
    """2D macro field (rho, ux, uy, _) per cell: rho = 1, ux = 0, uy seeded uniform noise."""
    N = W * H
    m = np.zeros((N, 4), dtype=np.float32)
    m[:, 0] = 1.0
    m[:, 2] = amplitude * uniform(seed, 1, N)
    return m.reshape(-1)
