"""D3Q19 and D2Q9 lattice tables and host-side helpers.

Mirrors src/lattice3d.ts:4-40 and src/lattice.ts:2-45 (velocity sets, weights, OPP, mirrors,
TRT pairs, flag bits, MAGIC_LAMBDA, trtLambda3, host equilibria).
"""
from __future__ import annotations

import numpy as np

# D3Q19 (src/lattice3d.ts:4-9): odd i and i + 1 are opposite and form TRT pairs.
CX = (0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0)
CY = (0, 0, 0, 1, -1, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 1, -1)
CZ = (0, 0, 0, 0, 0, 1, -1, 0, 0, 1, -1, 1, -1, 0, 0, -1, 1, -1, 1)
Q3 = 19
W = tuple(1 / 3 if i == 0 else (1 / 18 if i <= 6 else 1 / 36) for i in range(Q3))
OPP = tuple(0 if i == 0 else (i + 1 if i % 2 else i - 1) for i in range(Q3))


def _find(cx: int, cy: int, cz: int) -> int:
    for i in range(Q3):
        if CX[i] == cx and CY[i] == cy and CZ[i] == cz:
            return i
    raise ValueError(f"no direction ({cx}, {cy}, {cz})")


MIRROR_Y = tuple(_find(CX[i], -CY[i], CZ[i]) for i in range(Q3))
MIRROR_Z = tuple(_find(CX[i], CY[i], -CZ[i]) for i in range(Q3))
PAIRS = tuple((2 * k + 1, 2 * k + 2) for k in range(9))

FLAG_SOLID = 1 << 19
FLAG_INLET = 1 << 20
FLAG_OUTLET = 1 << 21

MAGIC_LAMBDA = 3 / 16  # src/lattice.ts:36


def trt_lambda3(tau: float) -> float:
    """TRT Lambda from the base tau: min(3/16, 50 (tau - 1/2)^2) (src/lattice3d.ts:29-31)."""
    return min(MAGIC_LAMBDA, 50 * (tau - 0.5) ** 2)


def equilibrium3(rho: float, ux: float, uy: float, uz: float) -> np.ndarray:
    """Unshifted D3Q19 equilibrium (src/lattice3d.ts:33-40)."""
    usq = 1.5 * (ux * ux + uy * uy + uz * uz)
    out = np.empty(Q3)
    for i in range(Q3):
        cu = 3 * (CX[i] * ux + CY[i] * uy + CZ[i] * uz)
        out[i] = W[i] * rho * (1 + cu + 0.5 * cu * cu - usq)
    return out


# D2Q9 (src/lattice.ts:2-7)
CX2 = (0, 1, 0, -1, 0, 1, -1, -1, 1)
CY2 = (0, 0, 1, 0, -1, 1, 1, -1, -1)
W2 = (4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36)
OPP2 = (0, 3, 4, 1, 2, 7, 8, 5, 6)
MIRROR_Y2 = (0, 1, 4, 3, 2, 8, 7, 6, 5)
Q2 = 9
PAIRS2 = ((1, 3), (2, 4), (5, 7), (6, 8))
FLAG2_SOLID = 1 << 9
FLAG2_INLET = 1 << 10
FLAG2_OUTLET = 1 << 11
BIDX_SHIFT = 12


class XMode:
    """src/lattice.ts:17-21"""
    Periodic = 0
    Wall = 1
    Open = 2


class YMode:
    """src/lattice.ts:23-28"""
    Periodic = 0
    NoSlip = 1
    Slip = 2
    MovingWall = 3


def equilibrium2(rho: float, ux: float, uy: float) -> np.ndarray:
    """Unshifted D2Q9 equilibrium (src/lattice.ts:38-45)."""
    usq = 1.5 * (ux * ux + uy * uy)
    out = np.empty(Q2)
    for i in range(Q2):
        cu = 3 * (CX2[i] * ux + CY2[i] * uy)
        out[i] = W2[i] * rho * (1 + cu + 0.5 * cu * cu - usq)
    return out
