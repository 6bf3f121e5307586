"""Lattice units (src/units.ts:1-24): Re -> tau with nu = (tau - 1/2) / 3 and the tau >= 0.51 clamp."""
from __future__ import annotations

import math
from dataclasses import dataclass

TAU_MIN = 0.51


@dataclass
class Derived:
    nu: float
    tau: float
    clamped: bool  # the requested Re needed tau below TAU_MIN
    effective_re: float
    mach: float


def derive_tau(re: float, u_lat: float, length: float) -> Derived:
    """src/units.ts:14-20"""
    nu = (u_lat * length) / re
    raw = 3 * nu + 0.5
    tau = max(raw, TAU_MIN)
    nu_eff = (tau - 0.5) / 3
    return Derived(nu=nu_eff, tau=tau, clamped=raw < TAU_MIN, effective_re=(u_lat * length) / nu_eff,
                   mach=u_lat * math.sqrt(3))


def max_reynolds(u_lat: float, length: float) -> float:
    """src/units.ts:22-24"""
    return (u_lat * length * 3) / (TAU_MIN - 0.5)
