"""Force-history analysis (src/analysis.ts:8-22) and the 3D page's coefficient and divergence
helpers (src/tunnel3d.ts:38-105)."""
from __future__ import annotations

import math

import numpy as np

from .geometry import empty_sdf3, add_sphere, add_box3, add_cylinder_z, add_wing, reference_area


def period_from_crossings(t, v):
    """Period from linearly interpolated upward crossings of the mean (src/analysis.ts:8-18).
    Returns (period, crossings) or None with fewer than three crossings."""
    v = list(v)
    t = list(t)
    m = sum(v) / len(v)
    times = []
    for k in range(1, len(v)):
        a = v[k - 1] - m
        b = v[k] - m
        if a < 0 and b >= 0:
            times.append(t[k - 1] + ((t[k] - t[k - 1]) * -a) / (b - a))
    if len(times) < 3:
        return None
    return (times[-1] - times[0]) / (len(times) - 1), len(times)


def mean(v) -> float:
    """src/analysis.ts:20-22"""
    v = list(v)
    return sum(v) / len(v)


def stream_function(ux, uy, W: int, H: int) -> np.ndarray:
    """psi[y * W + x]: u_x integrated (trapezoid) up the column x = 0, then -u_y along each row
    (src/analysis.ts:28-37). Solid cells should carry zero velocity."""
    ux = np.asarray(ux, dtype=np.float64).reshape(H, W)
    uy = np.asarray(uy, dtype=np.float64).reshape(H, W)
    psi = np.zeros((H, W))
    psi[1:, 0] = np.cumsum(0.5 * (ux[1:, 0] + ux[:-1, 0]))
    psi[:, 1:] = psi[:, :1] - np.cumsum(0.5 * (uy[:, 1:] + uy[:, :-1]), axis=1)
    return psi.reshape(-1)


def primary_vortex(psi, W: int, H: int):
    """Interior extremum of |psi|, refined by a parabola through its neighbours on each axis
    (src/analysis.ts:40-58). Returns (x, y, psi)."""
    p = np.asarray(psi, dtype=np.float64).reshape(H, W)
    inner = np.abs(p[1:H - 1, 1:W - 1])
    by, bx = np.unravel_index(int(np.argmax(inner)), inner.shape)
    by += 1
    bx += 1
    if abs(p[by, bx]) <= abs(p.reshape(-1)[1]):
        by, bx = divmod(1, W)  # no interior value beats the reference's starting index

    def refine(m, c, q):
        den = m - 2 * c + q
        return 0.0 if den == 0 else 0.5 * (m - q) / den

    x = bx + (refine(p[by, bx - 1], p[by, bx], p[by, bx + 1]) if 0 < bx < W - 1 else 0.0)
    y = by + (refine(p[by - 1, bx], p[by, bx], p[by + 1, bx]) if 0 < by < H - 1 else 0.0)
    return x, y, float(p[by, bx])


def coefficient_scale(u_target: float, area: float) -> float:
    """2 / (u^2 A), 0 without a body (src/tunnel3d.ts:75-77)."""
    return 2 / (u_target * u_target * area) if area > 0 else 0.0


def has_diverged(samples) -> bool:
    """Any non-finite force sample (src/tunnel3d.ts:97-99). Samples are dicts with fx, fy[, fz]."""
    for f in samples:
        for k in ("fx", "fy", "fz"):
            if k in f and f[k] is not None and not math.isfinite(f[k]):
                return True
    return False


def field_diverged(values) -> bool:
    """Any non-finite macro value (src/tunnel3d.ts:102-105)."""
    return not bool(np.all(np.isfinite(np.asarray(values))))


def build_body(obstacle: str, size_fraction: float, angle_deg: float, W: int, H: int, D: int,
               span_fraction: float = 0.6):
    """Obstacle SDF placed at (W/4, H/2, D/2) with its reference length and area
    (src/tunnel3d.ts:38-72). span_fraction sets the wing span as a fraction of D (0.6 on the page)."""
    sdf = empty_sdf3(W, H, D)
    L = size_fraction * H
    cx, cy, cz = W / 4, H / 2, D / 2
    a = angle_deg * math.pi / 180
    if obstacle == "sphere":
        add_sphere(sdf, W, H, D, cx, cy, cz, L / 2)
        half = [L / 2, L / 2, L / 2]
    elif obstacle == "cube":
        add_box3(sdf, W, H, D, cx, cy, cz, L / 2, L / 2, L / 2, -a)
        r = (L / 2) * (abs(math.cos(a)) + abs(math.sin(a)))
        half = [r, r, L / 2]
    elif obstacle == "cylinder":
        add_cylinder_z(sdf, W, H, D, cx, cy, L / 2)
        half = [L / 2, L / 2, D / 2]
    elif obstacle == "wing":
        add_wing(sdf, W, H, D, cx, cy, cz, L, span_fraction * D, a)
        half = [L / 2, L / 2, span_fraction * D / 2]
    elif obstacle == "none":
        return {"sdf": sdf, "lRef": L, "area": 0.0, "bounds": None}
    else:
        raise ValueError(obstacle)
    c = [cx, cy, cz]
    dims = [W, H, D]
    lo = [max(-0.5, c[k] - half[k] - 2) for k in range(3)]
    hi = [min(dims[k] - 0.5, c[k] + half[k] + 2) for k in range(3)]
    span = span_fraction * D if obstacle == "wing" else None
    return {"sdf": sdf, "lRef": L, "area": reference_area(obstacle, L, D, span), "bounds": (lo, hi)}
