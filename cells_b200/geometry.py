"""Signed distance fields for obstacles (host-side inputs of set_sdf), negative inside solids.

2D: src/geometry.ts:3-80 (emptySdf, addCircle, addBox, nacaPolygon, addPolygon).
3D: src/geometry3d.ts:8-99 (emptySdf3, addSphere, addBox3, addCylinderZ, addWing, referenceArea),
plus the star body of spherical-harmonic radius r(theta, phi) = r0 (1 + sum c_lm Y_lm) that the
reference lacks. Nodes sit at integer coordinates; the arrays are float32 like the reference's
Float32Array, and each stamp takes min(existing, d) within the shape's box grown by a 3-cell margin.
"""
from __future__ import annotations

import math

import numpy as np

FAR = 1e6  # src/geometry.ts:3
MARGIN = 3


# ---------------------------------------------------------------- 2D


def empty_sdf(W: int, H: int) -> np.ndarray:
    return np.full(W * H, FAR, dtype=np.float32)


def _stamp2(sdf: np.ndarray, W: int, H: int, box, d) -> None:
    x0 = max(0, math.floor(box[0]))
    y0 = max(0, math.floor(box[1]))
    x1 = min(W - 1, math.ceil(box[2]))
    y1 = min(H - 1, math.ceil(box[3]))
    if x1 < x0 or y1 < y0:
        return
    ys, xs = np.mgrid[y0:y1 + 1, x0:x1 + 1].astype(np.float64)
    v = d(xs, ys)
    view = sdf.reshape(H, W)
    cur = view[y0:y1 + 1, x0:x1 + 1].astype(np.float64)
    view[y0:y1 + 1, x0:x1 + 1] = np.minimum(cur, v).astype(np.float32)


def add_circle(sdf, W, H, cx, cy, r) -> None:
    """src/geometry.ts:23-25"""
    _stamp2(sdf, W, H, [cx - r - MARGIN, cy - r - MARGIN, cx + r + MARGIN, cy + r + MARGIN],
            lambda x, y: np.hypot(x - cx, y - cy) - r)


def add_box(sdf, W, H, cx, cy, hx, hy, angle=0.0) -> None:
    """Rectangle of half-extents (hx, hy) rotated counter-clockwise by angle (src/geometry.ts:28-39)."""
    c, s = math.cos(angle), math.sin(angle)
    R = math.hypot(hx, hy) + MARGIN

    def d(x, y):
        px = (x - cx) * c + (y - cy) * s
        py = -(x - cx) * s + (y - cy) * c
        qx = np.abs(px) - hx
        qy = np.abs(py) - hy
        return np.hypot(np.maximum(qx, 0), np.maximum(qy, 0)) + np.minimum(np.maximum(qx, qy), 0)

    _stamp2(sdf, W, H, [cx - R, cy - R, cx + R, cy + R], d)


def naca_polygon(x0, y0, chord, thickness, alpha, n=400):
    """NACA 4-digit symmetric section, closed trailing edge, leading edge at (x0, y0), pitched
    nose-up by alpha (src/geometry.ts:42-57). Returns an (M, 2) float64 array."""
    def half(t):
        return 5 * thickness * (0.2969 * math.sqrt(t) - 0.126 * t - 0.3516 * t * t + 0.2843 * t ** 3 - 0.1036 * t ** 4)

    pts = []
    for k in range(n + 1):
        t = (1 - math.cos(math.pi * k / n)) / 2
        pts.append((t, half(t)))
    for k in range(n - 1, 0, -1):
        t = (1 - math.cos(math.pi * k / n)) / 2
        pts.append((t, -half(t)))
    c, s = math.cos(-alpha), math.sin(-alpha)
    return np.array([(x0 + chord * (u * c - v * s), y0 + chord * (u * s + v * c)) for u, v in pts])


def polygon_distance(poly: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Signed distance to a closed polygon, even-odd inside test (src/geometry.ts:65-78)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    d2 = np.full(x.shape, np.inf)
    inside = np.zeros(x.shape, dtype=bool)
    n = len(poly)
    b = n - 1
    for a in range(n):
        ax, ay = poly[a]
        bx, by = poly[b]
        ex, ey = bx - ax, by - ay
        t = np.clip(((x - ax) * ex + (y - ay) * ey) / (ex * ex + ey * ey), 0, 1)
        dx = x - ax - t * ex
        dy = y - ay - t * ey
        d2 = np.minimum(d2, dx * dx + dy * dy)
        if ay != by:
            cross = ((ay > y) != (by > y)) & (x < (bx - ax) * (y - ay) / (by - ay) + ax)
        else:
            cross = np.zeros(x.shape, dtype=bool)
        inside ^= cross
        b = a
    d = np.sqrt(d2)
    return np.where(inside, -d, d)


def add_polygon(sdf, W, H, poly) -> None:
    """src/geometry.ts:59-80"""
    poly = np.asarray(poly, dtype=np.float64)
    mn = poly.min(axis=0)
    mx = poly.max(axis=0)
    _stamp2(sdf, W, H, [mn[0] - MARGIN, mn[1] - MARGIN, mx[0] + MARGIN, mx[1] + MARGIN],
            lambda x, y: polygon_distance(poly, x, y))


# ---------------------------------------------------------------- 3D


def empty_sdf3(W: int, H: int, D: int) -> np.ndarray:
    return np.full(W * H * D, FAR, dtype=np.float32)


def _stamp3(sdf, W, H, D, box, d) -> None:
    """src/geometry3d.ts:15-27: the box grows by MARGIN on every side before clipping."""
    x0 = max(0, math.floor(box[0] - MARGIN))
    y0 = max(0, math.floor(box[1] - MARGIN))
    z0 = max(0, math.floor(box[2] - MARGIN))
    x1 = min(W - 1, math.ceil(box[3] + MARGIN))
    y1 = min(H - 1, math.ceil(box[4] + MARGIN))
    z1 = min(D - 1, math.ceil(box[5] + MARGIN))
    if x1 < x0 or y1 < y0 or z1 < z0:
        return
    zs, ys, xs = np.mgrid[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1].astype(np.float64)
    v = d(xs, ys, zs)
    view = sdf.reshape(D, H, W)
    cur = view[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1].astype(np.float64)
    view[z0:z1 + 1, y0:y1 + 1, x0:x1 + 1] = np.minimum(cur, v).astype(np.float32)


def add_sphere(sdf, W, H, D, cx, cy, cz, r) -> None:
    """src/geometry3d.ts:29-31"""
    _stamp3(sdf, W, H, D, [cx - r, cy - r, cz - r, cx + r, cy + r, cz + r],
            lambda x, y, z: np.sqrt((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) - r)


def add_box3(sdf, W, H, D, cx, cy, cz, hx, hy, hz, angle_z=0.0) -> None:
    """Box of half-extents (hx, hy, hz) rotated about z through its centre (src/geometry3d.ts:34-46)."""
    c, s = math.cos(angle_z), math.sin(angle_z)
    R = math.hypot(hx, hy)

    def d(x, y, z):
        px = (x - cx) * c + (y - cy) * s
        py = -(x - cx) * s + (y - cy) * c
        qx = np.abs(px) - hx
        qy = np.abs(py) - hy
        qz = np.abs(z - cz) - hz
        outside = np.sqrt(np.maximum(qx, 0) ** 2 + np.maximum(qy, 0) ** 2 + np.maximum(qz, 0) ** 2)
        return outside + np.minimum(np.maximum(np.maximum(qx, qy), qz), 0)

    _stamp3(sdf, W, H, D, [cx - R, cy - R, cz - hz, cx + R, cy + R, cz + hz], d)


def add_cylinder_z(sdf, W, H, D, cx, cy, r) -> None:
    """Cylinder of radius r along z over the whole depth (src/geometry3d.ts:49-51)."""
    _stamp3(sdf, W, H, D, [cx - r, cy - r, 0, cx + r, cy + r, D - 1], lambda x, y, z: np.hypot(x - cx, y - cy) - r)


def add_wing(sdf, W, H, D, cx, cy, cz, chord, span, angle_z=0.0) -> None:
    """NACA0012 wing with flat tips, centred at (cx, cy, cz), pitched nose-up by angle_z about its
    mid-chord (src/geometry3d.ts:70-88). The section distance is cached as float32, as the reference
    caches it in a Float32Array before combining it with the span distance."""
    ox = cx - (chord / 2) * math.cos(angle_z)
    oy = cy + (chord / 2) * math.sin(angle_z)
    poly = naca_polygon(0, 0, chord, 0.12, angle_z, 200) + np.array([ox, oy])
    mn = poly.min(axis=0)
    mx = poly.max(axis=0)

    def d(x, y, z):
        d2 = polygon_distance(poly, x[0], y[0]).astype(np.float32).astype(np.float64)[None, :, :]
        dz = np.abs(z - cz) - span / 2
        return np.where((d2 < 0) | (dz < 0), np.maximum(d2, dz), np.hypot(d2, dz))

    _stamp3(sdf, W, H, D, [mn[0], mn[1], cz - span / 2, mx[0], mx[1], cz + span / 2], d)


def reference_area(obstacle: str, size: float, D: int, span: float | None = None) -> float:
    """Frontal area in cells^2 for the force coefficients (src/geometry3d.ts:91-99). The reference's
    wing area assumes the page's span of 0.6 D; pass span for any other wing."""
    if obstacle == "sphere":
        return math.pi * size * size / 4
    if obstacle == "cube":
        return size * size
    if obstacle == "cylinder":
        return size * D
    if obstacle == "wing":
        return size * (0.6 * D if span is None else span)
    if obstacle in ("none", None):
        return 0.0
    raise ValueError(obstacle)


# ---------------------------------------------------------------- star body (not in the reference)


def real_sph_harm(l: int, m: int, theta: np.ndarray, phi: np.ndarray) -> np.ndarray:
    """Orthonormal real spherical harmonic Y_lm(theta, phi) for l <= 3, theta the polar angle from +z."""
    from math import factorial, sqrt, pi

    x = np.cos(theta)
    am = abs(m)
    # associated Legendre P_l^|m|(x) without the Condon-Shortley phase, l <= 3
    s = np.sqrt(np.maximum(0.0, 1 - x * x))
    P = {
        (0, 0): np.ones_like(x),
        (1, 0): x, (1, 1): s,
        (2, 0): 0.5 * (3 * x * x - 1), (2, 1): 3 * x * s, (2, 2): 3 * s * s,
        (3, 0): 0.5 * (5 * x ** 3 - 3 * x), (3, 1): 1.5 * (5 * x * x - 1) * s, (3, 2): 15 * x * s * s,
        (3, 3): 15 * s ** 3,
    }[(l, am)]
    norm = sqrt((2 * l + 1) / (4 * pi) * factorial(l - am) / factorial(l + am))
    if m == 0:
        return norm * P
    if m > 0:
        return sqrt(2) * norm * P * np.cos(m * phi)
    return sqrt(2) * norm * P * np.sin(am * phi)


SH_INDEX = tuple((l, m) for l in range(4) for m in range(-l, l + 1))  # 16 (l, m) pairs


def star_radius(coef, theta, phi, r0=12.0):
    """r(theta, phi) = r0 (1 + sum_k coef[k] Y_{l_k m_k}(theta, phi)) over SH_INDEX."""
    s = np.zeros_like(np.asarray(theta, dtype=np.float64))
    for c, (l, m) in zip(coef, SH_INDEX):
        s = s + c * real_sph_harm(l, m, theta, phi)
    return r0 * (1 + s)


def add_star(sdf, W, H, D, cx, cy, cz, coef, r0=12.0) -> None:
    """Star-shaped body: signed radial distance |p - c| - r(theta, phi). This is the radial
    distance, not the Euclidean one; it has the right sign and zero set, and Bouzidi link fractions
    read it along lattice links, where it differs from the true distance by the surface's tilt."""
    coef = np.asarray(coef, dtype=np.float64)
    rmax = r0 * (1 + np.sum(np.abs(coef)) * 0.5 * math.sqrt(7 / math.pi)) + 1

    def d(x, y, z):
        dx, dy, dz = x - cx, y - cy, z - cz
        rr = np.sqrt(dx * dx + dy * dy + dz * dz)
        theta = np.arccos(np.clip(np.where(rr > 0, dz / np.maximum(rr, 1e-300), 1.0), -1, 1))
        phi = np.arctan2(dy, dx)
        return rr - star_radius(coef, theta, phi, r0)

    _stamp3(sdf, W, H, D, [cx - rmax, cy - rmax, cz - rmax, cx + rmax, cy + rmax, cz + rmax], d)
