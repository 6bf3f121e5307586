"""The star body's host functions in the library (cells3d_star_sdf, cells3d_star_coef_gradient)
against the numpy restatement of the same formulas in cells_b200.geometry. No GPU needed."""
import math

import numpy as np
import pytest

from cells_b200 import geometry as g
from cells_b200._lib import CellsError, star_coef_gradient, star_sdf


def _coef(seed):
    return np.random.default_rng(seed).normal(0, 0.05, 16)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_star_sdf_matches_numpy(seed):
    W, H, D = 48, 32, 28
    coef = _coef(seed)
    center = (14.3, 15.5, 13.0)
    a = g.empty_sdf3(W, H, D)
    g.add_sphere(a, W, H, D, 40, 8, 8, 3)  # a second body: the stamp keeps the minimum
    b = a.copy()
    g.add_star(a, W, H, D, *center, coef, 9.0)
    star_sdf(b, W, H, D, center, 9.0, coef)
    # libm and numpy may round the last double bit differently; after the float32 cast the values
    # agree to one float32 ulp
    assert np.allclose(a, b, rtol=0, atol=4e-6 * np.maximum(1.0, np.abs(a)).max())
    assert np.array_equal(a < 0, b < 0)
    assert np.count_nonzero(a != b) <= a.size // 1000


def test_star_sdf_sphere_is_radial_distance():
    W, H, D = 24, 24, 24
    coef = np.zeros(16)
    coef[0] = 0.25 * 2 * math.sqrt(math.pi)  # Y_00 = 1 / (2 sqrt(pi)): r = 8 * 1.25 = 10
    s = g.empty_sdf3(W, H, D)
    star_sdf(s, W, H, D, (12, 12, 12), 8.0, coef)
    z, y, x = np.mgrid[0:D, 0:H, 0:W]
    ref = (np.sqrt((x - 12.0) ** 2 + (y - 12.0) ** 2 + (z - 12.0) ** 2) - 10.0).astype(np.float32).ravel()
    assert np.allclose(s, ref, atol=1e-5)


@pytest.mark.parametrize("seed", [3, 4])
def test_star_coef_gradient_matches_numpy(seed):
    W, H, D = 40, 24, 20
    coef = _coef(seed)
    center = (11.0, 12.0, 10.0)
    rng = np.random.default_rng(seed + 10)
    dsdf = np.zeros(W * H * D)
    nodes = rng.choice(W * H * D, 500, replace=False)
    dsdf[nodes] = rng.normal(size=500)
    dsdf[(10 * H + 12) * W + 11] = 1.5  # the centre node itself (theta = 0, phi = 0)
    nodes = np.flatnonzero(dsdf)
    x, y, z = nodes % W, (nodes // W) % H, nodes // (W * H)
    dx, dy, dz = x - center[0], y - center[1], z - center[2]
    rr = np.sqrt(dx * dx + dy * dy + dz * dz)
    theta = np.arccos(np.clip(np.where(rr > 0, dz / np.maximum(rr, 1e-300), 1.0), -1, 1))
    phi = np.arctan2(dy, dx)
    jac = np.stack([-7.0 * g.real_sph_harm(l, m, theta, phi) for l, m in g.SH_INDEX], axis=1)
    want = dsdf[nodes] @ jac
    got = star_coef_gradient(dsdf, W, H, D, center, 7.0, coef)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_star_rejects_bad_input():
    s = g.empty_sdf3(8, 8, 8)
    with pytest.raises(CellsError):
        star_sdf(s, 8, 8, 8, (4, 4, 4), -1.0, np.zeros(16))
    with pytest.raises(CellsError):
        star_coef_gradient(np.zeros(512), 8, 8, 8, (4, 4, float("nan")), 3.0, np.zeros(16))
    with pytest.raises(ValueError):
        star_sdf(s, 8, 8, 8, (4, 4, 4), 3.0, np.zeros(15))
