"""Macro-field products on the GPU (speed / vorticity slices, tracer advection) against the oracle's
restatement of src/shaders/render3d.ts:33-65, 159-230, bit for bit on the same macro field.

The flow is a sphere tunnel run for a few hundred steps, so the field has a wake, a solid body and
the sponge; the oracle samples the macro field read back from the device, so the comparison checks
the sampling alone. The kernels are built without FMA contraction, like the oracle.
"""
import numpy as np
import pytest

from cells_b200 import Solver3D, geometry as g
from cells_b200.rng import perturbed_rest3
from oracle.oracle import advect, sample_slice

pytestmark = pytest.mark.gpu

W, H, D = 48, 32, 24


@pytest.fixture(scope="module")
def tunnel():
    s = Solver3D.create(W, H, D, precision="fp32", tau=0.56, uIn=0.08, spongeFraction=0.15, spongeTau=1.0,
                        absorb=0.02, forceEvery=0)
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 14, 16, 12, 5)
    s.setSdf(sdf)
    s.initField(perturbed_rest3(W, H, D, 1e-4, ux=0.08))
    s.run(300)
    yield s, s.readMacro().copy()
    s.destroy()


def same_bits(a, b):
    assert a.shape == b.shape
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), f"{np.count_nonzero(na != nb)} solid marks differ"
    bad = np.flatnonzero((a.view(np.uint32) != b.view(np.uint32)) & ~na)
    assert bad.size == 0, f"{bad.size} values differ, first {bad[:5]}: {a.reshape(-1)[bad[:5]]} vs {b.reshape(-1)[bad[:5]]}"


@pytest.mark.parametrize("mode", ["speed", "vorticity"])
@pytest.mark.parametrize("axis,pos,size", [(0, 14 / 47, None), (1, 0.5, None), (2, 0.5, None), (2, 0.37, (37, 23)),
                                           (0, 0.0, (19, 64)), (1, 1.0, (96, 48))])
def test_slice_matches_oracle(tunnel, mode, axis, pos, size):
    s, mac = tunnel
    got = s.sampleSlice(axis, pos, mode, 0.08, size)
    nv, nu = got.shape
    want = sample_slice(mac, W, H, D, axis, pos, {"speed": 0, "vorticity": 1}[mode], 0.08, nu, nv)
    same_bits(got, want)
    assert np.isfinite(got).any()
    # every slice but the inlet plane and the top row plane cuts the sphere
    assert np.isnan(got).any() == (not (axis == 0 and pos == 0.0) and not (axis == 1 and pos == 1.0))


def test_tracers_match_oracle_over_frames(tunnel):
    s, mac = tunnel
    rng = np.random.default_rng(20261203)
    n = 4096
    seeds = np.zeros((n, 4), dtype=np.float32)
    seeds[:, 0] = rng.uniform(0, W - 1, n)
    seeds[:, 1] = rng.uniform(0, H - 1, n)
    seeds[:, 2] = rng.uniform(0, D - 1, n)
    parts = np.zeros((n, 8), dtype=np.float32)
    parts[:, :4] = seeds
    want = parts.copy()
    for steps in (40.0, 15.0, 120.0):  # 4, 1 and 10 sub-steps (travel 3.2, 1.2 and 9.6 cells)
        s.advectTracers(seeds, parts, steps, 0.08)
        want = advect(mac, W, H, D, seeds, want, steps, 0.08)
        bad = np.flatnonzero(parts.view(np.uint32) != want.view(np.uint32))
        assert bad.size == 0, f"{bad.size} values differ after a frame of {steps} steps"
    # some tracers were restarted (those seeded in the sphere or swept out at the outlet)
    moved = np.linalg.norm(parts[:, :3] - seeds[:, :3], axis=1)
    assert (moved == 0).any() and (moved > 1).any()
