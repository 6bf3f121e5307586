"""Parity of the CUDA D3Q19 path (through the C ABI) with the CPU oracle on the same seeded inputs.

Two tolerances:
  * exact arithmetic (CELLS_ARITH_EXACT): the kernel rounds every operation as written, like the
    oracle, so stored populations must match bit for bit in every precision;
  * fast arithmetic (the default, FMA contraction): populations within 2e-6 absolute (f32 storage)
    after up to 30 steps; force samples within 1e-5 relative.
Force sums are f64 in both, in different orders: compared to 1e-9 relative in exact mode.
"""
import numpy as np
import pytest

from cells_b200 import Solver3D, geometry as g
from cells_b200.rng import perturbed_rest3
from oracle.oracle import OracleSolver3D, decode

pytestmark = pytest.mark.gpu

BASE = dict(tau=0.56, uIn=0.05, spongeFraction=0.15, spongeTau=1.0, absorb=0.02, forceEvery=1)


def pair(W, H, D, precision, exact, sdf, **kw):
    cfg = dict(BASE)
    cfg.update(kw)
    s = Solver3D.create(W, H, D, precision=precision, exactArithmetic=exact, **cfg)
    o = OracleSolver3D(W, H, D, precision, **cfg)
    s.setSdf(sdf)
    o.setSdf(sdf)
    m = perturbed_rest3(W, H, D, 1e-4, ux=cfg["uIn"])
    s.initField(m)
    o.initField(m)
    return s, o


def sphere_sdf(W, H, D, cx, cy, cz, r):
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, cx, cy, cz, r)
    return sdf


def assert_same(s, o, exact, tol=2e-6):
    a = s.readPopulations()
    b = o.populations()
    assert a.shape == b.shape
    if exact:
        bad = np.flatnonzero(a.view(f"u{a.itemsize}") != b.view(f"u{b.itemsize}"))
        assert bad.size == 0, f"{bad.size} populations differ, first at {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"
    else:
        da, db = decode(a, s.precision), decode(b, s.precision)
        err = np.max(np.abs(da - db))
        assert err <= tol, f"max population difference {err}"


def assert_forces(fs, fo, rel):
    assert [x["step"] for x in fs] == [x["step"] for x in fo]
    for a, b in zip(fs, fo):
        for k in ("fx", "fy", "fz"):
            scale = max(abs(b["fx"]), abs(b["fy"]), abs(b["fz"]), 1e-12)
            assert abs(a[k] - b[k]) <= rel * scale, (a, b)


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16", "fp64"])
def test_sphere_exact_all_precisions(precision):
    W, H, D = 24, 16, 12
    s, o = pair(W, H, D, precision, True, sphere_sdf(W, H, D, 8, 8, 6, 3))
    assert np.array_equal(s.readFlags(), o.flags)
    for n in (1, 4, 25):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


def test_sphere_fast_fp32_within_tolerance():
    W, H, D = 24, 16, 12
    s, o = pair(W, H, D, "fp32", False, sphere_sdf(W, H, D, 8, 8, 6, 3))
    for n in (1, 29):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, False, 2e-6)
    assert_forces(s.readForces(), o.readForces(), 1e-5)
    s.run(0)
    o.run(0)
    assert np.max(np.abs(s.readMacro() - o.readMacro())) < 1e-5
    s.destroy()


@pytest.mark.parametrize("precision,tol", [("fp16", 1e-4), ("bf16", 1e-3)])
def test_sphere_fast_16bit_within_storage_rounding(precision, tol):
    """Fast arithmetic with 16-bit storage (the x-pair path with the lean TRT form and saturating
    stores) stays within a few storage ulps of the exact oracle after 30 steps: FP16 x 2^15 has an
    ulp of about 3e-5 at |f - w| = 0.05, BF16 about 2.4e-4."""
    W, H, D = 32, 16, 12
    s, o = pair(W, H, D, precision, False, sphere_sdf(W, H, D, 10, 8, 6, 3))
    for n in (1, 29):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, False, tol)
    assert_forces(s.readForces(), o.readForces(), 2e-2)
    s.destroy()


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_smagorinsky_fixed_lambda_cylinder_touching_slip_faces(precision):
    """A spanwise cylinder meets both z faces: the slip-face bounce-back with its force branch (the
    16-bit kernels take the per-side face rows and the Smagorinsky pair collision)."""
    W, H, D = 20, 12, 10
    sdf = g.empty_sdf3(W, H, D)
    g.add_cylinder_z(sdf, W, H, D, 7, 6, 2.5)
    s, o = pair(W, H, D, precision, True, sdf, smagorinsky=0.1, lambda_=3 / 16)
    s.encodeSteps(20)
    o.encodeSteps(20)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


@pytest.mark.parametrize("precision", ["fp16", "bf16", "fp32"])
def test_odd_width_exact(precision):
    """An odd width: the one-cell-per-thread interior kernel instead of x-pairs (16-bit loads and
    the per-side face rows for 16-bit storage)."""
    W, H, D = 23, 14, 10
    s, o = pair(W, H, D, precision, True, sphere_sdf(W, H, D, 8, 7, 5, 3))
    for n in (1, 20):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


def test_odd_width_fast_fp32():
    """The one-cell-per-thread kernel in fast arithmetic (odd width): within 2e-6 of the oracle."""
    W, H, D = 23, 14, 10
    s, o = pair(W, H, D, "fp32", False, sphere_sdf(W, H, D, 8, 7, 5, 3))
    for n in (1, 29):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, False, 2e-6)
    assert_forces(s.readForces(), o.readForces(), 1e-5)
    s.destroy()


def test_odd_sizes_box_fp64():
    W, H, D = 19, 7, 5
    sdf = g.empty_sdf3(W, H, D)
    g.add_box3(sdf, W, H, D, 6, 3, 2, 1.5, 1.2, 1.0, 0.3)
    s, o = pair(W, H, D, "fp64", True, sdf, tau=0.8)
    s.encodeSteps(15)
    o.encodeSteps(15)
    assert_same(s, o, True)
    s.destroy()


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_body_touching_y_face_and_edges(precision):
    """A sphere cut by the y = 0 face and a box through a z edge: mirrored sources on solids and
    edge links (face cells of body rows go to the body role in every precision)."""
    W, H, D = 22, 10, 10
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 8, 0.5, 5, 3)
    g.add_box3(sdf, W, H, D, 14, 9, 9, 1.5, 1.5, 1.5)
    s, o = pair(W, H, D, precision, True, sdf)
    s.encodeSteps(12)
    o.encodeSteps(12)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


def test_moved_obstacle_refill():
    """setSdf after stepping: uncovered cells are refilled from fluid neighbours (aux3d.ts:83-99)."""
    W, H, D = 24, 12, 12
    s, o = pair(W, H, D, "fp32", True, sphere_sdf(W, H, D, 8, 6, 6, 3))
    s.encodeSteps(10)
    o.encodeSteps(10)
    moved = sphere_sdf(W, H, D, 11, 6, 6, 3)
    s.setSdf(moved)
    o.setSdf(moved)
    assert np.array_equal(s.readFlags(), o.flags)
    assert_same(s, o, True)
    s.encodeSteps(10)
    o.encodeSteps(10)
    assert_same(s, o, True)
    s.destroy()


def test_device_ramp_matches_host_ramp():
    """The device-side smoothstep ramp equals setting u(step) from the host before every step."""
    W, H, D = 20, 10, 8
    s, o = pair(W, H, D, "fp32", True, sphere_sdf(W, H, D, 6, 5, 4, 2), uIn=0.0)
    target, ramp = 0.08, 12
    s.setInletRamp("smoothstep", target, ramp, 1)
    for k in range(20):
        t = min(1.0, k / ramp)
        o.setInlet(target * (t * t * (3 - 2 * t)))
        o.encodeSteps(1)
    s.encodeSteps(20)
    assert_same(s, o, True)
    s.destroy()


def test_force_every_and_ring_on_device():
    W, H, D = 20, 10, 8
    s, o = pair(W, H, D, "fp32", True, sphere_sdf(W, H, D, 6, 5, 4, 2), forceEvery=3)
    s.encodeSteps(30)
    o.encodeSteps(30)
    fs, fo = s.readForces(), o.readForces()
    assert [x["step"] for x in fs] == list(range(3, 31, 3))
    assert_forces(fs, fo, 1e-9)
    s.destroy()


def test_mass_and_status():
    W, H, D = 24, 16, 12
    s, o = pair(W, H, D, "fp64", True, sphere_sdf(W, H, D, 8, 8, 6, 3))
    s.encodeSteps(7)
    o.encodeSteps(7)
    assert abs(s.mass() - o.mass()) <= 1e-9 * abs(o.mass())
    assert s.readStatus() == 0
    s.destroy()


def test_config_size_properties():
    """The 192x96x96 sphere workload of the benchmark: deterministic across runs, finite, no status."""
    W, H, D = 192, 96, 96
    sdf = sphere_sdf(W, H, D, 48, 48, 48, 8)
    res = []
    for _ in range(2):
        s = Solver3D.create(W, H, D, precision="fp32", tau=0.524, uIn=0.1, spongeFraction=0.15, absorb=0.02)
        s.setSdf(sdf)
        s.initField(perturbed_rest3(W, H, D, 1e-4))
        s.run(40)
        res.append((s.readForcesArray(), s.readMacro().copy(), s.readStatus(), s.mass()))
        s.destroy()
    (f0, m0, st0, ms0), (f1, m1, st1, ms1) = res
    assert st0 == 0 and st1 == 0
    assert np.array_equal(f0, f1) and np.array_equal(m0, m1) and ms0 == ms1
    assert np.all(np.isfinite(m0)) and f0.shape == (40, 4)


@pytest.mark.parametrize("every", [1, 3, 4])
def test_graph_replay_matches_oracle(every):
    """Long step runs replay cached CUDA graphs (128 steps each, one per phase of the parity and
    sampling period); a parameter change between replays rebuilds them."""
    W, H, D = 20, 10, 8
    s, o = pair(W, H, D, "fp32", True, sphere_sdf(W, H, D, 6, 5, 4, 2), forceEvery=every)
    for n in (5, 260, 131):
        s.encodeSteps(n)
        o.encodeSteps(n)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.setTau(0.6)
    o.setTau(0.6)
    s.encodeSteps(200)
    o.encodeSteps(200)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    assert s.launchCount() >= 596  # one step kernel per step, whether replayed from a graph or not
    s.destroy()


def test_state_snapshot_resumes_bit_for_bit():
    """saveState after 137 steps, loadState into a fresh solver with the same SDF: the next 150 steps
    (ramp still running) give the same populations as the uninterrupted run."""
    W, H, D = 24, 16, 12
    sdf = sphere_sdf(W, H, D, 8, 8, 6, 3)
    cfg = dict(BASE, uIn=0.0)
    s = Solver3D.create(W, H, D, precision="fp32", exactArithmetic=True, **cfg)
    s.setSdf(sdf)
    s.initField(perturbed_rest3(W, H, D, 1e-4))
    s.setInletRamp("smoothstep", 0.08, 200, 1)
    s.encodeSteps(137)
    snap = s.saveState()
    s.encodeSteps(150)
    t = Solver3D.create(W, H, D, precision="fp32", exactArithmetic=True, **cfg)
    t.setSdf(sdf)
    t.loadState(snap)
    t.encodeSteps(150)
    a, b = s.readPopulations(), t.readPopulations()
    solid = np.tile((s.readFlags() & (1 << 19)) != 0, 19)
    assert np.array_equal(a.view(np.uint32)[~solid], b.view(np.uint32)[~solid])
    assert t.step == s.step == 287
    s.destroy()
    t.destroy()


# ---------------------------------------------------------------- grids wider than one x tile
#
# The interior kernel is chosen per block from the tile's x range: tiles that end before the first
# absorbing column compile without the absorbing sources (ABS = false), tiles that do not hold the
# outlet column without its rules (OUT = false). At W = 200 the FP64 kernel takes 7 tiles of 32
# cells (tiles 0-4 ABS = OUT = false, tile 5 ABS only, tile 6 both) and the x-pair kernel of FP32
# and 16-bit storage 4 tiles of 64 cells (tiles 0-1 neither, tile 2 ABS only, tile 3 both). With
# absorb = 0 every tile has ABS = false and the last one OUT = true. The bodies sit in tiles of each
# kind, so body rows (the flag test of the pair kernel) occur in each too.

WIDE = (200, 12, 10)


def wide_sdf():
    W, H, D = WIDE
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 41, 6, 5, 3)      # FP64 tile 1, pair tile 0
    g.add_sphere(sdf, W, H, D, 99.5, 5, 4, 2.5)  # FP64 tile 3, pair tile 1, across two x tiles
    g.add_box3(sdf, W, H, D, 178, 7, 5, 2, 2, 2)  # FP64 tile 5, pair tile 2: inside the absorbing layer
    return sdf


@pytest.mark.parametrize("absorb", [0.02, 0.0])
@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16", "fp64"])
def test_multi_tile_exact(precision, absorb):
    W, H, D = WIDE
    s, o = pair(W, H, D, precision, True, wide_sdf(), absorb=absorb)
    info = s.info()
    tile = 32 if precision == "fp64" else 64  # x-pair tiles for f32 and 16-bit storage
    assert info["block_x"] == tile, info  # tile width in cells
    assert np.array_equal(s.readFlags(), o.flags)
    for n in (1, 4, 20):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


@pytest.mark.parametrize("precision,tol", [("fp32", 2e-6), ("fp16", 1e-4), ("bf16", 1e-3)])
def test_multi_tile_fast(precision, tol):
    W, H, D = WIDE
    s, o = pair(W, H, D, precision, False, wide_sdf())
    for n in (1, 29):
        s.encodeSteps(n)
        o.encodeSteps(n)
        assert_same(s, o, False, tol)
    assert_forces(s.readForces(), o.readForces(), 1e-5 if precision == "fp32" else 2e-2)
    s.destroy()


# ---------------------------------------------------------------- the 192x96x96 benchmark tunnel


def config2_pair(exact, precision="fp32"):
    """The benchmark's D3Q19 tunnel (192x96x96, sphere d = 16 at (48, 48, 48), Re 200, sponge over the
    last 15% with absorb 0.02) on the GPU and on the oracle, started at the inflow speed 0.1 with
    the seeded 1e-4 transverse perturbation."""
    from cells_b200.units import derive_tau

    W, H, D = 192, 96, 96
    tau = derive_tau(200, 0.1, 16).tau
    cfg = dict(tau=tau, uIn=0.1, spongeFraction=0.15, spongeTau=1.0, absorb=0.02, forceEvery=1)
    s = Solver3D.create(W, H, D, precision=precision, exactArithmetic=exact, **cfg)
    o = OracleSolver3D(W, H, D, precision, **cfg)
    sdf = sphere_sdf(W, H, D, 48, 48, 48, 8)
    m = perturbed_rest3(W, H, D, 1e-4, ux=0.1)
    for x in (s, o):
        x.setSdf(sdf)
        x.initField(m)
    return s, o


def velocity_l2(a, b):
    """Relative L2 norm of the velocity difference over the cells where b is fluid (rho != 0)."""
    a = a.reshape(-1, 4).astype(np.float64)
    b = b.reshape(-1, 4).astype(np.float64)
    fl = b[:, 3] != 0
    du = a[fl, :3] - b[fl, :3]
    return float(np.sqrt(np.sum(du * du) / np.sum(b[fl, :3] ** 2)))


def test_config2_exact_bit_for_bit():
    """50 steps of the 192x96x96 tunnel: every population bit-identical to the oracle, so the tiles
    of every interior variant at the benchmark's size (two 64-cell tiles without the absorbing layer
    or the outlet, one with both), the face rows and the body are all checked."""
    s, o = config2_pair(True)
    s.encodeSteps(50)
    o.encodeSteps(50)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


def test_config2_fast_against_oracle():
    """200 steps of the 192x96x96 tunnel with the fast (FMA-contracted) kernel against the exact
    oracle: populations within 2e-6, the velocity field's relative L2 difference <= 1e-4, every force
    sample within 1e-5 relative."""
    s, o = config2_pair(False)
    s.encodeSteps(200)
    o.encodeSteps(200)
    assert_same(s, o, False, 2e-6)
    assert_forces(s.readForces(), o.readForces(), 1e-5)
    s.run(0)
    o.run(0)
    l2 = velocity_l2(s.readMacro(), o.readMacro())
    print("velocity L2", l2)
    assert l2 <= 1e-4
    s.destroy()


def test_config2_fp16_fast_against_oracle():
    """The same tunnel with FP16 storage, 100 steps: populations within a few storage ulps (1e-4) of
    the exact FP16 oracle, velocity L2 <= 1e-3, force samples within 1e-2 relative (the drag passes
    through small values in the start-up transient, where storage rounding shows most)."""
    s, o = config2_pair(False, "fp16")
    s.encodeSteps(100)
    o.encodeSteps(100)
    assert_same(s, o, False, 1e-4)
    assert_forces(s.readForces(), o.readForces(), 1e-2)
    s.run(0)
    o.run(0)
    l2 = velocity_l2(s.readMacro(), o.readMacro())
    print("velocity L2", l2)
    assert l2 <= 1e-3
    s.destroy()


def test_prepare_steps_runs_nothing_and_graphs_match():
    """prepareSteps captures the step graphs ahead of a run without stepping: the state is unchanged
    and the prepared run matches the oracle bit for bit."""
    W, H, D = 20, 10, 8
    s, o = pair(W, H, D, "fp32", True, sphere_sdf(W, H, D, 6, 5, 4, 2), forceEvery=2)
    s.encodeSteps(3)
    o.encodeSteps(3)
    before = s.readPopulations().copy()
    s.prepareSteps(300)
    assert s.step == 3
    assert np.array_equal(s.readPopulations().view(np.uint32), before.view(np.uint32))
    s.encodeSteps(300)
    o.encodeSteps(300)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


def test_pinned_host_buffers_round_trip():
    """cells_host_alloc buffers as inputs and as the readMacro destination give the same results as
    pageable numpy arrays."""
    from cells_b200._lib import pinned_empty

    W, H, D = 32, 16, 12
    sdf = sphere_sdf(W, H, D, 10, 8, 6, 3)
    m = perturbed_rest3(W, H, D, 1e-4, ux=0.05)
    out = []
    for pinned in (False, True):
        s = Solver3D.create(W, H, D, precision="fp32", **BASE)
        sd, mc = sdf, m
        if pinned:
            sd = pinned_empty(sdf.size, np.float32)
            sd[:] = sdf
            mc = pinned_empty(m.size, np.float32)
            mc[:] = m
        s.setSdf(sd)
        s.initField(mc)
        s.run(20)
        dst = pinned_empty(4 * W * H * D, np.float32) if pinned else None
        out.append(s.readMacro(dst).copy())
        s.destroy()
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16"])
def test_face_pair_rows_exact(precision):
    """Face rows as x-pair tiles: a sphere cut by the z = 0 face near the outlet and a box on the
    y = H-1 face at the inlet, with the absorbing layer on, so the face tiles meet body rows, the
    inlet and outlet columns and the absorbing sources."""
    W, H, D = 24, 7, 6
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 19, 3, 0.5, 2.2)
    g.add_box3(sdf, W, H, D, 2, 6, 3, 1.5, 1.2, 1.2)
    s, o = pair(W, H, D, precision, True, sdf)
    s.encodeSteps(12)
    o.encodeSteps(12)
    assert_same(s, o, True)
    assert_forces(s.readForces(), o.readForces(), 1e-9)
    s.destroy()


@pytest.mark.parametrize("dims", [(20, 3, 6), (20, 6, 3), (20, 4, 4), (20, 3, 3)])
@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_thin_grids_exact(dims, precision):
    """Grids with one or two interior rows or planes: the face-pair tiles are off below three
    cells in y or z (the face blocks then take every face row) and cover single rows above it."""
    W, H, D = dims
    sdf = g.empty_sdf3(W, H, D)
    s, o = pair(W, H, D, precision, True, sdf)
    s.encodeSteps(10)
    o.encodeSteps(10)
    assert_same(s, o, True)
    s.destroy()
