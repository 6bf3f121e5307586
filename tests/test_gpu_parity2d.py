"""Parity of the CUDA D2Q9 path (through the C ABI) with the CPU oracle on the same seeded inputs.

Exact arithmetic (CELLS_ARITH_EXACT): every stored population must match the oracle bit for bit,
for every boundary kind of the reference's 2D solver (Zou-He inlet and outlet, slip, no-slip,
moving wall, periodic seams with Bouzidi links across them, walls), with Smagorinsky, absorbing
layers, body force and parabolic inflow, in f32 and f64, single tunnels and batches, per-step and
persistent launches. Fast arithmetic (FMA contraction): populations within 2e-6 absolute.
Force samples are f64 sums in different orders (tiles vs cell order): 1e-9 relative.
Flags are compared without the force-slot numbers, which the reference assigns in atomic order;
only whether a cell has a slot matters.
"""
import numpy as np
import pytest

from cells_b200 import Batch2D, Solver, geometry as g
from cells_b200.lattice3d import XMode, YMode
from cells_b200.rng import perturbed_rest2
from oracle.oracle import OracleSolver2D

pytestmark = pytest.mark.gpu

OPEN_TUNNEL = dict(left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip, tau=0.56, uIn=0.05,
                   spongeFraction=0.15, spongeTau=1.0, absorb=0.02, forceEvery=1)


def circle_sdf(W, H, cx, cy, r):
    sdf = g.empty_sdf(W, H)
    g.add_circle(sdf, W, H, cx, cy, r)
    return sdf


def make_pair(W, H, sdf, precision="fp32", exact=True, macro=None, **cfg):
    s = Solver.create(width=W, height=H, precision=precision, exactArithmetic=exact, **cfg)
    o = OracleSolver2D(W, H, precision=precision, **cfg)
    if sdf is not None:
        s.setSdf(sdf)
        o.setSdf(sdf)
    m = perturbed_rest2(W, H, 1e-4) if macro is None else macro
    s.initField(m)
    o.initField(m)
    return s, o


def same_flags(a, b):
    low = np.array_equal(a & 0xFFF, b & 0xFFF)
    slots = np.array_equal((a >> 12) != 0, (b >> 12) != 0)
    return low and slots


def assert_same(a, b, exact, tol=2e-6):
    assert a.shape == b.shape
    if exact:
        bad = np.flatnonzero(a.view(f"u{a.itemsize}") != b.view(f"u{b.itemsize}"))
        assert bad.size == 0, f"{bad.size} populations differ, first at {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"
    else:
        err = float(np.max(np.abs(a.astype(np.float64) - b.astype(np.float64))))
        assert err <= tol, f"max population difference {err}"


def assert_forces(fs, fo, rel=1e-9):
    assert [x["step"] for x in fs] == [x["step"] for x in fo]
    for a, b in zip(fs, fo):
        scale = max(abs(b["fx"]), abs(b["fy"]), 1e-12)
        assert abs(a["fx"] - b["fx"]) <= rel * scale and abs(a["fy"] - b["fy"]) <= rel * scale, (a, b)


def advance(s, o, n, ramp=None):
    """n steps on both; ramp(step) -> inlet speed set before each step, as runRamped does per chunk."""
    if ramp is None:
        s.encodeSteps(n)
        o.encodeSteps(n)
        return
    for _ in range(n):
        u = ramp(o.step)
        s.setInlet(u)
        o.update(uIn=u)
        s.encodeSteps(1)
        o.encodeSteps(1)


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_open_tunnel_cylinder_exact(precision):
    W, H = 96, 40
    s, o = make_pair(W, H, circle_sdf(W, H, 24, 20.3, 6), precision, **OPEN_TUNNEL)
    assert same_flags(s.readFlags(), o.flags)
    for n in (1, 5, 60):
        advance(s, o, n)
        assert_same(s.readPopulations(), o.populations(), True)
    assert_forces(s.readForces(), o.readForces())
    s.run(3)
    o.run(3)
    assert np.array_equal(s.readMacro().view(np.uint32), o.readMacro().view(np.uint32))
    s.destroy()


def test_open_tunnel_host_ramp_exact():
    W, H = 80, 32
    s, o = make_pair(W, H, circle_sdf(W, H, 20, 16.5, 5), **OPEN_TUNNEL)
    advance(s, o, 40, ramp=lambda st: 0.08 * min(1.0, st / 30))
    assert_same(s.readPopulations(), o.populations(), True)
    assert_forces(s.readForces(), o.readForces())
    s.destroy()


def test_device_ramp_matches_host_ramp():
    """set_inlet_ramp(smoothstep, update_every=7) equals setting the inlet per step on the host."""
    W, H = 64, 24
    s, o = make_pair(W, H, circle_sdf(W, H, 16, 12, 4), **OPEN_TUNNEL)
    s.setInletRamp("smoothstep", 0.1, 50, 7)

    def ramp(st):
        q = (st // 7) * 7
        t = min(1.0, q / 50)
        return 0.1 * (t * t * (3 - 2 * t))

    for _ in range(60):
        o.update(uIn=ramp(o.step))
        o.encodeSteps(1)
    s.encodeSteps(60)
    assert_same(s.readPopulations(), o.populations(), True)
    s.destroy()


def test_periodic_channel_seam_body_force_exact():
    """Periodic x with a body force and a cylinder cut by the seam: Bouzidi links across the seam."""
    W, H = 64, 32
    sdf = circle_sdf(W, H, 2.5, 15.5, 5)
    g.add_circle(sdf, W, H, 2.5 + W, 15.5, 5)
    cfg = dict(left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip, top=YMode.NoSlip, tau=0.8,
               bodyForce=(2e-6, 0.0), forceEvery=3)
    s, o = make_pair(W, H, sdf, **cfg)
    assert same_flags(s.readFlags(), o.flags)
    advance(s, o, 50)
    assert_same(s.readPopulations(), o.populations(), True)
    assert_forces(s.readForces(), o.readForces())
    s.run(1)
    o.run(1)
    assert np.array_equal(s.readMacro().view(np.uint32), o.readMacro().view(np.uint32))
    s.destroy()


def test_cavity_moving_lid_smagorinsky_exact():
    W = H = 48
    cfg = dict(left=XMode.Wall, right=XMode.Wall, bottom=YMode.NoSlip, top=YMode.MovingWall, tau=0.52, uLid=0.1,
               smagorinsky=0.1, forceEvery=0)
    s, o = make_pair(W, H, None, **cfg)
    advance(s, o, 80)
    assert_same(s.readPopulations(), o.populations(), True)
    s.destroy()


def test_parabolic_inlet_layer_noslip_exact():
    W, H = 120, 30
    cfg = dict(left=XMode.Open, right=XMode.Open, bottom=YMode.NoSlip, top=YMode.NoSlip, tau=0.6, uIn=0.06,
               parabolic=True, spongeFraction=0.1, absorb=0.1, inletLayerFraction=0.08, forceEvery=2)
    s, o = make_pair(W, H, circle_sdf(W, H, 30, 14.5, 4), **cfg)
    advance(s, o, 45)
    assert_same(s.readPopulations(), o.populations(), True)
    assert_forces(s.readForces(), o.readForces())
    s.destroy()


def test_update_and_moved_obstacle_refill_exact():
    """update(partial) mid-run, a moved obstacle (refill of uncovered cells), a brush stroke."""
    W, H = 72, 28
    s, o = make_pair(W, H, circle_sdf(W, H, 20, 14, 5), **OPEN_TUNNEL)
    advance(s, o, 20)
    s.update(tau=0.6, absorb=0.05, smagorinsky=0.12)
    o.update(tau=0.6, absorb=0.05, smagorinsky=0.12)
    sdf2 = circle_sdf(W, H, 23, 14, 5)
    s.setSdf(sdf2)
    o.setSdf(sdf2)
    assert same_flags(s.readFlags(), o.flags)
    advance(s, o, 15)
    s.brushStroke([(40, 10), (42, 11)], 3.0, False)
    for x, y in [(40, 10), (42, 11)]:
        o.brush(x, y, 3.0, False, rebuild=False)
    o._rebuild_flags()
    assert np.array_equal(s.readSdf().view(np.uint32), o.sdf.view(np.uint32))
    assert same_flags(s.readFlags(), o.flags)
    advance(s, o, 15)
    assert_same(s.readPopulations(), o.populations(), True)
    assert_forces(s.readForces(), o.readForces())
    s.destroy()


def test_fast_arithmetic_within_tolerance():
    W, H = 96, 40
    s, o = make_pair(W, H, circle_sdf(W, H, 24, 20.3, 6), exact=False, **OPEN_TUNNEL)
    advance(s, o, 30)
    assert_same(s.readPopulations(), o.populations(), False)
    assert_forces(s.readForces(), o.readForces(), rel=1e-4)
    s.destroy()


def batch_configs():
    return [
        dict(width=70, height=20, **OPEN_TUNNEL),
        dict(width=33, height=45, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip,
             top=YMode.NoSlip, tau=0.7, bodyForce=(1e-5, 0.0), forceEvery=2),
        dict(width=128, height=32, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip, tau=0.53,
             uIn=0.1, smagorinsky=0.1, spongeFraction=0.15, absorb=0.02, forceEvery=5),
    ]


def batch_sdfs(cfgs):
    out = []
    for c in cfgs:
        W, H = c["width"], c["height"]
        out.append(circle_sdf(W, H, W / 4, H / 2 + 0.3, max(2.0, H / 8)))
    return out


@pytest.mark.parametrize("launch", [None, (32, 2, False), (64, 4, False), (128, 1, True), (32, 8, True)])
def test_batch_matches_oracle_per_tunnel(launch):
    cfgs = batch_configs()
    b = Batch2D([dict(c, exactArithmetic=True) for c in cfgs])
    if launch is not None:
        b.setLaunch(*launch)
    oracles = []
    for t, c, sdf in zip(b.tunnels, cfgs, batch_sdfs(cfgs)):
        kw = {k: v for k, v in c.items() if k not in ("width", "height")}
        o = OracleSolver2D(c["width"], c["height"], **kw)
        t.setSdf(sdf)
        o.setSdf(sdf)
        m = perturbed_rest2(c["width"], c["height"], 1e-4)
        t.initField(m)
        o.initField(m)
        oracles.append(o)
    b.step(7)
    b.step(130)  # crosses a graph (or persistent chunk) boundary
    for o in oracles:
        o.encodeSteps(137)
    for t, o in zip(b.tunnels, oracles):
        assert_same(t.readPopulations(), o.populations(), True)
        assert_forces(t.readForces(), o.readForces())
    assert b.tunnels[0].readStatus() == 0
    b.destroy()


def test_batch_two_rows_per_thread_matches_oracle():
    """A batch of 4,096 tiles or more takes the kernel with two cell rows per thread; 2 tunnels of
    1000 x 253 (32 x 64 tiles of 32 x 4 threads each) reach it, with an odd height (the last row pair
    of a column has one row) and a width that is not a multiple of the tile."""
    W, H = 1000, 253
    cfgs = [dict(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                 tau=0.56, uIn=0.08, smagorinsky=0.1, spongeFraction=0.15, absorb=0.02, forceEvery=1),
            dict(width=W, height=H, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip,
                 top=YMode.NoSlip, tau=0.7, bodyForce=(1e-6, 0.0), forceEvery=3)]
    b = Batch2D([dict(c, exactArithmetic=True) for c in cfgs])
    b.setLaunch(32, 4, False)
    oracles = []
    for t, c in zip(b.tunnels, cfgs):
        sdf = circle_sdf(W, H, W / 4, H / 2 + 0.3, 12.0)
        kw = {k: v for k, v in c.items() if k not in ("width", "height")}
        o = OracleSolver2D(W, H, **kw)
        t.setSdf(sdf)
        o.setSdf(sdf)
        m = perturbed_rest2(W, H, 1e-4)
        t.initField(m)
        o.initField(m)
        oracles.append(o)
    b.step(3)
    b.step(100)  # one graph of 100 steps
    for o in oracles:
        o.encodeSteps(103)
    for t, o in zip(b.tunnels, oracles):
        assert_same(t.readPopulations(), o.populations(), True)
        assert_forces(t.readForces(), o.readForces())
    b.destroy()


@pytest.mark.parametrize("trial_steps", [40, 100])
def test_autotune_keeps_state_and_results(trial_steps):
    """Trials of 100 steps or more time graph replays (graphs rebuilt before the timed region), so
    both trial kinds run; the state is restored and later steps match an untuned batch."""
    cfgs = batch_configs()
    a = Batch2D([dict(c, exactArithmetic=True) for c in cfgs])
    ref = Batch2D([dict(c, exactArithmetic=True) for c in cfgs])
    for bb in (a, ref):
        for t, c, sdf in zip(bb.tunnels, cfgs, batch_sdfs(cfgs)):
            t.setSdf(sdf)
            t.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
        bb.step(11)
    before = [t.readPopulations() for t in a.tunnels]
    info = a.autotune(trial_steps)
    assert info["tile_x"] * info["tile_y"] in (64, 128, 256)
    for t, p in zip(a.tunnels, before):
        assert_same(t.readPopulations(), p, True)
    a.step(60)
    ref.step(60)
    for t, r in zip(a.tunnels, ref.tunnels):
        assert_same(t.readPopulations(), r.readPopulations(), True)
        assert t.step == r.step == 71
        fa, fr = t.readForces(), r.readForces()
        assert_forces(fa, fr)
    a.destroy()
    ref.destroy()


def test_mass_and_status():
    W, H = 64, 32
    s, o = make_pair(W, H, circle_sdf(W, H, 16, 16, 4), **OPEN_TUNNEL)
    advance(s, o, 10)
    assert abs(s.mass() - o.mass()) <= 1e-9 * abs(o.mass())
    assert s.readStatus() == 0
    s.destroy()
