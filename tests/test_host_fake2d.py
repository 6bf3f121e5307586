"""Host-side logic of the 2D C ABI on the fake device (no GPU, no kernels): the Params block as
writeParams packs it (src/solver.ts:180-197), the force ring's window and generation check (the
reference's fakeDevice() test, src/solver.test.ts:38-81), error conventions of create, and the
batch rules."""
import struct

import pytest

from cells_b200 import Batch2D, Solver, _lib
from cells_b200.lattice3d import XMode, YMode

FAKE = _lib.FAKE_DEVICE


def fake(**kw):
    c = dict(width=40, height=20, tau=0.6, device=FAKE)
    c.update(kw)
    return Solver.create(**c)


def test_params_block_follows_write_params():
    s = fake(left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.MovingWall, uIn=0.05, parabolic=True,
             spongeFraction=0.15, spongeTau=0.9, uLid=0.02, bodyForce=(1e-5, -2e-6), absorb=0.02,
             inletLayerFraction=0.08, smagorinsky=0.1)
    p = s.readParams()
    assert len(p) == 96
    u = struct.unpack("<24I", p)
    f = struct.unpack("<24f", p)
    assert u[:8] == (40, 20, 800, 7, 2, 2, 2, 3)  # groupsX = ceil(800 / 128)
    assert f[8] == pytest.approx(0.6, abs=1e-7) and f[9] == pytest.approx(3 / 16)
    assert f[10] == pytest.approx(0.01, rel=1e-6) and f[11] == pytest.approx(0.05, rel=1e-6)
    assert u[12] == 1
    assert f[13] == pytest.approx(39 * 0.85, rel=1e-6)
    assert f[14] == pytest.approx(0.9, rel=1e-6)  # max(spongeTau, tau)
    assert f[15] == pytest.approx(0.02, rel=1e-6)
    assert (f[16], f[17]) == (pytest.approx(1e-5, rel=1e-6), pytest.approx(-2e-6, rel=1e-6))
    assert u[18] == 1 and f[19] == pytest.approx(0.02, rel=1e-6)
    assert f[20] == pytest.approx(0.08 * 39, rel=1e-6)
    s.update(spongeFraction=0.0, bodyForce=(0.0, 0.0), tau=0.7)
    f = struct.unpack("<24f", s.readParams())
    u = struct.unpack("<24I", s.readParams())
    assert f[13] == 1e9 and u[18] == 0 and f[14] == pytest.approx(0.9, rel=1e-6)
    s.update(spongeTau=1.0)
    assert struct.unpack("<24f", s.readParams())[14] == pytest.approx(1.0)
    s.destroy()


def test_force_read_in_flight_across_reset_returns_nothing_and_keeps_alignment():
    """src/solver.test.ts:38-81 with the library's ring and generation check."""
    s = fake(forceEvery=4)
    s.fakeSetForce(99.0, 0.0)
    s.encodeSteps(4000)
    s.readForcesBegin()
    s.initField()  # step = 0 and resetForces, while the read is in flight
    s.fakeSetForce(1.0, 0.0)
    s.encodeSteps(40)
    assert s.readForcesEnd() == []
    s.fakeSetForce(2.0, 0.0)
    s.encodeSteps(400)
    samples = s.readForces()
    assert len(samples) == 110
    assert samples[0]["step"] == 4 and samples[0]["fx"] == 1.0
    assert samples[109]["step"] == 440 and samples[109]["fx"] == 2.0
    s.fakeSetForce(3.0, 0.0)
    s.encodeSteps(400)
    third = s.readForces()
    assert third[0]["step"] == 444 and third[0]["fx"] == 3.0
    s.destroy()


def test_ring_drops_overwritten_samples():
    s = fake(forceEvery=1)
    s.encodeSteps(8192 + 100)
    f = s.readForces()
    assert len(f) == 8192 and f[0]["step"] == 101 and f[-1]["step"] == 8292
    s.destroy()


def test_allocation_failure_frees_everything():
    before = _lib.lib().cells_fake_live_buffers()
    for at in (1, 2, 5, 8):
        with pytest.raises(_lib.CellsError) as e:
            fake(fakeFailAlloc=at)
        assert str(e.value).startswith("Solver allocation failed: ")
        assert e.value.status == _lib.CELLS_E_ALLOC
        assert _lib.lib().cells_fake_live_buffers() == before


def test_over_limit_fails_before_allocating():
    before = _lib.lib().cells_fake_live_buffers()
    with pytest.raises(_lib.CellsError) as e:
        fake(width=1000, height=1000, maxBufferBytes=1 << 20)
    assert str(e.value).startswith("Solver allocation failed: one distribution buffer needs 36000000 bytes")
    assert _lib.lib().cells_fake_live_buffers() == before


def test_bad_configs():
    with pytest.raises(_lib.CellsError) as e:
        fake(precision="fp16")
    assert e.value.status == _lib.CELLS_E_PRECISION_UNSUPPORTED
    with pytest.raises(_lib.CellsError):
        fake(tau=0.5)
    with pytest.raises(_lib.CellsError):
        fake(width=1)
    with pytest.raises(_lib.CellsError):
        fake(top=7)
    for wg in (32, 96, 512):
        with pytest.raises(_lib.CellsError) as e:
            fake(workgroupSize=wg)
        assert e.value.status == _lib.CELLS_E_INVALID
    for wg in (0, 64, 128, 256):
        fake(workgroupSize=wg).destroy()


def test_batch_rules():
    b = Batch2D([dict(width=64, height=16, tau=0.7, device=FAKE),
                 dict(width=100, height=25, tau=0.55, device=FAKE, forceEvery=2)])
    b.step(7)
    assert [t.step for t in b.tunnels] == [7, 7]
    assert [f["step"] for f in b.tunnels[1].readForces()] == [2, 4, 6]
    with pytest.raises(_lib.CellsError):
        b.tunnels[0].encodeSteps(1)  # a tunnel of a batch steps with the batch
    b.tunnels[0].initField()
    b.step(3)
    assert [t.step for t in b.tunnels] == [3, 10]
    info = b.info()
    assert info["tunnels"] == 2 and info["N"] == 64 * 16 + 100 * 25
    b.setLaunch(64, 2, False)
    assert b.info()["tile_x"] == 64
    with pytest.raises(_lib.CellsError):
        b.setLaunch(48, 2, False)
    with pytest.raises(_lib.CellsError):
        Batch2D([dict(width=64, height=16, tau=0.7, device=FAKE),
                 dict(width=64, height=16, tau=0.7, device=FAKE, precision="fp64")])
    b.destroy()


def test_update_cannot_change_grid():
    s = fake()
    with pytest.raises(_lib.CellsError):
        s.update(width=41)
    s.destroy()
