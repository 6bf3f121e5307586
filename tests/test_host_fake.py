"""Host-side logic of the C ABI on the fake device (no GPU, no kernels): parameter packing, the
error conventions of create, and the force ring's bookkeeping. These port the reference's
fakeDevice() tests, src/solver3d.test.ts:73-195 and src/solver.test.ts:38-81."""
import json
import os
import struct

import numpy as np
import pytest

from cells_b200 import Solver3D, _lib

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
CFG = dict(width=8, height=6, depth=4, tau=0.6, device=_lib.FAKE_DEVICE)


def fake(**kw):
    c = dict(CFG)
    c.update(kw)
    return Solver3D.create(**c)


def test_params_layout():
    k = GOLD["params_layout"]
    s = fake(uIn=0.0, spongeFraction=0.15)
    p = s.readParams()
    u = struct.unpack("<16I", p)
    f = struct.unpack("<16f", p)
    assert list(u[:4]) == k["u32_0_4"]
    assert abs(f[8] - 0.6) < 5e-7
    assert abs(f[12] - 7 * 0.85) < 5e-6
    s.setInlet(0.05)
    assert abs(struct.unpack("<16f", s.readParams())[11] - 0.05) < 5e-7
    s.setTau(0.7)
    assert abs(struct.unpack("<16f", s.readParams())[8] - 0.7) < 5e-7
    s.setSmagorinsky(0.16)
    assert abs(struct.unpack("<16f", s.readParams())[10] - 0.0256) < 5e-7
    assert s.cfg["smagorinsky"] == 0.16
    s.destroy()


def test_params_derivations():
    """spongeStart = 1e9 when off, tauSponge = max(spongeTau, tau), Lambda = trtLambda3(base tau)
    unless fixed (src/solver3d.ts:197-208)."""
    s = fake(tau=0.524)
    f = struct.unpack("<16f", s.readParams())
    assert f[12] == np.float32(1e9)
    assert f[13] == np.float32(1.0)
    assert f[9] == np.float32(50 * 0.024 ** 2)
    s.setLambda(0.1)
    assert struct.unpack("<16f", s.readParams())[9] == np.float32(0.1)
    s.setLambda(None)
    s.setTau(1.5)
    f = struct.unpack("<16f", s.readParams())
    assert f[13] == np.float32(1.5) and f[9] == np.float32(3 / 16)
    s.destroy()


def test_over_limit_fails_before_allocating():
    N = 8 * 6 * 4
    before = _lib.lib().cells_fake_live_buffers()
    with pytest.raises(_lib.CellsError) as e:
        fake(maxBufferBytes=19 * 4 * N - 1)
    assert e.value.status == _lib.CELLS_E_ALLOC
    assert str(e.value) == (f"Solver3D allocation failed: one distribution buffer needs {19 * 4 * N} bytes; "
                            f"this device allows {19 * 4 * N - 1} per buffer")
    assert _lib.lib().cells_fake_live_buffers() == before


@pytest.mark.parametrize("at", [1, 2, 5, 9])
def test_allocation_error_frees_everything(at):
    before = _lib.lib().cells_fake_live_buffers()
    with pytest.raises(_lib.CellsError) as e:
        fake(fakeFailAlloc=at)
    assert e.value.status == _lib.CELLS_E_ALLOC
    assert str(e.value).startswith("Solver3D allocation failed: fake out-of-memory")
    assert _lib.lib().cells_fake_live_buffers() == before


def test_destroy_frees_everything():
    before = _lib.lib().cells_fake_live_buffers()
    s = fake()
    assert _lib.lib().cells_fake_live_buffers() > before
    s.destroy()
    assert _lib.lib().cells_fake_live_buffers() == before


def test_unknown_precision_and_bad_grid():
    with pytest.raises(_lib.CellsError) as e:
        fake(precision="fp8")
    assert e.value.status == _lib.CELLS_E_PRECISION_UNSUPPORTED
    with pytest.raises(_lib.CellsError) as e:
        Solver3D.create(width=2, height=4, depth=4, device=_lib.FAKE_DEVICE)
    assert e.value.status == _lib.CELLS_E_INVALID


def test_buffer_sizes_follow_precision():
    """19 * b * N per distribution buffer (src/solver3d.test.ts:145-155), seen through the raw
    population access that needs exactly that many bytes."""
    N = 8 * 6 * 4
    for prec, b in (("fp16", 2), ("fp32", 4), ("bf16", 2), ("fp64", 8)):
        s = fake(precision=prec)
        assert s.readPopulations().nbytes == 19 * b * N
        s.destroy()


def test_force_ring_discards_read_overtaken_by_reset():
    """src/solver3d.test.ts:157-195: a read in flight across a reset returns nothing, and the samples
    after the reset keep their step numbers aligned (the reference resets step by hand there;
    initField resets step, parity and forces here)."""
    k = GOLD["force_ring_alignment"]
    s = fake(forceEvery=4)
    s.fakeSetForce(99, 198, 297)
    s.encodeSteps(4000)
    s.readForcesBegin()
    s.initField()  # step = 0, parity = 0, forces reset
    s.fakeSetForce(1, 2, 3)
    s.encodeSteps(40)
    assert s.readForcesEnd() == []
    s.fakeSetForce(2, 4, 6)
    s.encodeSteps(400)
    samples = s.readForces()
    assert len(samples) == k["expect_count"]
    assert samples[0] == {"step": 4, "fx": 1, "fy": 2, "fz": 3}
    assert samples[-1] == {"step": 440, "fx": 2, "fy": 4, "fz": 6}
    s.fakeSetForce(3, 6, 9)
    s.encodeSteps(400)
    third = s.readForces()
    assert third[0]["step"] == 444 and third[0]["fx"] == 3
    assert s.readForces() == []
    s.destroy()


def test_force_ring_drops_overwritten_samples():
    """Only the newest 8192 samples survive the ring (src/solver3d.ts:306)."""
    s = fake(forceEvery=1)
    s.fakeSetForce(1, 0, 0)
    s.encodeSteps(10000)
    samples = s.readForces()
    assert len(samples) == 8192
    assert samples[0]["step"] == 10000 - 8192 + 1 and samples[-1]["step"] == 10000
    s.encodeSteps(5)
    assert [x["step"] for x in s.readForces()] == [10001, 10002, 10003, 10004, 10005]
    s.destroy()


def test_force_every_zero_disables_sampling():
    s = fake(forceEvery=0)
    s.encodeSteps(100)
    assert s.readForces() == []
    s.destroy()


def test_state_snapshot_round_trip_and_checks():
    s = fake(forceEvery=2)
    s.setInletRamp("linear", 0.1, 300, 1)
    s.encodeSteps(7)
    snap = s.saveState()
    t = fake(forceEvery=2)
    t.loadState(snap)
    assert t.step == 7
    assert t.readParams() == s.readParams()
    assert t.readForces() == []
    with pytest.raises(_lib.CellsError):
        t.loadState(snap[:-1])
    with pytest.raises(_lib.CellsError):
        fake(width=9).loadState(snap)
    bad = bytearray(snap)
    bad[0] ^= 1
    with pytest.raises(_lib.CellsError):
        t.loadState(bytes(bad))
    s.destroy()
    t.destroy()


def test_field_products_check_their_arguments():
    s = fake(width=12, height=8, depth=6)
    out = s.sampleSlice(2, 0.5, "vorticity", 0.1)
    assert out.shape == (8, 12)
    for bad in (dict(axis=3), dict(pos=1.5), dict(mode="pressure"), dict(uRef=0.0), dict(size=(0, 4))):
        kw = dict(axis=0, pos=0.5, mode="speed", uRef=0.1, size=None)
        kw.update(bad)
        with pytest.raises(_lib.CellsError) as e:
            s.sampleSlice(**kw)
        assert e.value.status == _lib.CELLS_E_INVALID
    parts = np.zeros((4, 8), dtype=np.float32)
    s.advectTracers(np.zeros((4, 4), dtype=np.float32), parts, 10.0, 0.1)
    with pytest.raises(_lib.CellsError):
        s.advectTracers(np.zeros((4, 4), dtype=np.float32), parts, -1.0, 0.1)
    with pytest.raises(ValueError):
        s.advectTracers(np.zeros((3, 4), dtype=np.float32), parts, 1.0, 0.1)
    s.destroy()
