"""Failure detection on the GPU, tested without a GPU fault.

* Divergence: NaN populations written from the host into a running flow reach the momentum
  exchange and the macro field; the device status word records it (bit 1: a non-finite force
  sample, bit 2: a non-finite macro value), checkDiverged raises CELLS_E_DIVERGED, and the
  reference's host-side predicates (hasDiverged / fieldDiverged, src/tunnel3d.ts:97-105) agree.
  Re-initialising the flow, as the pages' recoverFromBlowup does, clears the status and the solver
  steps normally again.
* The persistent 2D kernel's grid barrier: a test hook makes every barrier wait for one arrival
  that never comes, so the bounded wait (one second) runs out; the kernel winds down, the call
  that waits for it raises CELLS_E_TIMEOUT, and after re-initialisation the batch gives the same
  populations as a batch that never failed.
"""
import time

import numpy as np
import pytest

from cells_b200 import Batch2D, Solver, Solver3D, analysis, geometry as g
from cells_b200._lib import CELLS_E_DIVERGED, CELLS_E_TIMEOUT, CellsError
from cells_b200.lattice3d import XMode, YMode
from cells_b200.rng import perturbed_rest2, perturbed_rest3

pytestmark = pytest.mark.gpu


def _poison_block(f, N, cells):
    """Sets every population of the given cells to NaN (f is the flat SoA array f[i * N + cell])."""
    for i in range(len(f) // N):
        f[i * N + cells] = np.nan


@pytest.mark.parametrize("precision", ["fp32", "fp16"])
def test_nan_populations_3d_set_status_and_diverged(precision):
    W, H, D = 32, 16, 12
    s = Solver3D.create(W, H, D, precision=precision, tau=0.56, uIn=0.05, spongeFraction=0.15, absorb=0.02,
                        forceEvery=1)
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 10, 8, 6, 3)
    s.setSdf(sdf)
    s.initField(perturbed_rest3(W, H, D, 1e-4, ux=0.05))
    s.encodeSteps(5)
    s.checkDiverged()
    assert s.readStatus() == 0 and not analysis.has_diverged(s.readForces())
    # NaN in a block of fluid cells upstream of the sphere, next to its surface
    N = W * H * D
    xs, ys, zs = np.meshgrid(np.arange(4, 7), np.arange(6, 11), np.arange(4, 9), indexing="ij")
    cells = (xs + W * (ys + H * zs)).ravel()
    f = s.readPopulations()
    _poison_block(f, N, cells)
    s.writePopulations(f)
    s.encodeSteps(4)
    assert analysis.has_diverged(s.readForces())
    assert s.readStatus() & 1
    s.run(0)  # macro refresh
    assert s.readStatus() & 2
    assert analysis.field_diverged(s.readMacro())
    with pytest.raises(CellsError) as e:
        s.checkDiverged()
    assert e.value.status == CELLS_E_DIVERGED
    assert "diverged" in str(e.value)
    # recover: a new flow clears the status word
    s.initField(perturbed_rest3(W, H, D, 1e-4, ux=0.05))
    assert s.readStatus() == 0
    s.run(20)
    s.checkDiverged()
    assert not analysis.has_diverged(s.readForces())
    assert not analysis.field_diverged(s.readMacro())
    s.destroy()


def test_nan_populations_2d_set_status_and_diverged():
    W, H = 96, 48
    s = Solver.create(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                      tau=0.56, uIn=0.05, forceEvery=1)
    sdf = g.empty_sdf(W, H)
    g.add_circle(sdf, W, H, 24, 24.3, 5)
    s.setSdf(sdf)
    s.initField(perturbed_rest2(W, H, 1e-4))
    s.encodeSteps(5)
    s.checkDiverged()
    N = W * H
    xs, ys = np.meshgrid(np.arange(15, 19), np.arange(20, 29), indexing="ij")
    f = s.readPopulations()
    _poison_block(f, N, (xs + W * ys).ravel())
    s.writePopulations(f)
    s.encodeSteps(4)
    assert analysis.has_diverged(s.readForces())
    s.run(0)
    assert s.readStatus() & 3 == 3
    with pytest.raises(CellsError) as e:
        s.checkDiverged()
    assert e.value.status == CELLS_E_DIVERGED
    s.initField(perturbed_rest2(W, H, 1e-4))
    assert s.readStatus() == 0
    s.run(20)
    s.checkDiverged()
    s.destroy()


def _barrier_batch():
    cfgs = [dict(width=96, height=40, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                 tau=0.56, uIn=0.05, forceEvery=1, exactArithmetic=True),
            dict(width=64, height=32, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip,
                 top=YMode.NoSlip, tau=0.7, bodyForce=(1e-5, 0.0), forceEvery=2, exactArithmetic=True)]
    b = Batch2D(cfgs)
    b.setLaunch(64, 2, True)  # persistent launches
    for t, c in zip(b.tunnels, cfgs):
        sdf = g.empty_sdf(c["width"], c["height"])
        g.add_circle(sdf, c["width"], c["height"], c["width"] / 4, c["height"] / 2 + 0.3, 4)
        t.setSdf(sdf)
        t.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
    return b, cfgs


def test_persistent_barrier_timeout_is_reported_and_recoverable():
    b, cfgs = _barrier_batch()
    b.step(12)
    b.synchronize()
    assert all(t.readStatus() == 0 for t in b.tunnels)
    b.setBarrierTest(1)
    t0 = time.perf_counter()
    with pytest.raises(CellsError) as e:
        b.step(12)
        b.synchronize()
    waited = time.perf_counter() - t0
    assert e.value.status == CELLS_E_TIMEOUT, str(e.value)
    assert waited < 30.0, waited  # one bounded wait of about a second, not a hang
    b.setBarrierTest(0)
    # re-initialise, then step beside a batch that never failed: same populations bit for bit
    ref, _ = _barrier_batch()
    for bb in (b, ref):
        for t, c in zip(bb.tunnels, cfgs):
            t.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
        bb.step(40)
        bb.synchronize()
    for t, r in zip(b.tunnels, ref.tunnels):
        a, c = t.readPopulations(), r.readPopulations()
        assert np.array_equal(a.view(np.uint32), c.view(np.uint32))
        assert t.readStatus() == 0
    b.destroy()
    ref.destroy()
