"""cells3d_mass_noalloc, the allocation-free mass reduction, against the handle's cells3d_mass.

Callers that cannot allocate device memory (a host or plugin framework that owns every device
buffer, a real-time loop) pass their own device buffers; this test plays such a caller. torch only holds
the caller's device buffers here. The two reductions sum the same f64 values in different orders,
so they agree to 1e-12 relative. The file name sorts last so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from cells_b200 import Solver3D, _lib, geometry as g
from cells_b200.rng import perturbed_rest3

pytestmark = pytest.mark.gpu

REL = 1e-12
TORCH_DTYPE = {"fp32": "float32", "fp16": "float16", "bf16": "int16", "fp64": "float64"}


def device_copy(torch, arr, dtype):
    host = torch.from_numpy(np.ascontiguousarray(arr).view(getattr(np, dtype) if dtype != "int16" else np.int16))
    return host.to("cuda")


def noalloc_mass(torch, pops, flags, n, precision, out, stream):
    rc = _lib.lib().cells3d_mass_noalloc(ctypes.c_void_p(pops.data_ptr()), ctypes.c_void_p(flags.data_ptr()), n,
                                         _lib.PRECISIONS[precision], ctypes.c_void_p(out.data_ptr()),
                                         ctypes.c_void_p(stream))
    return rc


@pytest.mark.parametrize("precision", ["fp32", "fp16", "bf16", "fp64"])
def test_noalloc_mass_matches_handle_mass_twice(precision):
    torch = pytest.importorskip("torch")
    W, H, D = 48, 24, 24
    N = W * H * D
    s = Solver3D.create(W, H, D, precision=precision, tau=0.56, uIn=0.05, spongeFraction=0.15, absorb=0.02)
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, 12, 12, 12, 4)
    s.setSdf(sdf)
    s.initField(perturbed_rest3(W, H, D, 1e-4, ux=0.05))
    stream = torch.cuda.current_stream().cuda_stream
    flags = device_copy(torch, s.readFlags().view(np.int32), "int32")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for steps in (5, 7):  # two calls in a row, on different states
        s.run(steps)
        want = s.mass()
        pops = device_copy(torch, s.readPopulations(), TORCH_DTYPE[precision])
        assert noalloc_mass(torch, pops, flags, N, precision, out, stream) == _lib.CELLS_OK
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= REL * abs(want), (got, want)
    s.destroy()


def test_noalloc_mass_rejects_grids_beyond_the_scratch():
    torch = pytest.importorskip("torch")
    tiny = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = _lib.lib().cells3d_mass_noalloc(ctypes.c_void_p(tiny.data_ptr()), ctypes.c_void_p(tiny.data_ptr()),
                                         8192 * 8192 + 1, _lib.FP32, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.CELLS_E_INVALID
    assert "exceed the maximum of 67108864" in _lib.lib().cells_last_error(None).decode()
