"""ctypes binding of libcells.so (the C ABI declared in include/cells.h).

The library is built in-tree (``cells_b200/libcells.so``) by ``__graft_entry__.build()``. There is
no fallback: importing a solver without the built library raises, so a missing extension can never
silently turn into a CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcells.so")

CELLS_OK = 0
CELLS_E_ALLOC = 1
CELLS_E_PRECISION_UNSUPPORTED = 2
CELLS_E_INVALID = 3
CELLS_E_CUDA = 4
CELLS_E_DIVERGED = 5
CELLS_E_TIMEOUT = 6

FP32, FP16, BF16, FP64 = 0, 1, 2, 3
PRECISIONS = {"fp32": FP32, "fp16": FP16, "bf16": BF16, "fp64": FP64}
BYTES_PER_POPULATION = {FP32: 4, FP16: 2, BF16: 2, FP64: 8}
FAKE_DEVICE = -2
RAMP_NONE, RAMP_LINEAR, RAMP_SMOOTHSTEP = 0, 1, 2
ARITH_FAST, ARITH_EXACT = 0, 1


class Cells3DConfig(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32), ("precision", C.c_int32),
        ("tau", C.c_double), ("lambda_", C.c_double), ("smagorinsky", C.c_double), ("u_in", C.c_double),
        ("sponge_fraction", C.c_double), ("sponge_tau", C.c_double), ("absorb", C.c_double),
        ("workgroup_size", C.c_int32), ("force_every", C.c_int32), ("device", C.c_int32),
        ("fake_fail_alloc", C.c_int32), ("max_buffer_bytes", C.c_uint64), ("arithmetic", C.c_int32),
        ("reserved1", C.c_int32),
    ]


class CellsForceSample(C.Structure):
    _fields_ = [("step", C.c_uint32), ("reserved", C.c_uint32), ("fx", C.c_double), ("fy", C.c_double),
                ("fz", C.c_double)]


class Cells3DInfo(C.Structure):
    _fields_ = [
        ("W", C.c_int32), ("H", C.c_int32), ("D", C.c_int32), ("precision", C.c_int32),
        ("N", C.c_int64), ("step", C.c_int64), ("block_x", C.c_int32), ("block_y", C.c_int32),
        ("force_every", C.c_int32), ("n_body_cells", C.c_int32),
    ]


class Cells2DConfig(C.Structure):
    _fields_ = [
        ("width", C.c_int32), ("height", C.c_int32), ("left", C.c_int32), ("right", C.c_int32),
        ("bottom", C.c_int32), ("top", C.c_int32), ("precision", C.c_int32), ("parabolic", C.c_int32),
        ("tau", C.c_double), ("lambda_", C.c_double), ("smagorinsky", C.c_double), ("u_in", C.c_double),
        ("u_lid", C.c_double), ("sponge_fraction", C.c_double), ("sponge_tau", C.c_double),
        ("body_force", C.c_double * 2), ("absorb", C.c_double), ("inlet_layer_fraction", C.c_double),
        ("workgroup_size", C.c_int32), ("force_every", C.c_int32), ("device", C.c_int32),
        ("fake_fail_alloc", C.c_int32), ("max_buffer_bytes", C.c_uint64), ("arithmetic", C.c_int32),
        ("reserved1", C.c_int32),
    ]


class Cells2DInfo(C.Structure):
    _fields_ = [
        ("W", C.c_int32), ("H", C.c_int32), ("precision", C.c_int32), ("force_every", C.c_int32),
        ("N", C.c_int64), ("step", C.c_int64), ("tile_x", C.c_int32), ("tile_y", C.c_int32),
        ("persistent", C.c_int32), ("tunnels", C.c_int32),
    ]


class Cells3DAdjointSpec(C.Structure):
    _fields_ = [("steps", C.c_int64), ("window_begin", C.c_int64), ("window_end", C.c_int64),
                ("checkpoint_every", C.c_int32), ("component", C.c_int32), ("scale", C.c_double)]


class CellsStar3D(C.Structure):
    _fields_ = [("cx", C.c_double), ("cy", C.c_double), ("cz", C.c_double), ("r0", C.c_double),
                ("coef", C.c_double * 16)]


class CellsError(RuntimeError):
    """A failed libcells call: ``status`` is the cells_status code, the message is the library's."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run __graft_entry__.build() (make -C cells_b200/csrc)")
    L = C.CDLL(LIB_PATH)
    P, I, D, I64, SZ = C.c_void_p, C.c_int, C.c_double, C.c_int64, C.c_size_t
    sig = {
        "cells3d_config_default": (None, [C.POINTER(Cells3DConfig)]),
        "cells3d_create": (I, [C.POINTER(Cells3DConfig), C.POINTER(P)]),
        "cells3d_destroy": (None, [P]),
        "cells_last_error": (C.c_char_p, [P]),
        "cells3d_set_tau": (I, [P, D]),
        "cells3d_set_smagorinsky": (I, [P, D]),
        "cells3d_set_inlet": (I, [P, D]),
        "cells3d_set_lambda": (I, [P, D]),
        "cells3d_set_inlet_ramp": (I, [P, I, D, I64, I64]),
        "cells3d_set_sdf": (I, [P, P, SZ]),
        "cells3d_init_field": (I, [P, P]),
        "cells3d_reset_forces": (I, [P]),
        "cells3d_step": (I, [P, I64]),
        "cells3d_prepare_steps": (I, [P, I64]),
        "cells3d_update_macro": (I, [P]),
        "cells3d_run": (I, [P, I64, I64]),
        "cells3d_synchronize": (I, [P]),
        "cells3d_read_macro": (I, [P, P]),
        "cells3d_read_forces": (I, [P, C.POINTER(CellsForceSample), SZ, C.POINTER(SZ)]),
        "cells3d_read_forces_begin": (I, [P]),
        "cells3d_read_forces_end": (I, [P, C.POINTER(CellsForceSample), SZ, C.POINTER(SZ)]),
        "cells3d_read_status": (I, [P, C.POINTER(C.c_uint32)]),
        "cells3d_check_diverged": (I, [P]),
        "cells3d_get_info": (I, [P, C.POINTER(Cells3DInfo)]),
        "cells3d_read_params": (I, [P, P]),
        "cells3d_mass": (I, [P, C.POINTER(D)]),
        "cells3d_read_populations": (I, [P, P, SZ]),
        "cells3d_write_populations": (I, [P, P, SZ]),
        "cells3d_read_flags": (I, [P, P, SZ]),
        "cells3d_sample_slice": (I, [P, I, D, I, D, I, I, P]),
        "cells_copy_roofline": (I, [I, I, I, I64, I, I, C.POINTER(D)]),
        "cells_host_alloc": (I, [SZ, C.POINTER(P)]),
        "cells_host_free": (None, [P]),
        "cells3d_advect_tracers": (I, [P, P, P, I, D, D]),
        "cells3d_timer_start": (I, [P]),
        "cells3d_timer_stop": (I, [P, C.POINTER(C.c_float)]),
        "cells3d_launch_count": (I, [P, C.POINTER(I64)]),
        "cells3d_fake_set_force": (I, [P, D, D, D]),
        "cells_fake_live_buffers": (I64, []),
        "cells3d_mass_noalloc": (I, [P, P, I64, C.c_int32, P, P]),
        "cells3d_adjoint_forward": (I, [P, C.POINTER(Cells3DAdjointSpec), C.POINTER(D)]),
        "cells3d_adjoint_backward": (I, [P, P, P, C.POINTER(D), P]),
        "cells3d_adjoint_release": (I, [P]),
        "cells3d_star_sdf": (I, [P, I, I, I, C.POINTER(CellsStar3D)]),
        "cells3d_star_coef_gradient": (I, [C.POINTER(CellsStar3D), I, I, I, P, P]),
        "cells3d_adjoint_backward_star": (I, [P, C.POINTER(CellsStar3D), P, C.POINTER(D)]),
        "cells3d_state_size": (I, [P, C.POINTER(SZ)]),
        "cells3d_save_state": (I, [P, P, SZ]),
        "cells3d_load_state": (I, [P, P, SZ]),
        # D2Q9 (Solver, src/solver.ts) and batches of 2D tunnels
        "cells2d_config_default": (None, [C.POINTER(Cells2DConfig)]),
        "cells2d_create": (I, [C.POINTER(Cells2DConfig), C.POINTER(P)]),
        "cells2d_destroy": (None, [P]),
        "cells2d_update": (I, [P, C.POINTER(Cells2DConfig)]),
        "cells2d_get_config": (I, [P, C.POINTER(Cells2DConfig)]),
        "cells2d_set_inlet": (I, [P, D]),
        "cells2d_set_inlet_ramp": (I, [P, I, D, I64, I64]),
        "cells2d_set_sdf": (I, [P, P, SZ]),
        "cells2d_brush": (I, [P, D, D, D, I, I]),
        "cells2d_brush_stroke": (I, [P, P, SZ, D, I]),
        "cells2d_read_sdf": (I, [P, P, SZ]),
        "cells2d_init_field": (I, [P, P]),
        "cells2d_reset_forces": (I, [P]),
        "cells2d_step": (I, [P, I64]),
        "cells2d_update_macro": (I, [P]),
        "cells2d_run": (I, [P, I64, I64]),
        "cells2d_synchronize": (I, [P]),
        "cells2d_read_macro": (I, [P, P]),
        "cells2d_read_forces": (I, [P, C.POINTER(CellsForceSample), SZ, C.POINTER(SZ)]),
        "cells2d_read_forces_begin": (I, [P]),
        "cells2d_read_forces_end": (I, [P, C.POINTER(CellsForceSample), SZ, C.POINTER(SZ)]),
        "cells2d_read_status": (I, [P, C.POINTER(C.c_uint32)]),
        "cells2d_check_diverged": (I, [P]),
        "cells2d_get_info": (I, [P, C.POINTER(Cells2DInfo)]),
        "cells2d_read_params": (I, [P, P]),
        "cells2d_mass": (I, [P, C.POINTER(D)]),
        "cells2d_read_populations": (I, [P, P, SZ]),
        "cells2d_write_populations": (I, [P, P, SZ]),
        "cells2d_read_flags": (I, [P, P, SZ]),
        "cells2d_timer_start": (I, [P]),
        "cells2d_timer_stop": (I, [P, C.POINTER(C.c_float)]),
        "cells2d_launch_count": (I, [P, C.POINTER(I64)]),
        "cells2d_fake_set_force": (I, [P, D, D]),
        "cells2d_batch_create": (I, [C.POINTER(Cells2DConfig), C.c_int32, C.POINTER(P)]),
        "cells2d_batch_destroy": (None, [P]),
        "cells2d_batch_tunnel": (I, [P, C.c_int32, C.POINTER(P)]),
        "cells2d_batch_step": (I, [P, I64]),
        "cells2d_batch_run": (I, [P, I64]),
        "cells2d_batch_synchronize": (I, [P]),
        "cells2d_batch_autotune": (I, [P, C.c_int32, C.POINTER(Cells2DInfo)]),
        "cells2d_batch_set_launch": (I, [P, C.c_int32, C.c_int32, C.c_int32]),
        "cells2d_batch_get_info": (I, [P, C.POINTER(Cells2DInfo)]),
        "cells2d_batch_set_barrier_test": (I, [P, C.c_int32]),
        "cells2d_batch_timer_start": (I, [P]),
        "cells2d_batch_timer_stop": (I, [P, C.POINTER(C.c_float)]),
        "cells2d_batch_launch_count": (I, [P, C.POINTER(I64)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status: int, handle=None) -> None:
    if status != CELLS_OK:
        msg = lib().cells_last_error(handle)
        raise CellsError(status, msg.decode() if msg else f"libcells status {status}")


def default_config3() -> Cells3DConfig:
    c = Cells3DConfig()
    lib().cells3d_config_default(C.byref(c))
    return c


def default_config2() -> Cells2DConfig:
    c = Cells2DConfig()
    lib().cells2d_config_default(C.byref(c))
    return c


def nan() -> float:
    return math.nan


def pinned_empty(n: int, dtype) -> "np.ndarray":
    """A 1-D numpy array of n elements in page-locked host memory (cells_host_alloc), freed when the
    array and every view of it are gone. Copies between it and the device take a direct DMA."""
    import weakref

    import numpy as np

    dt = np.dtype(dtype)
    nbytes = max(1, int(n) * dt.itemsize)
    ptr = C.c_void_p()
    st = lib().cells_host_alloc(nbytes, C.byref(ptr))
    if st != CELLS_OK:
        raise CellsError(st, (lib().cells_last_error(None) or b"").decode())
    buf = (C.c_byte * nbytes).from_address(ptr.value)
    weakref.finalize(buf, lib().cells_host_free, ptr.value)
    return np.frombuffer(buf, dtype=dt, count=int(n))


def star3d(center, r0: float, coef) -> CellsStar3D:
    """The CellsStar3D of a star body: centre (cx, cy, cz), base radius r0, 16 coefficients."""
    st = CellsStar3D()
    st.cx, st.cy, st.cz = (float(v) for v in center)
    st.r0 = float(r0)
    c = [float(v) for v in coef]
    if len(c) != 16:
        raise ValueError("a star body has 16 coefficients")
    for k in range(16):
        st.coef[k] = c[k]
    return st


def star_sdf(sdf, W: int, H: int, D: int, center, r0: float, coef) -> None:
    """Stamps the star body into the float32 SDF array in place (cells3d_star_sdf)."""
    import numpy as np

    if not (isinstance(sdf, np.ndarray) and sdf.dtype == np.float32 and sdf.flags.c_contiguous
            and sdf.size == W * H * D):
        raise ValueError("star_sdf needs a contiguous float32 array of W*H*D values")
    st = lib().cells3d_star_sdf(sdf.ctypes.data, W, H, D, C.byref(star3d(center, r0, coef)))
    if st != CELLS_OK:
        raise CellsError(st, (lib().cells_last_error(None) or b"").decode())


def star_coef_gradient(dsdf, W: int, H: int, D: int, center, r0: float, coef) -> "np.ndarray":
    """dJ/dcoef (16 float64) from dJ/dSDF (W*H*D float64) through cells3d_star_coef_gradient."""
    import numpy as np

    g = np.ascontiguousarray(dsdf, dtype=np.float64)
    if g.size != W * H * D:
        raise ValueError("dJ/dSDF needs W*H*D values")
    out = np.zeros(16, dtype=np.float64)
    st = lib().cells3d_star_coef_gradient(C.byref(star3d(center, r0, coef)), W, H, D, g.ctypes.data,
                                          out.ctypes.data)
    if st != CELLS_OK:
        raise CellsError(st, (lib().cells_last_error(None) or b"").decode())
    return out
