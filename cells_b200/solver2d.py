"""Solver: the reference's D2Q9 step API (src/solver.ts:50-340) over libcells.so, and Batch2D, many
independent 2D tunnels that advance in one kernel launch per step.

``Solver.create(width=..., height=..., left=..., ...)`` takes the SolverConfig keys of
src/solver.ts:15-40 (camelCase, as in the TypeScript); ``update(**partial)`` changes any of them
except the grid; ``initField(macro)`` takes (rho, ux, uy, _) per cell; ``readMacro`` returns
(rho, ux, uy, solid) per cell; ``readForces`` returns the samples since the last call as
``{step, fx, fy}``. Allocation failures raise CellsError with the message prefix
'Solver allocation failed: '.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import check, lib

HISTORY_LEN = 8192  # src/shaders/aux.ts:4

_DEFAULTS = dict(  # src/solver.ts:98-112
    left=0, right=0, bottom=0, top=0, lambda_=3 / 16, smagorinsky=0.0, uIn=0.0, parabolic=False, uLid=0.0,
    spongeFraction=0.0, spongeTau=1.0, bodyForce=(0.0, 0.0), absorb=0.0, inletLayerFraction=0.0,
    workgroupSize=0, forceEvery=1, precision="fp32", device=0, maxBufferBytes=0, fakeFailAlloc=0,
    exactArithmetic=False,
)
_PREC2 = {"fp32": _lib.FP32, "fp64": _lib.FP64}


def _to_config(cfg: dict) -> _lib.Cells2DConfig:
    c = _lib.default_config2()
    c.width, c.height = cfg["width"], cfg["height"]
    c.left, c.right, c.bottom, c.top = int(cfg["left"]), int(cfg["right"]), int(cfg["bottom"]), int(cfg["top"])
    if cfg["precision"] not in _PREC2:
        prec = _lib.PRECISIONS.get(cfg["precision"], -1)
    else:
        prec = _PREC2[cfg["precision"]]
    c.precision = prec
    c.parabolic = 1 if cfg["parabolic"] else 0
    c.tau = cfg["tau"]
    c.lambda_ = cfg["lambda_"]
    c.smagorinsky = cfg["smagorinsky"]
    c.u_in = cfg["uIn"]
    c.u_lid = cfg["uLid"]
    c.sponge_fraction = cfg["spongeFraction"]
    c.sponge_tau = cfg["spongeTau"]
    c.body_force[0], c.body_force[1] = cfg["bodyForce"]
    c.absorb = cfg["absorb"]
    c.inlet_layer_fraction = cfg["inletLayerFraction"]
    c.workgroup_size = cfg["workgroupSize"]
    c.force_every = cfg["forceEvery"]
    c.device = cfg["device"]
    c.fake_fail_alloc = cfg["fakeFailAlloc"]
    c.max_buffer_bytes = cfg["maxBufferBytes"]
    c.arithmetic = _lib.ARITH_EXACT if cfg["exactArithmetic"] else _lib.ARITH_FAST
    return c


def _full_config(kw: dict) -> dict:
    cfg = dict(_DEFAULTS)
    cfg.update(kw)
    for k in ("width", "height", "tau"):
        if k not in cfg:
            raise TypeError(f"SolverConfig needs {k}")
    cfg["bodyForce"] = tuple(cfg["bodyForce"])
    return cfg


_SAMPLE_DTYPE = np.dtype([("step", "<u4"), ("r", "<u4"), ("fx", "<f8"), ("fy", "<f8"), ("fz", "<f8")])


class Solver:
    """One D2Q9 TRT tunnel (a batch of one, or one tunnel of a Batch2D)."""

    def __init__(self, handle, cfg: dict, owner: bool = True, batch: "Optional[Batch2D]" = None):
        self._h = handle
        self._owner = owner
        self._batch = batch
        self.cfg = cfg
        self.W, self.H = cfg["width"], cfg["height"]
        self.N = self.W * self.H
        self.precision = cfg["precision"]
        self._fbuf = (_lib.CellsForceSample * HISTORY_LEN)()

    @staticmethod
    def create(**config) -> "Solver":
        cfg = _full_config(config)
        c = _to_config(cfg)
        h = C.c_void_p()
        check(lib().cells2d_create(C.byref(c), C.byref(h)), None)
        return Solver(h, cfg)

    def destroy(self) -> None:
        if self._h and self._owner:
            lib().cells2d_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    # ------------------------------------------------------------------ configuration
    def update(self, **changes) -> None:
        """update(partial), src/solver.ts:175-178."""
        cfg = dict(self.cfg)
        cfg.update(changes)
        cfg["bodyForce"] = tuple(cfg["bodyForce"])
        check(lib().cells2d_update(self._h, C.byref(_to_config(cfg))), self._h)
        self.cfg = cfg

    def setInlet(self, u: float) -> None:
        self.cfg["uIn"] = u
        check(lib().cells2d_set_inlet(self._h, u), self._h)

    def setInletRamp(self, kind: str, target: float, rampSteps: int, updateEvery: int = 1) -> None:
        """Device-side ramp (not in the reference): kind 'linear', 'smoothstep' or 'none'."""
        k = {"none": _lib.RAMP_NONE, "linear": _lib.RAMP_LINEAR, "smoothstep": _lib.RAMP_SMOOTHSTEP}[kind]
        check(lib().cells2d_set_inlet_ramp(self._h, k, target, rampSteps, updateEvery), self._h)

    # ------------------------------------------------------------------ geometry and state
    def setSdf(self, sdf: np.ndarray) -> None:
        a = np.ascontiguousarray(sdf, dtype=np.float32)
        check(lib().cells2d_set_sdf(self._h, a.ctypes.data, a.size), self._h)

    def readSdf(self) -> np.ndarray:
        out = np.empty(self.N, dtype=np.float32)
        check(lib().cells2d_read_sdf(self._h, out.ctypes.data, out.size), self._h)
        return out

    def brush(self, cx: float, cy: float, r: float, erase: bool, rebuild: bool = True) -> None:
        check(lib().cells2d_brush(self._h, cx, cy, r, 1 if erase else 0, 1 if rebuild else 0), self._h)

    def brushStroke(self, points: Sequence[Sequence[float]], r: float, erase: bool) -> None:
        a = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 2))
        check(lib().cells2d_brush_stroke(self._h, a.ctypes.data if a.size else None, a.shape[0], r,
                                         1 if erase else 0), self._h)

    def rebuildFlags(self) -> None:
        self.brushStroke([], 0.0, False)

    def initField(self, macro: Optional[np.ndarray] = None) -> None:
        """Equilibrium at the macro field (rho, ux, uy, _) per cell, or at rest."""
        if macro is None:
            check(lib().cells2d_init_field(self._h, None), self._h)
        else:
            m = np.ascontiguousarray(macro, dtype=np.float32)
            if m.size != 4 * self.N:
                raise ValueError("macro needs 4N floats")
            check(lib().cells2d_init_field(self._h, m.ctypes.data), self._h)

    def resetForces(self) -> None:
        check(lib().cells2d_reset_forces(self._h), self._h)

    # ------------------------------------------------------------------ stepping
    def encodeSteps(self, n: int) -> None:
        check(lib().cells2d_step(self._h, n), self._h)

    def encodeMacro(self) -> None:
        check(lib().cells2d_update_macro(self._h), self._h)

    def run(self, n: int, chunk: int = 500) -> None:
        check(lib().cells2d_run(self._h, n, chunk), self._h)

    def synchronize(self) -> None:
        check(lib().cells2d_synchronize(self._h), self._h)

    @property
    def step(self) -> int:
        return self.info()["step"]

    def info(self) -> dict:
        i = _lib.Cells2DInfo()
        check(lib().cells2d_get_info(self._h, C.byref(i)), self._h)
        return {k: getattr(i, k) for k, _ in i._fields_}

    # ------------------------------------------------------------------ readback
    def readMacro(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(4 * self.N, dtype=np.float32)
        check(lib().cells2d_read_macro(self._h, out.ctypes.data), self._h)
        return out

    def readForcesBegin(self) -> None:
        check(lib().cells2d_read_forces_begin(self._h), self._h)

    def readForcesEnd(self) -> list:
        n = C.c_size_t()
        check(lib().cells2d_read_forces_end(self._h, self._fbuf, HISTORY_LEN, C.byref(n)), self._h)
        b = self._fbuf
        return [{"step": b[k].step, "fx": b[k].fx, "fy": b[k].fy} for k in range(n.value)]

    def readForces(self) -> list:
        self.readForcesBegin()
        return self.readForcesEnd()

    def readForcesArray(self) -> np.ndarray:
        """readForces as an (n, 3) float64 array of (step, fx, fy)."""
        n = C.c_size_t()
        check(lib().cells2d_read_forces(self._h, self._fbuf, HISTORY_LEN, C.byref(n)), self._h)
        raw = np.frombuffer(self._fbuf, dtype=_SAMPLE_DTYPE, count=n.value)
        return np.stack([raw["step"].astype(np.float64), raw["fx"], raw["fy"]], axis=1)

    def readStatus(self) -> int:
        s = C.c_uint32()
        check(lib().cells2d_read_status(self._h, C.byref(s)), self._h)
        return s.value

    def checkDiverged(self) -> None:
        """Raises CellsError (status CELLS_E_DIVERGED) when a non-finite force sample or macro value
        was seen on the device since the last initField."""
        check(lib().cells2d_check_diverged(self._h), self._h)

    def readParams(self) -> bytes:
        buf = (C.c_uint8 * 96)()
        check(lib().cells2d_read_params(self._h, buf), self._h)
        return bytes(buf)

    def mass(self) -> float:
        v = C.c_double()
        check(lib().cells2d_mass(self._h, C.byref(v)), self._h)
        return v.value

    def _pop_dtype(self):
        return np.float64 if self.precision == "fp64" else np.float32

    def readPopulations(self) -> np.ndarray:
        out = np.empty(9 * self.N, dtype=self._pop_dtype())
        check(lib().cells2d_read_populations(self._h, out.ctypes.data, out.nbytes), self._h)
        return out

    def writePopulations(self, f: np.ndarray) -> None:
        a = np.ascontiguousarray(f, dtype=self._pop_dtype())
        check(lib().cells2d_write_populations(self._h, a.ctypes.data, a.nbytes), self._h)

    def readFlags(self) -> np.ndarray:
        out = np.empty(self.N, dtype=np.uint32)
        check(lib().cells2d_read_flags(self._h, out.ctypes.data, out.size), self._h)
        return out

    # ------------------------------------------------------------------ timing
    def timerStart(self) -> None:
        check(lib().cells2d_timer_start(self._h), self._h)

    def timerStop(self) -> float:
        ms = C.c_float()
        check(lib().cells2d_timer_stop(self._h, C.byref(ms)), self._h)
        return ms.value

    def launchCount(self) -> int:
        n = C.c_int64()
        check(lib().cells2d_launch_count(self._h, C.byref(n)), self._h)
        return n.value

    def fakeSetForce(self, fx: float, fy: float) -> None:
        check(lib().cells2d_fake_set_force(self._h, fx, fy), self._h)


class Batch2D:
    """Independent D2Q9 tunnels of different sizes stepped together: one launch per step for all
    of them (graph-replayed), or persistent launches, as the autotuner decides. ``tunnels[k]`` is
    a Solver for the per-tunnel calls; step with ``step(n)`` / ``run(n)`` on the batch."""

    def __init__(self, configs: Sequence[dict]):
        cfgs = [_full_config(c) for c in configs]
        arr = (_lib.Cells2DConfig * len(cfgs))(*[_to_config(c) for c in cfgs])
        h = C.c_void_p()
        check(lib().cells2d_batch_create(arr, len(cfgs), C.byref(h)), None)
        self._h = h
        self.tunnels = []
        for k, c in enumerate(cfgs):
            v = C.c_void_p()
            check(lib().cells2d_batch_tunnel(self._h, k, C.byref(v)), self._h)
            self.tunnels.append(Solver(v, c, owner=False, batch=self))

    def destroy(self) -> None:
        if self._h:
            for t in self.tunnels:
                t._h = None
            lib().cells2d_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def step(self, n: int) -> None:
        check(lib().cells2d_batch_step(self._h, n), self._h)

    def run(self, n: int) -> None:
        check(lib().cells2d_batch_run(self._h, n), self._h)

    def synchronize(self) -> None:
        check(lib().cells2d_batch_synchronize(self._h), self._h)

    def autotune(self, trialSteps: int = 100) -> dict:
        """Times trialSteps steps of every launch shape (9 block shapes x per-step graph replay or the
        persistent kernel) on a copy of the state, keeps the fastest and restores the state; returns
        the chosen shape (tile_x, tile_y, persistent)."""
        i = _lib.Cells2DInfo()
        check(lib().cells2d_batch_autotune(self._h, trialSteps, C.byref(i)), self._h)
        return {k: getattr(i, k) for k, _ in i._fields_}

    def setLaunch(self, tileX: int, tileY: int, persistent: bool) -> None:
        """Fixes the launch shape: tileX x tileY threads per block (64, 128 or 256); batches of 4,096
        tiles or more give each thread two cell rows."""
        check(lib().cells2d_batch_set_launch(self._h, tileX, tileY, 1 if persistent else 0), self._h)

    def info(self) -> dict:
        i = _lib.Cells2DInfo()
        check(lib().cells2d_batch_get_info(self._h, C.byref(i)), self._h)
        return {k: getattr(i, k) for k, _ in i._fields_}

    def setBarrierTest(self, extraArrivals: int) -> None:
        """Test hook of the persistent kernel's time-out path: with 1, every grid barrier of later
        persistent launches waits for an arrival that never comes, runs out after one second, and
        the call that waits for the launch raises CellsError (CELLS_E_TIMEOUT); 0 restores it."""
        check(lib().cells2d_batch_set_barrier_test(self._h, extraArrivals), self._h)

    def timerStart(self) -> None:
        check(lib().cells2d_batch_timer_start(self._h), self._h)

    def timerStop(self) -> float:
        ms = C.c_float()
        check(lib().cells2d_batch_timer_stop(self._h, C.byref(ms)), self._h)
        return ms.value

    def launchCount(self) -> int:
        n = C.c_int64()
        check(lib().cells2d_batch_launch_count(self._h, C.byref(n)), self._h)
        return n.value
