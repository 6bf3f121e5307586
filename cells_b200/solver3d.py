"""Solver3D: the reference's D3Q19 step API (src/solver3d.ts:42-320) over libcells.so.

Method names and behaviour follow the TypeScript class: ``create`` raises with the message prefix
'Solver3D allocation failed: ' when the buffers do not fit, ``setInlet`` takes an already-ramped
speed, ``run`` steps then refreshes the macro field and waits, ``readForces`` returns the samples
since the last call (dropping any the 8192-deep ring overwrote), ``readMacro`` returns (ux, uy, uz,
rho) per cell with rho = 0 in solids. Host buffers are numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, lib, star3d

HISTORY3_LEN = 8192  # src/shaders/aux3d.ts:5

_DEFAULTS = dict(  # src/solver3d.ts:110-119
    smagorinsky=0.0, uIn=0.0, spongeFraction=0.0, spongeTau=1.0, absorb=0.0, workgroupSize=0, forceEvery=1,
    lambda_=None, device=0, maxBufferBytes=0, fakeFailAlloc=0, exactArithmetic=False,
)


class Solver3D:
    """D3Q19 TRT wind tunnel on one CUDA device. Use ``Solver3D.create(**config)``."""

    def __init__(self, handle, cfg: dict):
        self._h = handle
        self.cfg = cfg
        info = _lib.Cells3DInfo()
        check(lib().cells3d_get_info(self._h, C.byref(info)), self._h)
        self.W, self.H, self.D, self.N = info.W, info.H, info.D, info.N
        self.precision = cfg["precision"]
        self._fbuf = (_lib.CellsForceSample * HISTORY3_LEN)()

    # ------------------------------------------------------------------ lifecycle
    @staticmethod
    def create(width: int, height: int, depth: int, precision: str = "fp32", tau: float = 0.6, **kw) -> "Solver3D":
        cfg = dict(_DEFAULTS)
        cfg.update(kw)
        cfg.update(width=width, height=height, depth=depth, precision=precision, tau=tau)
        c = _lib.default_config3()
        c.width, c.height, c.depth = width, height, depth
        if precision not in _lib.PRECISIONS:
            raise _lib.CellsError(_lib.CELLS_E_PRECISION_UNSUPPORTED, f"precision {precision} is not available")
        c.precision = _lib.PRECISIONS[precision]
        c.tau = tau
        c.lambda_ = math.nan if cfg["lambda_"] is None else cfg["lambda_"]
        c.smagorinsky = cfg["smagorinsky"]
        c.u_in = cfg["uIn"]
        c.sponge_fraction = cfg["spongeFraction"]
        c.sponge_tau = cfg["spongeTau"]
        c.absorb = cfg["absorb"]
        c.workgroup_size = cfg["workgroupSize"]
        c.force_every = cfg["forceEvery"]
        c.device = cfg["device"]
        c.fake_fail_alloc = cfg["fakeFailAlloc"]
        c.max_buffer_bytes = cfg["maxBufferBytes"]
        c.arithmetic = _lib.ARITH_EXACT if cfg["exactArithmetic"] else _lib.ARITH_FAST
        h = C.c_void_p()
        check(lib().cells3d_create(C.byref(c), C.byref(h)), None)
        return Solver3D(h, cfg)

    def destroy(self) -> None:
        if self._h:
            lib().cells3d_destroy(self._h)
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

    # ------------------------------------------------------------------ setters
    def setTau(self, tau: float) -> None:
        self.cfg["tau"] = tau
        check(lib().cells3d_set_tau(self._h, tau), self._h)

    def setSmagorinsky(self, cs: float) -> None:
        self.cfg["smagorinsky"] = cs
        check(lib().cells3d_set_smagorinsky(self._h, cs), self._h)

    def setInlet(self, u: float) -> None:
        self.cfg["uIn"] = u
        check(lib().cells3d_set_inlet(self._h, u), self._h)

    def setLambda(self, lam: Optional[float]) -> None:
        self.cfg["lambda_"] = lam
        check(lib().cells3d_set_lambda(self._h, math.nan if lam is None else lam), self._h)

    def setInletRamp(self, kind: str, target: float, rampSteps: int, updateEvery: int = 1) -> None:
        """Device-side ramp (not in the reference): kind 'linear', 'smoothstep' or 'none'."""
        k = {"none": _lib.RAMP_NONE, "linear": _lib.RAMP_LINEAR, "smoothstep": _lib.RAMP_SMOOTHSTEP}[kind]
        check(lib().cells3d_set_inlet_ramp(self._h, k, target, rampSteps, updateEvery), self._h)

    # ------------------------------------------------------------------ geometry and state
    def setSdf(self, sdf: np.ndarray) -> None:
        a = np.ascontiguousarray(sdf, dtype=np.float32)
        check(lib().cells3d_set_sdf(self._h, a.ctypes.data, a.size), self._h)

    def initField(self, macro: Optional[np.ndarray] = None) -> None:
        """Equilibrium at the inflow speed, or at the given (ux, uy, uz, rho) field (4N floats)."""
        if macro is None:
            check(lib().cells3d_init_field(self._h, None), self._h)
        else:
            m = np.ascontiguousarray(macro, dtype=np.float32)
            if m.size != 4 * self.N:
                raise ValueError("macro needs 4N floats")
            check(lib().cells3d_init_field(self._h, m.ctypes.data), self._h)

    def resetForces(self) -> None:
        check(lib().cells3d_reset_forces(self._h), self._h)

    # ------------------------------------------------------------------ stepping
    def encodeSteps(self, n: int) -> None:
        check(lib().cells3d_step(self._h, n), self._h)

    def prepareSteps(self, n: int) -> None:
        """Builds the CUDA graphs that encodeSteps(n) from the current step would replay, running
        nothing (no counterpart in the reference)."""
        check(lib().cells3d_prepare_steps(self._h, n), self._h)

    def encodeMacro(self) -> None:
        check(lib().cells3d_update_macro(self._h), self._h)

    def run(self, n: int, chunk: int = 500) -> None:
        check(lib().cells3d_run(self._h, n, chunk), self._h)

    def synchronize(self) -> None:
        check(lib().cells3d_synchronize(self._h), self._h)

    @property
    def step(self) -> int:
        info = _lib.Cells3DInfo()
        check(lib().cells3d_get_info(self._h, C.byref(info)), self._h)
        return info.step

    def info(self) -> dict:
        i = _lib.Cells3DInfo()
        check(lib().cells3d_get_info(self._h, C.byref(i)), self._h)
        return {k: getattr(i, k) for k, _ in i._fields_}

    # ------------------------------------------------------------------ readback
    def readMacro(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(4 * self.N, dtype=np.float32)
        check(lib().cells3d_read_macro(self._h, out.ctypes.data), self._h)
        return out

    def readForcesBegin(self) -> None:
        check(lib().cells3d_read_forces_begin(self._h), self._h)

    def readForcesEnd(self) -> list:
        n = C.c_size_t()
        check(lib().cells3d_read_forces_end(self._h, self._fbuf, HISTORY3_LEN, C.byref(n)), self._h)
        b = self._fbuf
        return [{"step": b[k].step, "fx": b[k].fx, "fy": b[k].fy, "fz": b[k].fz} for k in range(n.value)]

    def readForces(self) -> list:
        self.readForcesBegin()
        return self.readForcesEnd()

    def readForcesArray(self) -> np.ndarray:
        """readForces as an (n, 4) float64 array of (step, fx, fy, fz)."""
        n = C.c_size_t()
        check(lib().cells3d_read_forces(self._h, self._fbuf, HISTORY3_LEN, C.byref(n)), self._h)
        raw = np.frombuffer(self._fbuf, dtype=np.dtype([("step", "<u4"), ("r", "<u4"), ("fx", "<f8"), ("fy", "<f8"),
                                                         ("fz", "<f8")]), count=n.value)
        return np.stack([raw["step"].astype(np.float64), raw["fx"], raw["fy"], raw["fz"]], axis=1)

    def readStatus(self) -> int:
        s = C.c_uint32()
        check(lib().cells3d_read_status(self._h, C.byref(s)), self._h)
        return s.value

    def checkDiverged(self) -> None:
        """Raises CellsError (status CELLS_E_DIVERGED) when a non-finite force sample or macro value
        was seen on the device since the last initField (src/tunnel3d.ts:97-105)."""
        check(lib().cells3d_check_diverged(self._h), self._h)

    def readParams(self) -> bytes:
        buf = (C.c_uint8 * 64)()
        check(lib().cells3d_read_params(self._h, buf), self._h)
        return bytes(buf)

    def mass(self) -> float:
        v = C.c_double()
        check(lib().cells3d_mass(self._h, C.byref(v)), self._h)
        return v.value

    def _pop_dtype(self):
        return {"fp32": np.float32, "fp16": np.float16, "bf16": np.uint16, "fp64": np.float64}[self.precision]

    def readPopulations(self) -> np.ndarray:
        """The latest populations as stored (19 x N of the storage type; bf16 as raw uint16)."""
        out = np.empty(19 * self.N, dtype=self._pop_dtype())
        check(lib().cells3d_read_populations(self._h, out.ctypes.data, out.nbytes), self._h)
        return out

    def writePopulations(self, f: np.ndarray) -> None:
        a = np.ascontiguousarray(f, dtype=self._pop_dtype())
        check(lib().cells3d_write_populations(self._h, a.ctypes.data, a.nbytes), self._h)

    def readFlags(self) -> np.ndarray:
        out = np.empty(self.N, dtype=np.uint32)
        check(lib().cells3d_read_flags(self._h, out.ctypes.data, out.size), self._h)
        return out

    # ------------------------------------------------------------------ macro-field products
    FIELD_MODES = {"speed": 0, "vorticity": 1}
    _IN_PLANE = {0: (1, 2), 1: (0, 2), 2: (0, 1)}

    def sampleSlice(self, axis: int, pos: float, mode: str = "speed", uRef: float = 0.1,
                    size: Optional[tuple] = None) -> np.ndarray:
        """The slice view of src/shaders/render3d.ts:159-177 without a graphics pipeline: the field
        (speed / (1.6 uRef) or |curl u| / (0.3 uRef)) at the pixel centres of an (nv, nu) grid over
        the axis-aligned quad at pos * (dim - 1) on `axis`; NaN on solid nodes. The default size is
        the in-plane grid, one pixel per cell centre. Reads the macro field of the last run or
        updateMacro."""
        dims = (self.W, self.H, self.D)
        a, b = self._IN_PLANE[axis] if axis in self._IN_PLANE else (0, 0)
        nu, nv = size if size is not None else (dims[a], dims[b])
        out = np.empty((nv, nu), dtype=np.float32)
        check(lib().cells3d_sample_slice(self._h, axis, float(pos), self.FIELD_MODES.get(mode, -1), float(uRef),
                                         nu, nv, out.ctypes.data), self._h)
        return out

    def advectTracers(self, seeds: np.ndarray, particles: np.ndarray, steps: float, uRef: float = 0.1) -> None:
        """One frame of tracer advection (src/shaders/render3d.ts:196-230) over `steps` lattice steps:
        particles (count, 8) float32 = (x, y, z, 0, ux, uy, uz, 0), updated in place; seeds
        (count, 4) float32, where a tracer restarts when it leaves the box or enters a solid."""
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        if particles.dtype != np.float32 or not particles.flags.c_contiguous:
            raise ValueError("particles must be a C-contiguous float32 array")
        count = particles.size // 8
        if particles.size != 8 * count or seeds.size != 4 * count:
            raise ValueError("particles must hold 8 and seeds 4 floats per tracer")
        check(lib().cells3d_advect_tracers(self._h, seeds.ctypes.data, particles.ctypes.data, count, float(steps),
                                           float(uRef)), self._h)

    # ------------------------------------------------------------------ state save / restore
    def saveState(self) -> bytes:
        """Snapshot of the populations, step, parity, inlet speed and ramp (not the SDF or parameters)."""
        n = C.c_size_t()
        check(lib().cells3d_state_size(self._h, C.byref(n)), self._h)
        buf = (C.c_uint8 * n.value)()
        check(lib().cells3d_save_state(self._h, buf, n.value), self._h)
        return bytes(buf)

    def loadState(self, state: bytes) -> None:
        """Restores a saveState snapshot into a solver with the same grid, precision, config and SDF."""
        b = (C.c_uint8 * len(state)).from_buffer_copy(state)
        check(lib().cells3d_load_state(self._h, b, len(state)), self._h)

    # ------------------------------------------------------------------ discrete adjoint
    def adjointForward(self, steps: int, windowBegin: int, windowEnd: int, checkpointEvery: int = 100,
                       component: int = 0, scale: float = 1.0) -> float:
        """Steps `steps` steps with checkpoints and returns J = scale * mean force component over
        the window of step labels [windowBegin, windowEnd] (absolute step counts)."""
        spec = _lib.Cells3DAdjointSpec(steps, windowBegin, windowEnd, checkpointEvery, component, scale)
        j = C.c_double()
        check(lib().cells3d_adjoint_forward(self._h, C.byref(spec), C.byref(j)), self._h)
        return j.value

    def adjointBackward(self, terminal: Optional[np.ndarray] = None, wantAdjoint: bool = False) -> dict:
        """The backward sweep of the recorded run: dJ/dsdf (N float64), dJ/du_in, and optionally
        the adjoint of the initial populations (seeded with `terminal` at the final state)."""
        dsdf = np.zeros(self.N, dtype=np.float64)
        du = C.c_double()
        t = None
        if terminal is not None:
            t = np.ascontiguousarray(terminal, dtype=self._pop_dtype())
        out = np.empty(19 * self.N, dtype=self._pop_dtype()) if wantAdjoint else None
        check(lib().cells3d_adjoint_backward(self._h, None if t is None else t.ctypes.data, dsdf.ctypes.data,
                                             C.byref(du), None if out is None else out.ctypes.data), self._h)
        return {"dsdf": dsdf, "du": du.value, "adjoint": out}

    def adjointBackwardStar(self, center, r0: float, coef):
        """The backward sweep projected onto a star body's 16 coefficients
        (cells3d_adjoint_backward_star): (dJ/dcoef (16 float64), dJ/du_in)."""
        out = np.zeros(16, dtype=np.float64)
        du = C.c_double()
        check(lib().cells3d_adjoint_backward_star(self._h, C.byref(star3d(center, r0, coef)), out.ctypes.data,
                                                  C.byref(du)), self._h)
        return out, du.value

    def adjointRelease(self) -> None:
        check(lib().cells3d_adjoint_release(self._h), self._h)

    # ------------------------------------------------------------------ timing
    def timerStart(self) -> None:
        check(lib().cells3d_timer_start(self._h), self._h)

    def timerStop(self) -> float:
        ms = C.c_float()
        check(lib().cells3d_timer_stop(self._h, C.byref(ms)), self._h)
        return ms.value

    def launchCount(self) -> int:
        n = C.c_int64()
        check(lib().cells3d_launch_count(self._h, C.byref(n)), self._h)
        return n.value

    def fakeSetForce(self, fx: float, fy: float, fz: float) -> None:
        check(lib().cells3d_fake_set_force(self._h, fx, fy, fz), self._h)
