"""Python driver of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE ONLY.

Only tests, the smoke check and bench.py's CPU-baseline leg use this module; the product package
(cells_b200) never imports it. ``OracleSolver3D`` replays the host logic of the reference's
Solver3D (src/solver3d.ts:197-315: writeParams, setSdf/rebuildFlags, initField, encodeSteps, the
force ring) around the C restatement of the WGSL kernels in oracle/lbm3d.cpp, so a test can drive
the oracle and the CUDA solver through the same sequence of calls and compare the results.
Force samples are summed in f64 in cell order (the reference sums f32 slots in atomic order).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle.so")

PREC = {"fp32": 0, "fp16": 1, "bf16": 2, "fp64": 3}
DTYPE = {"fp32": np.float32, "fp16": np.float16, "bf16": np.uint16, "fp64": np.float64}
FLAG_SOLID = 1 << 19


class HostParams3(C.Structure):
    _fields_ = [("W", C.c_int32), ("H", C.c_int32), ("D", C.c_int32), ("pad", C.c_int32),
                ("tau", C.c_double), ("lambda_", C.c_double), ("smagC2", C.c_double), ("uIn", C.c_double),
                ("spongeStart", C.c_double), ("tauSponge", C.c_double), ("absorb", C.c_double)]


class HostParams2(C.Structure):
    _fields_ = [("W", C.c_int32), ("H", C.c_int32), ("left", C.c_int32), ("right", C.c_int32),
                ("bottom", C.c_int32), ("top", C.c_int32), ("parabolic", C.c_int32), ("forcing", C.c_int32),
                ("tau", C.c_double), ("lambda_", C.c_double), ("smagC2", C.c_double), ("uIn", C.c_double),
                ("spongeStart", C.c_double), ("tauSponge", C.c_double), ("uLid", C.c_double), ("fx", C.c_double),
                ("fy", C.c_double), ("absorb", C.c_double), ("inletLayer", C.c_double)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        HP = C.POINTER(HostParams3)
        L.oracle3d_step.argtypes = [C.c_int, HP, P, P, P, P, P]
        L.oracle3d_flags.argtypes = [C.c_int, HP, P, P, P, P, P, P]
        L.oracle3d_init.argtypes = [C.c_int, HP, P, P, P, P]
        L.oracle3d_macro.argtypes = [C.c_int, HP, P, P, P]
        L.oracle3d_mass.argtypes = [C.c_int, HP, P, P, C.POINTER(C.c_double)]
        L.oracle_trt_lambda3.argtypes = [C.c_double]
        L.oracle_trt_lambda3.restype = C.c_double
        L.oracle_codec_roundtrip.argtypes = [C.c_int, C.c_float]
        L.oracle_codec_roundtrip.restype = C.c_float
        L.oracle_num_threads.restype = C.c_int
        for fn in ("oracle3d_step", "oracle3d_flags", "oracle3d_init", "oracle3d_macro", "oracle3d_mass"):
            getattr(L, fn).restype = C.c_int
        I = C.c_int
        F = C.c_float
        L.oracle3d_sample_slice.argtypes = [P, I, I, I, I, F, I, F, I, I, P]
        L.oracle3d_sample_slice.restype = I
        L.oracle3d_advect.argtypes = [P, I, I, I, P, P, I, F, F]
        L.oracle3d_advect.restype = I
        HP2 = C.POINTER(HostParams2)
        L.oracle2d_step.argtypes = [C.c_int, HP2, P, P, P, P, P]
        L.oracle2d_run.argtypes = [C.c_int, HP2, P, P, C.c_int, C.c_longlong, P, P]
        L.oracle2d_flags.argtypes = [C.c_int, HP2, P, P, P, P, P]
        L.oracle2d_init.argtypes = [C.c_int, HP2, P, P, P]
        L.oracle2d_macro.argtypes = [C.c_int, HP2, P, P, P]
        L.oracle2d_mass.argtypes = [C.c_int, HP2, P, P, C.POINTER(C.c_double)]
        L.oracle2d_brush.argtypes = [C.c_int, C.c_int, P, C.c_double, C.c_double, C.c_double, C.c_int]
        for fn in ("oracle2d_step", "oracle2d_run", "oracle2d_flags", "oracle2d_init", "oracle2d_macro",
                   "oracle2d_mass", "oracle2d_brush"):
            getattr(L, fn).restype = C.c_int
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class OracleSolver3D:
    """The reference Solver3D's host logic over the CPU restatement of its kernels."""

    HISTORY_LEN = 8192

    def __init__(self, width, height, depth, precision="fp32", tau=0.6, lambda_=None, smagorinsky=0.0, uIn=0.0,
                 spongeFraction=0.0, spongeTau=1.0, absorb=0.0, forceEvery=1):
        self.W, self.H, self.D = width, height, depth
        self.N = width * height * depth
        self.precision = precision
        self.prec = PREC[precision]
        self.cfg = dict(tau=tau, lambda_=lambda_, smagorinsky=smagorinsky, uIn=uIn, spongeFraction=spongeFraction,
                        spongeTau=spongeTau, absorb=absorb, forceEvery=forceEvery)
        dt = DTYPE[precision]
        self.f = [np.zeros(19 * self.N, dtype=dt), np.zeros(19 * self.N, dtype=dt)]
        self.flags = np.zeros(self.N, dtype=np.uint32)
        self.touches = np.zeros(self.N, dtype=np.uint8)
        self.sdf = np.full(self.N, 1e6, dtype=np.float32)
        self.macro = np.zeros(4 * self.N, dtype=np.float32)
        self.cell_force = np.zeros(3 * self.N, dtype=np.float64)
        self.step = 0
        self.parity = 0
        self.samples = []  # (step, fx, fy, fz) produced since the last readForces
        self._rebuild_flags()

    # params exactly as writeParams derives them (src/solver3d.ts:197-208)
    def params(self) -> HostParams3:
        c = self.cfg
        p = HostParams3()
        p.W, p.H, p.D = self.W, self.H, self.D
        p.tau = c["tau"]
        p.lambda_ = c["lambda_"] if c["lambda_"] is not None else min(3 / 16, 50 * (c["tau"] - 0.5) ** 2)
        p.smagC2 = c["smagorinsky"] * c["smagorinsky"]
        p.uIn = c["uIn"]
        p.spongeStart = (self.W - 1) * (1 - c["spongeFraction"]) if c["spongeFraction"] > 0 else 1e9
        p.tauSponge = max(c["spongeTau"], c["tau"])
        p.absorb = c["absorb"]
        return p

    def setTau(self, tau):
        self.cfg["tau"] = tau

    def setSmagorinsky(self, cs):
        self.cfg["smagorinsky"] = cs

    def setInlet(self, u):
        self.cfg["uIn"] = u

    def _macro(self):
        p = self.params()
        lib().oracle3d_macro(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.flags), _ptr(self.macro))

    def _rebuild_flags(self):
        self._macro()
        p = self.params()
        lib().oracle3d_flags(self.prec, C.byref(p), _ptr(self.sdf), _ptr(self.flags), _ptr(self.touches),
                             _ptr(self.f[0]), _ptr(self.f[1]), _ptr(self.macro))

    def setSdf(self, sdf):
        self.sdf = np.ascontiguousarray(sdf, dtype=np.float32).copy()
        self._rebuild_flags()

    def initField(self, macro=None):
        p = self.params()
        m = None if macro is None else np.ascontiguousarray(macro, dtype=np.float32)
        lib().oracle3d_init(self.prec, C.byref(p), _ptr(self.f[0]), _ptr(self.f[1]), _ptr(self.flags), _ptr(m))
        self.step = 0
        self.parity = 0
        self.samples = []

    def encodeSteps(self, n):
        every = self.cfg["forceEvery"]
        for _ in range(n):
            p = self.params()
            sample = every > 0 and (self.step + 1) % every == 0
            self.cell_force[:] = 0
            lib().oracle3d_step(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.f[self.parity ^ 1]),
                                _ptr(self.flags), _ptr(self.sdf), _ptr(self.cell_force) if sample else None)
            self.parity ^= 1
            self.step += 1
            if sample:
                fsum = self.cell_force.reshape(-1, 3).sum(axis=0)
                self.samples.append((self.step, float(fsum[0]), float(fsum[1]), float(fsum[2])))

    def run(self, n, chunk=500):
        self.encodeSteps(n)
        self._macro()

    def readMacro(self):
        return self.macro.copy()

    def readForces(self):
        out = self.samples[-self.HISTORY_LEN:]
        self.samples = []
        return [{"step": s, "fx": a, "fy": b, "fz": c} for s, a, b, c in out]

    def populations(self):
        return self.f[self.parity]

    def mass(self):
        p = self.params()
        v = C.c_double()
        lib().oracle3d_mass(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.flags), C.byref(v))
        return v.value


class OracleSolver2D:
    """The reference Solver's host logic (src/solver.ts:50-340) over the CPU restatement of its
    kernels (oracle/lbm2d.cpp). Config keys follow SolverConfig (src/solver.ts:15-40)."""

    HISTORY_LEN = 8192
    DEFAULTS = dict(lambda_=3 / 16, smagorinsky=0.0, uIn=0.0, parabolic=False, uLid=0.0, spongeFraction=0.0,
                    spongeTau=1.0, bodyForce=(0.0, 0.0), absorb=0.0, inletLayerFraction=0.0, forceEvery=1)

    def __init__(self, width, height, left=0, right=0, bottom=0, top=0, tau=0.6, precision="fp32", **cfg):
        self.W, self.H = width, height
        self.N = width * height
        self.precision = precision
        self.prec = PREC[precision]
        if self.prec not in (0, 3):
            raise ValueError("the 2D oracle stores fp32 or fp64")
        self.cfg = dict(self.DEFAULTS)
        self.cfg.update(left=left, right=right, bottom=bottom, top=top, tau=tau)
        self.cfg.update(cfg)
        dt = DTYPE[precision]
        self.f = [np.zeros(9 * self.N, dtype=dt), np.zeros(9 * self.N, dtype=dt)]
        self.flags = np.zeros(self.N, dtype=np.uint32)
        self.sdf = np.full(self.N, 1e6, dtype=np.float32)
        self.macro = np.zeros(4 * self.N, dtype=np.float32)
        self.cell_force = np.zeros(2 * self.N, dtype=np.float64)
        self.step = 0
        self.parity = 0
        self.samples = []
        self._rebuild_flags()

    # writeParams, src/solver.ts:180-197
    def params(self) -> HostParams2:
        c = self.cfg
        p = HostParams2()
        p.W, p.H = self.W, self.H
        p.left, p.right, p.bottom, p.top = c["left"], c["right"], c["bottom"], c["top"]
        p.tau = c["tau"]
        p.lambda_ = c["lambda_"]
        p.smagC2 = c["smagorinsky"] * c["smagorinsky"]
        p.uIn = c["uIn"]
        p.parabolic = 1 if c["parabolic"] else 0
        p.spongeStart = (self.W - 1) * (1 - c["spongeFraction"]) if c["spongeFraction"] > 0 else 1e9
        p.tauSponge = max(c["spongeTau"], c["tau"])
        p.uLid = c["uLid"]
        p.fx, p.fy = c["bodyForce"]
        p.forcing = 1 if (c["bodyForce"][0] != 0 or c["bodyForce"][1] != 0) else 0
        p.absorb = c["absorb"]
        p.inletLayer = c["inletLayerFraction"] * (self.W - 1)
        return p

    def update(self, **changes):
        self.cfg.update(changes)

    def _macro(self):
        p = self.params()
        lib().oracle2d_macro(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.flags), _ptr(self.macro))

    def _rebuild_flags(self):
        self._macro()
        p = self.params()
        lib().oracle2d_flags(self.prec, C.byref(p), _ptr(self.sdf), _ptr(self.flags), _ptr(self.f[0]),
                             _ptr(self.f[1]), _ptr(self.macro))

    def setSdf(self, sdf):
        self.sdf = np.ascontiguousarray(sdf, dtype=np.float32).copy()
        self._rebuild_flags()

    def brush(self, cx, cy, r, erase, rebuild=True):
        lib().oracle2d_brush(self.W, self.H, _ptr(self.sdf), cx, cy, r, 1 if erase else 0)
        if rebuild:
            self._rebuild_flags()

    def initField(self, macro=None):
        if macro is None:
            macro = np.zeros(4 * self.N, dtype=np.float32)
            macro[0::4] = 1.0
        m = np.ascontiguousarray(macro, dtype=np.float32)
        self.macro = m.copy()
        p = self.params()
        lib().oracle2d_init(self.prec, C.byref(p), _ptr(m), _ptr(self.f[0]), _ptr(self.f[1]))
        self.step = 0
        self.parity = 0
        self.samples = []

    def encodeSteps(self, n):
        every = self.cfg["forceEvery"]
        if every <= 0:
            p = self.params()
            self.parity = lib().oracle2d_run(self.prec, C.byref(p), _ptr(self.f[0]), _ptr(self.f[1]), self.parity, n,
                                             _ptr(self.flags), _ptr(self.sdf))
            self.step += n
            return
        for _ in range(n):
            p = self.params()
            sample = (self.step + 1) % every == 0
            lib().oracle2d_step(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.f[self.parity ^ 1]),
                                _ptr(self.flags), _ptr(self.sdf), _ptr(self.cell_force) if sample else None)
            self.parity ^= 1
            self.step += 1
            if sample:
                fsum = self.cell_force.reshape(-1, 2).sum(axis=0)
                self.samples.append((self.step, float(fsum[0]), float(fsum[1])))

    def run(self, n, chunk=500):
        self.encodeSteps(n)
        self._macro()

    def readMacro(self):
        return self.macro.copy()

    def readForces(self):
        out = self.samples[-self.HISTORY_LEN:]
        self.samples = []
        return [{"step": s, "fx": a, "fy": b} for s, a, b in out]

    def populations(self):
        return self.f[self.parity]

    def mass(self):
        p = self.params()
        v = C.c_double()
        lib().oracle2d_mass(self.prec, C.byref(p), _ptr(self.f[self.parity]), _ptr(self.flags), C.byref(v))
        return v.value


def sample_slice(mac, W, H, D, axis, pos, mode, uRef, nu, nv):
    """The oracle's slice of a macro field (4N float32): (nv, nu) float32, NaN on solid nodes."""
    mac = np.ascontiguousarray(mac, dtype=np.float32)
    out = np.empty((nv, nu), dtype=np.float32)
    rc = lib().oracle3d_sample_slice(mac.ctypes.data, W, H, D, axis, pos, mode, uRef, nu, nv, out.ctypes.data)
    if rc != 0:
        raise ValueError("bad slice arguments")
    return out


def advect(mac, W, H, D, seeds, particles, steps, uRef):
    """The oracle's tracer frame: returns the advected copy of particles (count, 8) float32."""
    mac = np.ascontiguousarray(mac, dtype=np.float32)
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    out = np.array(particles, dtype=np.float32, copy=True, order="C")
    lib().oracle3d_advect(mac.ctypes.data, W, H, D, seeds.ctypes.data, out.ctypes.data, out.size // 8, steps, uRef)
    return out


def decode(f, precision):
    """Stored populations to float64 values (the codec's load)."""
    if precision == "fp16":
        return f.astype(np.float64) / 32768.0
    if precision == "bf16":
        return (f.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    return f.astype(np.float64)
