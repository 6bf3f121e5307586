"""The reference's 2D validation suite (src/cases.ts:61-427) on the CUDA solver, with its published
reference ranges and acceptance ranges unchanged, plus the 400x100 cylinder tunnel workload.

Each case returns ``{"name", "metrics": [{"name", "value", "ref", "accept", "pass"}], "pass",
"steps", "cells"}``. Cases drive the solver only through the public Solver API (create, setSdf,
initField, update, run, readForces, readMacro), as the reference's cases do.
"""
from __future__ import annotations

import math
import time
from typing import Callable, Optional

import numpy as np

from . import analysis, geometry as g
from .lattice3d import XMode, YMode
from .rng import perturbed_rest2
from .solver2d import Solver


def metric(name, value, ref, accept):
    return {"name": name, "value": float(value), "ref": list(ref), "accept": list(accept),
            "pass": bool(accept[0] <= value <= accept[1])}


def around(center, rel):
    return (center * (1 - rel), center * (1 + rel))


def result(name, metrics, steps, cells, **extra):
    r = {"name": name, "metrics": metrics, "pass": all(m["pass"] for m in metrics), "steps": steps, "cells": cells}
    r.update(extra)
    return r


def run_ramped(s: Solver, steps: int, u_target: float, ramp_steps: int, forces: list, chunk: int = 400):
    """The reference's runRamped (src/cases.ts:41-59): per chunk of 400 steps the inlet is set to
    the smoothstep ramp of the step count, then the forces are collected."""
    end = s.step + steps
    while s.step < end:
        r = min(1.0, s.step / ramp_steps)
        u = u_target * r * r * (3 - 2 * r)
        if u != s.cfg["uIn"]:
            s.update(uIn=u)
        s.run(min(chunk, end - s.step), chunk)
        forces.extend(s.readForces())
    return forces


def poiseuille(**kw):
    """Plane Poiseuille flow driven by a body force between no-slip walls (src/cases.ts:61-91)."""
    H, u_max = 32, 0.05
    metrics, steps = [], 0
    for tau in (0.6, 1.0, 1.5):
        nu = (tau - 0.5) / 3
        fx = 8 * nu * u_max / (H * H)
        s = Solver.create(width=4, height=H, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip,
                          top=YMode.NoSlip, tau=tau, bodyForce=(fx, 0.0), forceEvery=0, **kw)
        s.initField()
        n = math.ceil(10 * H * H / nu)
        s.run(n, 2000)
        steps += n
        m = s.readMacro()
        y = np.arange(H)
        e = fx / (2 * nu) * (y + 0.5) * (H - y - 0.5)
        got = m.reshape(H, 4, 4)[:, 1, 1].astype(np.float64)
        err = math.sqrt(float(np.sum((got - e) ** 2) / np.sum(e * e)))
        metrics.append(metric(f"L2 error, tau={tau}", err, (0, 0), (0, 2e-4)))
        s.destroy()
    return result("Plane Poiseuille", metrics, steps, 4 * H)


def taylor_green(**kw):
    """Decaying Taylor-Green vortex on periodic grids 32, 64, 128 (src/cases.ts:131-190)."""
    tau = 0.8
    nu = (tau - 0.5) / 3
    errors, ratios, steps = [], [], 0
    for n in (32, 64, 128):
        u0 = 0.04 * 32 / n
        k = 2 * math.pi / n
        s = Solver.create(width=n, height=n, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.Periodic,
                          top=YMode.Periodic, tau=tau, forceEvery=0, **kw)
        yy, xx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")

        def field(t):
            a = u0 * math.exp(-2 * nu * k * k * t)
            m = np.zeros((n, n, 4), dtype=np.float32)
            m[..., 0] = 1 - 0.75 * a * a * (np.cos(2 * k * xx) + np.cos(2 * k * yy))
            m[..., 1] = -a * np.cos(k * xx) * np.sin(k * yy)
            m[..., 2] = a * np.sin(k * xx) * np.cos(k * yy)
            return m.reshape(-1)

        s.initField(field(0))
        t = round(math.log(2) / (2 * nu * k * k))
        half = round(t / 2)
        s.run(half, 1000)
        mid = s.readMacro().astype(np.float64)
        s.run(t - half, 1000)
        end = s.readMacro().astype(np.float64)
        steps += t
        exact = field(t).astype(np.float64)
        sel = np.zeros(4, dtype=bool)
        sel[1:3] = True
        mask = np.tile(sel, n * n)
        errors.append(math.sqrt(float(np.sum((end[mask] - exact[mask]) ** 2) / np.sum(exact[mask] ** 2))))
        energy = lambda m: float(np.sum(m[1::4] ** 2 + m[2::4] ** 2))
        ratios.append(math.log(energy(mid) / energy(end)) / (4 * k * k * (t - half)) / nu)
        s.destroy()
    order = math.log2(errors[0] / errors[2]) / 2
    return result("Taylor-Green vortex", [
        metric("nu measured / nu (N=128)", ratios[2], (1, 1), (0.99, 1.01)),
        metric("velocity L2 error (N=128)", errors[2], (0, 0), (0, 0.01)),
        metric("convergence order 32 to 128", order, (2, 2), (1.8, math.inf)),
    ], steps, 128 * 128, errors=errors)


def periodic_seam(**kw):
    """A body cut by the periodic seam feels the same drag as in mid-domain (src/cases.ts:93-129)."""
    W, H, D, tau = 128, 64, 16, 0.8
    drag, steps = [], 0
    for cx in (W / 2 + D / 2 - 0.5, D / 2 - 0.5):
        s = Solver.create(width=W, height=H, left=XMode.Periodic, right=XMode.Periodic, bottom=YMode.NoSlip,
                          top=YMode.NoSlip, tau=tau, bodyForce=(2e-6, 0.0), forceEvery=100, **kw)
        sdf = g.empty_sdf(W, H)
        g.add_circle(sdf, W, H, cx, H / 2 - 0.5, D / 2)
        g.add_circle(sdf, W, H, cx + W, H / 2 - 0.5, D / 2)
        s.setSdf(sdf)
        s.initField()
        forces = []
        for _ in range(20):
            s.run(1000, 1000)
            forces.extend(s.readForces())
        steps += s.step
        drag.append(analysis.mean(f["fx"] for f in forces[-5:]))
        s.destroy()
    return result("Periodic seam invariance",
                  [metric("drag at seam / drag in middle", drag[1] / drag[0], (1, 1), (0.999, 1.001))], steps, W * H)


def _schafer_turek(D, re, force_every, u_max, **kw):
    W, H = 22 * D, round(4.1 * D)
    u_mean = 2 / 3 * u_max
    nu = u_mean * D / re
    cx, cy = 2 * D, 2 * D - 0.5
    s = Solver.create(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.NoSlip, top=YMode.NoSlip,
                      tau=3 * nu + 0.5, parabolic=True, uIn=0.0, forceEvery=force_every, spongeFraction=0.1,
                      spongeTau=1.0, absorb=0.1, **kw)
    sdf = g.empty_sdf(W, H)
    g.add_circle(sdf, W, H, cx, cy, D / 2)
    s.setSdf(sdf)
    s.initField()
    coef = lambda f: 2 * f / (u_mean * u_mean * D)
    return s, W, H, cx, cy, u_mean, coef


def schafer_turek_1(**kw):
    """Schafer-Turek 2D-1, steady flow at Re 20 (src/cases.ts:216-273)."""
    D, u_max = 40, 0.05
    s, W, H, cx, cy, u_mean, coef = _schafer_turek(D, 20, 50, u_max, **kw)
    forces, prev = [], math.inf
    for k in range(20):
        run_ramped(s, 10000, u_max, 5000, forces)
        cd = coef(analysis.mean(f["fx"] for f in forces[-20:]))
        if k >= 4 and abs(cd - prev) < 1e-4:
            break
        prev = cd
    last = forces[-20:]
    cd = coef(analysis.mean(f["fx"] for f in last))
    cl = coef(analysis.mean(f["fy"] for f in last))
    m = s.readMacro().reshape(H, W, 4).astype(np.float64)
    y0 = math.floor(cy)
    w = cy - y0
    rho_at = lambda x: (1 - w) * m[y0, x, 0] + w * m[y0 + 1, x, 0]
    ux_at = lambda x: (1 - w) * m[y0, x, 1] + w * m[y0 + 1, x, 1]
    xf, xb = cx - D / 2, cx + D / 2
    a, b = math.floor(xf), math.ceil(xb)
    p_front = rho_at(a) + (rho_at(a) - rho_at(a - 1)) * (xf - a)
    p_back = rho_at(b) + (rho_at(b) - rho_at(b + 1)) * (b - xb)
    dp = (p_front - p_back) / 3 / (u_mean * u_mean)
    la = math.nan
    for x in range(b, W - 1):
        u0, u1 = ux_at(x), ux_at(x + 1)
        if u0 < 0 <= u1:
            la = (x - u0 / (u1 - u0) - xb) / D
            break
    steps = s.step
    s.destroy()
    return result("Schafer-Turek 2D-1 (Re 20)", [
        metric("c_D", cd, (5.57, 5.59), around(5.58, 0.02)),
        metric("c_L", cl, (0.0104, 0.011), around(0.0107, 0.1)),
        metric("L_a / D", la, (0.842, 0.852), around(0.847, 0.03)),
        metric("dP / (rho U_mean^2)", dp, (0.1172 / 0.04, 0.1176 / 0.04), around(0.1174 / 0.04, 0.02)),
    ], steps, W * H)


def _periodic_window(s, forces, period, u, coef, min_amp, tol, checks):
    window, prev_amp = [], 0.0
    for k in range(checks):
        run_ramped(s, round(5 * period), u, 5000, forces)
        window = [f for f in forces if f["step"] > s.step - 5 * period]
        cls = [coef(f["fy"]) for f in window]
        amp = max(cls) - min(cls)
        if k >= 6 and amp > min_amp and abs(amp - prev_amp) < tol * amp:
            break
        prev_amp = amp
        del forces[:max(0, len(forces) - 20000)]
    return window


def schafer_turek_2(**kw):
    """Schafer-Turek 2D-2, periodic shedding at Re 100 (src/cases.ts:275-307)."""
    D, u_max = 40, 0.05
    s, W, H, cx, cy, u_mean, coef = _schafer_turek(D, 100, 5, u_max, **kw)
    period = D / (0.3 * u_mean)
    window = _periodic_window(s, [], period, u_max, coef, 0.5, 1e-3, 40)
    t = [f["step"] for f in window]
    cl = [coef(f["fy"]) for f in window]
    cd = [coef(f["fx"]) for f in window]
    p = analysis.period_from_crossings(t, cl)
    st = D / (p[0] * u_mean) if p else math.nan
    steps = s.step
    s.destroy()
    return result("Schafer-Turek 2D-2 (Re 100)", [
        metric("c_D,max", max(cd), (3.22, 3.24), around(3.23, 0.02)),
        metric("c_L,max", max(cl), (0.99, 1.01), around(1.0, 0.05)),
        metric("St", st, (0.295, 0.305), around(0.3, 0.02)),
    ], steps, W * H)


def unconfined_cylinder(**kw):
    """Cylinder at Re 100 in a 40D x 48D slip-walled tunnel (src/cases.ts:309-364): St 0.165 +- 4%,
    mean C_D 1.345 +- 5% over whole shedding periods."""
    D, lx, ly, xc, u = 32, 40, 48, 16, 0.05
    W, H = lx * D, ly * D
    nu = u * D / 100
    s = Solver.create(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                      tau=3 * nu + 0.5, forceEvery=5, spongeFraction=0.15, spongeTau=1.0, absorb=0.02, **kw)
    sdf = g.empty_sdf(W, H)
    g.add_circle(sdf, W, H, xc * D, H / 2 + 0.3, D / 2)
    s.setSdf(sdf)
    s.initField()
    coef = lambda f: 2 * f / (u * u * D)
    period = D / (0.165 * u)
    window = _periodic_window(s, [], period, u, coef, 0.3, 2e-3, 60)
    t = [f["step"] for f in window]
    p = analysis.period_from_crossings(t, [f["fy"] for f in window])
    st = D / (p[0] * u) if p else math.nan
    n = math.floor((t[-1] - t[0]) / p[0]) if p else 0
    span = [f for f in window if f["step"] > t[-1] - n * (p[0] if p else 0)]
    cd = coef(analysis.mean(f["fx"] for f in span))
    steps = s.step
    s.destroy()
    return result("Unconfined cylinder (Re 100)", [
        metric("St", st, (0.1643, 0.1670), around(0.165, 0.04)),
        metric("mean C_D", cd, (1.33, 1.36), around(1.345, 0.05)),
    ], steps, W * H)


def cavity(**kw):
    """Lid-driven cavity at Re 1000, primary vortex centre against Ghia (src/cases.ts:366-395)."""
    N, u = 128, 0.1
    nu = u * N / 1000
    s = Solver.create(width=N, height=N, left=XMode.Wall, right=XMode.Wall, bottom=YMode.NoSlip,
                      top=YMode.MovingWall, tau=3 * nu + 0.5, uLid=u, forceEvery=0, **kw)
    s.initField()
    v, prev = (0.0, 0.0, 0.0), (-1.0, -1.0)
    for k in range(40):
        s.run(20000, 2000)
        m = s.readMacro()
        v = analysis.primary_vortex(analysis.stream_function(m[1::4], m[2::4], N, N), N, N)
        if math.hypot(v[0] - prev[0], v[1] - prev[1]) < 0.01 and k >= 5:
            break
        prev = (v[0], v[1])
    steps = s.step
    s.destroy()
    return result("Ghia lid-driven cavity (Re 1000)", [
        metric("vortex x / L", (v[0] + 0.5) / N, (0.5313, 0.5313), (0.5213, 0.5413)),
        metric("vortex y / L", (v[1] + 0.5) / N, (0.5625, 0.5625), (0.5525, 0.5725)),
    ], steps, N * N)


def naca(**kw):
    """NACA0012 at Re 500, alpha 0 (src/cases.ts:397-427)."""
    c, u = 100, 0.1
    W, H = 16 * c, 8 * c
    nu = u * c / 500
    s = Solver.create(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                      tau=3 * nu + 0.5, forceEvery=50, spongeFraction=0.15, spongeTau=1.0, absorb=0.1,
                      inletLayerFraction=0.08, **kw)
    sdf = g.empty_sdf(W, H)
    g.add_polygon(sdf, W, H, g.naca_polygon(4 * c, H / 2 - 0.5, c, 0.12, 0.0))
    s.setSdf(sdf)
    s.initField()
    coef = lambda f: 2 * f / (u * u * c)
    forces, prev, cd = [], math.inf, math.nan
    for k in range(30):
        run_ramped(s, 10000, u, 5000, forces)
        cd = coef(analysis.mean(f["fx"] for f in forces[-20:]))
        if k >= 5 and abs(cd - prev) < 2e-4:
            break
        prev = cd
    steps = s.step
    s.destroy()
    return result("NACA0012 (Re 500, alpha 0)", [metric("C_D", cd, (0.1762, 0.178), around(0.1762, 0.05))],
                  steps, W * H)


CASES: dict[str, Callable] = {
    "poiseuille": poiseuille,
    "periodicSeam": periodic_seam,
    "taylorGreen": taylor_green,
    "schaferTurek1": schafer_turek_1,
    "schaferTurek2": schafer_turek_2,
    "unconfinedCylinder": unconfined_cylinder,
    "cavity": cavity,
    "naca": naca,
}


def run_case(key: str, **kw) -> dict:
    t0 = time.perf_counter()
    r = CASES[key](**kw)
    r["seconds"] = time.perf_counter() - t0
    return r


# ---------------------------------------------------------------- 64 batched NACA tunnels


def batched_naca_tunnels(count: int = 64, seed: Optional[int] = None):
    """Independent NACA0012 tunnels drawn from the seed: width log-uniform in [256, 1024], height
    width / 4, chord height / 5, angle of attack uniform in [-8, 12] degrees, Re uniform in
    [50, 400] (tau = 3 u chord / Re + 1/2, at least 0.51), Smagorinsky C_s = 0.1, inflow 0.1, the
    page's open tunnel (Zou-He inlet and outlet, slip walls, 15% sponge, absorb 0.02) with the
    section's leading edge at W/4 - chord/3 (src/app.ts:118-125). Returns [(config, sdf)]."""
    from .rng import SEED, uniform

    seed = SEED if seed is None else seed
    lw = uniform(seed, 11, count, math.log(256), math.log(1024))
    alpha = uniform(seed, 12, count, -8.0, 12.0)
    re = uniform(seed, 13, count, 50.0, 400.0)
    out = []
    for k in range(count):
        W = int(round(math.exp(float(lw[k]))))
        H = int(round(W / 4))
        chord = H / 5
        tau = max(3 * 0.1 * chord / float(re[k]) + 0.5, 0.51)
        cfg = dict(width=W, height=H, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                   tau=tau, smagorinsky=0.1, uIn=0.1, spongeFraction=0.15, spongeTau=1.0, absorb=0.02,
                   forceEvery=0)
        sdf = g.empty_sdf(W, H)
        g.add_polygon(sdf, W, H, g.naca_polygon(W / 4 - chord / 3, H / 2, chord, 0.12, math.radians(float(alpha[k]))))
        out.append((cfg, sdf))
    return out


def batched_naca_throughput(steps: int = 10000, device: int = 0, autotune: bool = True, warmup: int = 200,
                            count: int = 64) -> dict:
    """MLUPS of the batched tunnels stepped together (one Batch2D, CUDA-graph or persistent
    launches as the autotuner picks) and of the same tunnels stepped one at a time (one Solver
    each, graph-replayed), both timed with CUDA events on the solvers' streams; the final
    populations of each tunnel, batched and alone, are compared (how many are bit for bit equal,
    and the largest difference)."""
    from .solver2d import Batch2D

    tunnels = batched_naca_tunnels(count)
    cells = sum(c["width"] * c["height"] for c, _ in tunnels)
    b = Batch2D([dict(c, device=device) for c, _ in tunnels])
    for t, (c, sdf) in zip(b.tunnels, tunnels):
        t.setSdf(sdf)
        t.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
    launch = b.autotune(100) if autotune else b.info()
    b.step(warmup)
    b.synchronize()
    b.timerStart()
    b.step(steps)
    ms_batch = b.timerStop()
    batched = [t.readPopulations() for t in b.tunnels]
    b.destroy()
    ms_seq = 0.0
    identical, max_diff = 0, 0.0
    for (c, sdf), fb in zip(tunnels, batched):
        s = Solver.create(device=device, **c)
        s.setSdf(sdf)
        s.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
        s.encodeSteps(warmup)
        s.synchronize()
        s.timerStart()
        s.encodeSteps(steps)
        ms_seq += s.timerStop()
        fs = s.readPopulations()
        s.destroy()
        # the same tunnel after the same steps, batched and alone
        identical += int(np.array_equal(fb.view(np.uint32), fs.view(np.uint32)))
        max_diff = max(max_diff, float(np.max(np.abs(fb.astype(np.float64) - fs.astype(np.float64)))))
    return {"tunnels": count, "cells": cells, "steps": steps, "batched_mlups": cells * steps / (ms_batch * 1e3),
            "sequential_mlups": cells * steps / (ms_seq * 1e3), "speedup": ms_seq / ms_batch,
            "batched_ms": ms_batch, "sequential_ms": ms_seq,
            "bitwise_identical_tunnels": identical, "max_population_diff": max_diff,
            "finite": bool(all(np.all(np.isfinite(f)) for f in batched)),
            "launch": {"tile": [launch["tile_x"], launch["tile_y"]], "persistent": bool(launch["persistent"])}}


# ---------------------------------------------------------------- the 400 x 100 cylinder tunnel


CYLINDER_TUNNEL = dict(width=400, height=100, left=XMode.Open, right=XMode.Open, bottom=YMode.Slip, top=YMode.Slip,
                       tau=0.56, lambda_=3 / 16, smagorinsky=0.0, spongeFraction=0.15, spongeTau=1.0, absorb=0.02,
                       forceEvery=1)


def cylinder_tunnel_inputs():
    """D2Q9 400x100, cylinder of diameter 20 at (80, 50.5), Re 100 (tau 0.56), Zou-He inlet ramped
    linearly to 0.1 over 3000 steps, Zou-He outlet, slip walls, 15% outlet sponge; from rest with a
    seeded transverse perturbation of amplitude 1e-4. Returns (config, sdf, macro)."""
    W, H = 400, 100
    sdf = g.empty_sdf(W, H)
    g.add_circle(sdf, W, H, 80, 50.5, 10)
    return dict(CYLINDER_TUNNEL), sdf, perturbed_rest2(W, H, 1e-4)


def cylinder_ramp(step: int) -> float:
    return 0.1 * min(1.0, step / 3000)


def cylinder_coefficients(forces, u=0.1, D=20, skip=10000):
    """C_D averaged over whole C_L periods after `skip` steps, C_L amplitude, St = D / (period u)."""
    fs = [f for f in forces if f["step"] > skip]
    t = [f["step"] for f in fs]
    cl = [2 * f["fy"] / (u * u * D) for f in fs]
    cd = [2 * f["fx"] / (u * u * D) for f in fs]
    p = analysis.period_from_crossings(t, cl)
    if not p:
        return {"C_D": analysis.mean(cd), "C_L_amp": 0.5 * (max(cl) - min(cl)), "St": math.nan}
    n = math.floor((t[-1] - t[0]) / p[0])
    sel = [k for k in range(len(t)) if t[k] > t[-1] - n * p[0]]
    return {"C_D": analysis.mean(cd[k] for k in sel), "C_L_amp": 0.5 * (max(cl) - min(cl)),
            "C_L_rms": math.sqrt(analysis.mean(c * c for c in cl)), "St": D / (p[0] * u)}


def cylinder_tunnel(steps: int = 20000, device: int = 0, exact: bool = False,
                    on_chunk: Optional[Callable] = None) -> dict:
    """Runs the 400x100 cylinder tunnel with the device-side linear ramp and returns the force
    traces, C_D / C_L / St, the final macro field and the throughput."""
    cfg, sdf, macro = cylinder_tunnel_inputs()
    s = Solver.create(device=device, exactArithmetic=exact, **cfg)
    s.setSdf(sdf)
    s.initField(macro)
    s.setInletRamp("linear", 0.1, 3000, 1)
    s.synchronize()
    t0 = time.perf_counter()
    forces = []
    done = 0
    while done < steps:
        k = min(2000, steps - done)
        s.encodeSteps(k)
        forces.extend(s.readForces())
        done += k
        if on_chunk:
            on_chunk(s)
    s.run(0)
    dt = time.perf_counter() - t0
    m = s.readMacro()
    s.destroy()
    out = cylinder_coefficients(forces)
    out.update(forces=forces, macro=m, seconds=dt, mlups=400 * 100 * steps / dt / 1e6)
    return out
