"""3D validation and precision workloads on the CUDA solver.

* ``sphere_fp16``: the reference's sphereFp16 case (src/cases3d.ts:11-81): a sphere of diameter 16 at
  Re 100 on 192x96x96, FP32 and FP16 storage each run in blocks of 2000 steps (smoothstep inlet ramp
  over 3000 steps set per chunk of 400, forces every 4 steps) until C_D changes by less than 1e-4
  between blocks; gate: C_D of FP16 within 1% of FP32. BF16 and FP64 are added beside them.
* ``sphere_wake``: the 3D page's sphere (size fraction 0.2 of the height, 19.2 cells, at (W/4, H/2,
  D/2) of 192x96x96; u = 0.1 smoothstep-ramped over 3000 steps; sponge 0.15, absorb 0.02; forces
  every 4 steps; from rest, src/app3d.ts:18-20,182,314-315, src/tunnel3d.ts:38-72) at a given Re,
  for the wake regimes the reference reports (README.md:73): at Re 250 a steady wake that leans to
  one side (C_L 0.063), at Re 300 shedding with St 0.135.
* ``precision_sweep``: four obstacles (sphere D=20, cube edge 18, spanwise cylinder D=16, NACA0012
  wing chord 40 over the full span at 6 degrees) at Re 200 on 256x128x128, stored as FP32, FP16
  and BF16 with FP32 arithmetic, 4000 steps; time-averaged C_D and C_L over steps 2000..4000 and the
  relative velocity L2 over fluid cells at step 4000, each against an FP64 run of the same kernel on
  the same grid and on the 128x64x64 grid with lengths halved (same Re and u).
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import analysis, geometry as g
from .rng import perturbed_rest3
from .solver3d import Solver3D
from .units import derive_tau


def smoothstep(t):
    return t * t * (3 - 2 * t)


def sphere_fp16(precisions=("fp32", "fp16", "bf16", "fp64"), device=0, grid=(192, 96, 96), max_blocks=15):
    W, H, D = grid
    d, u = 16, 0.1
    tau = derive_tau(100, u, d).tau
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, W / 4, H / 2, D / 2, d / 2)
    scale = 2 / (u * u * g.reference_area("sphere", d, D))
    cd, steps = {}, {}
    for prec in precisions:
        s = Solver3D.create(W, H, D, precision=prec, tau=tau, spongeFraction=0.15, spongeTau=1.0, absorb=0.02,
                            forceEvery=4, device=device)
        s.setSdf(sdf)
        s.initField()
        prev = math.nan
        for k in range(1, max_blocks + 1):
            block = []
            end = k * 2000
            while s.step < end:
                s.setInlet(u * smoothstep(min(1.0, s.step / 3000)))
                s.run(min(400, end - s.step), 400)
                block.extend(f["fx"] for f in s.readForces())
            c = analysis.mean(block) * scale
            cd[prec] = c
            if k >= 5 and abs(c - prev) / abs(prev) < 1e-4:
                break
            prev = c
        steps[prec] = s.step
        s.destroy()
    ref = cd["fp32"]
    return {"name": "Sphere C_D, FP16 vs FP32 (Re 100)", "C_D": cd, "steps": steps,
            "rel_vs_fp32": {p: abs(v - ref) / abs(ref) for p, v in cd.items()},
            "pass": abs(cd["fp16"] - ref) / abs(ref) <= 0.01 if "fp16" in cd else None}


OBSTACLES = (("sphere", 20, 0.0), ("cube", 18, 0.0), ("cylinder", 16, 0.0), ("wing", 40, 6.0))


def _body(kind, size, angle_deg, W, H, D):
    cx, cy, cz = W / 4, H / 2, D / 2
    sdf = g.empty_sdf3(W, H, D)
    a = math.radians(angle_deg)
    if kind == "sphere":
        g.add_sphere(sdf, W, H, D, cx, cy, cz, size / 2)
        area = g.reference_area("sphere", size, D)
    elif kind == "cube":
        g.add_box3(sdf, W, H, D, cx, cy, cz, size / 2, size / 2, size / 2, 0.0)
        area = g.reference_area("cube", size, D)
    elif kind == "cylinder":
        g.add_cylinder_z(sdf, W, H, D, cx, cy, size / 2)
        area = g.reference_area("cylinder", size, D)
    else:
        g.add_wing(sdf, W, H, D, cx, cy, cz, size, D, a)
        area = g.reference_area("wing", size, D, span=D)
    return sdf, area


def _run(kind, size, angle, grid, precision, steps, device, u=0.1, re=200.0):
    W, H, D = grid
    sdf, area = _body(kind, size, angle, W, H, D)
    tau = max(derive_tau(re, u, size).tau, 0.51)
    s = Solver3D.create(W, H, D, precision=precision, tau=tau, uIn=0.0, spongeFraction=0.15, spongeTau=1.0,
                        absorb=0.02, forceEvery=1, device=device)
    s.setSdf(sdf)
    s.initField(perturbed_rest3(W, H, D, 1e-4))
    s.setInletRamp("linear", u, 3000 * steps // 4000, 1)
    s.encodeSteps(steps)
    f = s.readForcesArray()
    s.run(0)
    m = s.readMacro().reshape(-1, 4)
    s.destroy()
    scale = 2 / (u * u * area)
    sel = f[:, 0] > steps // 2
    return {"C_D": scale * float(np.mean(f[sel, 1])), "C_L": scale * float(np.mean(f[sel, 2])), "macro": m,
            "tau": tau}


def _vel_l2(a, b):
    fluid = (b[:, 3] != 0) & (a[:, 3] != 0)
    du = a[fluid, :3].astype(np.float64) - b[fluid, :3].astype(np.float64)
    return math.sqrt(float(np.sum(du * du)) / float(np.sum(b[fluid, :3].astype(np.float64) ** 2)))


def precision_sweep(device=0, grid=(256, 128, 128), steps=4000, obstacles=OBSTACLES,
                    precisions=("fp32", "fp16", "bf16")):
    W, H, D = grid
    half = (W // 2, H // 2, D // 2)
    out = []
    for kind, size, angle in obstacles:
        t0 = time.perf_counter()
        ref = _run(kind, size, angle, grid, "fp64", steps, device)
        ref_half = _run(kind, size / 2, angle, half, "fp64", steps // 2, device)
        row = {"obstacle": kind, "size": size, "tau": ref["tau"], "fp64": {"C_D": ref["C_D"], "C_L": ref["C_L"]},
               "fp64_half_grid": {"C_D": ref_half["C_D"], "C_L": ref_half["C_L"]}}
        for prec in precisions:
            r = _run(kind, size, angle, grid, prec, steps, device)
            row[prec] = {"C_D": r["C_D"], "C_L": r["C_L"],
                         "C_D_err_vs_fp64": abs(r["C_D"] - ref["C_D"]) / abs(ref["C_D"]),
                         "C_L_abs_err_vs_fp64": abs(r["C_L"] - ref["C_L"]),
                         "C_D_err_vs_fp64_half_grid": abs(r["C_D"] - ref_half["C_D"]) / abs(ref_half["C_D"]),
                         "vel_L2_vs_fp64": _vel_l2(r["macro"], ref["macro"])}
        row["seconds"] = time.perf_counter() - t0
        out.append(row)
    return out


def sweep_table(rows) -> str:
    """The precision sweep as a markdown table: per obstacle and storage, C_D and C_L (mean over the
    second half of the run), the relative C_D error and absolute C_L error against the FP64 run on
    the same grid, the relative C_D difference to the FP64 run on the half grid, and the relative
    velocity L2 difference at the last step."""
    out = ["| obstacle | storage | C_D | C_L | C_D err vs FP64 | C_L abs err vs FP64 | C_D vs FP64 half grid "
           "| velocity L2 vs FP64 |", "|---|---|---|---|---|---|---|---|"]
    for r in rows:
        out.append(f"| {r['obstacle']} ({r['size']:g}) | FP64 | {r['fp64']['C_D']:.5f} | {r['fp64']['C_L']:.5f} "
                   f"| — | — | {abs(r['fp64']['C_D'] - r['fp64_half_grid']['C_D']) / abs(r['fp64_half_grid']['C_D']):.2e} "
                   f"| — |")
        for prec in ("fp32", "fp16", "bf16"):
            if prec not in r:
                continue
            e = r[prec]
            out.append(f"| | {prec.upper()} | {e['C_D']:.5f} | {e['C_L']:.5f} | {e['C_D_err_vs_fp64']:.2e} "
                       f"| {e['C_L_abs_err_vs_fp64']:.2e} | {e['C_D_err_vs_fp64_half_grid']:.2e} "
                       f"| {e['vel_L2_vs_fp64']:.2e} |")
    return "\n".join(out)


def sphere_wake(re: float, steps: int = 40000, precision: str = "fp32", device: int = 0, grid=(192, 96, 96)) -> dict:
    """The 3D page's sphere at Reynolds number re (module docstring). Returns the side-force
    coefficients C_y and C_z averaged over the second half of the run (the page's C_L readout is
    C_y over the second half of its force history), their magnitude, C_D over the same half, and the
    Strouhal number of the side force with the larger oscillation over the last 15,000 steps."""
    W, H, D = grid
    body = analysis.build_body("sphere", 0.2, 0.0, W, H, D)
    L, u = body["lRef"], 0.1
    tau = derive_tau(re, u, L).tau
    s = Solver3D.create(W, H, D, precision=precision, tau=tau, uIn=0.0, spongeFraction=0.15, spongeTau=1.0,
                        absorb=0.02, forceEvery=4, device=device)
    s.setSdf(body["sdf"])
    s.initField()
    s.setInletRamp("smoothstep", u, 3000, 1)
    chunks = []
    done = 0
    while done < steps:
        k = min(20000, steps - done)  # the ring holds 8192 samples, 32,768 steps at every 4th
        s.encodeSteps(k)
        done += k
        chunks.append(s.readForcesArray())
    s.destroy()
    f = np.concatenate(chunks)
    scale = 2 / (u * u * body["area"])
    half = f[f[:, 0] > steps / 2]
    cy, cz = scale * float(np.mean(half[:, 2])), scale * float(np.mean(half[:, 3]))
    tail = f[f[:, 0] > steps - 15000]
    comp = 2 if np.ptp(tail[:, 2]) >= np.ptp(tail[:, 3]) else 3
    p = analysis.period_from_crossings(list(tail[:, 0]), list(tail[:, comp]))
    st = L / (p[0] * u) if p else math.nan
    return {"re": re, "tau": tau, "steps": steps, "precision": precision, "L": L,
            "C_D": scale * float(np.mean(half[:, 1])), "C_y": cy, "C_z": cz, "C_side": math.hypot(cy, cz),
            "side_amplitude": [scale * float(np.ptp(tail[:, 2])) / 2, scale * float(np.ptp(tail[:, 3])) / 2],
            "St": st, "St_component": "y" if comp == 2 else "z"}
