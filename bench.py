#!/usr/bin/env python
"""D3Q19 wind-tunnel step throughput on B200 (MLUPS and fraction of the HBM roofline).

Workload (default): the D3Q19 TRT tunnel at 192x96x96 with FP32 storage, a sphere of diameter 16
at (48, 48, 48) as an SDF with Bouzidi walls, equilibrium inlet ramped linearly to u = 0.1 over
3000 steps (device-side ramp), copy-and-relax outlet, slip side faces, outlet sponge over the last
15% with absorb 0.02, Re 200 (tau = 0.524, Lambda = 50 (tau - 1/2)^2), start from rest with a seeded
1e-4 velocity perturbation, forces sampled every step. Inputs are synthetic (seed 20261203).

One step = one fused step kernel over the whole grid. The two distribution buffers (2 x 134 MB)
exceed the 126 MB L2, so every timed step streams from HBM without an explicit flush.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
  python bench.py --precision-sweep    (sphere, cube, spanwise cylinder, NACA wing x FP32/FP16/BF16)

With --gpus N under torchrun every rank runs an independent replica on its own GPU (the path does
not shard: replicas only); value is the whole-job MLUPS from the max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "D3Q19 MLUPS + % HBM peak, FP16 vs FP32 store at C_D err≤1%; adjoint cost/fwd"
BYTES_PER_CELL = {"fp32": 152, "fp16": 76, "bf16": 76, "fp64": 304}
FALLBACK_HBM_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(workload: str):
    """dram bytes per launch of the step kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(workload)
    except Exception:
        return None


class ClockSampler:
    """SM clocks and throttle reasons read through NVML (read-only queries) while the timed region
    runs: one sample as it starts, one every 2 ms from a thread, one as it ends, so even a
    millisecond-long region has samples taken during it."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.nv = None
        self.handle = None
        self.thread = None
        self.stop = None

    def _sample(self):
        nv, h = self.nv, self.handle
        try:
            sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
            self.samples.append((sm, smax, bits))
        except Exception:
            pass

    def _loop(self):
        while not self.stop.wait(0.002):
            self._sample()

    def __enter__(self):
        import threading

        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.handle = nv.nvmlDeviceGetHandleByIndex(self.gpu)
            self._sample()
            self.stop = threading.Event()
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
        except Exception:
            self.nv = None
        return self

    def __exit__(self, *exc):
        if self.nv is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            self._sample()
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        reasons = set()
        for _, _, bits in self.samples:
            for name, attr in self.REASONS:
                if bits & getattr(self.nv, attr, 0):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(x[0] for x in self.samples),
                "sm_max_mhz": max(x[1] for x in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": "NVML, 2 ms period plus the start and end of the region"}


def physical_gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# ---------------------------------------------------------------- workload


def tunnel_setup(W, H, D, precision, device, tau=None, exact=False):
    from cells_b200 import Solver3D, geometry as g
    from cells_b200.rng import perturbed_rest3
    from cells_b200.units import derive_tau

    d = 16 * H / 96  # sphere diameter 16 on the 96-high grid; scaled with the grid
    tau = derive_tau(200, 0.1, d).tau if tau is None else tau
    s = Solver3D.create(W, H, D, precision=precision, tau=tau, uIn=0.0, spongeFraction=0.15, spongeTau=1.0,
                        absorb=0.02, forceEvery=1, device=device, exactArithmetic=exact)
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, W / 4, H / 2, D / 2, d / 2)
    macro = perturbed_rest3(W, H, D, 1e-4)
    return s, sdf, macro, tau


def copy_roofline(device: int, precision: str, n: int, launches: int = 300, flags: bool = False) -> dict:
    """The reference's copy roofline (src/bench.ts:61-95) at this size: the 19 population arrays
    copied between two buffers with no arithmetic, timed with CUDA events; GB/s counts the
    population bytes (19 loads and 19 stores per cell), as the step's roofline does."""
    import ctypes as C

    from cells_b200 import _lib

    ms = C.c_double()
    _lib.check(_lib.lib().cells_copy_roofline(device, _lib.PRECISIONS[precision], 19, n, launches, int(flags),
                                              C.byref(ms)))
    gbps = 2 * 19 * _lib.BYTES_PER_POPULATION[_lib.PRECISIONS[precision]] * n / (ms.value * 1e-3) / 1e9
    return {"ms_per_launch": round(ms.value, 5), "gbps": round(gbps, 1)}


def time_steps(s, warmup: int, steps: int):
    s.encodeSteps(warmup)
    s.prepareSteps(steps)  # the step graphs the timed run replays, captured outside the timed region
    s.synchronize()
    s.readForces()
    l0 = s.launchCount()
    s.timerStart()
    s.encodeSteps(steps)
    ms = s.timerStop()
    launches = s.launchCount() - l0
    s.readForces()
    return ms, launches


def run_e2e(s, sdf, macro, steps: int, chunk: int = 100):
    """The reference's caller pattern (src/cases.ts:41-59) through the public API with host buffers:
    setSdf and initField from host arrays, then per chunk setInlet (host-ramped), run(chunk) and
    readForces, and readMacro at the end. Wall clock, synchronised on the device. The SDF, the
    initial macro field and the macro readback live in pinned host memory (cells_host_alloc),
    allocated and filled before the timed region."""
    import numpy as np

    from cells_b200._lib import pinned_empty

    sdf_h = pinned_empty(sdf.size, np.float32)
    sdf_h[:] = sdf
    macro_h = pinned_empty(macro.size, np.float32)
    macro_h[:] = macro
    out_h = pinned_empty(macro.size, np.float32)
    sdf, macro = sdf_h, macro_h
    s.synchronize()
    h2d = d2h = 0
    t0 = time.perf_counter()
    s.setSdf(sdf)
    h2d += sdf.nbytes
    s.initField(macro)
    h2d += macro.nbytes
    forces = 0
    done = 0
    while done < steps:
        k = min(chunk, steps - done)
        t = min(1.0, done / 3000)
        s.setInlet(0.1 * t)
        h2d += 8
        s.run(k, k)
        f = s.readForcesArray()
        forces += len(f)
        d2h += 32 * len(f)
        done += k
    m = s.readMacro(out_h)
    d2h += m.nbytes
    dt = time.perf_counter() - t0
    assert np.all(np.isfinite(m))
    return dt, h2d, d2h


def precision_cd(device, steps=5000, grid=(192, 96, 96)):
    """C_D of the sphere tunnel (mean over the last 1000 of `steps` steps) per storage precision,
    and its relative error against the FP64 run of the same kernel and grid."""
    import numpy as np

    W, H, D = grid
    d = 16 * H / 96
    scale = 2 / (0.1 * 0.1 * np.pi * d * d / 4)
    out = {}
    for prec in ("fp64", "fp32", "fp16", "bf16"):
        s, sdf, macro, _ = tunnel_setup(W, H, D, prec, device=device)
        s.setSdf(sdf)
        s.initField(macro)
        s.setInletRamp("linear", 0.1, 3000, 1)
        s.encodeSteps(steps)
        f = s.readForcesArray()
        s.destroy()
        out[prec] = scale * float(np.mean(f[f[:, 0] > steps - 1000, 1]))
    ref = out["fp64"]
    return {"workload": f"D3Q19 {W}x{H}x{D} sphere d={d:g} Re200, {steps} steps, C_D over the last 1000",
            "C_D": {k: round(v, 6) for k, v in out.items()},
            "rel_err_vs_fp64": {k: abs(v - ref) / abs(ref) for k, v in out.items() if k != "fp64"}}


def adjoint_cost(device):
    """Wall times of the shape gradient on the 128x64x64 star-body drag problem (FP32, 6000 steps,
    checkpoints every 100): the recording forward run (StarDrag.forward: the body's SDF on the host,
    setSdf, initField, adjoint_forward), the backward sweep (recompute from checkpoints + adjoint
    steps) and the host chain rule to the 16 coefficients, for a handle's first gradient and for a
    second one with other coefficients (the handle keeps its checkpoint block); against one plain
    forward run of the 6000 steps and against a forward evaluation of J that includes building and
    setting the body. cost_ratio is the sweep alone over the plain run."""
    from cells_b200.adjoint import StarDrag
    from cells_b200.rng import SEED, normal

    p = StarDrag(precision="fp32", device=device)
    s = p.solver
    times = []
    for k, coef in enumerate((0.02 * normal(SEED, 17, 16), 0.02 * normal(SEED, 18, 16))):
        s.synchronize()
        t0 = time.perf_counter()
        J = p.forward(coef)
        s.synchronize()
        t_rec = time.perf_counter() - t0
        t0 = time.perf_counter()
        r = s.adjointBackward()
        t_bwd = time.perf_counter() - t0
        t0 = time.perf_counter()
        dcoef, du = p.coefficient_gradient(r)
        t_chain = time.perf_counter() - t0
        times.append((J, t_rec, t_bwd, t_chain, du))
    # one plain forward run of the same steps, and a forward evaluation that builds the body too
    s.initField(p.macro)
    s.setInletRamp("linear", 0.1, p.ramp_steps, 1)
    s.synchronize()
    t0 = time.perf_counter()
    s.encodeSteps(p.steps)
    s.synchronize()
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    s.setSdf(p.sdf(0.02 * normal(SEED, 18, 16)))
    s.initField(p.macro)
    s.setInletRamp("linear", 0.1, p.ramp_steps, 1)
    s.encodeSteps(p.steps)
    s.readForces()
    s.synchronize()
    t_eval = time.perf_counter() - t0
    p.destroy()
    (J, r1, b1, c1, du), (_, r2, b2, c2, _) = times
    return {"workload": "star body r0=12 at 128x64x64, Re150, 6000 steps, K=100, FP32", "J": J,
            "forward_s": t_fwd, "forward_evaluation_s": t_eval,
            "first": {"recording_forward_s": r1, "backward_s": b1, "chain_rule_s": c1},
            "second": {"recording_forward_s": r2, "backward_s": b2, "chain_rule_s": c2},
            "cost_ratio": b1 / t_fwd,
            "total_gradient_ratio": (r1 + b1 + c1) / t_fwd,
            "total_gradient_ratio_second": (r2 + b2 + c2) / t_fwd,
            "gradient_over_forward_evaluation": (r2 + b2 + c2) / t_eval, "dJ_du": du}


def cpu_baseline(W, H, D, precision="fp32", budget_s=12.0, max_steps=400):
    """The oracle (C++ restatement of the reference's kernels) on the host cores, OpenMP."""
    from cells_b200 import geometry as g
    from cells_b200.rng import perturbed_rest3
    from cells_b200.units import derive_tau
    from oracle.oracle import OracleSolver3D, lib as olib

    d = 16 * H / 96
    tau = derive_tau(200, 0.1, d).tau
    o = OracleSolver3D(W, H, D, precision, tau=tau, uIn=0.0, spongeFraction=0.15, absorb=0.02, forceEvery=1)
    sdf = g.empty_sdf3(W, H, D)
    g.add_sphere(sdf, W, H, D, W / 4, H / 2, D / 2, d / 2)
    o.setSdf(sdf)
    o.initField(perturbed_rest3(W, H, D, 1e-4))
    o.setInlet(0.1)
    t0 = time.perf_counter()
    o.encodeSteps(1)
    one = time.perf_counter() - t0
    k = max(1, min(max_steps, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.encodeSteps(k)
    dt = time.perf_counter() - t0
    N = W * H * D
    return {"value": N * k / dt / 1e6, "unit": "MLUPS", "cores": int(olib().oracle_num_threads()), "kind": "port",
            "sample": f"{k} full D3Q19 steps of the {W}x{H}x{D} {precision} sphere tunnel on the CPU oracle "
                      f"(OpenMP), {dt:.1f} s"}


# ---------------------------------------------------------------- main


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32")
    ap.add_argument("--grid", default="192x96x96")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, variants and the CPU baseline")
    ap.add_argument("--profile", action="store_true", help="short run for ncu: warmup + steps only, no extras")
    ap.add_argument("--profile-adjoint", action="store_true",
                    help="short run for ncu of the discrete adjoint: the 128x64x64 star body over --steps steps "
                         "(checkpoints every 100), forward then backward sweep")
    ap.add_argument("--profile2d", action="store_true",
                    help="short run for ncu of the 2D step kernel: the 64 batched NACA tunnels, one launch per "
                         "step (tile 32 x 2), warmup + steps")
    ap.add_argument("--precision-sweep", action="store_true",
                    help="the four-obstacle precision sweep at 256x128x128 (FP32, FP16, BF16 against FP64 on the same "
                         "grid and on 128x64x64); prints one JSON line and a markdown table")
    args = ap.parse_args()
    if args.precision_sweep:
        from cells_b200 import cases3d

        rows = cases3d.precision_sweep()
        print(json.dumps({"precision_sweep": rows}), flush=True)
        print(cases3d.sweep_table(rows), flush=True)
        return
    if args.profile_adjoint:
        from cells_b200.adjoint import StarDrag
        from cells_b200.rng import SEED, normal

        n = max(200, (args.steps // 100) * 100)
        p = StarDrag(precision="fp32", device=0, steps=n, ramp_steps=n // 2, window=(n // 2, n))
        J = p.forward(0.02 * normal(SEED, 17, 16))
        p.backward()
        p.solver.synchronize()
        p.destroy()
        print(json.dumps({"profile_adjoint": "done", "steps": n, "J": J}))
        return
    if args.profile2d:
        from cells_b200 import cases2d
        from cells_b200.rng import perturbed_rest2
        from cells_b200.solver2d import Batch2D

        tunnels = cases2d.batched_naca_tunnels(64)
        b = Batch2D([dict(c, device=0) for c, _ in tunnels])
        for t, (c, sdf) in zip(b.tunnels, tunnels):
            t.setSdf(sdf)
            t.initField(perturbed_rest2(c["width"], c["height"], 1e-4))
        b.setLaunch(32, 2, False)
        b.step(max(3, args.warmup) + args.steps)
        b.synchronize()
        b.destroy()
        print(json.dumps({"profile2d": "done", "steps": max(3, args.warmup) + args.steps}))
        return
    W, H, D = (int(v) for v in args.grid.lower().split("x"))
    N = W * H * D
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist  # plumbing only: a barrier and a max over ranks
        from datetime import timedelta

        dist.init_process_group(backend="gloo", timeout=timedelta(seconds=120))
    workload = f"D3Q19 {W}x{H}x{D} {args.precision} sphere d=16 Re200 tunnel"

    if args.impl == "reference":
        if rank == 0:
            cb = cpu_baseline(W, H, D, args.precision, budget_s=60.0, max_steps=max(1, args.steps))
            line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "MLUPS", "n_gpus": args.gpus,
                    "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                    "config": {"workload": workload, "grid": [W, H, D], "storage": args.precision,
                               "note": "the reference is TypeScript+WGSL for browser WebGPU, which cannot run here; "
                                       "its kernels' C++ restatement (oracle/) runs on the host cores instead"},
                    "cpu_baseline": cb,
                    "e2e": {"value": cb["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    s, sdf, macro, tau = tunnel_setup(W, H, D, args.precision, device=local)
    s.setSdf(sdf)
    s.initField(macro)
    s.setInletRamp("linear", 0.1, 3000, 1)
    if dist is not None:
        dist.barrier()
    with ClockSampler(physical_gpu_index(local)) as clocks:
        ms, launches = time_steps(s, max(3, args.warmup), args.steps)
    clk = clocks.summary()
    if dist is not None:
        import torch

        t = torch.tensor([ms], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    mlups = world * N * args.steps / (ms * 1e3)
    per_gpu_mlups = N * args.steps / (ms * 1e3)
    hbm, peak_kind = peaks()
    achieved = per_gpu_mlups * 1e6 * BYTES_PER_CELL[args.precision] / 1e9
    traffic = profiled_traffic(workload)
    info = s.info()
    copy = copy_roofline(local, args.precision, N)
    copy["step_frac"] = round(achieved / copy["gbps"], 4)
    line = {
        "metric": METRIC, "value": round(mlups, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if args.precision != "fp64" else "f64", "data": "synthetic",
        "config": {"workload": workload, "grid": [W, H, D], "storage": args.precision, "tau": tau,
                   "parallelism": f"replicas{world}", "l2": "inputs larger than L2 (2 x 134 MB populations)",
                   "block": [info["block_x"], info["block_y"]], "body_cells": info["n_body_cells"]},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                     "frac": round(achieved / hbm, 4), "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_cell": BYTES_PER_CELL[args.precision]},
        "copy_roofline": copy,
        "gpu_launches": launches,
        "clocks": clk,
    }
    if not args.no_extras and not args.profile:
        e2e_steps = 1000  # fixed: the public-API loop of 10 chunks of 100 steps, whatever --steps is
        dt, h2d, d2h = run_e2e(s, sdf, macro, e2e_steps)
        line["e2e"] = {"value": round(N * e2e_steps / dt / 1e6 * world, 1), "unit": "MLUPS",
                       "h2d_bytes_per_step": h2d / e2e_steps, "d2h_bytes_per_step": d2h / e2e_steps,
                       "steps": e2e_steps, "calls": "setSdf, initField, (setInlet, run(100), readForces) x k, readMacro",
                       "host_buffers": "pinned (cells_host_alloc)"}
        s.destroy()
        def variant(prec, grid, steps):
            v, vsdf, vmac, _ = tunnel_setup(*grid, prec, device=local)
            v.setSdf(vsdf)
            v.initField(vmac)
            v.setInletRamp("linear", 0.1, 3000, 1)
            vms, _ = time_steps(v, 100, steps)
            v.destroy()
            vn = grid[0] * grid[1] * grid[2]
            vm = vn * steps / (vms * 1e3)
            vcopy = copy_roofline(local, prec, vn)
            return {"storage": prec, "grid": list(grid), "steps": steps, "mlups": round(vm, 1),
                    "hbm_frac": round(vm * 1e6 * BYTES_PER_CELL[prec] / 1e9 / hbm, 4),
                    "copy_gbps": vcopy["gbps"],
                    "copy_frac": round(vm * 1e6 * BYTES_PER_CELL[prec] / 1e9 / vcopy["gbps"], 4)}

        line["variants"] = [variant(prec, (W, H, D), 1000) for prec in ("fp16", "bf16", "fp64")]
        # the targets' own workload: the 256x128x128 step in FP32 and 16-bit storage, CUDA events
        big = {prec: variant(prec, (256, 128, 128), 2000) for prec in ("fp32", "fp16", "bf16")}
        line["targets_256x128x128"] = {
            "workload": "D3Q19 256x128x128 sphere tunnel (d = 21.3, Re 200), 2000 timed steps after 100",
            "fp32": big["fp32"], "fp16": big["fp16"], "bf16": big["bf16"],
            "fp16_over_fp32": round(big["fp16"]["mlups"] / big["fp32"]["mlups"], 4),
            "bf16_over_fp32": round(big["bf16"]["mlups"] / big["fp32"]["mlups"], 4),
            "targets": "HBM frac >= 0.75 in FP32 and FP16; FP16 >= 1.8x FP32"}
        from cells_b200 import cases2d

        line["precision_cd"] = precision_cd(local)
        b2 = cases2d.batched_naca_throughput(10000, device=local)
        b2["hbm_frac"] = round(b2["batched_mlups"] * 1e6 * 72 / 1e9 / hbm, 4)
        line["batched2d"] = b2
        c2 = cases2d.cylinder_tunnel(20000, device=local)
        line["cylinder2d"] = {"workload": "D2Q9 400x100 cylinder D=20 Re100, 20000 steps", "mlups": c2["mlups"],
                              "C_D": c2["C_D"], "C_L_amp": c2["C_L_amp"], "St": c2["St"]}
        line["adjoint"] = adjoint_cost(local)
        if rank == 0 and world == 1:
            line["cpu_baseline"] = cpu_baseline(W, H, D, args.precision)
    else:
        s.destroy()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
