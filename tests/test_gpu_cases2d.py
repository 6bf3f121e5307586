"""The 2D workloads on the GPU against the reference's own acceptance ranges and the oracle.

* The 400x100 cylinder tunnel (D = 20 at (80, 50.5), Re 100, linear ramp to 0.1 over 3000 steps,
  20,000 steps): exact arithmetic reproduces the oracle's force trace and final field bit for bit;
  fast arithmetic keeps C_D, the C_L amplitude and St within 1% of the oracle's.
* The eight validation cases of src/cases.ts with their acceptance ranges unchanged: plane
  Poiseuille, Taylor-Green, periodic-seam invariance, Schafer-Turek 2D-1 and 2D-2, the unconfined
  cylinder (St 0.165 +- 4%, mean C_D 1.345 +- 5%), the Ghia lid-driven cavity and NACA0012 at Re 500.
"""
import math

import numpy as np
import pytest

from cells_b200 import cases2d
from oracle.oracle import OracleSolver2D

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_cylinder():
    cfg, sdf, macro = cases2d.cylinder_tunnel_inputs()
    W, H = cfg.pop("width"), cfg.pop("height")
    o = OracleSolver2D(W, H, **cfg)
    o.setSdf(sdf)
    o.initField(macro)
    forces = []
    for step in range(20000):
        o.update(uIn=cases2d.cylinder_ramp(step))
        o.encodeSteps(1)
        if step % 2000 == 1999:
            forces.extend(o.readForces())
    o.run(0)
    out = cases2d.cylinder_coefficients(forces)
    out.update(forces=forces, macro=o.readMacro(), populations=o.populations().copy())
    return out


def test_cylinder_tunnel_exact_is_bit_identical_to_oracle(oracle_cylinder):
    got = cases2d.cylinder_tunnel(20000, exact=True)
    ref = oracle_cylinder
    assert [f["step"] for f in got["forces"]] == [f["step"] for f in ref["forces"]]
    for a, b in zip(got["forces"], ref["forces"]):
        scale = max(abs(b["fx"]), abs(b["fy"]), 1e-12)
        assert abs(a["fx"] - b["fx"]) <= 1e-9 * scale and abs(a["fy"] - b["fy"]) <= 1e-9 * scale
    assert np.array_equal(got["macro"].view(np.uint32), ref["macro"].view(np.uint32))


def test_cylinder_tunnel_fast_within_one_percent(oracle_cylinder):
    got = cases2d.cylinder_tunnel(20000, exact=False)
    ref = oracle_cylinder
    print("GPU", {k: got[k] for k in ("C_D", "C_L_amp", "St", "mlups")}, "oracle",
          {k: ref[k] for k in ("C_D", "C_L_amp", "St")})
    assert math.isfinite(ref["St"]) and ref["C_L_amp"] > 0.1  # the wake sheds
    for k in ("C_D", "C_L_amp", "St"):
        assert abs(got[k] - ref[k]) <= 0.01 * abs(ref[k]), (k, got[k], ref[k])


@pytest.mark.parametrize("key", ["poiseuille", "taylorGreen", "periodicSeam", "schaferTurek1", "schaferTurek2",
                                 "cavity", "naca"])
def test_reference_validation_case(key):
    r = cases2d.run_case(key)
    print(r["name"], [(m["name"], m["value"]) for m in r["metrics"]], f"{r['seconds']:.1f} s")
    assert r["pass"], r["metrics"]


def test_unconfined_cylinder_reference_ranges():
    r = cases2d.run_case("unconfinedCylinder")
    print(r["name"], [(m["name"], m["value"]) for m in r["metrics"]], r["steps"], f"{r['seconds']:.1f} s")
    assert r["pass"], r["metrics"]
