"""3D precision checks on the GPU.

* The reference's sphereFp16 case (src/cases3d.ts:11-81): Re 100 sphere at 192x96x96, C_D of FP16
  storage within 1% of FP32 (the reference's gate), run to convergence; the FP32 C_D within 1% of
  the reference's published 1.156 for this case (README.md:71).
* The sphere of the precision sweep (D = 20, Re 200, 256x128x128, 4000 steps): C_D of FP32 and FP16
  storage within 1% of the FP64 run of the same kernel and grid. BF16 (8-bit mantissa) is measured
  at about 1.5% and held to 3%.
"""
import pytest

from cells_b200 import cases3d

pytestmark = pytest.mark.gpu


def test_sphere_fp16_reference_gate():
    r = cases3d.sphere_fp16(precisions=("fp32", "fp16"))
    print(r)
    assert r["pass"], r
    assert abs(r["C_D"]["fp32"] - 1.156) <= 0.01 * 1.156, r["C_D"]


def test_sphere_precisions_within_one_percent_of_fp64():
    rows = cases3d.precision_sweep(obstacles=(("sphere", 20, 0.0),))
    row = rows[0]
    print(row)
    for prec, tol in (("fp32", 1e-3), ("fp16", 0.01), ("bf16", 0.03)):
        assert row[prec]["C_D_err_vs_fp64"] <= tol, (prec, row[prec])
