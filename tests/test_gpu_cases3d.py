"""3D precision checks on the GPU.

* The reference's sphereFp16 case (src/cases3d.ts:11-81): Re 100 sphere at 192x96x96, C_D of FP16
  storage within 1% of FP32 (the reference's gate), run to convergence; the FP32 C_D within 1% of
  the reference's published 1.156 for this case (README.md:71).
* The sphere wake regimes the reference reports for its page's sphere (README.md:73): a steady
  leaning wake at Re 250 with side-force coefficient 0.063, shedding at Re 300 with St 0.135.
* The precision sweep (sphere D = 20, cube edge 18, spanwise cylinder D = 16, NACA0012 wing chord 40
  at 6 degrees; Re 200, 256x128x128, 4000 steps), each obstacle in FP32, FP16 x 2^15 and BF16
  storage against the FP64 run of the same kernel and grid: C_D of FP32 within 1e-4 relative and
  its velocity field within 1e-4 relative L2; FP16 C_D within 1% and velocity L2 within 1e-2. BF16
  (8-bit significand) measures 1.5-2.6% on C_D and is held to 4%.
"""
import pytest

from cells_b200 import cases3d

pytestmark = pytest.mark.gpu


def test_sphere_fp16_reference_gate():
    r = cases3d.sphere_fp16(precisions=("fp32", "fp16"))
    print(r)
    assert r["pass"], r
    assert abs(r["C_D"]["fp32"] - 1.156) <= 0.01 * 1.156, r["C_D"]


def test_precision_sweep_all_obstacles_against_fp64():
    rows = cases3d.precision_sweep()
    print(cases3d.sweep_table(rows))
    assert [r["obstacle"] for r in rows] == ["sphere", "cube", "cylinder", "wing"]
    for row in rows:
        for prec, cd_tol, l2_tol in (("fp32", 1e-4, 1e-4), ("fp16", 0.01, 1e-2), ("bf16", 0.04, 0.1)):
            e = row[prec]
            assert e["C_D_err_vs_fp64"] <= cd_tol, (row["obstacle"], prec, e)
            assert e["vel_L2_vs_fp64"] <= l2_tol, (row["obstacle"], prec, e)


def test_sphere_wake_re250_steady_leaning_wake():
    """The page's sphere (19.2 cells at 192x96x96, from rest, FP32) at Re 250: the wake is steady and
    leans to one side; the reference reports C_L 0.063 there (README.md:73; published 0.062). The
    side force here settles on the lattice diagonal (C_y = C_z), so its magnitude is compared."""
    r = cases3d.sphere_wake(250, 40000)
    print(r)
    assert max(r["side_amplitude"]) < 1e-3, r  # steady
    assert abs(r["C_side"] - 0.063) <= 0.05 * 0.063, r


def test_sphere_wake_re300_sheds_at_reference_strouhal():
    """The same sphere at Re 300 sheds; the reference reports St 0.135 (README.md:73; published
    0.137) after about 30,000 steps from rest."""
    r = cases3d.sphere_wake(300, 50000)
    print(r)
    assert max(r["side_amplitude"]) > 5e-3, r  # shedding
    assert abs(r["St"] - 0.135) <= 0.02 * 0.135, r
