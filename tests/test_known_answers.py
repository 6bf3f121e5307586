"""Known answers from the reference's own unit tests (tests/golden/known_answers.json) checked
against the host helpers, the lattice tables and the oracle. CPU only."""
import json
import math
import os

import numpy as np
import pytest

from cells_b200 import analysis, geometry as g, lattice3d as L, units
from oracle import oracle as O

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def close(a, b, digits):
    # vitest toBeCloseTo(x, d): |a - b| < 10^-d / 2
    return abs(a - b) < 10 ** (-digits) / 2


def test_d3q19_weights_and_isotropy():
    C = [L.CX, L.CY, L.CZ]
    assert len(L.CX) == L.Q3
    assert close(sum(L.W), 1, 12)
    for a in range(3):
        assert close(sum(L.W[i] * C[a][i] for i in range(L.Q3)), 0, 12)
        for b in range(3):
            m2 = sum(L.W[i] * C[a][i] * C[b][i] for i in range(L.Q3))
            assert close(m2, 1 / 3 if a == b else 0, 12)


def test_d3q19_opp_mirrors_pairs():
    C = [L.CX, L.CY, L.CZ]
    for i in range(L.Q3):
        assert L.OPP[L.OPP[i]] == i
        for a in range(3):
            assert C[a][L.OPP[i]] == -C[a][i]
        assert L.MIRROR_Y[L.MIRROR_Y[i]] == i
        assert (L.CX[L.MIRROR_Y[i]], L.CY[L.MIRROR_Y[i]], L.CZ[L.MIRROR_Y[i]]) == (L.CX[i], -L.CY[i], L.CZ[i])
        assert (L.CX[L.MIRROR_Z[i]], L.CY[L.MIRROR_Z[i]], L.CZ[L.MIRROR_Z[i]]) == (L.CX[i], L.CY[i], -L.CZ[i])
    seen = set()
    for a, b in L.PAIRS:
        assert b == L.OPP[a] and a < b
        seen |= {a, b}
    assert sorted(seen) == list(range(1, 19))


def test_device_mirror_tables_match_lattice():
    """The constexpr tables in cells_b200/csrc/d3q19.cuh equal the lattice's mirrors."""
    src = open(os.path.join(os.path.dirname(__file__), "..", "cells_b200", "csrc", "d3q19.cuh")).read()

    def table(name):
        body = src[src.index(name):]
        body = body[body.index("{", body.index("v[Q3]")) + 1:body.index("}", body.index("v[Q3]"))]
        return tuple(int(t) for t in body.split(","))

    assert table("mirror_y3") == L.MIRROR_Y
    assert table("mirror_z3") == L.MIRROR_Z
    assert table("cx3") == L.CX and table("cy3") == L.CY and table("cz3") == L.CZ


def test_flag_bits():
    dirs = ((1 << 19) - 1) & ~1
    for f in (L.FLAG_SOLID, L.FLAG_INLET, L.FLAG_OUTLET):
        assert f & dirs == 0 and 0 < f < 2 ** 32
    assert L.FLAG_SOLID & L.FLAG_INLET == 0 and L.FLAG_SOLID & L.FLAG_OUTLET == 0 and L.FLAG_INLET & L.FLAG_OUTLET == 0


def test_trt_lambda3_host_and_oracle():
    for c in GOLD["trtLambda3"]["cases"]:
        want = eval(c["expect_expr"]) if "expect_expr" in c else c["expect"]
        for fn in (L.trt_lambda3, O.lib().oracle_trt_lambda3):
            got = fn(c["tau"])
            if c.get("exact"):
                assert got == want
            else:
                assert close(got, want, c["digits"])


def test_equilibrium_moments():
    for rho, ux, uy, uz in GOLD["equilibrium3_moments"]["cases"]:
        f = L.equilibrium3(rho, ux, uy, uz)
        assert close(f.sum(), rho, 6)
        assert close(sum(f[i] * L.CX[i] for i in range(19)), rho * ux, 6)
        assert close(sum(f[i] * L.CY[i] for i in range(19)), rho * uy, 6)
        assert close(sum(f[i] * L.CZ[i] for i in range(19)), rho * uz, 6)
    rho, ux, uy = GOLD["equilibrium2_moments"]["case"]
    f = L.equilibrium2(rho, ux, uy)
    assert close(f.sum(), rho, 12)
    assert close(sum(f[i] * L.CX2[i] for i in range(9)), rho * ux, 12)
    assert close(sum(f[i] * L.CY2[i] for i in range(9)), rho * uy, 12)


def test_derive_tau():
    k = GOLD["deriveTau"]
    d = units.derive_tau(100, 0.1, 40)
    assert close(d.tau, k["plain"]["tau"], 10) and d.clamped is False
    c = units.derive_tau(1e5, 0.1, 40)
    assert c.clamped is True and c.tau == 0.51
    assert close(c.effective_re, units.max_reynolds(0.1, 40), 6)


def test_period_from_crossings():
    t = [k * 0.7 for k in range(5000)]
    v = [0.3 + math.sin(2 * math.pi * s / 123.4) for s in t]
    assert close(analysis.period_from_crossings(t, v)[0], 123.4, 2)
    assert analysis.period_from_crossings([0, 1, 2], [1, 2, 3]) is None


def test_circle_and_naca_sdf():
    s = g.empty_sdf(20, 20)
    g.add_circle(s, 20, 20, 10, 10, 4)
    assert close(s[10 * 20 + 10], -4, 2) and close(s[10 * 20 + 16], 2, 2)
    W, H = 200, 60
    s = g.empty_sdf(W, H)
    poly = g.naca_polygon(50, 30, 100, 0.12, 0)
    g.add_polygon(s, W, H, poly)
    assert s[30 * W + 80] < -5 and s[30 * W + 40] > 9
    assert close(poly[:, 1].max() - poly[:, 1].min(), 12, 1)


def _at(sdf, W, H, x, y, z):
    return sdf[x + W * (y + H * z)]


def _trilinear(sdf, W, H, x, y, z):
    x0, y0, z0 = math.floor(x), math.floor(y), math.floor(z)
    tx, ty, tz = x - x0, y - y0, z - z0
    v = 0.0
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = (tx if dx else 1 - tx) * (ty if dy else 1 - ty) * (tz if dz else 1 - tz)
                v += w * _at(sdf, W, H, x0 + dx, y0 + dy, z0 + dz)
    return v


def test_sdf3_shapes():
    W, H, D = 32, 24, 20
    s = g.empty_sdf3(W, H, D)
    g.add_sphere(s, W, H, D, 16, 12, 10, 4)
    assert close(_at(s, W, H, 16, 12, 10), -4, 6) and close(_at(s, W, H, 22, 12, 10), 2, 6)
    assert _at(s, W, H, 29, 12, 10) == g.FAR
    s = g.empty_sdf3(W, H, D)
    a = math.pi / 6
    g.add_box3(s, W, H, D, 16, 12, 10, 8, 1, 1, a)
    assert _trilinear(s, W, H, 16 + 6 * math.cos(a), 12 + 6 * math.sin(a), 10) < 0
    assert _trilinear(s, W, H, 16 + 6 * math.cos(-a), 12 + 6 * math.sin(-a), 10) > 0
    s = g.empty_sdf3(W, H, D)
    g.add_cylinder_z(s, W, H, D, 16, 12, 3)
    assert close(_at(s, W, H, 16, 12, 0), -3, 6) and close(_at(s, W, H, 16, 12, D - 1), -3, 6)


def test_wing_pivot_and_tips():
    W, H, D = 32, 24, 20
    s = g.empty_sdf3(W, H, D)
    cx, cy, cz, chord, span = 16, 12, 10, 19.2, 12
    a = 20 * math.pi / 180
    g.add_wing(s, W, H, D, cx, cy, cz, chord, span, a)
    d = (math.cos(a), -math.sin(a))
    lo, hi, off = math.inf, -math.inf, 0.0
    for y in range(H):
        for x in range(W):
            if _at(s, W, H, x, y, cz) >= 0:
                continue
            along = (x - cx) * d[0] + (y - cy) * d[1]
            lo, hi = min(lo, along), max(hi, along)
            off = max(off, abs(-(x - cx) * d[1] + (y - cy) * d[0]))
    assert _trilinear(s, W, H, cx, cy, cz) < 0
    assert -chord / 2 <= lo < -chord / 2 + 1.5
    assert chord / 2 - 3 < hi <= chord / 2
    assert off < 0.06 * chord + 1
    s = g.empty_sdf3(W, H, D)
    cx, cy, cz, chord, span = 16, 12, 10, 16, 12
    g.add_wing(s, W, H, D, cx, cy, cz, chord, span, 0)
    x = round(cx - chord / 2 + 0.3 * chord)
    assert close(_at(s, W, H, x, cy, cz + span // 2 + 1), 1, 1)
    assert close(_at(s, W, H, x, cy, cz - span // 2 - 1), 1, 1)
    assert _at(s, W, H, x, cy, cz) < 0


def test_reference_area_and_coefficients():
    for c in GOLD["referenceArea"]["cases"]:
        v = g.reference_area(c["obstacle"], c["size"], c["D"])
        assert v == c["value"] if c.get("exact") else close(v, c["value"], c["digits"])
    assert close(analysis.coefficient_scale(0.1, 100), 2, 12)
    assert analysis.coefficient_scale(0.1, 0) == 0


def test_build_body_sphere():
    W, H, D = 192, 96, 96
    b = analysis.build_body("sphere", 0.2, 0, W, H, D)
    assert b["sdf"][W // 4 + W * (H // 2 + H * (D // 2))] < 0
    assert close(b["lRef"], 19.2, 6) and close(b["area"], math.pi * 19.2 * 19.2 / 4, 6)
    lo, hi = b["bounds"]
    assert close(lo[0], W / 4 - 9.6 - 2, 6) and close(hi[1], H / 2 + 9.6 + 2, 6) and close(lo[2], D / 2 - 9.6 - 2, 6)
    flat = analysis.build_body("cube", 0.2, 0, W, H, D)["bounds"]
    turned = analysis.build_body("cube", 0.2, 20, W, H, D)["bounds"]
    assert turned[1][0] - turned[0][0] > flat[1][0] - flat[0][0]
    assert close(turned[1][2] - turned[0][2], flat[1][2] - flat[0][2], 6)
    none = analysis.build_body("none", 0.2, 0, 16, 8, 8)
    assert close(none["lRef"], 0.2 * 8, 12) and none["area"] == 0 and none["bounds"] is None
    assert np.all(none["sdf"] == g.FAR)


def test_divergence_predicates():
    assert analysis.has_diverged([]) is False
    assert analysis.has_diverged([{"fx": 1, "fy": -2}, {"fx": 1e30, "fy": 0, "fz": 3}]) is False
    assert analysis.has_diverged([{"fx": 1, "fy": 2}, {"fx": math.nan, "fy": 0}]) is True
    assert analysis.has_diverged([{"fx": 1, "fy": math.inf}]) is True
    assert analysis.has_diverged([{"fx": 1, "fy": 2, "fz": -math.inf}]) is True
    assert analysis.field_diverged(np.array([1, 0.1, 0, 0, 1, 0.1, 0, 0], dtype=np.float32)) is False
    assert analysis.field_diverged(np.array([1, 0.1, np.nan, 0], dtype=np.float32)) is True
    assert analysis.field_diverged(np.array([np.inf, 0, 0, 0], dtype=np.float32)) is True


@pytest.mark.parametrize("prec", [1, 2])
def test_codec_round_trips(prec):
    """FP16 x 2^15 with the +-1.99 clamp (src/shaders/common3d.ts:52-63) and bf16 round trips."""
    lib = O.lib()
    for v in [0.0, 1e-3, -0.0123, 0.3333, 1.5, -1.98]:
        r = lib.oracle_codec_roundtrip(prec, v)
        tol = (2.0 ** -11 if prec == 1 else 2.0 ** -8) * max(abs(v), 2.0 ** -15)
        assert abs(r - v) <= tol
    if prec == 1:
        assert abs(lib.oracle_codec_roundtrip(1, 5.0) - 1.99) < 1e-3  # clamped before the store
        assert abs(lib.oracle_codec_roundtrip(1, -5.0) + 1.99) < 1e-3
