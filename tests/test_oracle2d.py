"""The 2D oracle against the reference's own acceptance tests (CPU only).

The reference holds no golden vectors for step results; what pins its 2D step is its validation
suite (src/cases.ts). The two cases that run in seconds on the CPU are ported here unchanged and
run on the oracle (oracle/lbm2d.cpp): plane Poiseuille (src/cases.ts:61-91, L2 error below 2e-4 for
tau in {0.6, 1.0, 1.5}) and the Taylor-Green vortex (src/cases.ts:131-190: viscosity within 1%,
velocity L2 below 1% at N = 128, convergence order at least 1.8). The D2Q9 equilibrium moments
follow src/analysis.test.ts:65-73.
"""
import math

import numpy as np
import pytest

from cells_b200.lattice3d import CX2, CY2, XMode, YMode, equilibrium2
from oracle.oracle import OracleSolver2D


def test_d2q9_equilibrium_moments():
    f = equilibrium2(1.1, 0.05, -0.02)
    assert abs(f.sum() - 1.1) < 1e-12
    assert abs(sum(f[i] * CX2[i] for i in range(9)) - 1.1 * 0.05) < 1e-12
    assert abs(sum(f[i] * CY2[i] for i in range(9)) - 1.1 * -0.02) < 1e-12


def poiseuille_error(tau, precision="fp32"):
    H, u_max = 32, 0.05
    nu = (tau - 0.5) / 3
    fx = 8 * nu * u_max / (H * H)
    s = OracleSolver2D(4, H, XMode.Periodic, XMode.Periodic, YMode.NoSlip, YMode.NoSlip, tau=tau,
                       precision=precision, bodyForce=(fx, 0.0), forceEvery=0)
    s.initField()
    n = math.ceil(10 * H * H / nu)
    s.run(n, 2000)
    m = s.readMacro()
    num = den = 0.0
    for y in range(H):
        e = fx / (2 * nu) * (y + 0.5) * (H - y - 0.5)
        num += (float(m[(y * 4 + 1) * 4 + 1]) - e) ** 2
        den += e * e
    return math.sqrt(num / den)


@pytest.mark.parametrize("tau", [0.6, 1.0, 1.5])
def test_poiseuille_reference_acceptance(tau):
    assert poiseuille_error(tau) < 2e-4


def taylor_green(n, precision="fp32"):
    tau = 0.8
    nu = (tau - 0.5) / 3
    u0 = 0.04 * 32 / n
    k = 2 * math.pi / n
    s = OracleSolver2D(n, n, XMode.Periodic, XMode.Periodic, YMode.Periodic, YMode.Periodic, tau=tau,
                       precision=precision, forceEvery=0)

    def field(t):
        a = u0 * math.exp(-2 * nu * k * k * t)
        y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        m = np.zeros((n, n, 4), dtype=np.float32)
        m[..., 0] = 1 - 0.75 * a * a * (np.cos(2 * k * x) + np.cos(2 * k * y))
        m[..., 1] = -a * np.cos(k * x) * np.sin(k * y)
        m[..., 2] = a * np.sin(k * x) * np.cos(k * y)
        return m.reshape(-1)

    s.initField(field(0))
    t = round(math.log(2) / (2 * nu * k * k))
    energy = lambda m: float(np.sum(m[1::4].astype(np.float64) ** 2 + m[2::4].astype(np.float64) ** 2))
    s.run(round(t / 2))
    mid = s.readMacro()
    s.run(t - round(t / 2))
    end = s.readMacro()
    exact = field(t)
    num = den = 0.0
    for c in (1, 2):
        num += float(np.sum((end[c::4].astype(np.float64) - exact[c::4]) ** 2))
        den += float(np.sum(exact[c::4].astype(np.float64) ** 2))
    dt = t - round(t / 2)
    nu_measured = math.log(energy(mid) / energy(end)) / (4 * k * k * dt)
    return math.sqrt(num / den), nu_measured / nu


def test_taylor_green_reference_acceptance():
    errors = []
    ratio = None
    for n in (32, 64, 128):
        err, ratio = taylor_green(n)
        errors.append(err)
    order = math.log2(errors[0] / errors[2]) / 2
    assert 0.99 <= ratio <= 1.01
    assert errors[2] < 0.01
    assert order >= 1.8


def test_fp64_oracle_agrees_with_fp32():
    e32 = poiseuille_error(1.0, "fp32")
    e64 = poiseuille_error(1.0, "fp64")
    assert e64 < 2e-4 and abs(e32 - e64) < 1e-4
