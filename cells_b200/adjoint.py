"""Shape and inflow gradients of a tunnel's drag through the discrete adjoint (no counterpart in the
reference): a forward/backward pair in the style of an autograd Function.

``StarDrag.forward(coef, u)`` builds the star body r(theta, phi) = r0 (1 + sum_k coef_k Y_k) (16
real spherical harmonics, l <= 3), runs the D3Q19 tunnel from rest with the inlet ramped to u, and
returns J = C_D averaged over the objective window. ``StarDrag.backward()`` returns dJ/dcoef (16)
and dJ/du from one backward sweep of the recorded run: dJ/dsdf from the library, contracted with
dsdf/dcoef_k = -r0 Y_k(theta, phi) at each node, and dJ/du_in plus the explicit -2 J / u of the
coefficient's 1/u^2. ``finite_difference`` gives the central differences of the same J (FP64 runs by
default) for checking.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence

import numpy as np

from . import geometry as g
from ._lib import star_coef_gradient, star_sdf
from .rng import perturbed_rest3
from .solver3d import Solver3D
from .units import derive_tau


class StarDrag:
    """C_D of a star-shaped body in the D3Q19 tunnel. Defaults: 128x64x64, body centred at
    (W/4, H/2, D/2) with r0 = 12 (D = 24), Re 150 (tau 0.548), inlet ramped linearly to u over 3000
    steps, 6000 steps with C_D averaged over step labels 4000..6000, checkpoints every 100 steps,
    15% outlet sponge with absorb 0.02."""

    def __init__(self, W=128, H=64, D=64, r0=12.0, re=150.0, u=0.1, ramp_steps=3000, steps=6000,
                 window=(4000, 6000), checkpoint_every=100, precision="fp32", device=0, exact=False,
                 sponge=0.15, absorb=0.02, perturbation=1e-4):
        self.W, self.H, self.D = W, H, D
        self.r0 = r0
        self.center = (W / 4, H / 2, D / 2)
        self.tau = derive_tau(re, u, 2 * r0).tau
        self.u0 = u
        self.ramp_steps = ramp_steps
        self.steps = steps
        self.window = window
        self.K = checkpoint_every
        self.area = math.pi * r0 * r0
        self.solver = Solver3D.create(W, H, D, precision=precision, tau=self.tau, uIn=0.0, spongeFraction=sponge,
                                      spongeTau=1.0, absorb=absorb, forceEvery=0, device=device,
                                      exactArithmetic=exact)
        self.macro = perturbed_rest3(W, H, D, perturbation)
        self._coef = None
        self._u = None
        self._J = None
        self._sdf = None

    def sdf(self, coef) -> np.ndarray:
        s = g.empty_sdf3(self.W, self.H, self.D)
        star_sdf(s, self.W, self.H, self.D, self.center, self.r0, coef)
        return s

    def scale(self, u) -> float:
        return 2.0 / (u * u * self.area)

    def forward(self, coef: Sequence[float], u: Optional[float] = None) -> float:
        u = self.u0 if u is None else u
        s = self.solver
        self._coef = np.asarray(coef, dtype=np.float64)
        self._u = u
        self._sdf = self.sdf(self._coef)
        s.setSdf(self._sdf)
        s.initField(self.macro)
        s.setInletRamp("linear", u, self.ramp_steps, 1)
        self._J = s.adjointForward(self.steps, self.window[0], self.window[1], self.K, 0, self.scale(u))
        return self._J

    def backward(self):
        """(dJ/dcoef (16,), dJ/du) of the last forward: the adjoint sweep and the chain rule to the
        coefficients in one library call (cells3d_adjoint_backward_star)."""
        if self._J is None:
            raise RuntimeError("backward needs a forward first")
        dcoef, du = self.solver.adjointBackwardStar(self.center, self.r0, self._coef)
        return dcoef, du - 2.0 * self._J / self._u

    def coefficient_gradient(self, r):
        """(dJ/dcoef (16,), dJ/du) from the sweep's result r (Solver3D.adjointBackward): dJ/dsdf times
        the SDF's derivative by the coefficients (cells3d_star_coef_gradient), and dJ/du with the
        coefficient scale's own dependence on u."""
        dcoef = star_coef_gradient(r["dsdf"], self.W, self.H, self.D, self.center, self.r0, self._coef)
        du = r["du"] - 2.0 * self._J / self._u
        return dcoef, du

    def destroy(self):
        self.solver.destroy()


def finite_difference(problem_factory, coef, u, h=1e-4, which: Optional[Sequence[int]] = None):
    """Central differences of J = StarDrag.forward over the coefficients in `which` (indices 0..15,
    16 = u). problem_factory() returns the StarDrag to evaluate with (FP64 for the reference check).
    Returns (gradient dict, solidity flips dict)."""
    p = problem_factory()
    base = p.sdf(coef) < 0
    grads, flips = {}, {}
    which = list(range(17)) if which is None else list(which)
    for k in which:
        vals = []
        nflip = 0
        for sgn in (1, -1):
            c = np.array(coef, dtype=np.float64)
            uu = u
            if k < 16:
                c[k] += sgn * h
                nflip += int(np.count_nonzero((p.sdf(c) < 0) != base))
            else:
                uu = u + sgn * h
            vals.append(p.forward(c, uu))
        grads[k] = (vals[0] - vals[1]) / (2 * h)
        flips[k] = nflip
    p.destroy()
    return grads, flips
