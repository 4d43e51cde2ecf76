"""A differentiable steady solve for PyTorch: J(hsrc, ln lambda) with its gradient from the GPU
adjoint (h2g_adjoint), as a torch.autograd.Function.  No reference counterpart (the reference has
no gradients); the wrapped forward is PBiCGSTAB! + RB-GS (src/NonUniform.jl:248-350) on the
reference's operator.

    J = (sum_c w_c theta_c^p)^(1/p),    A(lambda) theta = b(hsrc)   (steady, calRHS! b)
    lambda_c = lambda0_c * exp(lnlam_c) on the interior; an isothermal guard copies its scaled
    interior neighbour (apply_boundary_conditions!, src/boundary_conditions.jl:198-205)

backward returns dJ/dhsrc and dJ/dlnlam per cell (zero on the guards, which the model does not
use) times the incoming gradient.  Inputs and gradients are float64 tensors of the grid's shape
(MX, MY, MZ) indexed [i, j, k] like the reference's arrays.  The library keys every cell's
conductivity in 7 bits, so lambda may take at most 127 distinct values over the grid: per-band or
per-material parameters fit (the 13 log-scales of h2_b200.adjoint give at most 84), a field of
per-cell values does not (H2GError, status UNSUPPORTED).  The gradient is per cell either way.
The Julia counterpart is the ChainRulesCore rrule in julia/H2GPURules.jl.
"""
from __future__ import annotations

import numpy as np
import torch

from . import adjoint as A
from .model import ISOTHERMAL, _face
from .nonuniform import Solver


class HotspotProblem:
    """The fixed data of the objective: a Solver with the grid set (steady), the base conductivity
    lam0 and mask (guard layers included, boundary conditions applied), the starting temperature
    theta0, the boundary set `bcs` (six (type, T, q, h, T_inf) tuples, x-, x+, y-, y+, z-, z+), the
    weights w (e.g. A.silicon_weights), the exponent p and the solver tolerance."""

    def __init__(self, solver: Solver, lam0, mask, theta0, bcs, weights, p: float = 8.0, tol: float = 1e-12):
        self.s = solver
        self.lam0 = np.asfortranarray(lam0, dtype=np.float64)
        self.mask = np.asfortranarray(mask, dtype=np.float64)
        self.theta0 = np.asfortranarray(theta0, dtype=np.float64)
        self.bcs = list(bcs)
        self.w = np.asfortranarray(weights, dtype=np.float64)
        self.p = float(p)
        self.tol = float(tol)

    def lam(self, lnlam: np.ndarray) -> np.ndarray:
        lam = self.lam0.copy(order="F")
        inner = (slice(1, -1),) * 3
        lam[inner] *= np.exp(lnlam[inner])
        for f, bc in enumerate(self.bcs):
            if bc[0] == ISOTHERMAL:
                g, i = _face(lam, f)
                lam[g] = lam[i]
        return lam

    def prepare(self, hsrc: np.ndarray, lnlam: np.ndarray):
        """Fields, heat source, start temperature and b = calRHS! of (hsrc, lambda) on the device."""
        s = self.s
        s.set_fields(self.lam(lnlam), self.mask)
        s.set_hsrc(np.asfortranarray(hsrc, dtype=np.float64))
        s.set_theta(self.theta0)
        s.calrhs(self.bcs, zero_b=True)

    def value(self) -> float:
        st, res = self.s.solve("pbicgstab", tol=self.tol, maxItr=20_000, smoother="gs")
        if not res.isconverged:
            raise RuntimeError(f"forward solve did not converge (status {st})")
        th = self.s.get_theta()
        return float(np.sum(self.w * th ** self.p) ** (1.0 / self.p))


def _np(t: torch.Tensor) -> np.ndarray:
    return np.asfortranarray(t.detach().to("cpu", torch.float64).numpy())


class HotspotNorm(torch.autograd.Function):
    """J = HotspotNorm.apply(hsrc, lnlam, problem); J.backward() gives hsrc.grad, lnlam.grad."""

    @staticmethod
    def forward(ctx, hsrc: torch.Tensor, lnlam: torch.Tensor, problem: HotspotProblem):
        problem.prepare(_np(hsrc), _np(lnlam))
        if ctx.needs_input_grad[0] or ctx.needs_input_grad[1]:
            J, gh, gl, rf, ra = A.steady_gradient(problem.s, problem.w, problem.p, tol=problem.tol)
            if not (rf.isconverged and ra.isconverged):
                raise RuntimeError("forward or adjoint solve did not converge")
            dev = hsrc.device
            ctx.save_for_backward(torch.from_numpy(np.ascontiguousarray(gh)).to(dev),
                                  torch.from_numpy(np.ascontiguousarray(gl)).to(dev))
        else:
            J = problem.value()
        return torch.tensor(J, dtype=torch.float64, device=hsrc.device)

    @staticmethod
    def backward(ctx, gJ: torch.Tensor):
        gh, gl = ctx.saved_tensors
        return gJ * gh, gJ * gl, None


def hotspot_norm(hsrc: torch.Tensor, lnlam: torch.Tensor, problem: HotspotProblem) -> torch.Tensor:
    return HotspotNorm.apply(hsrc, lnlam, problem)
