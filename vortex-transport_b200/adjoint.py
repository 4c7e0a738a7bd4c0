"""torch.autograd bridge to the discrete adjoint of the RK4 stepper.

`rk4_run(U0, solver, dt, nsteps)` is U(T) as a differentiable function of
U(0): its forward is vt_adjoint_forward (the same kernels as vt_step_rk4, with
binomial checkpoints kept in device memory) and its backward is
vt_adjoint_backward (the exact transpose of the linearised step). Used for
gradient checks and for recovering vortex parameters from a final state; the
stepping itself never runs in torch.

The loss of the inverse problems is the mass-weighted misfit
    J = 1/2 sum_e detJ_e sum_c (U - U*)_{e,:,c}^T M_ref (U - U*)_{e,:,c},
and `vortex_ic` restates the reference's nodal vortex initial condition
(Element.cpp:124-179) in torch, so dJ/d(eps, M, x0, y0) follows by the chain
rule through dJ/dU(0).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import Problem, Solver, default_vortex


class _RK4Run(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U0, solver, dt, nsteps, nsnapshots):
        torch.cuda.current_stream(U0.device).synchronize()
        U0c = U0.detach().to(torch.float64).contiguous()
        solver.upload_device(U0c.data_ptr())
        solver.adjoint_forward(dt, nsteps, nsnapshots)
        UT = torch.empty_like(U0c)
        solver.download_device(UT.data_ptr())
        ctx.solver = solver
        return UT

    @staticmethod
    def backward(ctx, grad):
        return ctx.solver.adjoint_backward(grad.contiguous()), None, None, None, None


def rk4_run(U0: torch.Tensor, solver: Solver, dt: float, nsteps: int, nsnapshots: int | None = None):
    """U(T) after nsteps RK4 steps from U0 (a (K, Np, 4) float64 CUDA tensor on
    the solver's device), differentiable in U0. nsnapshots (default: every
    step) bounds the checkpoint states kept in device memory."""
    return _RK4Run.apply(U0, solver, float(dt), int(nsteps), int(nsnapshots or nsteps))


def mass_matrix(problem: Problem) -> np.ndarray:
    """M_ref, the reference mass matrix (the inverse of minv_ref)."""
    return np.linalg.inv(problem.array("minv_ref"))


def mass_weighted_loss(U: torch.Tensor, target: torch.Tensor, detj: torch.Tensor, M: torch.Tensor):
    d = U - target
    Md = torch.einsum("ij,ejc->eic", M, d)
    return 0.5 * torch.sum(detj[:, None, None] * d * Md)


def vortex_ic(nodes: torch.Tensor, epsilon, M_infty, x0, y0, base=None) -> torch.Tensor:
    """Nodal isentropic-vortex state at the (K, Np, 2) physical nodes, the
    formula of the host initial condition at t = 0 with p_infty = 1/(gamma M^2)
    (the free stream at unit speed and Mach M). The parameters may be tensors
    that require grad."""
    c = base or default_vortex()
    g = c.gamma
    x, y = nodes[..., 0], nodes[..., 1]
    dx, dy = x - x0, y - y0
    f0 = 1.0 - (dx * dx + dy * dy) / (c.rc * c.rc)
    f1 = 1.0 - epsilon * epsilon * (g - 1) * M_infty * M_infty * torch.exp(f0) / (8.0 * math.pi ** 2)
    f2 = epsilon * (c.U_infty ** 2 + c.V_infty ** 2) * torch.exp(f0 / 2.0) / (2.0 * math.pi * c.rc)
    p_infty = 1.0 / (g * M_infty * M_infty)
    rho = c.rho_infty * f1 ** (1.0 / (g - 1.0))
    u = c.U_infty - f2 * dy
    v = c.V_infty + f2 * dx
    p = p_infty * f1 ** (g / (g - 1.0))
    E = p / (rho * (g - 1.0)) + (u * u + v * v) / 2.0
    return torch.stack([rho, rho * u, rho * v, rho * E], dim=-1)
