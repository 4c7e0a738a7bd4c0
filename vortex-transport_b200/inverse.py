"""Batched inverse problem: recover each vortex's strength, Mach number and
centre (eps, M, x0, y0) from its state after `steps` RK4 steps.

All instances share one mesh (a batch group), so every loss evaluation is one
batched forward sweep and one batched reverse sweep (vt_batch_adjoint_*: one
launch per stage for all instances). The loss of instance i is the
mass-weighted misfit J_i = 1/2 ||U_i(T) - U*_i(T)||_M; dJ_i/dtheta_i follows
from dJ_i/dU_i(0) (the adjoint) through the torch initial condition. Each
instance runs its own L-BFGS on the host (two-loop recursion, Armijo
backtracking, curvature pairs kept only when s.y > 0); the instances' trial
points are evaluated together. The parameters are scaled very differently (M
sets the background pressure, p = 1/(gamma M^2), and its gradient is ~1e4
times the others'), so the two-loop recursion starts from the inverse
Gauss-Newton diagonal 1 / ||dU(0)/dtheta_k||_M^2 instead of a scalar.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import Batch, Problem, make_params
from .adjoint import mass_matrix, vortex_ic

PARAMS = ("epsilon", "M_infty", "x0", "y0")
# box keeping every trial state physical (M and eps bound the vortex depth)
LOWER = np.array([0.05, 0.25, -3.0, -3.0])
UPPER = np.array([0.6, 0.8, 3.0, 3.0])


def true_parameters(n: int = 128, seed: int = 5) -> np.ndarray:
    """(n, 4) seeded true parameters: eps ~ U[0.15, 0.45], M ~ U[0.3, 0.6],
    centre ~ U[-1.5, 1.5]^2."""
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0.15, 0.45, n), rng.uniform(0.3, 0.6, n),
                     rng.uniform(-1.5, 1.5, n), rng.uniform(-1.5, 1.5, n)], axis=1)


def perturbed_guess(theta: np.ndarray, seed: int = 6) -> np.ndarray:
    """The initial guess: eps +- 0.05, M +- 0.05, centre +- 0.3 (seeded)."""
    rng = np.random.default_rng(seed)
    d = rng.uniform(-1.0, 1.0, theta.shape) * np.array([0.05, 0.05, 0.3, 0.3])
    return np.clip(theta + d, LOWER, UPPER)


@dataclass
class History:
    it: list = field(default_factory=list)
    loss: list = field(default_factory=list)
    err: list = field(default_factory=list)


class BatchedInverse:
    """n instances of the vortex on one side x side mesh of order p."""

    def __init__(self, theta_true: np.ndarray, side: int = 64, p: int = 2, steps: int = 300,
                 dt: float = 1.5e-4, nsnapshots: int | None = None, integration_order: int = 10,
                 device: int = 0):
        self.n = theta_true.shape[0]
        self.steps, self.dt = steps, dt
        self.nsnapshots = nsnapshots or steps
        self.problem = Problem(make_params(side, side, p=p, integration_order=integration_order, time_step=dt))
        self.batch = Batch([self.problem] * self.n, device=device)
        self.batch.set_dt(np.full(self.n, dt))
        self.dev = torch.device("cuda", device)
        self.nodes = torch.tensor(self.problem.array("nodes_phys"), device=self.dev)
        self.detj = torch.tensor(self.problem.array("detj"), device=self.dev)
        self.M = torch.tensor(mass_matrix(self.problem), device=self.dev)
        self.theta_true = np.array(theta_true, dtype=np.float64)
        self.evaluations = 0
        self.gpu_seconds = 0.0
        with torch.no_grad():
            self._upload(self._ic(torch.tensor(self.theta_true, device=self.dev)))
        self.batch.rk4(steps)
        self.target = self._download()

    def _ic(self, th: torch.Tensor) -> torch.Tensor:
        c = [th[:, k, None, None] for k in range(4)]
        return vortex_ic(self.nodes[None], c[0], c[1], c[2], c[3])

    def _upload(self, U0: torch.Tensor) -> None:
        U0 = U0.detach().contiguous()
        for i in range(self.n):
            self.batch.upload_device(i, U0[i])

    def _download(self) -> torch.Tensor:
        K, Np = self.batch.shapes[0]
        out = torch.empty((self.n, K, Np, 4), dtype=torch.float64, device=self.dev)
        for i in range(self.n):
            self.batch.download_device(i, out[i])
        return out

    def loss_and_grad(self, theta: np.ndarray):
        """Per-instance losses (n,) and gradients (n, 4) at theta (n, 4)."""
        th = torch.tensor(theta, device=self.dev, requires_grad=True)
        U0 = self._ic(th)
        t0 = time.perf_counter()
        self._upload(U0)
        self.batch.adjoint_forward(self.steps, self.nsnapshots)
        UT = self._download()
        d = UT - self.target
        Md = torch.einsum("ij,nejc->neic", self.M, d)
        w = self.detj[None, :, None, None]
        J = 0.5 * torch.sum(w * d * Md, dim=(1, 2, 3))
        gT = (w * Md).contiguous()
        lam = self.batch.adjoint_backward([gT[i] for i in range(self.n)])
        self.gpu_seconds += time.perf_counter() - t0
        self.evaluations += 1
        g, = torch.autograd.grad(U0, th, grad_outputs=torch.stack(lam))
        return J.detach().cpu().numpy(), g.cpu().numpy()

    def gauss_newton_diagonal(self, theta: np.ndarray) -> np.ndarray:
        """(n, 4): ||dU_i(0)/dtheta_ik||^2 in the mass-weighted norm."""
        th = torch.tensor(theta, device=self.dev)
        out = np.empty_like(theta)
        w = self.detj[None, :, None, None]
        for k in range(4):
            e = torch.zeros_like(th)
            e[:, k] = 1.0
            _, v = torch.func.jvp(self._ic, (th,), (e,))
            out[:, k] = torch.sum(w * v * torch.einsum("ij,nejc->neic", self.M, v), dim=(1, 2, 3)).cpu().numpy()
        return out

    def solve(self, theta0: np.ndarray, iterations: int = 50, memory: int = 8, c1: float = 1e-4,
              ftol: float = 1e-20, max_evaluations: int | None = None, history: History | None = None):
        """Independent L-BFGS per instance, at most `iterations` accepted steps
        each; an instance stops early once its loss is below ftol times its
        starting loss, or when backtracking stalls. Returns (theta, loss,
        accepted steps) per instance."""
        n = self.n
        x = np.clip(np.array(theta0, dtype=np.float64), LOWER, UPPER)
        h0 = 1.0 / np.maximum(self.gauss_newton_diagonal(x), 1e-300)
        f, g = self.loss_and_grad(x)
        f_start = f.copy()
        stop = np.zeros(n, dtype=bool)
        S = [[] for _ in range(n)]
        Y = [[] for _ in range(n)]
        done = np.zeros(n, dtype=int)
        alpha = np.ones(n)
        d = np.zeros_like(x)
        fresh = np.ones(n, dtype=bool)  # a new direction is needed
        max_evaluations = max_evaluations or 4 * iterations
        while (~stop & (done < iterations)).any() and self.evaluations < max_evaluations:
            for i in np.nonzero(fresh & ~stop & (done < iterations))[0]:
                q = g[i].copy()
                a = []
                for s_, y_ in zip(reversed(S[i]), reversed(Y[i])):
                    r = 1.0 / (y_ @ s_)
                    a.append(r * (s_ @ q))
                    q -= a[-1] * y_
                q *= h0[i]
                for (s_, y_), ai in zip(zip(S[i], Y[i]), reversed(a)):
                    r = 1.0 / (y_ @ s_)
                    q += s_ * (ai - r * (y_ @ q))
                d[i] = -q
                if d[i] @ g[i] >= 0:  # not a descent direction: scaled steepest descent
                    d[i] = -h0[i] * g[i]
                alpha[i] = 1.0
                fresh[i] = False
            active = ~stop & (done < iterations)
            xt = np.where(active[:, None], np.clip(x + alpha[:, None] * d, LOWER, UPPER), x)
            ft, gt = self.loss_and_grad(xt)
            for i in np.nonzero(active)[0]:
                if ft[i] <= f[i] + c1 * (g[i] @ (xt[i] - x[i])):
                    s_, y_ = xt[i] - x[i], gt[i] - g[i]
                    if s_ @ y_ > 1e-300:
                        S[i].append(s_)
                        Y[i].append(y_)
                        if len(S[i]) > memory:
                            S[i].pop(0)
                            Y[i].pop(0)
                    x[i], f[i], g[i] = xt[i], ft[i], gt[i]
                    done[i] += 1
                    fresh[i] = True
                    stop[i] = f[i] <= ftol * f_start[i]
                else:
                    alpha[i] *= 0.5
                    stop[i] = alpha[i] < 1e-8  # stalled
            if history is not None:
                history.it.append(int(done.min()))
                history.loss.append(float(f.sum()))
                history.err.append(float(np.abs(x - self.theta_true).max()))
        return x, f, done

    def close(self):
        self.batch.close()
