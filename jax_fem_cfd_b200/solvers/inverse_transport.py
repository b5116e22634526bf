"""Differentiable inverse transport: a passive scalar (solvers/passive_transport.py
:64-97) carried by the flow of a wall-bounded unit square, with the flow's
nodal initial velocity as the unknown.

    loss(U_0) = sum_i m_i (phi_T,i - target_i)^2

with m the lumped nodal mass, phi_T the scalar after `steps` time steps of the
4-step flow step and the transport step, phi_0 the indicator of
[0.4, 0.6] x [0.2, 0.4] and the target a sum of three Gaussian blobs
(sigma 0.05) at seeded centres. The gradient is the hand-written adjoint of
solvers/adjoint.py (Step and Transport), chained by `rollout` with a
checkpoint every `ckpt` steps. The reference has no counterpart: it would
differentiate its JAX time loop with jax.grad.
"""
import numpy as np
import torch

from .adjoint import deferred_status, rollout


class InverseTransport:
    """The problem on an n x n Q1 mesh of the unit square, all walls no-slip,
    pinned pressure (rho = 1, mu = nu). The initial velocity is the
    parameter; `initial_velocity()` gives the seeded N(0, 0.1) start in FP32."""

    def __init__(self, n=128, steps=150, nu=1e-3, D=1e-4, dt=0.01, ckpt=10, supg=True, tol=1e-10, seed=0):
        from ..serving import cavity_config
        from ..setup import regular_mesh as rm
        from ..setup import simulation as sim
        _, timestep, coords, *rest = sim.setup(cavity_config(n))
        self.solver = timestep.solver
        self.ud = self.solver.u_full(rest[-1])
        self.nconn = rm.create_mesh_2d(n, n, 1.0, 1.0)[1]
        self.n, self.steps, self.nu, self.D, self.dt = n, steps, nu, D, dt
        self.ckpt, self.supg, self.tol, self.seed = ckpt, supg, tol, seed
        nn = self.solver.nn
        x, y = coords[:, 0], coords[:, 1]
        self.phi0 = ((x >= 0.4) & (x <= 0.6) & (y >= 0.2) & (y <= 0.4)).to(torch.float64)
        rng = np.random.default_rng(seed)
        target = torch.zeros(nn, dtype=torch.float64, device=coords.device)
        for cx, cy in rng.uniform(0.2, 0.8, size=(3, 2)):
            target += torch.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * 0.05 ** 2))
        self.target = target
        self.mass = self.solver.ctx.element_data()[6][:nn].clone()
        self.P0 = torch.zeros(nn, dtype=torch.float64, device=coords.device)

    def initial_velocity(self):
        g = torch.Generator(device="cpu").manual_seed(self.seed)
        u = 0.1 * torch.randn(self.solver.ndim * self.solver.nn, generator=g, dtype=torch.float32)
        return u.to(self.target.device)

    def final_scalar(self, U0, ckpt=None):
        state = rollout(self.solver, self.nconn, U0.to(torch.float64), self.P0, self.steps, self.dt, 1.0, self.nu,
                        self.ud, ckpt=self.ckpt if ckpt is None else ckpt, tol=self.tol, phi0=self.phi0, D=self.D,
                        supg=self.supg)
        return state[2]

    def loss(self, U0, ckpt=None):
        """The loss as a 0-d tensor (differentiable in U0). The solves' statuses
        are read once, at the end, unless an enclosing block defers them."""
        with deferred_status():
            return (self.mass * (self.final_scalar(U0, ckpt) - self.target) ** 2).sum()

    def value_and_grad(self, U0, ckpt=None):
        """(loss, d loss / d U0) with U0's dtype for the gradient."""
        u = U0.detach().clone().requires_grad_(True)
        with deferred_status():
            L = (self.mass * (self.final_scalar(u, ckpt) - self.target) ** 2).sum()
            L.backward()
        return float(L.detach()), u.grad
