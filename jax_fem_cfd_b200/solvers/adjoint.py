"""Adjoint of the pressure-projection stage of the 4-step time step.

The stage (solvers/standard.py:156-163, steps 5-7 of fem_step4) maps the
intermediate velocity U* to

    P = A+ k (D U* - F_p)                   k = rho / dt, A+ the pinned pressure solve
    U = U* - c M^-1 G P,  U = U_d on gamma_d     c = dt / rho, M the lumped mass

with D = G^T (divergence_element_mult is sum_i G_i^T u_i, gradient_element_mult
is [G_1 p; ...]). A+ solves A P = rhs with the gamma_p rows of A and rhs
zeroed and P = 0 on gamma_p, which is symmetric on the free nodes. The stage is
affine in U*, and its reverse (vector-Jacobian product) for output gradients
(g_U, g_P) is

    g_U' = g_U with gamma_d rows zeroed
    w    = g_P - c D (M^-1 g_U'),  w = 0 on gamma_p
    lam  = A+ w                     (the adjoint solve: the same pinned MG-PCG)
    g_U* = g_U' + k G lam

`Projection` puts this behind torch.autograd (the analogue of jax.custom_vjp).
It covers the projection stage only: the momentum solve (transposed BiCGSTAB
with Ce(U_n)^T and the linearisation of Ce in U_n) is not part of it. Pinned
pressure (set_zeroP) only. No reference counterpart: the reference
differentiates with jax.grad.
"""
import torch

from .. import _lib
from ..context import ptr, stream


def _solver_masks(solver):
    ctx = solver.ctx
    pm = solver.pmask.to(torch.bool)
    dm = solver.dmask.to(torch.bool) if solver.dmask is not None else None
    return ctx, pm, dm


def _pressure(solver, rhs, tol):
    """A+ rhs: the pinned MG-PCG pressure solve of the solver's context from 0."""
    ctx, pm, _ = _solver_masks(solver)
    r = rhs.clone()
    r[pm] = 0.0
    x = torch.zeros_like(r)
    it = torch.zeros(1, dtype=torch.int32, device=r.device)
    st = torch.zeros(1, dtype=torch.int32, device=r.device)
    _lib.call("fem_pressure_solve", ctx.handle, ptr(r), ptr(x), float(tol), 0.0, 1000, solver.precond, 0, 1, ptr(it),
              ptr(st), stream())
    if int(st.item()) != 0:
        raise _lib.FemError(f"pressure solve status {int(st.item())}")
    return x


def _grad(solver, p):
    y = torch.empty(solver.ndim * solver.nn, dtype=torch.float64, device=p.device)
    _lib.call("fem_grad_apply", solver.ctx.handle, ptr(p), None, ptr(y), stream())
    return y


def _div(solver, u):
    y = torch.empty(solver.nn, dtype=torch.float64, device=u.device)
    _lib.call("fem_div_apply", solver.ctx.handle, ptr(u), None, ptr(y), stream())
    return y


class Projection(torch.autograd.Function):
    """(U*, ...) -> (U, P) of the projection stage; backward is its adjoint."""

    @staticmethod
    def forward(fctx, U_star, solver, dt, rho, U_d_full, F_p, tol=1e-12):
        if not solver.cfg.set_zeroP:
            raise ValueError("Projection covers the pinned-pressure (set_zeroP) form only")
        ctx, pm, dm = _solver_masks(solver)
        M = ctx.element_data()[6]
        k, c = rho / dt, dt / rho
        U_star = U_star.detach().to(torch.float64).contiguous()
        rhs = k * (_div(solver, U_star) - (F_p if F_p is not None else 0.0))
        P = _pressure(solver, rhs, tol)
        U = U_star - c * _grad(solver, P) / M
        if dm is not None:
            U[dm] = U_d_full[dm]
        fctx.solver, fctx.k, fctx.c, fctx.tol = solver, k, c, tol
        return U, P

    @staticmethod
    def backward(fctx, gU, gP):
        solver, k, c, tol = fctx.solver, fctx.k, fctx.c, fctx.tol
        ctx, pm, dm = _solver_masks(solver)
        M = ctx.element_data()[6]
        gU = (gU if gU is not None else torch.zeros(solver.ndim * solver.nn, dtype=torch.float64,
                                                     device=M.device)).contiguous().clone()
        if dm is not None:
            gU[dm] = 0.0
        w = (gP.contiguous().clone() if gP is not None else torch.zeros(solver.nn, dtype=torch.float64,
                                                                        device=M.device))
        w = w - c * _div(solver, (gU / M).contiguous())
        w[pm] = 0.0
        lam = _pressure(solver, w, tol)
        return gU + k * _grad(solver, lam), None, None, None, None, None, None
