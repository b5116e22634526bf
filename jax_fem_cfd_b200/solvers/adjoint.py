"""Adjoints of the two linear stages of the 4-step time step: the pressure
projection and the momentum solve (for a fixed convection operator).

The projection (solvers/standard.py:156-163, steps 5-7 of fem_step4) maps the
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

`Projection` puts this behind torch.autograd (the analogue of jax.custom_vjp);
pinned pressure (set_zeroP) only.

`MomentumSolve` is the momentum solve of solvers/standard.py:14-43 for a fixed
operator A = (rho/dt) Me + theta (rho Ce(U_n) + mu Le) with identity rows on
gamma_d (A_m = P_f A + P_d), as a function of its right-hand side. Its reverse
is the adjoint solve A_m^T lam = g: A^T = (rho/dt) Me + theta (rho Ce^T + mu Le)
(Me, Le symmetric, Ce^T element by element), and the identity rows become
identity columns, so lam_f solves the masked transposed system with rhs
(g_f, 0) and lam_d = g_d - (A^T lam_f)_d. The dependence of Ce on U_n (the
linearisation of convection) enters through `Step`, below; the transport
adjoint is not built. No reference counterpart: the
reference differentiates with jax.grad.

`rollout` chains Steps with checkpoints every `ckpt` steps (recomputation in
the backward pass). `Step` is one whole 4-step time step (U_n, P_n) -> (U_{n+1}, P_{n+1}) of a
wall-bounded pinned-pressure problem (solvers/standard.py:148-165, theta = 1/2,
Ce(U_n) with beta = 1/2, F = 0, F_p = 0): the rhs
(rho/dt) Me U_n - (1 - theta)(rho Ce(U_n) + mu Le) U_n - G P_n (U_d on gamma_d),
the momentum solve, U* = U_hat + (dt/rho) G P_n / M, the projection. Its
reverse chains the adjoints above with the velocity side of the convection
operator: Ce(U) is linear in U, and d/dU <a, Ce(U) b> (conv_vjp_u) is a sum
over elements and Gauss points of w A_c (N_k d_d B_c + beta d_d N_k B_c), where
A_c, B_c are a_c, b_c interpolated at the Gauss point.
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


def _ebe(solver, x, alpha, A, beta=0.0, B=None, transB=0):
    """(alpha A + beta B_e) x per velocity component (fem_ebe_apply)."""
    y = torch.empty_like(x)
    _lib.call("fem_ebe_apply", solver.ctx.handle, solver.ndim, ptr(x), ptr(y), float(alpha), ptr(A), float(beta),
              ptr(B), int(transB), 0.0, None, stream())
    return y


def conv_vjp_u(solver, nconn, a, b, beta):
    """d/dU <a, Ce(U) b> (a, b: ndim*nn vectors, Ce acting on each component)."""
    wq, N, Nd = solver.ctx.element_data()[:3]
    nd, nn = solver.ndim, solver.nn
    w = wq.reshape(-1)
    ae = a.view(nd, nn)[:, nconn]  # (c, e, i)
    be = b.view(nd, nn)[:, nconn]
    A = torch.einsum("qi,cei->ceq", N, ae)
    B = torch.einsum("qi,cei->ceq", N, be)
    dB = torch.einsum("qdi,cei->ceqd", Nd, be)
    s_ = torch.einsum("ceq,ceqd->eqd", A, dB)
    t_ = torch.einsum("ceq,ceq->eq", A, B)
    ge = torch.einsum("q,qk,eqd->edk", w, N, s_) + beta * torch.einsum("q,qdk,eq->edk", w, Nd, t_)
    out = torch.zeros(nd, nn, dtype=torch.float64, device=a.device)
    idx = nconn.reshape(-1)
    for d in range(nd):
        out[d].index_add_(0, idx, ge[:, d, :].reshape(-1))
    return out.reshape(-1)


def _bicgstab(solver, Ksh, beta, B, mask, rhs, tol):
    ctx = solver.ctx
    x = torch.zeros_like(rhs)
    it = torch.zeros(1, dtype=torch.int32, device=rhs.device)
    st = torch.zeros(1, dtype=torch.int32, device=rhs.device)
    _lib.call("fem_bicgstab_solve", ctx.handle, solver.ndim, 1.0, ptr(Ksh), float(beta), ptr(B), 0.0, None, ptr(mask),
              ptr(rhs), ptr(x), float(tol), 0.0, 0, ptr(it), ptr(st), stream())
    if int(st.item()) != 0:
        raise _lib.FemError(f"BiCGSTAB status {int(st.item())}")
    return x


class MomentumSolve(torch.autograd.Function):
    """rhs -> U_hat = A_m^-1 rhs for a fixed Ce(U_n); backward is the adjoint solve."""

    @staticmethod
    def forward(fctx, rhs, solver, Ce_all, rho, mu, dt, theta=0.5, tol=1e-13):
        ctx = solver.ctx
        Me, Le = ctx.element_data()[3], ctx.element_data()[4]
        Ksh = ((rho / dt) * Me + (theta * mu) * Le).reshape(-1).contiguous()
        Ce = Ce_all.to(torch.float64).contiguous()
        x = _bicgstab(solver, Ksh, theta * rho, Ce, solver.dmask, rhs.detach().to(torch.float64).contiguous(), tol)
        fctx.solver, fctx.Ksh, fctx.Ce, fctx.beta, fctx.tol = solver, Ksh, Ce, theta * rho, tol
        return x

    @staticmethod
    def backward(fctx, g):
        solver, Ksh, Ce, beta, tol = fctx.solver, fctx.Ksh, fctx.Ce, fctx.beta, fctx.tol
        nen = int(round(Ksh.numel() ** 0.5))
        CeT = Ce.reshape(-1, nen, nen).transpose(1, 2).contiguous()
        g = g.contiguous()
        dm = solver.dmask.to(torch.bool) if solver.dmask is not None else None
        b = g.clone()
        if dm is not None:
            b[dm] = 0.0
        lam = _bicgstab(solver, Ksh, beta, CeT, solver.dmask, b, tol)
        if dm is not None:
            y = torch.empty_like(lam)
            _lib.call("fem_ebe_apply", solver.ctx.handle, solver.ndim, ptr(lam), ptr(y), 1.0, ptr(Ksh), float(beta),
                      ptr(CeT), 0, 0.0, None, stream())
            lam[dm] = g[dm] - y[dm]
        return lam, None, None, None, None, None, None, None


def _projection_vjp(solver, gU, gP, k, c, tol):
    ctx, pm, dm = _solver_masks(solver)
    M = ctx.element_data()[6]
    gU = gU.contiguous().clone()
    if dm is not None:
        gU[dm] = 0.0
    w = gP.contiguous().clone() - c * _div(solver, (gU / M).contiguous())
    w[pm] = 0.0
    return gU + k * _grad(solver, _pressure(solver, w, tol))


class Step(torch.autograd.Function):
    """(U_n, P_n) -> (U_{n+1}, P_{n+1}) of one 4-step time step; backward is its adjoint."""

    @staticmethod
    def forward(fctx, U_n, P_n, solver, nconn, dt, rho, mu, U_d_full, tol=1e-13):
        if not solver.cfg.set_zeroP:
            raise ValueError("Step covers the pinned-pressure (set_zeroP) form only")
        theta, beta = 0.5, 0.5
        ctx, pm, dm = _solver_masks(solver)
        Me, Le, M = ctx.element_data()[3].reshape(-1), ctx.element_data()[4].reshape(-1), ctx.element_data()[6]
        Un = U_n.detach().to(torch.float64).contiguous()
        Pn = P_n.detach().to(torch.float64).contiguous()
        Ce = torch.empty(solver.ctx.ne * Me.numel(), dtype=torch.float64, device=Un.device)
        _lib.call("fem_convection_build", ctx.handle, ptr(Un), beta, None, None, None, ptr(Ce), stream())
        rhs = (_ebe(solver, Un, rho / dt, Me) - (1 - theta) * _ebe(solver, Un, mu, Le, rho, Ce)
               - _grad(solver, Pn))
        if dm is not None:
            rhs[dm] = U_d_full[dm]
        Ksh = ((rho / dt) * Me + (theta * mu) * Le).contiguous()
        Uh = _bicgstab(solver, Ksh, theta * rho, Ce, solver.dmask, rhs, tol)
        c, k = dt / rho, rho / dt
        Us = Uh + c * _grad(solver, Pn) / M
        P = _pressure(solver, k * _div(solver, Us), tol)
        U = Us - c * _grad(solver, P) / M
        if dm is not None:
            U[dm] = U_d_full[dm]
        fctx.save = (solver, nconn, Un, Ce, Ksh, Uh, dt, rho, mu, tol)
        return U, P

    @staticmethod
    def backward(fctx, gU, gP):
        solver, nconn, Un, Ce, Ksh, Uh, dt, rho, mu, tol = fctx.save
        theta, beta = 0.5, 0.5
        ctx, pm, dm = _solver_masks(solver)
        Me, Le, M = ctx.element_data()[3].reshape(-1), ctx.element_data()[4].reshape(-1), ctx.element_data()[6]
        nd, nn = solver.ndim, solver.nn
        c, k = dt / rho, rho / dt
        gU = gU if gU is not None else torch.zeros(nd * nn, dtype=torch.float64, device=Un.device)
        gP = gP if gP is not None else torch.zeros(nn, dtype=torch.float64, device=Un.device)
        gUs = _projection_vjp(solver, gU, gP, k, c, tol)            # through the projection
        gPn = c * _div(solver, (gUs / M).contiguous())              # U* = U_hat + c G P_n / M
        # the adjoint momentum solve (identity rows become identity columns)
        nen = int(round(Ksh.numel() ** 0.5))
        CeT = Ce.view(-1, nen, nen).transpose(1, 2).contiguous()
        b = gUs.clone()
        if dm is not None:
            b[dm] = 0.0
        lam = _bicgstab(solver, Ksh, theta * rho, CeT, solver.dmask, b, tol)  # = lam_f (0 on gamma_d)
        # rhs = (rho/dt) Me U_n - (1 - theta)(rho Ce(U_n) + mu Le) U_n - G P_n, U_d on gamma_d
        gUn = (_ebe(solver, lam, rho / dt, Me) - (1 - theta) * _ebe(solver, lam, mu, Le, rho, Ce, 1)
               - (1 - theta) * rho * conv_vjp_u(solver, nconn, lam, Un, beta))
        gPn = gPn - _div(solver, lam)
        # the operator's dependence on U_n: U_hat = A(U_n)^-1 rhs, dA = theta rho Ce(dU) on the free rows
        gUn = gUn - theta * rho * conv_vjp_u(solver, nconn, lam, Uh, beta)
        return gUn, gPn, None, None, None, None, None, None, None


def rollout(solver, nconn, U0, P0, steps, dt, rho, mu, U_d_full, ckpt=10, tol=1e-13):
    """`steps` time steps of Step from (U0, P0), differentiable end to end. With
    gradients enabled and ckpt > 0, every chunk of `ckpt` steps is a checkpoint
    (torch.utils.checkpoint): only the chunk boundaries are kept, and a chunk's
    steps are recomputed when the backward pass reaches it."""
    from torch.utils.checkpoint import checkpoint

    def chunk(u, p, n):
        for _ in range(n):
            u, p = Step.apply(u, p, solver, nconn, dt, rho, mu, U_d_full, tol)
        return u, p

    u, p = U0, P0
    done = 0
    while done < steps:
        n = min(ckpt, steps - done) if ckpt > 0 else steps - done
        if ckpt > 0 and torch.is_grad_enabled():
            u, p = checkpoint(chunk, u, p, n, use_reentrant=False)
        else:
            u, p = chunk(u, p, n)
        done += n
    return u, p
