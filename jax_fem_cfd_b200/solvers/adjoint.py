"""Adjoints of the two linear stages of the 4-step time step: the pressure
projection and the momentum solve (for a fixed convection operator).

The projection (solvers/standard.py:156-163, steps 5-7 of fem_step4) maps the
intermediate velocity U* to

    P = A+ k (D U* - F_p)                   k = rho / dt, A+ the pinned pressure solve
    U = U* - c M^-1 G P,  U = U_d on gamma_d     c = dt / rho, M the lumped mass

with D = G^T (divergence_element_mult is sum_i G_i^T u_i, gradient_element_mult
is [G_1 p; ...]). A+ solves A P = rhs with the gamma_p rows of A and rhs
zeroed and P = 0 on gamma_p (set_zeroP), or, for mean-zero pressure, is
C S C with C = I - 1 1^T / n the centring and S the solve on the mean-zero
subspace; both are symmetric. The stage is affine in U*, and its reverse
(vector-Jacobian product) for output gradients (g_U, g_P) is

    g_U' = g_U with gamma_d rows zeroed
    w    = g_P - c D (M^-1 g_U'),  w = 0 on gamma_p (pinned)
    lam  = A+ w                     (the adjoint solve: the same MG-PCG)
    g_U* = g_U' + k G lam

`Projection` puts this behind torch.autograd (the analogue of jax.custom_vjp).

`MomentumSolve` is the momentum solve of solvers/standard.py:14-43 for a fixed
operator A = (rho/dt) Me + theta (rho Ce(U_n) + mu Le) with identity rows on
gamma_d (A_m = P_f A + P_d), as a function of its right-hand side. Its reverse
is the adjoint solve A_m^T lam = g: A^T = (rho/dt) Me + theta (rho Ce^T + mu Le)
(Me, Le symmetric, Ce^T element by element), and the identity rows become
identity columns, so lam_f solves the masked transposed system with rhs
(g_f, 0) and lam_d = g_d - (A^T lam_f)_d. The dependence of Ce on U_n (the
linearisation of convection) enters through `Step`, below, and the passive
scalar's step through `Transport`. No reference counterpart: the reference
differentiates with jax.grad.

`rollout` chains Steps with checkpoints every `ckpt` steps (recomputation in
the backward pass). `Step` is one whole 4-step time step (U_n, P_n) -> (U_{n+1}, P_{n+1}) of a
wall-bounded pinned-pressure or a periodic mean-zero problem (solvers/standard.py:148-165, theta = 1/2,
Ce(U_n) with beta = 1/2, F = 0, F_p = 0): the rhs
(rho/dt) Me U_n - (1 - theta)(rho Ce(U_n) + mu Le) U_n - G P_n (U_d on gamma_d),
the momentum solve, U* = U_hat + (dt/rho) G P_n / M, the projection. Its
reverse chains the adjoints above with the velocity side of the convection
operator: Ce(U) is linear in U, and d/dU <a, Ce(U) b> (conv_vjp_u) is a sum
over elements and Gauss points of w A_c (N_k d_d B_c + beta d_d N_k B_c), where
A_c, B_c are a_c, b_c interpolated at the Gauss point.
"""
import contextlib

import torch

from .. import _lib
from ..context import ptr, stream

# Device int32 flags of the open deferred_status blocks. Process-wide, not per
# thread: the autograd engine runs the backward functions of CUDA tensors on its
# own device thread, which has to see the flag of the block around backward().
# So deferred blocks are for one thread at a time.
_DEFERRED = []


@contextlib.contextmanager
def deferred_status():
    """Inside the block, the solves here do not read their status back on the
    host after each call (which waits for the device). Each status is folded
    into one device flag instead, read once when the block ends, and a failure
    anywhere inside raises FemError then. Blocks nest; they are process-wide
    (see _DEFERRED), so only one thread at a time may use them."""
    flag = torch.zeros(1, dtype=torch.int32, device=torch.device("cuda", torch.cuda.current_device()))
    _DEFERRED.append(flag)
    try:
        yield
    finally:
        _DEFERRED.pop()
    if int(flag.item()) != 0:
        raise _lib.FemError("a solve inside the deferred-status block failed (status flags "
                            f"{int(flag.item()):#x})")


def _check(st, what):
    if _DEFERRED:
        _DEFERRED[-1].bitwise_or_(st[:1])
    elif int(st.item()) != 0:
        raise _lib.FemError(f"{what} status {int(st.item())}")


def _solver_masks(solver):
    ctx = solver.ctx
    pm = solver.pmask.to(torch.bool)
    dm = solver.dmask.to(torch.bool) if solver.dmask is not None else None
    return ctx, pm, dm


def _pressure(solver, rhs, tol):
    """A+ rhs: the pressure solve of the solver's context from 0. Pinned
    (set_zeroP): gamma_p rows of rhs zeroed and P = 0 there. Mean-zero: rhs
    centred, the solve on the mean-zero subspace and P centred
    (solvers/standard.py:104-125), i.e. P = C S C rhs with C = I - 1 1^T / n."""
    ctx, pm, _ = _solver_masks(solver)
    pinned = bool(solver.cfg.set_zeroP)
    r = rhs.clone()
    if pinned:
        r.masked_fill_(pm, 0.0)
    x = torch.zeros_like(r)
    it = torch.zeros(1, dtype=torch.int32, device=r.device)
    st = torch.zeros(1, dtype=torch.int32, device=r.device)
    _lib.call("fem_pressure_solve", ctx.handle, ptr(r), ptr(x), float(tol), 0.0, 1000, solver.precond,
              0 if pinned else 1, 1, ptr(it), ptr(st), stream())
    _check(st, "pressure solve")
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
        ctx, pm, dm = _solver_masks(solver)
        M = ctx.element_data()[6]
        k, c = rho / dt, dt / rho
        U_star = U_star.detach().to(torch.float64).contiguous()
        rhs = k * (_div(solver, U_star) - (F_p if F_p is not None else 0.0))
        P = _pressure(solver, rhs, tol)
        U = U_star - c * _grad(solver, P) / M
        if dm is not None:
            U = torch.where(dm, U_d_full, U)
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
            gU.masked_fill_(dm, 0.0)
        w = (gP.contiguous().clone() if gP is not None else torch.zeros(solver.nn, dtype=torch.float64,
                                                                        device=M.device))
        w = w - c * _div(solver, (gU / M).contiguous())
        if solver.cfg.set_zeroP:
            w.masked_fill_(pm, 0.0)
        lam = _pressure(solver, w, tol)
        return gU + k * _grad(solver, lam), None, None, None, None, None, None


def _ebe(solver, x, alpha, A, beta=0.0, B=None, transB=0, ncomp=None):
    """(alpha A + beta B_e) x per component (fem_ebe_apply); ncomp defaults to the
    velocity's."""
    y = torch.empty_like(x)
    _lib.call("fem_ebe_apply", solver.ctx.handle, ncomp or solver.ndim, ptr(x), ptr(y), float(alpha), ptr(A),
              float(beta), ptr(B), int(transB), 0.0, None, stream())
    return y


def conv_vjp_u(solver, nconn, a, b, beta):
    """d/dU <a, Ce(U) b> (a, b: ndim*nn vectors, Ce acting on each component),
    by fem_conv_vjp."""
    a, b = a.detach().contiguous(), b.detach().contiguous()
    y = torch.empty(solver.ndim * solver.nn, dtype=torch.float64, device=a.device)
    _lib.call("fem_conv_vjp", solver.ctx.handle, solver.ndim, ptr(a), ptr(b), float(beta), ptr(y), stream())
    return y


def _bicgstab(solver, Ksh, beta, B, mask, rhs, tol, ncomp=None):
    ctx = solver.ctx
    x = torch.zeros_like(rhs)
    it = torch.zeros(1, dtype=torch.int32, device=rhs.device)
    st = torch.zeros(1, dtype=torch.int32, device=rhs.device)
    _lib.call("fem_bicgstab_solve", ctx.handle, ncomp or solver.ndim, 1.0, ptr(Ksh), float(beta), ptr(B), 0.0, None,
              ptr(mask), ptr(rhs), ptr(x), float(tol), 0.0, 0, ptr(it), ptr(st), stream())
    _check(st, "BiCGSTAB")
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
            b.masked_fill_(dm, 0.0)
        lam = _bicgstab(solver, Ksh, beta, CeT, solver.dmask, b, tol)
        if dm is not None:
            y = torch.empty_like(lam)
            _lib.call("fem_ebe_apply", solver.ctx.handle, solver.ndim, ptr(lam), ptr(y), 1.0, ptr(Ksh), float(beta),
                      ptr(CeT), 0, 0.0, None, stream())
            lam = torch.where(dm, g - y, lam)
        return lam, None, None, None, None, None, None, None


def _projection_vjp(solver, gU, gP, k, c, tol):
    ctx, pm, dm = _solver_masks(solver)
    M = ctx.element_data()[6]
    gU = gU.contiguous().clone()
    if dm is not None:
        gU.masked_fill_(dm, 0.0)
    w = gP.contiguous().clone() - c * _div(solver, (gU / M).contiguous())
    if solver.cfg.set_zeroP:
        w.masked_fill_(pm, 0.0)
    return gU + k * _grad(solver, _pressure(solver, w, tol))


class Step(torch.autograd.Function):
    """(U_n, P_n) -> (U_{n+1}, P_{n+1}) of one 4-step time step; backward is its adjoint."""

    @staticmethod
    def forward(fctx, U_n, P_n, solver, nconn, dt, rho, mu, U_d_full, tol=1e-13):
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
            rhs = torch.where(dm, U_d_full, rhs)
        Ksh = ((rho / dt) * Me + (theta * mu) * Le).contiguous()
        Uh = _bicgstab(solver, Ksh, theta * rho, Ce, solver.dmask, rhs, tol)
        c, k = dt / rho, rho / dt
        Us = Uh + c * _grad(solver, Pn) / M
        P = _pressure(solver, k * _div(solver, Us), tol)
        U = Us - c * _grad(solver, P) / M
        if dm is not None:
            U = torch.where(dm, U_d_full, U)
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
            b.masked_fill_(dm, 0.0)
        lam = _bicgstab(solver, Ksh, theta * rho, CeT, solver.dmask, b, tol)  # = lam_f (0 on gamma_d)
        # rhs = (rho/dt) Me U_n - (1 - theta)(rho Ce(U_n) + mu Le) U_n - G P_n, U_d on gamma_d
        gUn = (_ebe(solver, lam, rho / dt, Me) - (1 - theta) * _ebe(solver, lam, mu, Le, rho, Ce, 1)
               - (1 - theta) * rho * conv_vjp_u(solver, nconn, lam, Un, beta))
        gPn = gPn - _div(solver, lam)
        # the operator's dependence on U_n: U_hat = A(U_n)^-1 rhs, dA = theta rho Ce(dU) on the free rows
        gUn = gUn - theta * rho * conv_vjp_u(solver, nconn, lam, Uh, beta)
        return gUn, gPn, None, None, None, None, None, None, None


def transport_elements(solver, Un, U, dt, D, supg, transpose=False):
    """(E_k, B_k), (ne, nen, nen) each: the per-element parts of the transport
    step's operators (solvers/passive_transport.py:14-62 with the matrices of
    :80-88), built on the device by fem_transport_elements. The lhs is
    A = K_A + E_k and the rhs operator B = K_B + B_k, with the shared
    K_A = Me/dt + (D/2) Le and K_B = Me/dt - (D/2) Le. With SUPG:
        E_k = Mtau/dt + (Ce(U) + Ctau)/2,   B_k = Mtau/dt - (Ce(U_n) + Ctau)/2,
        Ctau = tau Ct(U_n),  Mtau = tau Ce(U_n)^T,  tau = tau(U_n, Ce(U), Ct(U_n)),
    without it E_k = Ce(U)/2 and B_k = -Ce(U_n)/2; Ce has beta = 1
    (core/element_calc.py:165-185), Ct = sum_q w dN^T (u u^T) dN (:188-200),
    tau the r = 2 blend of :202-229. transpose=True returns each block
    transposed."""
    ctx = solver.ctx
    nen = ctx.element_data()[3].shape[-1]
    Un, U = (t.detach().to(torch.float64).contiguous() for t in (Un, U))
    Ek = torch.empty(ctx.ne, nen, nen, dtype=torch.float64, device=Un.device)
    Bk = torch.empty_like(Ek)
    _lib.call("fem_transport_elements", ctx.handle, ptr(Un), ptr(U), float(dt), float(D), int(bool(supg)),
              int(bool(transpose)), ptr(Ek), ptr(Bk), stream())
    return Ek, Bk


def transport_vjp(solver, Un, U, lam, phin, phi, dt, D, supg):
    """(d/dU_n, d/dU) of <lam, B(U_n) phi_n - A(U_n, U) phi> (the velocity
    dependence of Ce, Ctau, Mtau and tau in the operators of
    transport_elements) by the fem_transport_vjp kernels."""
    ctx = solver.ctx
    gUn, gU = torch.empty_like(Un), torch.empty_like(U)
    _lib.call("fem_transport_vjp", ctx.handle, ptr(Un), ptr(U), ptr(lam), ptr(phin), ptr(phi), float(dt), float(D),
              int(bool(supg)), ptr(gUn), ptr(gU), stream())
    return gUn, gU


class Transport(torch.autograd.Function):
    """(U_n, U, phi_n[, phi_d]) -> phi_{n+1}: the passive-scalar step of
    solvers/passive_transport.py:64-97 (fem_transport_phi); backward is its
    adjoint. phi solves A_m phi = r with A_m = P_f A + P_d (identity rows on
    gamma_d_phi), r_f = (B phi_n)_f, r_d = phi_d. For an output gradient g:
        A_m^T lam = g        (masked transposed BiCGSTAB, as in MomentumSolve)
        g_phi_n = B^T (P_f lam),   g_phi_d = lam on gamma_d_phi,
        g_U_n, g_U = d/dU <P_f lam, B(U_n, U) phi_n - A(U_n, U) phi>
    the transposed element matrices from fem_transport_elements and the last
    line from fem_transport_vjp (the shared parts of A and B do not depend on
    the velocity)."""

    @staticmethod
    def forward(fctx, U_n, U, phi_n, phid_full, solver, nconn, dt, D, supg=False, phi_mask=None, tol=1e-13):
        if (phi_mask is None) != (phid_full is None):
            raise ValueError("phi_mask and phid_full go together")
        ctx = solver.ctx
        Un, Uc, pn = (t.detach().to(torch.float64).contiguous() for t in (U_n, U, phi_n))
        pd = phid_full.detach().to(torch.float64).contiguous() if phid_full is not None else None
        phi = torch.empty_like(pn)
        it = torch.zeros(1, dtype=torch.int32, device=pn.device)
        st = torch.zeros(1, dtype=torch.int32, device=pn.device)
        _lib.call("fem_transport_phi", ctx.handle, ptr(Un), ptr(Uc), ptr(pn), float(dt), float(D), int(bool(supg)),
                  ptr(phi_mask), ptr(pd), float(tol), ptr(phi), ptr(it), ptr(st), stream())
        _check(st, "transport BiCGSTAB")
        fctx.save = (solver, nconn, Un, Uc, pn, phi, dt, D, supg, phi_mask, tol)
        return phi

    @staticmethod
    def backward(fctx, g):
        solver, nconn, Un, Uc, pn, phi, dt, D, supg, phi_mask, tol = fctx.save
        ctx = solver.ctx
        Me, Le = ctx.element_data()[3], ctx.element_data()[4]
        EkT, BkT = transport_elements(solver, Un, Uc, dt, D, supg, transpose=True)
        KA = (Me / dt + 0.5 * D * Le).reshape(-1).contiguous()
        KB = (Me / dt - 0.5 * D * Le).reshape(-1).contiguous()
        m = phi_mask.to(torch.bool) if phi_mask is not None else None
        g = g.contiguous()
        b = g.clone()
        if m is not None:
            b.masked_fill_(m, 0.0)
        lam = _bicgstab(solver, KA, 1.0, EkT, phi_mask, b, tol, ncomp=1)   # lam_f, 0 on gamma_d_phi
        g_phid = None
        if m is not None:
            lam_d = g - _ebe(solver, lam, 1.0, KA, 1.0, EkT, ncomp=1)
            g_phid = torch.where(m, lam_d, torch.zeros_like(lam_d))
        g_phin = _ebe(solver, lam, 1.0, KB, 1.0, BkT, ncomp=1)
        gUn, gU = transport_vjp(solver, Un, Uc, lam, pn, phi, dt, D, supg)
        return gUn, gU, g_phin, g_phid, None, None, None, None, None, None, None


def rollout(solver, nconn, U0, P0, steps, dt, rho, mu, U_d_full, ckpt=10, tol=1e-13, phi0=None, D=0.0, supg=False,
            phi_mask=None, phid_full=None):
    """`steps` time steps of Step from (U0, P0), differentiable end to end, and
    with phi0 given the passive scalar carried along by Transport (the order of
    solvers/passive_transport.py:64-97: the flow step, then phi from U_n and
    U_{n+1}); returns (U, P) or (U, P, phi). With gradients enabled and
    ckpt > 0, every chunk of `ckpt` steps is a checkpoint
    (torch.utils.checkpoint): only the chunk boundaries are kept, and a chunk's
    steps are recomputed when the backward pass reaches it."""
    from torch.utils.checkpoint import checkpoint

    def chunk(n, u, p, *phi):
        for _ in range(n):
            u1, p = Step.apply(u, p, solver, nconn, dt, rho, mu, U_d_full, tol)
            if phi:
                phi = (Transport.apply(u, u1, phi[0], phid_full, solver, nconn, dt, D, supg, phi_mask, tol),)
            u = u1
        return (u, p) + phi

    state = (U0, P0) + ((phi0,) if phi0 is not None else ())
    done = 0
    while done < steps:
        n = min(ckpt, steps - done) if ckpt > 0 else steps - done
        if ckpt > 0 and torch.is_grad_enabled():
            state = checkpoint(chunk, n, *state, use_reentrant=False)
        else:
            state = chunk(n, *state)
        done += n
    return state
