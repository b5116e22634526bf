"""Krylov solvers (oracle restatement of utils/jax_iterative_solvers.py).

Same loop conditions, initial values, breakdown codes and tolerance rule
``r.r <= max(tol^2 b.b, atol^2)`` as the reference's vendored JAX solvers.
Test infrastructure only."""
import numpy as np


def _vdot(x, y):
    return float(np.dot(x, y))


def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """utils/jax_iterative_solvers.py:87-120 (_cg_solve) via cg :214 / _isolve :174.

    Returns (x, iters). With M=None the loop condition uses gamma = r.z (z = r);
    otherwise it recomputes r.r (:97)."""
    if x0 is None:
        x0 = np.zeros_like(b)
    if maxiter is None:
        maxiter = 10 * b.size
    bs = _vdot(b, b)
    atol2 = max(tol ** 2 * bs, atol ** 2)
    prec = M if M is not None else (lambda r: r)
    x = x0.copy()
    r = b - A(x)
    z = prec(r)
    p = z
    gamma = _vdot(r, z)
    k = 0
    while True:
        rs = gamma if M is None else _vdot(r, r)
        if not (rs > atol2 and k < maxiter):
            break
        Ap = A(p)
        alpha = gamma / _vdot(p, Ap)
        x = x + alpha * p
        r = r - alpha * Ap
        z = prec(r)
        gamma_ = _vdot(r, z)
        beta = gamma_ / gamma
        p = z + beta * p
        gamma = gamma_
        k += 1
    return x, k


def bicgstab(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """utils/jax_iterative_solvers.py:123-167 (_bicgstab_solve) via bicgstab :685.

    Breakdown: iteration count -11 when omega or alpha is 0, -10 when rho is 0
    (:156-157); the loop stops on k < 0."""
    if x0 is None:
        x0 = np.zeros_like(b)
    if maxiter is None:
        maxiter = 10 * b.size
    prec = M if M is not None else (lambda r: r)
    bs = _vdot(b, b)
    atol2 = max(tol ** 2 * bs, atol ** 2)
    x = x0.copy()
    r = b - A(x)
    rhat = r
    alpha = omega = rho = 1.0
    p = q = r
    k = 0
    while _vdot(r, r) > atol2 and k < maxiter and k >= 0:
        rho_ = _vdot(rhat, r)
        beta = rho_ / rho * alpha / omega
        p = r + beta * (p - omega * q)
        phat = prec(p)
        q = A(phat)
        alpha = rho_ / _vdot(rhat, q)
        s = r - alpha * q
        exit_early = _vdot(s, s) < atol2
        shat = prec(s)
        t = A(shat)
        omega = _vdot(t, s) / _vdot(t, t)
        if exit_early:
            x = x + alpha * phat
            r = s
        else:
            x = x + (alpha * phat + omega * shat)
            r = s - omega * t
        k_ = -11 if (omega == 0 or alpha == 0) else k + 1
        k = -10 if rho_ == 0 else k_
        rho = rho_
    return x, k
