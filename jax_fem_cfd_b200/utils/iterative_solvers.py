"""CG and BiCGSTAB with the call signatures of jax_fem_cfd
utils/jax_iterative_solvers.py:214 cg and :685 bicgstab, for arbitrary matvec
callables on device tensors. The loop control is the reference's (tolerance
rule r.r <= max(tol^2 b.b, atol^2), PCG condition on r.r, BiCGSTAB breakdown
codes -10 / -11); vector updates and dot products are libfemb200 kernels with
the convergence test read back once per iteration. The solvers' own
time-step paths do not use these: they run the same loops device-resident in
one persistent launch each."""
import ctypes

import torch

from .. import _lib
from ..context import Context, Mesh, f64, ptr, stream

_BLAS = {}


def _handle():
    dev = torch.cuda.current_device()
    c = _BLAS.get(dev)
    if c is None:
        c = _BLAS[dev] = Context(Mesh(0, False, 1, 1))
    return c.handle


def _dot(x, y):
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    _lib.call("fem_dot", _handle(), ptr(x), ptr(y), int(x.numel()), ptr(out), stream())
    return out


def _axpby(a, x, b, y):
    _lib.call("fem_axpby", _handle(), float(a), ptr(x), float(b), ptr(y), int(y.numel()), stream())
    return y


def _lin(a, x, b, y):
    out = y.clone()
    return _axpby(a, x, b, out)


def cg(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """utils/jax_iterative_solvers.py:87-120 semantics; returns (x, iters)."""
    b = f64(b)
    x = torch.zeros_like(b) if x0 is None else f64(x0).clone()
    maxiter = 10 * b.numel() if maxiter is None else maxiter
    bs = float(_dot(b, b))
    atol2 = max(tol ** 2 * bs, atol ** 2)
    prec = (lambda r: r) if M is None else M
    r = _lin(-1.0, f64(A(x)), 1.0, b)
    z = f64(prec(r))
    p = z.clone()
    gamma = float(_dot(r, z))
    k = 0
    while True:
        rs = gamma if M is None else float(_dot(r, r))
        if not (rs > atol2 and k < maxiter):
            break
        Ap = f64(A(p))
        alpha = gamma / float(_dot(p, Ap))
        _axpby(alpha, p, 1.0, x)
        _axpby(-alpha, Ap, 1.0, r)
        z = f64(prec(r))
        gamma_ = float(_dot(r, z))
        beta = gamma_ / gamma
        p = _lin(1.0, z, beta, p)
        gamma = gamma_
        k += 1
    return x, k


def bicgstab(A, b, x0=None, *, tol=1e-5, atol=0.0, maxiter=None, M=None):
    """utils/jax_iterative_solvers.py:123-167 semantics; returns (x, k) with k
    negative on breakdown."""
    b = f64(b)
    x = torch.zeros_like(b) if x0 is None else f64(x0).clone()
    maxiter = 10 * b.numel() if maxiter is None else maxiter
    prec = (lambda v: v) if M is None else M
    bs = float(_dot(b, b))
    atol2 = max(tol ** 2 * bs, atol ** 2)
    r = _lin(-1.0, f64(A(x)), 1.0, b)
    rhat = r.clone()
    alpha = omega = rho = 1.0
    p, q = r.clone(), r.clone()
    k = 0
    while float(_dot(r, r)) > atol2 and k < maxiter and k >= 0:
        rho_ = float(_dot(rhat, r))
        beta = rho_ / rho * alpha / omega
        p = _lin(-omega, q, 1.0, p)
        p = _lin(1.0, r, beta, p)
        phat = f64(prec(p))
        q = f64(A(phat))
        alpha = rho_ / float(_dot(rhat, q))
        s = _lin(-alpha, q, 1.0, r)
        exit_early = float(_dot(s, s)) < atol2
        shat = f64(prec(s))
        t = f64(A(shat))
        omega = float(_dot(t, s)) / float(_dot(t, t))
        _axpby(alpha, phat, 1.0, x)
        if exit_early:
            r = s
        else:
            _axpby(omega, shat, 1.0, x)
            r = _lin(-omega, t, 1.0, s)
        k_ = -11 if (omega == 0 or alpha == 0) else k + 1
        k = -10 if rho_ == 0 else k_
        rho = rho_
    return x, k
