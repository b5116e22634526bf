"""Element-by-element matvecs (drop-in for core/element_mult.py).

Each call is one node-centric libfemb200 kernel over the structured mesh of
``nconn`` (implicit connectivity, deterministic summation, no atomics)."""
from .. import _lib
from ..context import context_for, empty, f64, ptr, stream
from ..setup.regular_mesh import mesh_of


def _ebe(x, nconn, nn, ncomp, alpha, A, beta=0.0, B=None, transB=0, gamma=0.0, C=None):
    ctx = context_for(mesh_of(nconn, nn))
    xs = f64(x)
    y = empty(ncomp * ctx.nn)
    _lib.call("fem_ebe_apply", ctx.handle, int(ncomp), ptr(xs), ptr(y), float(alpha),
              ptr(f64(A)) if A is not None else None, float(beta), ptr(f64(B)) if B is not None else None,
              int(transB), float(gamma), ptr(f64(C)) if C is not None else None, stream())
    return y


def consistent_mass_mult(S, Me, nconn, nn, ndim):
    """core/element_mult.py:11: M S per component (3D supported; the reference's
    ndim == 3 branch raises NameError at :26)."""
    return _ebe(S, nconn, nn, ndim, 1.0, Me)


def laplacian_element_mult(P, Le, nconn, nn):
    """core/element_mult.py:38."""
    return _ebe(P, nconn, nn, 1, 1.0, Le)


def gradient_element_mult(P, Ge, nconn, nn, ndim):
    """core/element_mult.py:51: [G_1 P; ...; G_ndim P]."""
    ctx = context_for(mesh_of(nconn, nn))
    y = empty(ndim * ctx.nn)
    _lib.call("fem_grad_apply", ctx.handle, ptr(f64(P)), ptr(f64(Ge)), ptr(y), stream())
    return y


def divergence_element_mult(U, Ge, nconn, nn, ndim):
    """core/element_mult.py:133: sum_i G_i^T u_i."""
    ctx = context_for(mesh_of(nconn, nn))
    y = empty(ctx.nn)
    _lib.call("fem_div_apply", ctx.handle, ptr(f64(U)), ptr(f64(Ge)), ptr(y), stream())
    return y


def visc_conv_mult(U, Ce_all, Le, mu, rho, nconn, nn, ndim):
    """core/element_mult.py:79: (rho Ce_e + mu Le) u_c."""
    return _ebe(U, nconn, nn, ndim, mu, Le, rho, Ce_all)


def stabilized_visc_conv_mult(U, Ce_all, Se_all, Le, mu, rho, nconn, nn, ndim):
    """core/element_mult.py:106: (rho Ce_e + mu Le + Se_e) u_c."""
    return _ebe(U, nconn, nn, ndim, mu, Le, rho, Ce_all, 0, 1.0, Se_all)


def scalar_visc_conv_mult(phi, Ce_all, Le, D, nconn, nn):
    """core/element_mult.py:159: (Ce_e + D Le) phi."""
    return _ebe(phi, nconn, nn, 1, D, Le, 1.0, Ce_all)


def scalar_stabilized_visc_conv_mult(phi, Ce_all, Se_all, Le, D, nconn, nn):
    """core/element_mult.py:174: (Ce_e + D Le + Se_e) phi."""
    return _ebe(phi, nconn, nn, 1, D, Le, 1.0, Ce_all, 0, 1.0, Se_all)


def scalar_consistent_mass_SUPG_mult(phi, Me_tau_all, Me, nconn, nn):
    """core/element_mult.py:190: (Me + Me_tau_e) phi."""
    return _ebe(phi, nconn, nn, 1, 1.0, Me, 1.0, Me_tau_all)
