"""Element-by-element matvecs (oracle restatement of core/element_mult.py):
gather x[nconn] -> per-element dense product -> scatter-add in element order.
Test infrastructure only."""
import numpy as np

from .element import _assemble


def _shared(A, x, nconn, nn):
    return _assemble(np.einsum("ab,eb->ea", A, x[nconn]), nconn, nn)


def _per_elem(Ae, x, nconn, nn):
    return _assemble(np.einsum("eab,eb->ea", Ae, x[nconn]), nconn, nn)


def consistent_mass_mult(S, Me, nconn, nn, ndim):
    """core/element_mult.py:11-36. The ndim==3 branch of the reference raises
    NameError (y_result undefined, :26); the third component is build-defined."""
    return np.concatenate([_shared(Me, S[c * nn:(c + 1) * nn], nconn, nn) for c in range(ndim)])


def laplacian_element_mult(P, Le, nconn, nn):
    """core/element_mult.py:38-49: y = sum_e P_e^T Le P_e x."""
    return _shared(Le, P, nconn, nn)


def gradient_element_mult(P, Ge, nconn, nn, ndim):
    """core/element_mult.py:51-77: [G_1 P; ...; G_ndim P]."""
    return np.concatenate([_shared(Ge[i], P, nconn, nn) for i in range(ndim)])


def visc_conv_mult(U, Ce_all, Le, mu, rho, nconn, nn, ndim):
    """core/element_mult.py:79-104: (rho Ce_e + mu Le) u_c for each component c."""
    K = rho * Ce_all + (mu * Le)[None]
    return np.concatenate([_per_elem(K, U[c * nn:(c + 1) * nn], nconn, nn) for c in range(ndim)])


def stabilized_visc_conv_mult(U, Ce_all, Se_all, Le, mu, rho, nconn, nn, ndim):
    """core/element_mult.py:106-131."""
    K = rho * Ce_all + (mu * Le)[None] + Se_all
    return np.concatenate([_per_elem(K, U[c * nn:(c + 1) * nn], nconn, nn) for c in range(ndim)])


def divergence_element_mult(U, Ge, nconn, nn, ndim):
    """core/element_mult.py:133-157: sum_i Ge_i^T u_i."""
    out = _shared(Ge[0].T, U, nconn, nn)
    for i in range(1, ndim):
        out = out + _shared(Ge[i].T, U[i * nn:(i + 1) * nn], nconn, nn)
    return out


def scalar_visc_conv_mult(phi, Ce_all, Le, D, nconn, nn):
    """core/element_mult.py:159-172: (Ce_e + D Le) phi."""
    return _per_elem(Ce_all + (D * Le)[None], phi, nconn, nn)


def scalar_stabilized_visc_conv_mult(phi, Ce_all, Se_all, Le, D, nconn, nn):
    """core/element_mult.py:174-188: (Ce_e + D Le + Se_e) phi."""
    return _per_elem(Ce_all + (D * Le)[None] + Se_all, phi, nconn, nn)


def scalar_consistent_mass_SUPG_mult(phi, Me_tau_all, Me, nconn, nn):
    """core/element_mult.py:190-201: (Me + Me_tau_e) phi."""
    return _per_elem(Me[None] + Me_tau_all, phi, nconn, nn)
