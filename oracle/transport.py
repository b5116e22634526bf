"""NS step followed by a Crank-Nicolson (SUPG) advection-diffusion step for a
passive scalar (oracle restatement of solvers/passive_transport.py).
Test infrastructure only."""
import numpy as np

from . import element as ecalc
from . import emult
from . import standard
from .solvers import bicgstab


def _dirichlet(rhs, x, gamma, val):
    rhs = rhs.copy()
    rhs[gamma] = val
    x0 = x.copy()
    x0[gamma] = val
    return rhs, x0


def update_phi_SUPG(phi_n, nconn, Mtau_all_n, Ctau_all_n, Me, Ce_all, Ce_all_n, Le, D, dt, nn,
                    gamma_d_phi, phi_d, tol):
    """solvers/passive_transport.py:14-36."""
    mask = None
    if gamma_d_phi is not None:
        mask = np.zeros(nn, dtype=bool)
        mask[gamma_d_phi] = True

    def lhs(phi):
        res = ((1 / dt) * emult.scalar_consistent_mass_SUPG_mult(phi, Mtau_all_n, Me, nconn, nn)
               + 0.5 * emult.scalar_stabilized_visc_conv_mult(phi, Ce_all, Ctau_all_n, Le, D, nconn, nn))
        return np.where(mask, phi, res) if mask is not None else res

    rhs = ((1 / dt) * emult.scalar_consistent_mass_SUPG_mult(phi_n, Mtau_all_n, Me, nconn, nn)
           - 0.5 * emult.scalar_stabilized_visc_conv_mult(phi_n, Ce_all_n, Ctau_all_n, Le, D, nconn, nn))
    x0 = phi_n
    if gamma_d_phi is not None:
        rhs, x0 = _dirichlet(rhs, phi_n, gamma_d_phi, phi_d)
    return bicgstab(lhs, rhs, x0=x0, tol=tol)


def update_phi(phi_n, nconn, Me, Ce_all, Ce_all_n, Le, D, dt, nn, gamma_d_phi, phi_d, tol):
    """solvers/passive_transport.py:39-61."""
    mask = None
    if gamma_d_phi is not None:
        mask = np.zeros(nn, dtype=bool)
        mask[gamma_d_phi] = True

    def lhs(phi):
        res = ((1 / dt) * emult.consistent_mass_mult(phi, Me, nconn, nn, 1)
               + 0.5 * emult.scalar_visc_conv_mult(phi, Ce_all, Le, D, nconn, nn))
        return np.where(mask, phi, res) if mask is not None else res

    rhs = ((1 / dt) * emult.consistent_mass_mult(phi_n, Me, nconn, nn, 1)
           - 0.5 * emult.scalar_visc_conv_mult(phi_n, Ce_all_n, Le, D, nconn, nn))
    x0 = phi_n
    if gamma_d_phi is not None:
        rhs, x0 = _dirichlet(rhs, phi_n, gamma_d_phi, phi_d)
    return bicgstab(lhs, rhs, x0=x0, tol=tol)


def timestep(U_n, P_n, M, Le, Ge, rho, mu, dt, nconn, wq, N, Nderiv, gamma_d, U_d, gamma_p, F_p, nn, ndim,
             stab, p_precond, p_M_op, tol, set_zeroP, F, phi_n, gamma_d_phi, phi_d, D, Me, phi_S_func,
             phi_SUPG):
    """solvers/passive_transport.py:64-97."""
    Ce_n = ecalc.conservative_convec_elem_calc(nconn, U_n, wq, N, Nderiv, nn, ndim, 0.5)
    U_hat, U_iters = standard.solve_momentum(U_n, P_n, Me, Le, Ge, Ce_n, rho, mu, dt, nconn, nn, ndim,
                                             gamma_d, U_d, F, tol, 0.5, 1)
    U_star = U_hat + ((dt / rho) * emult.gradient_element_mult(P_n, Ge, nconn, nn, ndim) / M)
    P, P_iters = standard.solve_pressure(U_star, P_n, Le, Ge, rho, dt, nconn, nn, ndim, gamma_p, F_p,
                                         set_zeroP, p_precond, p_M_op, tol, gamma=0)
    U = U_star - ((dt / rho) * emult.gradient_element_mult(P, Ge, nconn, nn, ndim) / M)
    if gamma_d is not None:
        U = U.copy()
        U[gamma_d] = U_d
    Ce1_n = ecalc.conservative_convec_elem_calc(nconn, U_n, wq, N, Nderiv, nn, ndim, 1)
    Ce1 = ecalc.conservative_convec_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim, 1)
    if phi_SUPG:
        Ct_n = ecalc.Ctau_tilde_elem_calc(nconn, U_n, wq, N, Nderiv, nn, ndim)
        tau_n = ecalc.calculate_tau(nconn, U_n, Ce1, Ct_n, N, nn, ndim, D, dt, r=2)
        Ctau = tau_n[:, None, None] * Ct_n
        Mtau = tau_n[:, None, None] * Ce1_n.transpose(0, 2, 1)
        phi, phi_iters = update_phi_SUPG(phi_n, nconn, Mtau, Ctau, Me, Ce1, Ce1_n, Le, D, dt, nn,
                                         gamma_d_phi, phi_d, tol)
    else:
        phi, phi_iters = update_phi(phi_n, nconn, Me, Ce1, Ce1_n, Le, D, dt, nn, gamma_d_phi, phi_d, tol)
    return U, P, phi, U_iters, P_iters, phi_iters


def setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, gamma_d_phi, mesh_func, config):
    """solvers/passive_transport.py:100-180."""
    mc = config.mesh_config
    ns, ade = config.solver_config.NS_config, config.solver_config.ADE_config
    ndim = len(mc.num_elem)
    shape_func, boundary_shapefunc = standard.shape_funcs_for(ndim, mc.shape_func_ord)
    wq, N, Nderiv = shape_func(node_coords[nconn[0]])
    M, Me = ecalc.lumped_mass_matrix(nconn, wq, N, nn, ndim)
    Le = ecalc.laplacian_element_calc(wq, Nderiv)
    Ge = ecalc.gradient_element_calc(wq, N, Nderiv, ndim)
    if ns.pressure_precond == "approx_inv":
        L_diag = ecalc.laplacian_diag(Le, nconn, nn)

        def M_op(r, nconn):
            # passive_transport.py:147-149 keeps the D1x / D1L values on gamma_p
            D1x = r / L_diag
            D1L = emult.laplacian_element_mult(D1x, Le, nconn, nn) / L_diag
            D1L[gamma_p] = D1x[gamma_p]
            t = emult.laplacian_element_mult(D1L, Le, nconn, nn)
            t[gamma_p] = D1L[gamma_p]
            return 3 * D1x - 3 * D1L + t / L_diag
    else:
        M_op = standard.make_pressure_M_op(ns, mc, Le, nconn, nn, gamma_p, mesh_func, shape_func)

    def compute_loaded(U_d, S_func, t_n, t):
        return standard.compute(node_coords, bconn, nvec, boundary_shapefunc, gamma_d, U_d, nn, ndim, S_func,
                                Me, nconn, t_n, t)

    def timestep_loaded(U_n, P_n, phi_n, dt, rho, mu, D, U_d, phi_d, F_p, F, phi_S_func):
        return timestep(U_n, P_n, M, Le, Ge, rho, mu, dt, nconn, wq, N, Nderiv, gamma_d, U_d, gamma_p, F_p,
                        nn, ndim, ns.streamline_diff, ns.pressure_precond, M_op, ns.solver_tol, ns.set_zeroP, F,
                        phi_n, gamma_d_phi, phi_d, D, Me, phi_S_func, ade.phi_SUPG)

    return compute_loaded, timestep_loaded
