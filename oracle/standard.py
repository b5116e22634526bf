"""Incompressible NS 4-step projection (oracle restatement of solvers/standard.py).
Test infrastructure only."""
from functools import partial

import numpy as np

from . import element as ecalc
from . import emult
from . import multigrid as mg
from . import shape as shapefunc
from .solvers import bicgstab, cg


def solve_momentum(U_n, P_n, Me, Le, Ge, Ce_all_n, rho, mu, dt, nconn, nn, ndim, gamma_d, U_d, F,
                   tol, theta, gamma):
    """solvers/standard.py:14-43: theta-scheme momentum solve, Dirichlet rows = identity."""
    mask = None
    if gamma_d is not None:
        mask = np.zeros(U_n.shape[0], dtype=bool)
        mask[gamma_d] = True

    def lhs(U):
        res = ((rho / dt) * emult.consistent_mass_mult(U, Me, nconn, nn, ndim)
               + theta * emult.visc_conv_mult(U, Ce_all_n, Le, mu, rho, nconn, nn, ndim))
        if mask is not None:
            res = np.where(mask, U, res)
        return res

    rhs = (((rho / dt) * emult.consistent_mass_mult(U_n, Me, nconn, nn, ndim))
           - gamma * emult.gradient_element_mult(P_n, Ge, nconn, nn, ndim)
           - (1 - theta) * emult.visc_conv_mult(U_n, Ce_all_n, Le, mu, rho, nconn, nn, ndim) + F)
    if gamma_d is not None:
        rhs = rhs.copy()
        rhs[gamma_d] = U_d
        x0 = U_n.copy()
        x0[gamma_d] = U_d
    else:
        x0 = U_n
    return bicgstab(lhs, rhs, x0=x0, tol=tol)


def solve_pressure(U_star, P_n, Le, Ge, rho, dt, nconn, nn, ndim, gamma_p, F_p, set_zeroP, precond,
                   M_op, tol, gamma):
    """solvers/standard.py:85-125: PPE by (P)CG, pinned rows zeroed or mean-zero."""

    def lhs(P):
        res = emult.laplacian_element_mult(P, Le, nconn, nn)
        if set_zeroP:
            res[gamma_p] = 0
        return res

    if gamma == 1:
        rhs = ((rho / dt) * (emult.divergence_element_mult(U_star, Ge, nconn, nn, ndim) - F_p)
               + emult.laplacian_element_mult(P_n, Le, nconn, nn))
    else:
        rhs = (rho / dt) * (emult.divergence_element_mult(U_star, Ge, nconn, nn, ndim) - F_p)
    if set_zeroP:
        rhs = rhs.copy()
        rhs[gamma_p] = 0
        x0 = P_n.copy()
        x0[gamma_p] = 0
    else:
        rhs = rhs - np.mean(rhs)
        x0 = P_n
    if precond == "approx_inv":
        M_op = partial(M_op, nconn=nconn)
    P, it = cg(lhs, rhs, x0=x0, tol=tol, maxiter=1000, M=M_op)
    P = P.copy()
    if set_zeroP:
        P[gamma_p] = 0
    else:
        P = P - np.mean(P)
    return P, it


def four_step_timestep(U_n, P_n, M, Me, Le, Ge, rho, mu, dt, nconn, nn, ndim, wq, N, Nderiv, gamma_d, U_d,
                       gamma_p, F_p, F, set_zeroP, p_precond, p_M_op, tol, theta):
    """solvers/standard.py:148-165 (Choi et al. 4-step projection)."""
    Ce = ecalc.conservative_convec_elem_calc(nconn, U_n, wq, N, Nderiv, nn, ndim, 0.5)
    U_hat, U_iters = solve_momentum(U_n, P_n, Me, Le, Ge, Ce, rho, mu, dt, nconn, nn, ndim, gamma_d, U_d, F,
                                    tol, theta, gamma=1)
    U_star = U_hat + ((dt / rho) * emult.gradient_element_mult(P_n, Ge, nconn, nn, ndim) / M)
    P, P_iters = solve_pressure(U_star, P_n, Le, Ge, rho, dt, nconn, nn, ndim, gamma_p, F_p, set_zeroP,
                                p_precond, p_M_op, tol, gamma=0)
    U = U_star - ((dt / rho) * emult.gradient_element_mult(P, Ge, nconn, nn, ndim) / M)
    if gamma_d is not None:
        U = U.copy()
        U[gamma_d] = U_d
    return U, P, U_iters, P_iters


def three_step_timestep(U_n, P_n, M, Me, Le, Ge, rho, mu, dt, nconn, nn, ndim, wq, N, Nderiv, gamma_d, U_d,
                        gamma_p, F_p, F, set_zeroP, p_precond, p_M_op, tol, theta, gamma):
    """solvers/standard.py:127-146."""
    Ce = ecalc.conservative_convec_elem_calc(nconn, U_n, wq, N, Nderiv, nn, ndim, 0.5)
    U_star, U_iters = solve_momentum(U_n, P_n, Me, Le, Ge, Ce, rho, mu, dt, nconn, nn, ndim, gamma_d, U_d, F,
                                     tol, theta, gamma)
    P, P_iters = solve_pressure(U_star, P_n, Le, Ge, rho, dt, nconn, nn, ndim, gamma_p, F_p, set_zeroP,
                                p_precond, p_M_op, tol, gamma)
    dP = P if gamma == 0 else P - P_n
    U = U_star - ((dt / rho) * emult.gradient_element_mult(dP, Ge, nconn, nn, ndim) / M)
    if gamma_d is not None:
        U = U.copy()
        U[gamma_d] = U_d
    return U, P, U_iters, P_iters


def compute(node_coords, bconn, nvec, boundary_shapefunc, gamma_d, U_d, nn, ndim, S_func, Me, nconn, t_n, t):
    """solvers/standard.py:167-188: F_p = int_Gd q u_d.n ; F = Me (S_n + S)/2."""
    F, F_p = 0, 0
    if gamma_d is not None:
        if ndim == 2:
            F_p = ecalc.u_dot_n_boundary_integral_1d(bconn, nvec, gamma_d, U_d, nn, node_coords,
                                                     boundary_shapefunc)
        else:
            F_p = ecalc.u_dot_n_boundary_integral_2d(bconn, nvec, gamma_d, U_d, nn, node_coords,
                                                     boundary_shapefunc)
    if S_func is not None:
        S = (S_func(t_n) + S_func(t)) / 2
        F = emult.consistent_mass_mult(S, Me, nconn, nn, ndim)
    return F_p, F


def shape_funcs_for(ndim, order):
    if ndim == 2:
        return ((shapefunc.quad4_shape_functions, shapefunc.lin2_shape_functions) if order == 1
                else (shapefunc.quad9_shape_functions, shapefunc.lin3_shape_functions))
    return shapefunc.hex8_shape_functions, shapefunc.quad4_shape_functions


def make_pressure_M_op(NS_config, mesh_config, Le, nconn, nn, gamma_p, mesh_func, shape_func):
    """solvers/standard.py:219-247 (jacobi / approx_inv / multigrid preconditioners)."""
    prec = NS_config.pressure_precond
    if prec == "jacobi":
        L_diag = ecalc.laplacian_diag(Le, nconn, nn)
        return lambda r: r / L_diag
    if prec == "approx_inv":
        L_diag = ecalc.laplacian_diag(Le, nconn, nn)

        def op(r, nconn):
            D1x = r / L_diag
            D1L = emult.laplacian_element_mult(D1x, Le, nconn, nn) / L_diag
            D1L[gamma_p] = 0
            t = emult.laplacian_element_mult(D1L, Le, nconn, nn)
            t[gamma_p] = 0
            return 3 * D1x - 3 * D1L + t / L_diag
        return op
    if prec == "multigrid" and len(mesh_config.num_elem) == 3:
        # build-defined 3D extension (oracle/multigrid3d.py)
        from . import multigrid3d as mg3
        levels = mg3.multigrid3d_setup(mesh_config.num_elem, NS_config.final_multigrid_mesh,
                                       mesh_config.domain_size, NS_config.outlet_faces)

        def op3(r):
            return mg3.v_cycle3d(r, levels)
        op3.levels = levels
        return op3
    if prec == "multigrid":
        data = mg.multigrid_setup(mesh_config.num_elem, NS_config.final_multigrid_mesh,
                                  mesh_config.domain_size, NS_config.outlet_faces, mesh_func, shape_func,
                                  mesh_config.shape_func_ord, mesh_config.partial_dirichlet)
        lvl_nums, Le_lvls, nconn_lvls, L_diag_lvls, gamma_p_lvls = data

        def op(r):
            return mg.v_cycle(r, lvl_nums, Le_lvls, nconn_lvls, L_diag_lvls, gamma_p_lvls,
                              NS_config.solver_tol, mesh_config.periodic, NS_config.set_zeroP)
        op.mg_data = data
        return op
    return None


def setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, mesh_func, config):
    """solvers/standard.py:191-267: returns (compute_loaded, timestep_loaded)."""
    mc, ns = config.mesh_config, config.solver_config
    ndim = len(mc.num_elem)
    shape_func, boundary_shapefunc = shape_funcs_for(ndim, mc.shape_func_ord)
    wq, N, Nderiv = shape_func(node_coords[nconn[0]])
    M, Me = ecalc.lumped_mass_matrix(nconn, wq, N, nn, ndim)
    Le = ecalc.laplacian_element_calc(wq, Nderiv)
    Ge = ecalc.gradient_element_calc(wq, N, Nderiv, ndim)
    M_op = make_pressure_M_op(ns, mc, Le, nconn, nn, gamma_p, mesh_func, shape_func)

    def compute_loaded(U_d, S_func, t_n, t):
        return compute(node_coords, bconn, nvec, boundary_shapefunc, gamma_d, U_d, nn, ndim, S_func, Me,
                       nconn, t_n, t)

    def timestep_loaded(U_n, P_n, dt, rho, mu, U_d, F_p, F):
        return four_step_timestep(U_n, P_n, M, Me, Le, Ge, rho, mu, dt, nconn, nn, ndim, wq, N, Nderiv,
                                  gamma_d, U_d, gamma_p, F_p, F, ns.set_zeroP, ns.pressure_precond, M_op,
                                  ns.solver_tol, 0.5)

    timestep_loaded.M_op = M_op
    timestep_loaded.data = dict(M=M, Me=Me, Le=Le, Ge=Ge, wq=wq, N=N, Nderiv=Nderiv)
    return compute_loaded, timestep_loaded
