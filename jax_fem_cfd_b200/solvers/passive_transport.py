"""NS step followed by a Crank-Nicolson (optionally SUPG) advection-diffusion
step of a passive scalar (drop-in for jax_fem_cfd solvers/passive_transport.py)."""
import numpy as np
import torch

from .. import _lib
from ..context import f64, i64, make_mask, ptr, scatter_set, stream
from ..setup.regular_mesh import mesh_of
from .standard import NSSolver


def setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, gamma_d_phi, mesh_func, config):
    """solvers/passive_transport.py:100-180: (compute_loaded, timestep_loaded)
    with timestep_loaded(U_n, P_n, phi_n, dt, rho, mu, D, U_d, phi_d, F_p, F, phi_S_func)."""
    mc = config.mesh_config
    ns, ade = config.solver_config.NS_config, config.solver_config.ADE_config
    if ns.pressure_precond == "approx_inv":
        ns = type(ns)(**{**ns.__dict__, "pressure_precond": "approx_inv_pt"})
    solver = NSSolver(mesh_of(nconn, nn), gamma_d, gamma_p, bconn, nvec, ns, mc)
    ctx = solver.ctx
    Me = ctx.element_data()[3]
    phi_mask = make_mask(gamma_d_phi, ctx.nn) if gamma_d_phi is not None else None
    phi_status = torch.zeros(1, dtype=torch.int32, device=ctx.dev)

    def compute_loaded(U_d, S_func, t_n, t):
        F_p, F = 0, 0
        if gamma_d is not None:
            F_p = solver.boundary_flux(U_d)
        if S_func is not None:
            S = torch.empty(ctx.ndim * ctx.nn, dtype=torch.float64, device=ctx.dev)
            _lib.call("fem_axpby", ctx.handle, 0.5, ptr(f64(S_func(t_n))), 0.0, ptr(S), S.numel(), stream())
            _lib.call("fem_axpby", ctx.handle, 0.5, ptr(f64(S_func(t))), 1.0, ptr(S), S.numel(), stream())
            F = torch.empty_like(S)
            _lib.call("fem_ebe_apply", ctx.handle, ctx.ndim, ptr(S), ptr(F), 1.0, ptr(Me.reshape(-1)), 0.0, None, 0,
                      0.0, None, stream())
        return F_p, F

    def timestep_loaded(U_n, P_n, phi_n, dt, rho, mu, D, U_d, phi_d, F_p, F, phi_S_func):
        """solvers/passive_transport.py:64-97."""
        U_n, phi_n = f64(U_n), f64(phi_n)
        U, P, ui, pi = solver.step(U_n, P_n, dt, rho, mu, U_d, F_p, F)
        phid_full = None
        if gamma_d_phi is not None:
            phid_full = torch.zeros(ctx.nn, dtype=torch.float64, device=ctx.dev)
            scatter_set(phid_full, gamma_d_phi, phi_d)
        phi = torch.empty_like(phi_n)
        it = torch.empty(1, dtype=torch.int32, device=ctx.dev)
        _lib.call("fem_transport_phi", ctx.handle, ptr(U_n), ptr(U), ptr(phi_n), float(dt), float(D),
                  int(bool(ade.phi_SUPG)), ptr(phi_mask), ptr(phid_full), float(ns.solver_tol), ptr(phi), ptr(it),
                  ptr(phi_status), stream())
        return U, P, phi, ui, pi, it[0]

    timestep_loaded.solver = solver
    return compute_loaded, timestep_loaded
