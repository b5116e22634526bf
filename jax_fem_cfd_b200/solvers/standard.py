"""Incompressible Navier-Stokes 4-step projection (drop-in for jax_fem_cfd
solvers/standard.py).

setup_solver returns (compute_loaded, timestep_loaded) with the reference's
call signatures. One time step is: Ce build, momentum rhs, one persistent
BiCGSTAB launch, U*, PPE rhs, one persistent (P)CG launch (multigrid V-cycles
inside it), projection. Iteration counts come back as 0-d int32 device tensors
like the reference's device scalars."""
import math

import numpy as np
import torch

from .. import _lib
from ..context import Context, f64, i64, make_mask, ptr, scatter_set, stream
from ..core import multigrid as mg
from ..setup.regular_mesh import mesh_of


# mixed-precision pressure solve: FP32 multigrid-PCG iterations per FP64
# refinement cycle, and the cap on cycles. Two inner iterations with ~2 cycles
# per solve were the fastest on B200 (3D channel 151.7 steps/s at 2, 135.3 at 4;
# Taylor-Green 256^2 Q2 548 at 2, 413 at 4), at the same error against FP64.
MIXED_INNER, MIXED_CYCLES = 2, 10


class NSSolver:
    """Device-resident state of one NS problem: context, boundary sets,
    multigrid hierarchy, cached Dirichlet vectors."""

    def __init__(self, mesh, gamma_d, gamma_p, bconn, nvec, solver_cfg, mesh_cfg):
        self.ctx = Context(mesh)
        self.mesh, self.cfg, self.mcfg = mesh, solver_cfg, mesh_cfg
        ctx = self.ctx
        self.nn, self.ndim = ctx.nn, ctx.ndim
        self.dmask = make_mask(gamma_d, self.ndim * self.nn) if gamma_d is not None else None
        gp = np.array([0]) if (gamma_p is None or isinstance(gamma_p, int)) else gamma_p
        self.pmask = make_mask(gp, self.nn)
        self.gamma_d = i64(gamma_d) if gamma_d is not None else None
        ctx.set_bc(self.dmask, self.pmask, solver_cfg.set_zeroP)
        self.precond = _lib.PREC[solver_cfg.pressure_precond]
        if solver_cfg.pressure_precond == "multigrid":
            nlev = int(math.log2(mesh.nex // solver_cfg.final_multigrid_mesh[0])) + 1
            pins = mg.level_pin_sets(mesh, nlev, solver_cfg.outlet_faces, mesh_cfg.partial_dirichlet,
                                     mesh_cfg.shape_func_ord)
            self.hier = mg.Hierarchy(ctx, nlev, pins, solver_cfg.solver_tol)
        precision = getattr(solver_cfg, "precision", "fp64")
        _lib.call("fem_ctx_set_precision", ctx.handle, _lib.PRECISION[precision], MIXED_INNER, MIXED_CYCLES)
        self.bconn = bconn.to(torch.int32).contiguous() if bconn is not None else None
        self.nvec = f64(nvec).reshape(-1) if nvec is not None else None
        self.iters = torch.zeros(2, dtype=torch.int32, device=ctx.dev)
        self.status = torch.zeros(2, dtype=torch.int32, device=ctx.dev)
        self._ud_key = None
        self._ud_full = None

    def u_full(self, U_d):
        """ndim*nn vector holding U_d on gamma_d (cached per U_d tensor version)."""
        if self.gamma_d is None:
            return None
        key = (U_d.data_ptr(), U_d._version) if isinstance(U_d, torch.Tensor) else None
        if key is None or key != self._ud_key:
            full = torch.zeros(self.ndim * self.nn, dtype=torch.float64, device=self.ctx.dev)
            self._ud_full = scatter_set(full, self.gamma_d, U_d)
            self._ud_key = key
        return self._ud_full

    def boundary_flux(self, U_d):
        """F_p = int_Gamma_d q u_d . n (core/element_calc.py:111-135 / 137-163)."""
        F_p = torch.empty(self.nn, dtype=torch.float64, device=self.ctx.dev)
        _lib.call("fem_boundary_flux", self.ctx.handle, ptr(self.bconn), ptr(self.nvec), int(self.bconn.shape[0]),
                  int(self.bconn.shape[1]), ptr(self.u_full(U_d)), ptr(F_p), stream())
        return F_p

    def step(self, U_n, P_n, dt, rho, mu, U_d, F_p, F, out=None):
        U_n, P_n = f64(U_n), f64(P_n)
        Uo = torch.empty_like(U_n) if out is None else out[0]
        Po = torch.empty_like(P_n) if out is None else out[1]
        Fp = None if (F_p is None or isinstance(F_p, (int, float))) else f64(F_p)
        Fv = None if (F is None or isinstance(F, (int, float))) else f64(F)
        iters = torch.empty(2, dtype=torch.int32, device=self.ctx.dev)
        _lib.call("fem_step4", self.ctx.handle, ptr(U_n), ptr(P_n), float(dt), float(rho), float(mu),
                  ptr(self.u_full(U_d) if U_d is not None else None), ptr(Fp), ptr(Fv), float(self.cfg.solver_tol),
                  self.precond, ptr(Uo), ptr(Po), ptr(iters), ptr(self.status), stream())
        return Uo, Po, iters[0], iters[1]


def setup_solver(node_coords, nconn, bconn, nvec, gamma_d, gamma_p, nn, mesh_func, config):
    """solvers/standard.py:191-267: returns (compute_loaded, timestep_loaded)."""
    mc, ns = config.mesh_config, config.solver_config
    solver = NSSolver(mesh_of(nconn, nn), gamma_d, gamma_p, bconn, nvec, ns, mc)
    ctx = solver.ctx
    Me = ctx.element_data()[3]

    def compute_loaded(U_d, S_func, t_n, t):
        """solvers/standard.py:167-188: (F_p, F); zeros when absent."""
        F_p, F = 0, 0
        if gamma_d is not None:
            F_p = solver.boundary_flux(U_d)
        if S_func is not None:
            S = torch.empty(ctx.ndim * ctx.nn, dtype=torch.float64, device=ctx.dev)
            Sn, S1 = f64(S_func(t_n)), f64(S_func(t))
            _lib.call("fem_axpby", ctx.handle, 0.5, ptr(Sn), 0.0, ptr(S), int(S.numel()), stream())
            _lib.call("fem_axpby", ctx.handle, 0.5, ptr(S1), 1.0, ptr(S), int(S.numel()), stream())
            F = torch.empty_like(S)
            _lib.call("fem_ebe_apply", ctx.handle, ctx.ndim, ptr(S), ptr(F), 1.0, ptr(Me.reshape(-1)), 0.0, None, 0,
                      0.0, None, stream())
        return F_p, F

    def timestep_loaded(U_n, P_n, dt, rho, mu, U_d, F_p, F):
        """solvers/standard.py:264-265 -> four_step_timestep (:148-165)."""
        return solver.step(U_n, P_n, dt, rho, mu, U_d, F_p, F)

    timestep_loaded.solver = solver
    compute_loaded.solver = solver
    return compute_loaded, timestep_loaded


def _solver_for(nconn, nn, gamma_d, gamma_p, set_zeroP, precond, tol):
    """A cached NSSolver for the module-level reference-signature functions."""
    from ..setup.simulation import SimpleMeshConfig, StandardSolverConfig
    mesh = mesh_of(nconn, nn)
    gd = None if gamma_d is None else i64(gamma_d)
    key = (mesh, None if gd is None else (gd.data_ptr(), gd.numel()),
           gamma_p if isinstance(gamma_p, int) else (None if gamma_p is None else i64(gamma_p).cpu().numpy().tobytes()),
           bool(set_zeroP), precond, float(tol))
    s = _SOLVERS.get(key)
    if s is None:
        fmg = [max(1, mesh.nex // (mesh.nex & -mesh.nex)), 1] if precond == "multigrid" else None
        if precond == "multigrid":
            k = 0
            while (mesh.nex >> (k + 1)) >= 4 and (mesh.ney >> (k + 1)) >= 4 and ((mesh.nex >> (k + 1)) << (k + 1)) == mesh.nex:
                k += 1
            fmg = [mesh.nex >> k, mesh.ney >> k]
        cfg = StandardSolverConfig([], [], [], False, tol, set_zeroP, precond, fmg)
        mcfg = SimpleMeshConfig([mesh.nex, mesh.ney], [mesh.lx, mesh.ly], 2 if mesh.kind == 1 else 1, mesh.periodic)
        gp = gamma_p if not isinstance(gamma_p, int) else np.array([gamma_p])
        if len(_SOLVERS) > 8:
            _SOLVERS.clear()
        s = _SOLVERS[key] = NSSolver(mesh, gd, gp, None, None, cfg, mcfg)
    return s


_SOLVERS = {}


def solve_momentum(U_n, P_n, Me, Le, Ge, Ce_all_n, rho, mu, dt, nconn, nn, ndim, gamma_d, U_d, F, tol, theta, gamma):
    """solvers/standard.py:14-43: theta-scheme momentum solve by one persistent
    BiCGSTAB launch; Dirichlet rows are identity rows (where(mask, U, AU))."""
    from ..core import element_mult as em
    mesh = mesh_of(nconn, nn)
    s = _solver_for(nconn, nn, gamma_d, 0, True, None, tol)
    ctx = s.ctx
    N = ndim * ctx.nn
    rhs = em.consistent_mass_mult(U_n, Me, nconn, nn, ndim)
    gp = em.gradient_element_mult(P_n, Ge, nconn, nn, ndim)
    vc = em.visc_conv_mult(U_n, Ce_all_n, Le, mu, rho, nconn, nn, ndim)
    h = ctx.handle
    _lib.call("fem_axpby", h, -float(gamma), ptr(gp), rho / dt, ptr(rhs), N, stream())
    _lib.call("fem_axpby", h, -(1 - theta), ptr(vc), 1.0, ptr(rhs), N, stream())
    if F is not None and not isinstance(F, (int, float)):
        _lib.call("fem_axpby", h, 1.0, ptr(f64(F)), 1.0, ptr(rhs), N, stream())
    x = f64(U_n).clone()
    mask = None
    if gamma_d is not None:
        scatter_set(rhs, gamma_d, U_d)
        scatter_set(x, gamma_d, U_d)
        mask = s.dmask
    # A = (rho/dt) Me + theta (rho Ce + mu Le): shared part combined on the device
    Ksh = torch.empty_like(f64(Me).reshape(-1))
    _lib.call("fem_axpby", h, rho / dt, ptr(f64(Me).reshape(-1)), 0.0, ptr(Ksh), Ksh.numel(), stream())
    _lib.call("fem_axpby", h, theta * mu, ptr(f64(Le).reshape(-1)), 1.0, ptr(Ksh), Ksh.numel(), stream())
    iters = torch.empty(1, dtype=torch.int32, device=ctx.dev)
    _lib.call("fem_bicgstab_solve", h, int(ndim), 1.0, ptr(Ksh), theta * rho, ptr(f64(Ce_all_n)), 0.0, None,
              ptr(mask), ptr(rhs), ptr(x), float(tol), 0.0, 0, ptr(iters), ptr(s.status), stream())
    return x, iters[0]


def solve_pressure(U_star, P_n, Le, Ge, rho, dt, nconn, nn, ndim, gamma_p, F_p, set_zeroP, precond, M_op, tol,
                   gamma):
    """solvers/standard.py:85-125: PPE by one persistent (P)CG launch. The
    preconditioner is named by ``precond`` ("jacobi", "approx_inv",
    "multigrid" or None); M_op is not called (its device form is built here)."""
    from ..core import element_mult as em
    s = _solver_for(nconn, nn, None, gamma_p, set_zeroP, precond, tol)
    ctx = s.ctx
    rhs = em.divergence_element_mult(U_star, Ge, nconn, nn, ndim)
    h = ctx.handle
    if F_p is not None and not isinstance(F_p, (int, float)):
        _lib.call("fem_axpby", h, -1.0, ptr(f64(F_p)), 1.0, ptr(rhs), ctx.nn, stream())
    _lib.call("fem_axpby", h, 0.0, ptr(rhs), rho / dt, ptr(rhs), ctx.nn, stream())
    if gamma == 1:
        lp = em.laplacian_element_mult(P_n, Le, nconn, nn)
        _lib.call("fem_axpby", h, 1.0, ptr(lp), 1.0, ptr(rhs), ctx.nn, stream())
    x = f64(P_n).clone()
    if set_zeroP:
        gp = np.array([0]) if isinstance(gamma_p, int) else gamma_p
        scatter_set(rhs, gp, 0.0)
        scatter_set(x, gp, 0.0)
    iters = torch.empty(1, dtype=torch.int32, device=ctx.dev)
    _lib.call("fem_pressure_solve", h, ptr(rhs), ptr(x), float(tol), 0.0, 1000, _lib.PREC[precond],
              0 if set_zeroP else 1, 1, ptr(iters), ptr(s.status), stream())
    return x, iters[0]


def compute(node_coords, bconn, nvec, boundary_shapefunc, gamma_d, U_d, nn, ndim, S_func, Me, nconn, t_n, t):
    """solvers/standard.py:167-188."""
    from ..core import element_calc as ec
    from ..core import element_mult as em
    F, F_p = 0, 0
    if gamma_d is not None:
        fn = ec.u_dot_n_boundary_integral_1d if ndim == 2 else ec.u_dot_n_boundary_integral_2d
        F_p = fn(bconn, nvec, gamma_d, U_d, nn, node_coords, boundary_shapefunc, nconn=nconn)
    if S_func is not None:
        S = f64(S_func(t_n)).clone()
        ctx_h = _solver_for(nconn, nn, None, 0, True, None, 1e-8).ctx.handle
        _lib.call("fem_axpby", ctx_h, 0.5, ptr(f64(S_func(t))), 0.5, ptr(S), S.numel(), stream())
        F = em.consistent_mass_mult(S, Me, nconn, nn, ndim)
    return F_p, F
