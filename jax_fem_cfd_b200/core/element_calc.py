"""Element matrices and assembled diagonals (drop-in for core/element_calc.py).
All arithmetic runs in libfemb200 kernels on the device."""
import torch

from .. import _lib
from ..context import context_for, empty, f64, i64, ptr, stream
from ..setup.regular_mesh import mesh_of


def _quad(wq, N, Nderiv):
    wq, N, dN = f64(wq).reshape(-1), f64(N), f64(Nderiv)
    nq, nen = N.shape
    dim = dN.shape[1]
    return wq, N.reshape(-1), dN.reshape(-1), nq, nen, dim


def _matrices(wq, N, Nderiv):
    wq, N, dN, nq, nen, dim = _quad(wq, N, Nderiv)
    Me, Le, Lo, Ge = empty(nen * nen), empty(nen * nen), empty(nen * nen), empty(dim * nen * nen)
    _lib.call("fem_element_matrices", nq, nen, dim, ptr(wq), ptr(N), ptr(dN), ptr(Me), ptr(Le), ptr(Lo), ptr(Ge),
              stream())
    return Me.view(nen, nen), Le.view(nen, nen), Lo.view(nen, nen), Ge.view(dim, nen, nen)


def lumped_mass_matrix(nconn, wq, N, nn, ndim):
    """core/element_calc.py:9: (M tiled ndim times, Me). Nderiv is not needed for
    Me; a zero derivative table of the right shape is passed."""
    Nt = f64(N)
    dN = torch.zeros((Nt.shape[0], 1, Nt.shape[1]), dtype=torch.float64, device=Nt.device)
    Me, _, _, _ = _matrices(wq, Nt, dN)
    ctx = context_for(mesh_of(nconn, nn))
    M = empty(ndim * int(nn))
    _lib.call("fem_assemble_diag", ctx.handle, ptr(Me), None, int(ndim), ptr(M), None, stream())
    return M, Me


def laplacian_element_calc(wq, Nderiv):
    """core/element_calc.py:27: Le = sum_q w dN^T dN."""
    dN = f64(Nderiv)
    N = torch.zeros((dN.shape[0], dN.shape[2]), dtype=torch.float64, device=dN.device)
    return _matrices(wq, N, dN)[1]


def gradient_element_calc(wq, N, Nderiv, ndim):
    """core/element_calc.py:34: Ge[i] = sum_q w N (x) dN_i."""
    return _matrices(wq, N, Nderiv)[3]


def laplacian_diag(Le, nconn, nn):
    """core/element_calc.py:99: assembled diag(L)."""
    ctx = context_for(mesh_of(nconn, nn))
    Ld = empty(int(nn))
    _lib.call("fem_assemble_diag", ctx.handle, None, ptr(f64(Le)), 1, None, ptr(Ld), stream())
    return Ld


def conservative_convec_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim, beta):
    """core/element_calc.py:165: Ce_e = sum_q w N (x) (u_q . dN) + beta sum_q w (div u)_q N (x) N."""
    ctx = context_for(mesh_of(nconn, nn))
    wq_, N_, dN_, nq, nen, dim = _quad(wq, N, Nderiv)
    Ce = empty(ctx.ne * nen * nen)
    _lib.call("fem_convection_build", ctx.handle, ptr(f64(U)), float(beta), ptr(wq_), ptr(N_), ptr(dN_), ptr(Ce),
              stream())
    return Ce.view(ctx.ne, nen, nen)


def convection_element_calc(nconn, U, wq, N, Nderiv, nn, ndim):
    """core/element_calc.py:42 (advective form, beta = 0)."""
    return conservative_convec_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim, 0.0)


def Ctau_tilde_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim):
    """core/element_calc.py:188: sum_q w dN^T (u u^T) dN."""
    ctx = context_for(mesh_of(nconn, nn))
    wq_, N_, dN_, nq, nen, dim = _quad(wq, N, Nderiv)
    Ct = empty(ctx.ne * nen * nen)
    _lib.call("fem_ctau_tilde_build", ctx.handle, ptr(f64(U)), ptr(wq_), ptr(N_), ptr(dN_), ptr(Ct), stream())
    return Ct.view(ctx.ne, nen, nen)


def calculate_tau(nconn, U, Ce_all, Ctau_tilde_all, N, nn, ndim, D, dt, r):
    """core/element_calc.py:202: per-element SUPG tau (r-norm blend)."""
    ctx = context_for(mesh_of(nconn, nn))
    tau = empty(ctx.ne)
    _lib.call("fem_supg_tau", ctx.handle, ptr(f64(U)), ptr(f64(Ce_all)), ptr(f64(Ctau_tilde_all)), float(D),
              float(dt), float(r), ptr(f64(N).reshape(-1)), ptr(tau), stream())
    return tau


def _u_full(gamma_d, U_d, length):
    from ..context import scatter_set
    out = torch.zeros(int(length), dtype=torch.float64, device=f64(U_d).device)
    return scatter_set(out, gamma_d, U_d)


def u_dot_n_boundary_integral_1d(bconn, nvec, gamma_d, U_d, nn, node_coords, shapefunc=None, nconn=None):
    """core/element_calc.py:111: F = assemble over boundary edges of int N (u_d . n)."""
    from ..setup.regular_mesh import mesh_of as _m
    b = i64(bconn).view(-1, bconn.shape[-1] if hasattr(bconn, "shape") else 2)
    ctx = context_for(_m(nconn, nn)) if nconn is not None else _ctx_from_coords(node_coords, nn)
    return _flux(ctx, b, nvec, gamma_d, U_d, nn)


def u_dot_n_boundary_integral_2d(bconn, nvec, gamma_d, U_d, nn, node_coords, shapefunc=None, nconn=None):
    """Build-defined 3D face integral (the reference's :137 handles only faces in
    the (z, y) plane, TODO at :149): in-plane axes are those orthogonal to n."""
    from ..setup.regular_mesh import mesh_of as _m
    b = i64(bconn).view(-1, 4)
    ctx = context_for(_m(nconn, nn)) if nconn is not None else _ctx_from_coords(node_coords, nn)
    return _flux(ctx, b, nvec, gamma_d, U_d, nn)


def _flux(ctx, b, nvec, gamma_d, U_d, nn):
    Uf = _u_full(gamma_d, U_d, ctx.ndim * int(nn))
    b32 = b.to(torch.int32).contiguous()
    nv = f64(nvec).reshape(-1)
    F = empty(int(nn))
    _lib.call("fem_boundary_flux", ctx.handle, ptr(b32), ptr(nv), int(b32.shape[0]), int(b32.shape[1]), ptr(Uf),
              ptr(F), stream())
    return F


def _ctx_from_coords(node_coords, nn):
    raise ValueError("pass nconn= so the boundary integral can locate its mesh")
