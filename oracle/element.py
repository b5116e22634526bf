"""Element matrices and assembled diagonals (oracle restatement of
core/element_calc.py). Test infrastructure only."""
import numpy as np


def _assemble(vals, nconn, nn):
    """jax.ops.segment_sum(vals.flatten(), nconn.flatten(), nn): scatter-add in
    flattened (element-major) order."""
    out = np.zeros(nn, dtype=np.result_type(vals, np.float64))
    np.add.at(out, np.asarray(nconn).ravel(), np.asarray(vals).ravel())
    return out


def lumped_mass_matrix(nconn, wq, N, nn, ndim):
    """core/element_calc.py:9-25: Me = sum_q w N (x) N; M = assemble(rowsum Me), tiled ndim."""
    Me = np.sum((N * wq)[:, :, None] @ N[:, None, :], axis=0)
    Ml = np.sum(Me, axis=1)
    M = _assemble(np.tile(Ml, nconn.shape[0]), nconn, nn)
    return np.concatenate([M] * ndim), Me


def laplacian_element_calc(wq, Nderiv):
    """core/element_calc.py:27-32: Le = sum_q w dN^T dN."""
    return np.sum((Nderiv * wq[:, :, None]).transpose(0, 2, 1) @ Nderiv, axis=0)


def gradient_element_calc(wq, N, Nderiv, ndim):
    """core/element_calc.py:34-40: Ge[i] = sum_q w N (x) dN_i."""
    return np.stack([np.sum((N * wq)[:, :, None] @ Nderiv[:, i, :][:, None, :], axis=0)
                     for i in range(ndim)], axis=0)


def laplacian_diag(Le, nconn, nn):
    """core/element_calc.py:99-109."""
    return _assemble(np.tile(np.diag(Le), nconn.shape[0]), nconn, nn)


def _elem_fields(nconn, U, nn, ndim):
    """U[nconn + nn*i] stacked to (ne, I, ndim)."""
    return np.stack([U[nconn + nn * i] for i in range(ndim)], axis=-1)


def conservative_convec_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim, beta):
    """core/element_calc.py:165-185: Ce = sum_q w N (x) (u_q . dN) + beta sum_q w (div u)_q N (x) N."""
    Ul = _elem_fields(nconn, U, nn, ndim)                        # (e, I, d)
    Uq = np.einsum("qI,eId->eqd", N, Ul)                           # (e, q, d)
    CeA = np.einsum("qa,eqd,qdb->eab", N * wq, Uq, Nderiv)
    divq = np.einsum("qdI,eId->eq", Nderiv, Ul)                    # (e, q)
    CeD = np.einsum("qa,eq,qb->eab", N * wq, divq, N)
    return CeA + beta * CeD


def convection_element_calc(nconn, U, wq, N, Nderiv, nn, ndim):
    """core/element_calc.py:42-54 (advective form only)."""
    Ul = _elem_fields(nconn, U, nn, ndim)
    Uq = np.einsum("qI,eId->eqd", N, Ul)
    return np.einsum("qa,eqd,qdb->eab", N * wq, Uq, Nderiv)


def Ctau_tilde_elem_calc(nconn, U, wq, N, Nderiv, nn, ndim):
    """core/element_calc.py:188-200: sum_q w dN^T (u u^T) dN."""
    Ul = _elem_fields(nconn, U, nn, ndim)
    Uq = np.einsum("qI,eId->eqd", N, Ul)
    return np.einsum("qda,eqd,eqk,qkb->eab", Nderiv * wq[:, :, None], Uq, Uq, Nderiv)


def calculate_tau(nconn, U, Ce_all, Ctau_tilde_all, N, nn, ndim, D, dt, r):
    """core/element_calc.py:202-229 (per-element SUPG tau, r-norm blend)."""
    D = D + 1e-6
    Ul = _elem_fields(nconn, U, nn, ndim)
    Uq = np.einsum("qI,eId->eqd", N, Ul)
    ce_n = np.sqrt(np.sum(Ce_all ** 2, axis=(1, 2)))
    kt_n = np.sqrt(np.sum(Ctau_tilde_all ** 2, axis=(1, 2)))
    un2 = np.mean(np.sum(Uq ** 2, axis=2), axis=1)
    Re = (un2 * ce_n) / (D * kt_n)
    tau1 = ce_n / kt_n
    tau2 = dt / 2
    tau3 = tau1 * Re
    return (1 / (tau1 ** r) + 1 / (tau2 ** r) + 1 / (tau3 ** r)) ** (-1 / r)


def u_dot_n_boundary_integral_1d(bconn, nvec, gamma_d, U_d, nn, node_coords, shapefunc):
    """core/element_calc.py:111-135: F = assemble(int_edge N (U_q . n))."""
    ui = np.searchsorted(gamma_d, bconn)
    vi = np.searchsorted(gamma_d, bconn + nn)
    U = np.stack([U_d[ui], U_d[vi]], axis=-1)                      # (be, I, 2)
    Fe = np.zeros(bconn.shape, dtype=np.float64)
    for ie in range(bconn.shape[0]):
        wq, N, _ = shapefunc(node_coords[bconn[ie]])
        Uq = N @ U[ie]
        Fe[ie] = (N * wq).T @ np.sum(nvec[ie][None, :] * Uq, axis=1)
    return _assemble(Fe, bconn, nn)


def u_dot_n_boundary_integral_2d(bconn, nvec, gamma_d, U_d, nn, node_coords, shapefunc):
    """Build-defined 3D face integral. The reference (core/element_calc.py:137-163)
    only handles faces whose in-plane coordinates are (z, y) (TODO at :149); here
    the two in-plane coordinates are the ones orthogonal to the face normal."""
    ui = np.searchsorted(gamma_d, bconn)
    vi = np.searchsorted(gamma_d, bconn + nn)
    wi = np.searchsorted(gamma_d, bconn + 2 * nn)
    U = np.stack([U_d[ui], U_d[vi], U_d[wi]], axis=-1)
    Fe = np.zeros(bconn.shape, dtype=np.float64)
    for ie in range(bconn.shape[0]):
        nrm = np.asarray(nvec[ie])
        axes = [d for d in range(3) if nrm[d] == 0]
        wq, N, _ = shapefunc(node_coords[bconn[ie]][:, axes])
        Uq = N @ U[ie]
        Fe[ie] = (N * np.abs(wq)).T @ np.sum(nrm[None, :] * Uq, axis=1)
    return _assemble(Fe, bconn, nn)
