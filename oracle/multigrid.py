"""Geometric multigrid V-cycle for the pressure Poisson problem (oracle
restatement of core/multigrid.py). Test infrastructure only."""
import numpy as np

from . import element as ecalc
from .emult import laplacian_element_mult
from .solvers import cg


def multigrid_setup(num_elem, num_elemf, domain_size, outlet_faces, mesh_func, shapefunc,
                    shape_func_ord, partial_dirichlet):
    """core/multigrid.py:9-88. Levels N = log2(nex/nexf) + 1 (from x only, :12);
    ney halves in lockstep (:80). Returns (lvl_nums, Le_lvls, nconn_lvls,
    L_diag_lvls, gamma_p_lvls) with cumulative offsets [nn, nnx, nny, ne, np]."""
    nex, ney = num_elem
    N = int(np.log2(nex // num_elemf[0])) + 1
    nen = 4 if shape_func_ord == 1 else 9
    lvl = np.zeros((N + 1, 5), dtype=np.int64)
    Le_lvls = np.zeros((N, 2, nen, nen))
    nconns, diags, gps = [], [], []
    for i in range(N):
        node_coords, nconn, surfnodes, bconns, _ = mesh_func(nex, ney, *domain_size)
        wq, _, Nderiv = shapefunc(node_coords[nconn[0]])
        nn = node_coords.shape[0]
        nnx, nny = (nex + 1, ney + 1) if shape_func_ord == 1 else (2 * nex + 1, 2 * ney + 1)
        outlet = []
        if outlet_faces:
            for face in outlet_faces:
                outlet.append(surfnodes[face])
        if partial_dirichlet:
            for face, (s, e, kind) in partial_dirichlet.items():
                fn, fb = surfnodes[face], bconns[face]
                nfe = fb.shape[0]
                si, ei = round(s * nfe), round(e * nfe)
                if shape_func_ord == 2:
                    si, ei = 2 * si, 2 * ei
                if kind == "outlet":
                    outlet.append(fn[:si])
                    outlet.append(fn[ei + 1:])
        gamma_p = np.unique(np.concatenate(outlet)) if outlet else np.array([0])
        Le = ecalc.laplacian_element_calc(wq, Nderiv)
        Ld = ecalc.laplacian_diag(Le, nconn, nn)
        lvl[i + 1] = [lvl[i, 0] + nn, nnx, nny, lvl[i, 3] + nex * ney, lvl[i, 4] + gamma_p.shape[0]]
        Le_lvls[i, 0] = Le
        Le_lvls[i, 1] = Le - np.diag(np.diag(Le))
        nconns.append(nconn)
        diags.append(Ld)
        gps.append(gamma_p)
        nex, ney = nex // 2, ney // 2
    lvl_nums = tuple(tuple(int(x) for x in row) for row in lvl)
    return lvl_nums, Le_lvls, np.concatenate(nconns), np.concatenate(diags), np.concatenate(gps)


def _periodic_full(x, ny, nx):
    """Re-insert the dropped periodic row/column (core/multigrid.py:96-102, 148-154)."""
    xr = x.reshape(ny - 1, nx - 1)
    full = np.zeros((ny, nx))
    full[:-1, :-1] = xr
    full[:-1, -1] = xr[:, 0]
    full[-1, :-1] = xr[0, :]
    full[-1, -1] = xr[0, 0]
    return full


def interpolation_operator(xH, nnH_x, nnH_y, nnh_x, nnh_y, periodic):
    """core/multigrid.py:90-140: lattice-bilinear prolongation coarse -> fine."""
    H = _periodic_full(xH, nnH_y, nnH_x) if periodic else xH.reshape(nnH_y, nnH_x)
    h = np.zeros((nnh_y, nnh_x))
    h[0::2, 0::2] = H
    h[0::2, 1:-1:2] = 0.5 * H[:, :-1] + 0.5 * H[:, 1:]
    h[1:-1:2, 0::2] = 0.5 * H[:-1, :] + 0.5 * H[1:, :]
    h[1:-1:2, 1:-1:2] = 0.25 * H[:-1, :-1] + 0.25 * H[:-1, 1:] + 0.25 * H[1:, :-1] + 0.25 * H[1:, 1:]
    if periodic:
        h = h[:-1, :-1]
    return h.ravel()


def restriction_operator(xh, nnh_x, nnh_y, nnH_x, nnH_y, periodic):
    """core/multigrid.py:142-212: R = I^T on the full (duplicated-periodic) lattice,
    no 1/4 factor; corner, edge and interior formulas as the reference writes them."""
    f = _periodic_full(xh, nnh_y, nnh_x) if periodic else xh.reshape(nnh_y, nnh_x)
    X, Y = nnh_x, nnh_y
    H = np.zeros((nnH_y, nnH_x))
    H[0, 0] = f[0, 0] + 0.5 * (f[0, 1] + f[1, 0]) + 0.25 * f[1, 1]
    H[0, -1] = f[0, X - 1] + 0.5 * (f[0, X - 2] + f[1, X - 1]) + 0.25 * f[1, X - 2]
    H[-1, 0] = f[Y - 1, 0] + 0.5 * (f[Y - 2, 0] + f[Y - 1, 1]) + 0.25 * f[Y - 2, 1]
    H[-1, -1] = f[Y - 1, X - 1] + 0.5 * (f[Y - 1, X - 2] + f[Y - 2, X - 1]) + 0.25 * f[Y - 2, X - 2]
    vi = 2 * np.arange(1, nnH_y - 1)
    hj = 2 * np.arange(1, nnH_x - 1)
    H[1:-1, 0] = f[vi, 0] + 0.5 * (f[vi + 1, 0] + f[vi - 1, 0] + f[vi, 1]) + 0.25 * (f[vi + 1, 1] + f[vi - 1, 1])
    H[1:-1, -1] = (f[vi, X - 1] + 0.5 * (f[vi + 1, X - 1] + f[vi - 1, X - 1] + f[vi, X - 2])
                   + 0.25 * (f[vi + 1, X - 2] + f[vi - 1, X - 2]))
    H[0, 1:-1] = f[0, hj] + 0.5 * (f[0, hj + 1] + f[0, hj - 1] + f[1, hj]) + 0.25 * (f[1, hj + 1] + f[1, hj - 1])
    H[-1, 1:-1] = (f[Y - 1, hj] + 0.5 * (f[Y - 1, hj + 1] + f[Y - 1, hj - 1] + f[Y - 2, hj])
                   + 0.25 * (f[Y - 2, hj + 1] + f[Y - 2, hj - 1]))
    V, Hh = vi[:, None], hj[None, :]
    H[1:-1, 1:-1] = (f[V, Hh] + 0.5 * (f[V + 1, Hh] + f[V - 1, Hh] + f[V, Hh + 1] + f[V, Hh - 1])
                     + 0.25 * (f[V + 1, Hh + 1] + f[V + 1, Hh - 1] + f[V - 1, Hh + 1] + f[V - 1, Hh - 1]))
    if periodic:
        H = H[:-1, :-1]
    return H.ravel()


def single_jacobi_iter(x, rhs, Le_off, L_diag, gamma_p, nconn, nn, set_zeroP):
    """core/multigrid.py:214-228: one weighted (omega = 2/3) Jacobi sweep."""
    omega = 2 / 3
    x = x.copy()
    if set_zeroP:
        x[gamma_p] = 0
    off = laplacian_element_mult(x, Le_off, nconn, nn)
    x = omega * (rhs - off) / L_diag + (1 - omega) * x
    if set_zeroP:
        x[gamma_p] = 0
    else:
        x = x - np.mean(x)
    return x


def v_cycle(rhs, lvl_nums, Le_lvls, nconn_lvls, L_diag_lvls, gamma_p_lvls, tol, periodic, set_zeroP):
    """core/multigrid.py:231-330: one V-cycle from x = 0 (pre-smooth, restrict,
    coarse CG or one Jacobi, prolong, post-smooth)."""
    L = lvl_nums
    N = len(L) - 1
    x_l = np.zeros(L[-1][0])
    r_l = np.zeros(L[-1][0])
    r_l[0:L[1][0]] = rhs
    for n in range(N - 1):
        nc = nconn_lvls[L[n][3]:L[n + 1][3]]
        nnh = L[n + 1][0] - L[n][0]
        D = L_diag_lvls[L[n][0]:L[n + 1][0]]
        if set_zeroP:
            gp = gamma_p_lvls[L[n][4]:L[n + 1][4]]
            rh = r_l[L[n][0]:L[n + 1][0]].copy()
            rh[gp] = 0
            xh = 2 / 3 * rh / D
            xh[gp] = 0
            Lx = laplacian_element_mult(xh, Le_lvls[n, 0], nc, nnh)
            Lx[gp] = 0
            rH = rh - Lx
            rH = restriction_operator(rH, L[n + 1][1], L[n + 1][2], L[n + 2][1], L[n + 2][2], periodic)
        else:
            rh = r_l[L[n][0]:L[n + 1][0]]
            rh = rh - np.mean(rh)
            xh = 2 / 3 * rh / D
            xh = xh - np.mean(xh)
            rH = rh - laplacian_element_mult(xh, Le_lvls[n, 0], nc, nnh)
            rH = rH - np.mean(rH)
            rH = restriction_operator(rH, L[n + 1][1], L[n + 1][2], L[n + 2][1], L[n + 2][2], periodic)
            rH = rH - np.mean(rH)
        x_l[L[n][0]:L[n + 1][0]] = xh
        r_l[L[n + 1][0]:L[n + 2][0]] = rH
    nc_N = nconn_lvls[L[N - 1][3]:L[N][3]]
    nn_N = L[N][0] - L[N - 1][0]
    if set_zeroP:
        gpN = gamma_p_lvls[L[N - 1][4]:L[N][4]]

        def op(x):
            y = laplacian_element_mult(x, Le_lvls[N - 1, 0], nc_N, nn_N)
            y[gpN] = 0
            return y

        rN = r_l[L[N - 1][0]:L[N][0]].copy()
        rN[gpN] = 0
        xN, _ = cg(op, rN, tol=tol, maxiter=1000)
        xN = xN.copy()
        xN[gpN] = 0
    else:
        rN = r_l[L[N - 1][0]:L[N][0]]
        rN = rN - np.mean(rN)
        xN = single_jacobi_iter(np.zeros(rN.shape[0]), rN, Le_lvls[N - 1, 1],
                                L_diag_lvls[L[N - 1][0]:L[N][0]], 0, nc_N, nn_N, False)
    x_l[L[N - 1][0]:L[N][0]] = xN
    for n in range(N - 2, -1, -1):
        nc = nconn_lvls[L[n][3]:L[n + 1][3]]
        gp = gamma_p_lvls[L[n][4]:L[n + 1][4]]
        nnh = L[n + 1][0] - L[n][0]
        rh = r_l[L[n][0]:L[n + 1][0]]
        xH = interpolation_operator(x_l[L[n + 1][0]:L[n + 2][0]], L[n + 2][1], L[n + 2][2],
                                    L[n + 1][1], L[n + 1][2], periodic)
        if not set_zeroP:
            xH = xH - np.mean(xH)
        xh = x_l[L[n][0]:L[n + 1][0]] + xH
        xh = single_jacobi_iter(xh, rh, Le_lvls[n, 1], L_diag_lvls[L[n][0]:L[n + 1][0]],
                                gp, nc, nnh, set_zeroP)
        x_l[L[n][0]:L[n + 1][0]] = xh
    return x_l[0:L[1][0]].copy()
