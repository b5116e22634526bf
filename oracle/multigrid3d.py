"""Geometric multigrid for the hex8 pressure Poisson problem (oracle).

TEST INFRASTRUCTURE ONLY. BUILD-DEFINED EXTENSION: the reference refuses 3D
multigrid (setup/simulation.py:75-76), so there is no reference run to pin
this file to. It extends the reference's 2D scheme (core/multigrid.py) to hex8
lattices and is the specification the CUDA path is checked against:

- levels (core/multigrid.py:9-88 in 3D): N = log2(nex / nexf) + 1 levels, every
  axis halved in lockstep; each level re-discretises the Laplacian on its own
  hex8 mesh (Le from the hex8 shape functions, core/element_calc.py:27-32);
  gamma_p per level = the outlet-face nodes of that level's mesh, or node 0;
- transfers: lattice-trilinear prolongation P and R = P^T (the 3D form of
  core/multigrid.py:90-212: weights 1, 1/2, 1/4, 1/8, no scaling);
- smoother: Chebyshev iteration of degree `deg` (3) on D^-1 A over the
  interval [lo, hi] * lambda, lambda = a power-iteration estimate of the
  largest eigenvalue of D^-1 A (restricted to the free nodes), from a fixed
  hashed start vector; the same polynomial before and after the coarse
  correction, so the V-cycle is symmetric (a valid CG preconditioner);
  Chebyshev recurrence as in Saad, Iterative Methods for Sparse Linear
  Systems, 2nd ed., Algorithm 12.1;
- coarsest level: solved exactly, by the inverse of its matrix with the
  gamma_p rows and columns replaced by the identity;
- pinned form only (gamma_p rows zeroed, as the reference's set_zeroP branch):
  3D meshes are never periodic, and a pure-Neumann 3D problem is refused.

Operators are assembled as scipy.sparse matrices from the same element
matrices (the sum order differs from the element-by-element scatter only by
rounding)."""
import numpy as np
import scipy.sparse as sp

from . import element as ecalc
from . import mesh as omesh
from . import shape as oshape

CHEB_DEGREE = 3
CHEB_LO, CHEB_HI = 0.2, 1.1    # Chebyshev interval as fractions of the estimated lambda_max
POWER_ITERS = 40               # power iterations for lambda_max of D^-1 A per level


def hashed_start(n):
    """Start vector of the power iteration: ((i * 2654435761) mod 2^32) / 2^32 - 1/2."""
    i = np.arange(n, dtype=np.uint64)
    return ((i * np.uint64(2654435761)) % np.uint64(2 ** 32)).astype(np.float64) / 4294967296.0 - 0.5


def assembled(Le, nconn, nn):
    """Sparse assembled matrix sum_e P_e^T Le P_e."""
    ne, nen = nconn.shape
    rows = np.repeat(nconn, nen, axis=1).ravel()
    cols = np.tile(nconn, (1, nen)).ravel()
    vals = np.tile(Le.ravel(), ne)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nn, nn))


class Level:
    pass


def level_count(num_elem, num_elemf):
    """N = log2(nex / nexf) + 1 (core/multigrid.py:12), all axes in lockstep."""
    return int(np.log2(num_elem[0] // num_elemf[0])) + 1


def multigrid3d_setup(num_elem, num_elemf, domain_size, outlet_faces, deg=CHEB_DEGREE, lo=CHEB_LO, hi=CHEB_HI,
                      power_iters=POWER_ITERS):
    nex, ney, nez = num_elem
    lx, ly, lz = domain_size
    N = level_count(num_elem, num_elemf)
    levels = []
    for i in range(N):
        nc, nconn, surf, _, _ = omesh.create_mesh_3d(nex, ney, nez, lx, ly, lz)
        nn = nc.shape[0]
        wq, _, Nderiv = oshape.hex8_shape_functions(nc[nconn[0]])
        Le = ecalc.laplacian_element_calc(wq, Nderiv)
        L = Level()
        L.dims = (nex + 1, ney + 1, nez + 1)
        L.nn = nn
        L.A = assembled(Le, nconn, nn)
        L.D = ecalc.laplacian_diag(Le, nconn, nn)
        gp = np.unique(np.concatenate([surf[f] for f in outlet_faces])) if outlet_faces else np.array([0])
        L.gp = gp
        L.free = np.ones(nn, dtype=bool)
        L.free[gp] = False
        L.invDm = np.where(L.free, 1.0 / L.D, 0.0)
        levels.append(L)
        nex, ney, nez = nex // 2, ney // 2, nez // 2
    for L in levels[:-1]:
        lam = power_lambda(L, power_iters)
        L.lam = lam
        L.bounds = (lo * lam, hi * lam)
        L.deg = deg
    C = levels[-1]
    Ad = C.A.toarray()
    Ad[C.gp, :] = 0.0
    Ad[:, C.gp] = 0.0
    Ad[C.gp, C.gp] = 1.0
    C.Ainv = np.linalg.inv(Ad)
    return levels


def apply_A(L, x):
    """L x with the gamma_p rows zeroed."""
    y = L.A @ x
    y[L.gp] = 0.0
    return y


def power_lambda(L, iters):
    """Largest eigenvalue of D^-1 A on the free nodes: ||w|| / ||v|| of the last of
    `iters` normalised power steps w = D^-1 A v, from the hashed start vector."""
    v = hashed_start(L.nn)
    v[L.gp] = 0.0
    lam = 0.0
    for _ in range(iters):
        w = L.invDm * (L.A @ v)
        nw, nv = np.sqrt(np.dot(w, w)), np.sqrt(np.dot(v, v))
        lam = nw / nv
        v = w / nw
    return lam


def cheb_coeffs(L):
    """(theta, delta, [(a_k, b_k)]): d_1 = b_1 D^-1 r_0, d_k = a_k d_{k-1} + b_k D^-1 r_{k-1}."""
    lo, hi = L.bounds
    theta, delta = (hi + lo) / 2, (hi - lo) / 2
    sigma = theta / delta
    rho_old = 1.0 / sigma
    co = [(0.0, 1.0 / theta)]
    for _ in range(1, L.deg):
        rho = 1.0 / (2.0 * sigma - rho_old)
        co.append((rho * rho_old, 2.0 * rho / delta))
        rho_old = rho
    return co


def chebyshev(L, b, x0):
    """deg Chebyshev steps on A x = b (gamma_p rows zeroed) from x0 (None: 0)."""
    co = cheb_coeffs(L)
    x = np.zeros(L.nn) if x0 is None else x0.copy()
    d = None
    for k, (a, bk) in enumerate(co):
        res = b - apply_A(L, x) if (k > 0 or x0 is not None) else b.copy()
        res[L.gp] = 0.0
        d = bk * (L.invDm * res) if k == 0 else a * d + bk * (L.invDm * res)
        x = x + d
    return x


def prolong3d(xH, dH, dh):
    """Trilinear interpolation from the (NX, NY, NZ) lattice to the (2NX-1, ...) lattice."""
    NX, NY, NZ = dH
    nx, ny, nz = dh
    H = xH.reshape(NZ, NY, NX)
    # along x
    a = np.zeros((NZ, NY, nx))
    a[:, :, 0::2] = H
    a[:, :, 1::2] = 0.5 * (H[:, :, :-1] + H[:, :, 1:])
    b = np.zeros((NZ, ny, nx))
    b[:, 0::2, :] = a
    b[:, 1::2, :] = 0.5 * (a[:, :-1, :] + a[:, 1:, :])
    c = np.zeros((nz, ny, nx))
    c[0::2] = b
    c[1::2] = 0.5 * (b[:-1] + b[1:])
    return c.ravel()


def _restrict_axis(f, axis):
    f = np.moveaxis(f, axis, 0)
    out = f[0::2].copy()
    out[:-1] += 0.5 * f[1::2]
    out[1:] += 0.5 * f[1::2]
    return np.moveaxis(out, 0, axis)


def restrict3d(xh, dh):
    """R = P^T of prolong3d."""
    nx, ny, nz = dh
    f = xh.reshape(nz, ny, nx)
    for ax in (2, 1, 0):
        f = _restrict_axis(f, ax)
    return f.ravel()


def v_cycle3d(r, levels):
    """One V-cycle from x = 0 in the pinned form of core/multigrid.py:231-330."""
    N = len(levels)
    rl, xl = [None] * N, [None] * N
    rl[0] = r.copy()
    for n in range(N - 1):
        L = levels[n]
        rh = rl[n].copy()
        rh[L.gp] = 0.0
        x = chebyshev(L, rh, None)
        t = rh - apply_A(L, x)
        t[L.gp] = 0.0
        xl[n] = x
        rl[n + 1] = restrict3d(t, L.dims)
    C = levels[-1]
    rc = rl[-1].copy()
    rc[C.gp] = 0.0
    xl[-1] = C.Ainv @ rc
    for n in range(N - 2, -1, -1):
        L = levels[n]
        x = xl[n] + prolong3d(xl[n + 1], levels[n + 1].dims, L.dims)
        x[L.gp] = 0.0
        rh = rl[n].copy()
        rh[L.gp] = 0.0
        xl[n] = chebyshev(L, rh, x)
    return xl[0]
