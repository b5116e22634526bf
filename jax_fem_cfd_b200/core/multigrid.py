"""Geometric multigrid (drop-in for core/multigrid.py).

multigrid_setup returns the reference's tuple (lvl_nums, Le_lvls, nconn_lvls,
L_diag_lvls, gamma_p_lvls) plus a device hierarchy handle; v_cycle runs one
V-cycle as a single persistent cooperative kernel (coarse levels inside one CTA)."""
import math

import numpy as np
import torch

from .. import _lib
from ..context import Context, Mesh, empty, f64, make_mask, ptr, stream
from ..setup.regular_mesh import mesh_of


def level_meshes(mesh: Mesh, nlev):
    if mesh.ndim == 3:
        return [Mesh(mesh.kind, False, mesh.nex >> l, mesh.ney >> l, mesh.nez >> l, mesh.lx, mesh.ly, mesh.lz)
                for l in range(nlev)]
    return [Mesh(mesh.kind, mesh.periodic, mesh.nex >> l, mesh.ney >> l, 1, mesh.lx, mesh.ly) for l in range(nlev)]


def _face_nodes_3d(m: Mesh):
    """Node lists of the hex8 faces [D, R, T, L, F, B] (setup/regular_mesh.py:80-96)."""
    nnx, nny, nnz = m.nex + 1, m.ney + 1, m.nez + 1
    zoff = np.arange(nnz) * nnx * nny
    return [np.tile(np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(1, nny + 1) - 1, nnz) + np.repeat(zoff, nny),
            np.tile(nnx * (nny - 1) + np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(nny), nnz) + np.repeat(zoff, nny),
            np.arange(nnx * nny), nnx * nny * (nnz - 1) + np.arange(nnx * nny)]


def _face_nodes_2d(m: Mesh):
    s = 2 if m.kind == 1 else 1
    nnx, nny = s * m.nex + 1, s * m.ney + 1
    return [np.arange(nnx), nnx * np.arange(1, nny + 1) - 1, nnx * (nny - 1) + np.arange(nnx), nnx * np.arange(nny)]


def level_pin_sets(mesh: Mesh, nlev, outlet_faces, partial_dirichlet, shape_func_ord):
    """gamma_p of every level (core/multigrid.py:35-62): outlet face nodes plus
    partial-Dirichlet remainders; [0] when there are none. hex8 meshes (the 3D
    extension) take the outlet faces of each level's box."""
    out = []
    for m in level_meshes(mesh, nlev):
        nodes = []
        surf = None if m.periodic else (_face_nodes_3d(m) if m.ndim == 3 else _face_nodes_2d(m))
        if outlet_faces:
            for f in outlet_faces:
                nodes.append(surf[f])
        if partial_dirichlet:
            for f, (s0, e0, kind) in partial_dirichlet.items():
                fn = surf[f]
                nfe = (len(fn) - 1) // (2 if shape_func_ord == 2 else 1)
                si, ei = round(s0 * nfe), round(e0 * nfe)
                if shape_func_ord == 2:
                    si, ei = 2 * si, 2 * ei
                if kind == "outlet":
                    nodes.append(fn[:si])
                    nodes.append(fn[ei + 1:])
        out.append(np.unique(np.concatenate(nodes)) if nodes else np.array([0]))
    return out


class Hierarchy:
    """Device multigrid hierarchy of a context (fem_ctx_setup_multigrid)."""

    def __init__(self, ctx: Context, nlev, pin_sets, coarse_tol):
        self.ctx, self.nlev = ctx, nlev
        masks = [make_mask(p, m.counts()[0]) for p, m in zip(pin_sets, level_meshes(ctx.mesh, nlev))]
        cat = torch.cat(masks)
        ctx.setup_multigrid(nlev, cat, coarse_tol)
        self._masks = cat
        self.coarse_tol = float(coarse_tol)
        self.set_zeroP = None
        self.lvl_nums = self._lvl_nums(pin_sets)

    def _lvl_nums(self, pin_sets):
        rows = [[0, 0, 0, 0, 0]]
        for l in range(self.nlev):
            nn, nnx, nny, nex, ney = self.ctx.level_info(l)
            p = rows[-1]
            rows.append([p[0] + nn, nnx, nny, p[3] + nex * ney, p[4] + len(pin_sets[l])])
        return tuple(tuple(r) for r in rows)


def multigrid_setup(num_elem, num_elemf, domain_size, outlet_faces, mesh_func, shapefunc, shape_func_ord,
                    partial_dirichlet):
    """core/multigrid.py:9: levels N = log2(nex / nexf) + 1. Returns (lvl_nums,
    Le_lvls, nconn_lvls, L_diag_lvls, gamma_p_lvls); the device hierarchy is
    attached to nconn_lvls as ``fem_hierarchy``."""
    nex, ney = num_elem
    N = int(math.log2(nex // num_elemf[0])) + 1
    coords, nconn, *_ = mesh_func(nex, ney, *domain_size)
    mesh = mesh_of(nconn)
    ctx = Context(mesh)
    pins = level_pin_sets(mesh, N, outlet_faces, partial_dirichlet, shape_func_ord)
    H = Hierarchy(ctx, N, pins, 1e-8)
    nen = ctx.nen
    Le_lvls = torch.zeros((N, 2, nen, nen), dtype=torch.float64, device=coords.device)
    diags, nconns = [], []
    from . import element_calc as ec
    from .shape_functions import quad4_shape_functions, quad9_shape_functions
    sf = quad4_shape_functions if shape_func_ord == 1 else quad9_shape_functions
    for l, m in enumerate(level_meshes(mesh, N)):
        c, nc, *_ = mesh_func(m.nex, m.ney, *domain_size)
        wq, Nq, dN = sf(c[nc[0]])
        _, Le, Le_off, _ = ec._matrices(wq, Nq, dN)
        Le_lvls[l, 0] = Le
        Le_lvls[l, 1] = Le_off
        diags.append(ec.laplacian_diag(Le, nc, c.shape[0]))
        nconns.append(nc)
    gp = torch.as_tensor(np.concatenate(pins)).to(coords.device)
    nconn_lvls = torch.cat(nconns)
    nconn_lvls.fem_hierarchy = H
    return H.lvl_nums, Le_lvls, nconn_lvls, torch.cat(diags), gp


def interpolation_operator(xH, nnH_x, nnH_y, nnh_x, nnh_y, periodic):
    """core/multigrid.py:90: lattice-bilinear prolongation."""
    n = (nnh_x - 1) * (nnh_y - 1) if periodic else nnh_x * nnh_y
    out = empty(n)
    _lib.call("fem_lattice_interpolate", int(nnH_x), int(nnH_y), int(nnh_x), int(nnh_y), int(bool(periodic)),
              ptr(f64(xH)), ptr(out), stream())
    return out


def restriction_operator(xh, nnh_x, nnh_y, nnH_x, nnH_y, periodic):
    """core/multigrid.py:142: R = I^T, no 1/4 factor."""
    n = (nnH_x - 1) * (nnH_y - 1) if periodic else nnH_x * nnH_y
    out = empty(n)
    _lib.call("fem_lattice_restrict", int(nnh_x), int(nnh_y), int(nnH_x), int(nnH_y), int(bool(periodic)),
              ptr(f64(xh)), ptr(out), stream())
    return out


def v_cycle(rhs, lvl_nums, Le_lvls, nconn_lvls, L_diag_lvls, gamma_p_lvls, tol, periodic, set_zeroP):
    """core/multigrid.py:231: one V-cycle from x = 0 as a single persistent
    kernel. The device hierarchy travels on nconn_lvls (set by multigrid_setup)."""
    H = getattr(nconn_lvls, "fem_hierarchy", None)
    if H is None:
        raise ValueError("nconn_lvls must come from jax_fem_cfd_b200 multigrid_setup")
    ctx = H.ctx
    if H.coarse_tol != float(tol):
        ctx.setup_multigrid(H.nlev, H._masks, float(tol))
        H.coarse_tol = float(tol)
    if H.set_zeroP != bool(set_zeroP):
        ctx.set_bc(None, H._masks[:ctx.nn], bool(set_zeroP))
        H.set_zeroP = bool(set_zeroP)
    z = empty(ctx.nn)
    _lib.call("fem_mg_vcycle", ctx.handle, ptr(f64(rhs)), ptr(z), stream())
    return z
