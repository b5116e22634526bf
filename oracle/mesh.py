"""Structured mesh generators (oracle restatement of setup/regular_mesh.py).

Node (i, j[, k]) -> k*nnx*nny + j*nnx + i; element connectivity counter-clockwise;
faces ordered [D, R, T, L(, F, B)]. Test infrastructure only.
"""
import numpy as np


def create_mesh_2d(nex, ney, lx, ly):
    """setup/regular_mesh.py:6-44 (quad4, non-periodic)."""
    nnx, nny = nex + 1, ney + 1
    dx, dy = lx / nex, ly / ney
    i, j = np.meshgrid(np.arange(nnx), np.arange(nny))
    node_coords = np.stack([i.ravel() * dx, j.ravel() * dy], axis=1)
    ie, je = np.meshgrid(np.arange(nex), np.arange(ney))
    ie, je = ie.ravel(), je.ravel()
    nconn = np.stack([je * nnx + ie, je * nnx + ie + 1, (je + 1) * nnx + ie + 1,
                      (je + 1) * nnx + ie], axis=1).astype(np.int64)
    surf = [np.arange(nnx), nnx * np.arange(1, nny + 1) - 1,
            nnx * (nny - 1) + np.arange(nnx), nnx * np.arange(nny)]
    bconns = [np.stack([s[:-1], s[1:]], axis=1) for s in surf]
    normals = np.array([[0, -1], [1, 0], [0, 1], [-1, 0]])
    nvecs = [np.tile(normals[f], (bconns[f].shape[0], 1)) for f in range(4)]
    return node_coords, nconn, surf, bconns, nvecs


def create_mesh_2d_quad9(nex, ney, lx, ly):
    """setup/regular_mesh.py:108-146 (quad9, non-periodic)."""
    nnx, nny = 2 * nex + 1, 2 * ney + 1
    dx, dy = lx / nex, ly / ney
    i, j = np.meshgrid(np.arange(nnx), np.arange(nny))
    node_coords = np.stack([i.ravel() * dx / 2, j.ravel() * dy / 2], axis=1)
    e = np.arange(nex * ney)
    ie, je = e % nex, e // nex
    nconn = np.stack([2 * ie + 2 * je * nnx, 2 * ie + 1 + 2 * je * nnx, 2 * ie + 2 + 2 * je * nnx,
                      2 * ie + 2 + (2 * je + 1) * nnx, 2 * ie + 2 + (2 * je + 2) * nnx,
                      2 * ie + 1 + (2 * je + 2) * nnx, 2 * ie + (2 * je + 2) * nnx,
                      2 * ie + (2 * je + 1) * nnx, 2 * ie + 1 + (2 * je + 1) * nnx],
                     axis=1).astype(np.int64)
    surf = [np.arange(0, nnx), np.arange(nnx - 1, nnx * nny, nnx),
            np.arange(nnx * (nny - 1), nnx * nny), np.arange(0, nnx * nny, nnx)]
    bconns = [np.stack([s[:-2:2], s[1:-1:2], s[2::2]], axis=1) for s in surf]
    normals = np.array([[0, -1], [1, 0], [0, 1], [-1, 0]])
    nvecs = [np.tile(normals[f], (bconns[f].shape[0], 1)) for f in range(4)]
    return node_coords, nconn, surf, bconns, nvecs


def create_periodic_mesh_2d(nex, ney, lx, ly):
    """setup/regular_mesh.py:150-181 (quad4, periodic; duplicate nodes dropped)."""
    nnx, nny = nex, ney
    dx, dy = lx / nex, ly / ney
    i, j = np.meshgrid(np.arange(nnx), np.arange(nny))
    node_coords = np.stack([i.ravel() * dx, j.ravel() * dy], axis=1)
    e = np.arange(nex * ney)
    ie, je = e % nex, e // nex
    nconn = np.stack([ie + je * nnx, (ie + 1) % nnx + je * nnx,
                      (ie + 1) % nnx + ((je + 1) % nny) * nnx, ie + ((je + 1) % nny) * nnx],
                     axis=1).astype(np.int64)
    return node_coords, nconn, None, None, None


def create_periodic_mesh_2d_quad9(nex, ney, lx, ly):
    """setup/regular_mesh.py:183-219 (quad9, periodic; duplicate nodes dropped)."""
    nnx, nny = 2 * nex, 2 * ney
    dx, dy = lx / nex, ly / ney
    i, j = np.meshgrid(np.arange(nnx), np.arange(nny))
    node_coords = np.stack([i.ravel() * dx / 2, j.ravel() * dy / 2], axis=1)
    e = np.arange(nex * ney)
    ie, je = e % nex, e // nex
    nconn = np.stack([2 * ie + 2 * je * nnx, 2 * ie + 1 + 2 * je * nnx,
                      (2 * ie + 2) % nnx + 2 * je * nnx, (2 * ie + 2) % nnx + (2 * je + 1) * nnx,
                      (2 * ie + 2) % nnx + ((2 * je + 2) % nny) * nnx,
                      2 * ie + 1 + ((2 * je + 2) % nny) * nnx, 2 * ie + ((2 * je + 2) % nny) * nnx,
                      2 * ie + (2 * je + 1) * nnx, 2 * ie + 1 + (2 * je + 1) * nnx],
                     axis=1).astype(np.int64)
    return node_coords, nconn, None, None, None


def create_mesh_3d(nex, ney, nez, lx, ly, lz):
    """setup/regular_mesh.py:46-104 (hex8)."""
    nnx, nny, nnz = nex + 1, ney + 1, nez + 1
    dx, dy, dz = lx / nex, ly / ney, lz / nez
    k, j, i = np.meshgrid(np.arange(nnz), np.arange(nny), np.arange(nnx), indexing="ij")
    node_coords = np.stack([i.ravel() * dx, j.ravel() * dy, k.ravel() * dz], axis=1)
    ke, je, ie = np.meshgrid(np.arange(nez), np.arange(ney), np.arange(nex), indexing="ij")
    ie, je, ke = ie.ravel(), je.ravel(), ke.ravel()
    base = [je * nnx + ie, je * nnx + ie + 1, (je + 1) * nnx + ie + 1, (je + 1) * nnx + ie]
    nconn = np.stack([ke * nnx * nny + b for b in base] + [(ke + 1) * nnx * nny + b for b in base],
                     axis=1).astype(np.int64)
    n3 = nconn.reshape(nez, ney, nex, 8)
    # Same index expressions as regular_mesh.py:73-78. Where the scalar and the
    # list index are separated by a slice (faces D, T, F, B) numpy/JAX advanced
    # indexing moves the list axis first, so those rows are NOT per-face quads;
    # bconns_3d_faces() gives the geometric face quads used by the 3D extension.
    bconns = [n3[:, 0, :, [0, 1, 5, 4]].reshape(-1, 4),
              n3[:, :, -1, [1, 5, 6, 2]].reshape(-1, 4),
              n3[:, -1, :, [3, 2, 6, 7]].reshape(-1, 4),
              n3[:, :, 0, [0, 4, 7, 3]].reshape(-1, 4),
              n3[0, :, :, [0, 1, 2, 3]].reshape(-1, 4),
              n3[-1, :, :, [4, 5, 6, 7]].reshape(-1, 4)]
    zoff = np.arange(nnz) * nnx * nny
    surf = [np.tile(np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(1, nny + 1) - 1, nnz) + np.repeat(zoff, nny),
            np.tile(nnx * (nny - 1) + np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(nny), nnz) + np.repeat(zoff, nny),
            np.arange(nnx * nny), nnx * nny * (nnz - 1) + np.arange(nnx * nny)]
    normals = np.array([[0, -1, 0], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, 0, -1], [0, 0, 1]])
    nvecs = [np.tile(normals[f], (bconns[f].shape[0], 1)) for f in range(6)]
    return node_coords, nconn, surf, bconns, nvecs


def bconns_3d_faces(nex, ney, nez):
    """Build-defined (no reference counterpart): geometric boundary quads of a
    hex8 box per face [D, R, T, L, F, B], each row one face quad (4 nodes)."""
    nnx, nny = nex + 1, ney + 1
    ke, je, ie = np.meshgrid(np.arange(nez), np.arange(ney), np.arange(nex), indexing="ij")
    base = [je * nnx + ie, je * nnx + ie + 1, (je + 1) * nnx + ie + 1, (je + 1) * nnx + ie]
    nconn = np.stack([ke * nnx * nny + b for b in base] + [(ke + 1) * nnx * nny + b for b in base],
                     axis=-1)
    return [nconn[:, 0, :][..., [0, 1, 5, 4]].reshape(-1, 4),
            nconn[:, :, -1][..., [1, 5, 6, 2]].reshape(-1, 4),
            nconn[:, -1, :][..., [3, 2, 6, 7]].reshape(-1, 4),
            nconn[:, :, 0][..., [0, 4, 7, 3]].reshape(-1, 4),
            nconn[0][..., [0, 1, 2, 3]].reshape(-1, 4),
            nconn[-1][..., [4, 5, 6, 7]].reshape(-1, 4)]
