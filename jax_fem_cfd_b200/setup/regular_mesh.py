"""Structured meshes (drop-in for jax_fem_cfd setup/regular_mesh.py).

node_coords and nconn are generated on the device by fem_mesh_generate; the
returned nconn tensor carries its mesh descriptor (``nconn.fem_mesh``) so the
element-product entry points can use implicit connectivity. Face node lists,
boundary connectivities and normals are small index arrays built on the host."""
import numpy as np
import torch

from .. import _lib
from ..context import KIND_HEX, KIND_Q1, KIND_Q2, Mesh, device, i64, stream, ptr


def _generate(mesh):
    nn, ne, nen = mesh.counts()
    dim = mesh.ndim
    coords = torch.empty((nn, dim), dtype=torch.float64, device=device())
    nconn = torch.empty((ne, nen), dtype=torch.int64, device=device())
    d = mesh.desc()
    import ctypes
    _lib.call("fem_mesh_generate", ctypes.byref(d), ptr(coords), ptr(nconn), stream())
    nconn.fem_mesh = mesh
    return coords, nconn


def _dev(a):
    return i64(np.asarray(a))


def _faces_2d(nnx, nny, quad9):
    surf = [np.arange(nnx), nnx * np.arange(1, nny + 1) - 1, nnx * (nny - 1) + np.arange(nnx), nnx * np.arange(nny)]
    if quad9:
        bcs = [np.stack([s[:-2:2], s[1:-1:2], s[2::2]], axis=1) for s in surf]
    else:
        bcs = [np.stack([s[:-1], s[1:]], axis=1) for s in surf]
    normals = np.array([[0, -1], [1, 0], [0, 1], [-1, 0]])
    nv = [np.tile(normals[f], (bcs[f].shape[0], 1)) for f in range(4)]
    return surf, bcs, nv


def create_mesh_2d(num_elem_x, num_elem_y, domain_size_x, domain_size_y):
    """setup/regular_mesh.py:6 — quad4, node (i, j) -> j*nnx + i, faces [D, R, T, L]."""
    mesh = Mesh(KIND_Q1, False, int(num_elem_x), int(num_elem_y), 1, float(domain_size_x), float(domain_size_y))
    coords, nconn = _generate(mesh)
    surf, bcs, nv = _faces_2d(num_elem_x + 1, num_elem_y + 1, False)
    return coords, nconn, [_dev(s) for s in surf], [_dev(b) for b in bcs], [_dev(v) for v in nv]


def create_mesh_2d_quad9(nex, ney, Lx, Ly):
    """setup/regular_mesh.py:108 — quad9."""
    mesh = Mesh(KIND_Q2, False, int(nex), int(ney), 1, float(Lx), float(Ly))
    coords, nconn = _generate(mesh)
    surf, bcs, nv = _faces_2d(2 * nex + 1, 2 * ney + 1, True)
    return coords, nconn, [_dev(s) for s in surf], [_dev(b) for b in bcs], [_dev(v) for v in nv]


def create_periodic_mesh_2d(nex, ney, Lx, Ly):
    """setup/regular_mesh.py:150 — quad4, periodic (duplicate nodes dropped)."""
    coords, nconn = _generate(Mesh(KIND_Q1, True, int(nex), int(ney), 1, float(Lx), float(Ly)))
    return coords, nconn, None, None, None


def create_periodic_mesh_2d_quad9(nex, ney, Lx, Ly):
    """setup/regular_mesh.py:183 — quad9, periodic."""
    coords, nconn = _generate(Mesh(KIND_Q2, True, int(nex), int(ney), 1, float(Lx), float(Ly)))
    return coords, nconn, None, None, None


def hex_faces(nex, ney, nez):
    """Face node lists and geometric face quads of a hex8 box [D, R, T, L, F, B]
    (surface lists as regular_mesh.py:82-89; quads per face for the 3D flux)."""
    nnx, nny, nnz = nex + 1, ney + 1, nez + 1
    zoff = np.arange(nnz) * nnx * nny
    surf = [np.tile(np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(1, nny + 1) - 1, nnz) + np.repeat(zoff, nny),
            np.tile(nnx * (nny - 1) + np.arange(nnx), nnz) + np.repeat(zoff, nnx),
            np.tile(nnx * np.arange(nny), nnz) + np.repeat(zoff, nny),
            np.arange(nnx * nny), nnx * nny * (nnz - 1) + np.arange(nnx * nny)]
    ke, je, ie = np.meshgrid(np.arange(nez), np.arange(ney), np.arange(nex), indexing="ij")
    base = [je * nnx + ie, je * nnx + ie + 1, (je + 1) * nnx + ie + 1, (je + 1) * nnx + ie]
    nc = np.stack([ke * nnx * nny + b for b in base] + [(ke + 1) * nnx * nny + b for b in base], axis=-1)
    quads = [nc[:, 0, :][..., [0, 1, 5, 4]].reshape(-1, 4), nc[:, :, -1][..., [1, 5, 6, 2]].reshape(-1, 4),
             nc[:, -1, :][..., [3, 2, 6, 7]].reshape(-1, 4), nc[:, :, 0][..., [0, 4, 7, 3]].reshape(-1, 4),
             nc[0][..., [0, 1, 2, 3]].reshape(-1, 4), nc[-1][..., [4, 5, 6, 7]].reshape(-1, 4)]
    normals = np.array([[0, -1, 0], [1, 0, 0], [0, 1, 0], [-1, 0, 0], [0, 0, -1], [0, 0, 1]])
    nv = [np.tile(normals[f], (quads[f].shape[0], 1)) for f in range(6)]
    return surf, quads, nv


def create_mesh_3d(ne_x, ne_y, ne_z, domain_size_x, domain_size_y, domain_size_z):
    """setup/regular_mesh.py:46 — hex8. The reference's D/T/F/B bconn index
    expressions (:73-78) reorder axes; here every face's bconn row is one
    geometric face quad (the 3D boundary integral is build-defined)."""
    mesh = Mesh(KIND_HEX, False, int(ne_x), int(ne_y), int(ne_z), float(domain_size_x), float(domain_size_y),
                float(domain_size_z))
    coords, nconn = _generate(mesh)
    surf, quads, nv = hex_faces(ne_x, ne_y, ne_z)
    return coords, nconn, [_dev(s) for s in surf], [_dev(q) for q in quads], [_dev(v) for v in nv]


def mesh_of(nconn, nn=None):
    """The structured Mesh behind a connectivity tensor: the descriptor attached
    by the generators above, else recognised from the values of nconn (any of
    the five regular_mesh.py families). Unstructured connectivity raises."""
    m = getattr(nconn, "fem_mesh", None)
    if m is not None:
        return m
    cache = _INFER.get(id(nconn))
    if cache is not None and cache[0] is nconn:
        return cache[1]
    a = nconn.detach().cpu().numpy() if isinstance(nconn, torch.Tensor) else np.asarray(nconn)
    ne, nen = a.shape
    nn = int(nn) if nn is not None else int(a.max()) + 1
    cands = []
    if nen == 4:
        nnx = int(a[0, 3] - a[0, 0])
        if nnx > 1 and nn % nnx == 0:
            cands.append(Mesh(KIND_Q1, False, nnx - 1, nn // nnx - 1))
        nnx = int(a[0, 3])
        if nnx > 0 and nn % nnx == 0:
            cands.append(Mesh(KIND_Q1, True, nnx, nn // nnx))
    elif nen == 9:
        nnx = int(a[0, 3] - 2)
        if nnx > 2 and nn % nnx == 0:
            nny = nn // nnx
            if nnx % 2 == 1:
                cands.append(Mesh(KIND_Q2, False, (nnx - 1) // 2, (nny - 1) // 2))
            else:
                cands.append(Mesh(KIND_Q2, True, nnx // 2, nny // 2))
    elif nen == 8:
        nnx = int(a[0, 3] - a[0, 0])
        nnxy = int(a[0, 4] - a[0, 0])
        if nnx > 1 and nnxy % nnx == 0 and nn % nnxy == 0:
            cands.append(Mesh(KIND_HEX, False, nnx - 1, nnxy // nnx - 1, nn // nnxy - 1))
    for m in cands:
        if m.nex < 1 or m.ney < 1 or m.nez < 1:
            continue
        try:
            mnn, mne, men = m.counts()
        except _lib.FemError:
            continue
        if (mnn, mne, men) != (nn, ne, nen):
            continue
        _, ref = _generate(m)
        if torch.equal(ref.cpu(), torch.as_tensor(a)):
            _INFER[id(nconn)] = (nconn, m)
            return m
    raise ValueError("nconn is not one of the structured meshes of regular_mesh.py; "
                     "unstructured connectivity is not supported by the B200 path")


_INFER = {}
