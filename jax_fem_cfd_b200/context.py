"""Device contexts, mesh descriptors and tensor plumbing over the C ABI.

torch provides device memory and the current stream; every arithmetic step is a
libfemb200 kernel. A context owns the mesh-resident element data and solver
workspace of one structured mesh (setup/regular_mesh.py lattices)."""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import FemError

KIND_Q1, KIND_Q2, KIND_HEX = _lib.FEM_KIND_Q1_2D, _lib.FEM_KIND_Q2_2D, _lib.FEM_KIND_HEX8


def require_cuda():
    if not torch.cuda.is_available():
        raise FemError("jax_fem_cfd_b200 needs a CUDA device (B200, sm_100a); there is no CPU fallback")


def device():
    require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _from_dlpack(x):
    """Zero-copy torch view of a foreign DLPack producer (e.g. a JAX array)."""
    if not isinstance(x, (torch.Tensor, np.ndarray)) and hasattr(x, "__dlpack__"):
        return torch.from_dlpack(x)
    return x


def f64(x):
    """Contiguous float64 CUDA tensor view/copy of x (numpy, list, scalar, tensor
    or DLPack producer)."""
    x = _from_dlpack(x)
    if isinstance(x, torch.Tensor):
        if x.device.type != "cuda":
            x = x.to(device(), non_blocking=True)
        if x.dtype != torch.float64:
            x = x.to(torch.float64)
        return x.contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.float64)).to(device()).contiguous()


def i64(x):
    x = _from_dlpack(x)
    if isinstance(x, torch.Tensor):
        if x.device.type != "cuda":
            x = x.to(device())
        return x.to(torch.int64).contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.int64)).to(device()).contiguous()


def empty(n, dtype=torch.float64):
    return torch.empty(n, dtype=dtype, device=device())


@dataclass(frozen=True)
class Mesh:
    """Structured mesh of regular_mesh.py: kind, periodicity, element counts, box."""
    kind: int
    periodic: bool
    nex: int
    ney: int
    nez: int = 1
    lx: float = 1.0
    ly: float = 1.0
    lz: float = 1.0

    def desc(self):
        return _lib.MeshDesc(self.kind, int(self.periodic), self.nex, self.ney, self.nez, self.lx, self.ly, self.lz)

    def counts(self):
        nn, ne, nen = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        d = self.desc()
        _lib.call("fem_mesh_counts", ctypes.byref(d), ctypes.byref(nn), ctypes.byref(ne), ctypes.byref(nen))
        return nn.value, ne.value, nen.value

    @property
    def ndim(self):
        return 3 if self.kind == KIND_HEX else 2

    @property
    def lattice(self):
        """Full lattice extents (nnx, nny) incl. the periodic duplicate (lvl_nums entries)."""
        s = 2 if self.kind == KIND_Q2 else 1
        return s * self.nex + 1, s * self.ney + 1


class Context:
    """Owns a fem_ctx: element data, boundary sets, multigrid hierarchy, workspace."""

    def __init__(self, mesh: Mesh):
        require_cuda()
        _lib.load()
        self.mesh = mesh
        self.dev = device()
        h = ctypes.c_void_p()
        d = mesh.desc()
        _lib.call("fem_ctx_create", ctypes.byref(d), self.dev.index or 0, ctypes.byref(h))
        self.handle = h
        dims = [ctypes.c_int() for _ in range(5)]
        _lib.call("fem_ctx_dims", h, *[ctypes.byref(x) for x in dims])
        self.nn, self.ne, self.nen, self.ndim, self.nq = [x.value for x in dims]
        self.nlev = 1
        self._edata = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize()
                _lib.load().fem_ctx_destroy(h)
            except Exception:
                pass
            self.handle = None

    def element_data(self):
        """(wq, N, Nderiv, Me, Le, Ge, M_lumped, L_diag) device tensors."""
        if self._edata is None:
            nq, nen, nd, nn = self.nq, self.nen, self.ndim, self.nn
            wq, N, dN = empty(nq), empty(nq * nen), empty(nq * nd * nen)
            Me, Le, Ge = empty(nen * nen), empty(nen * nen), empty(nd * nen * nen)
            M, Ld = empty(nd * nn), empty(nn)
            _lib.call("fem_ctx_element_data", self.handle, ptr(wq), ptr(N), ptr(dN), ptr(Me), ptr(Le), ptr(Ge),
                      ptr(M), ptr(Ld), stream())
            self._edata = (wq.view(nq, 1), N.view(nq, nen), dN.view(nq, nd, nen), Me.view(nen, nen),
                           Le.view(nen, nen), Ge.view(nd, nen, nen), M, Ld)
        return self._edata

    def set_bc(self, dmask, pmask, set_zeroP):
        self._dmask, self._pmask = dmask, pmask
        _lib.call("fem_ctx_set_bc", self.handle, ptr(dmask), ptr(pmask), int(bool(set_zeroP)), stream())

    def setup_multigrid(self, nlev, level_pmasks, coarse_tol):
        torch.cuda.current_stream().synchronize()
        _lib.call("fem_ctx_setup_multigrid", self.handle, int(nlev), ptr(level_pmasks), float(coarse_tol),
                  stream())
        self.nlev = nlev

    def level_info(self, level):
        v = [ctypes.c_int() for _ in range(5)]
        _lib.call("fem_ctx_level_info", self.handle, level, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)


_CTX_CACHE = {}


def context_for(mesh: Mesh) -> Context:
    """Shared per-mesh context for the standalone element-product entry points."""
    ctx = _CTX_CACHE.get(mesh)
    if ctx is None:
        if len(_CTX_CACHE) > 16:
            _CTX_CACHE.clear()
        ctx = _CTX_CACHE[mesh] = Context(mesh)
    return ctx


def make_mask(idx, length):
    """uint8 device mask with ones at idx (int indices)."""
    m = torch.empty(int(length), dtype=torch.uint8, device=device())
    if idx is None:
        _lib.call("fem_make_mask", None, 0, int(length), ptr(m), stream())
        return m
    ix = i64(idx)
    _lib.call("fem_make_mask", ptr(ix), int(ix.numel()), int(length), ptr(m), stream())
    return m


def scatter_set(out, idx, vals):
    """out.at[idx].set(vals) in place (vals tensor or scalar)."""
    ix = i64(idx)
    if isinstance(vals, (int, float)):
        _lib.call("fem_scatter", ptr(ix), None, float(vals), int(ix.numel()), ptr(out), stream())
    else:
        v = f64(vals).reshape(-1)
        if v.numel() == 1 and ix.numel() != 1:
            v = v.expand(ix.numel()).contiguous()
        _lib.call("fem_scatter", ptr(ix), ptr(v), 0.0, int(ix.numel()), ptr(out), stream())
    return out
