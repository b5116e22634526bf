"""fem_boundary_flux_noalloc against fem_boundary_flux, through the C ABI.

The no-allocation entry point serves callers that must not allocate device
memory during a call, for example a host framework that hands out every device
byte through its own allocator. It keeps its per-face scratch in a fixed array
inside the library instead of in the context. Both entry points evaluate the
faces with the same kernel and sum each node's entries in face order, so on
the same inputs they agree bit for bit (the test allows relative 1e-14). Two
calls in a row check that reusing the shared array, which keeps the first
call's values, still gives correct results; a free-memory reading before and
after further calls checks that they allocate nothing.

This file is collected last, so a run that stops at the first failure has run
every other test before it."""
import ctypes
import os
import re

import numpy as np
import pytest
import torch

from tests.conftest import ROOT

pytestmark = pytest.mark.gpu

TOL = 1e-14


def _face_limit():
    with open(os.path.join(ROOT, "include", "fem_b200.h")) as f:
        return int(re.search(r"#define FEM_NOALLOC_FACE_VALUES (\d+)", f.read()).group(1))


def _channel_solver(order):
    import jax_fem_cfd_b200.setup.simulation as gsim
    cfg = gsim.Config(mesh="simple", solver="standard",
                      mesh_config=gsim.SimpleMeshConfig(num_elem=[16, 8], domain_size=[2.0, 1.0],
                                                        shape_func_ord=order, periodic=False),
                      solver_config=gsim.StandardSolverConfig(dirichlet_faces=[0, 2, 3], symmetry_faces=[],
                                                              outlet_faces=[1], streamline_diff=False,
                                                              solver_tol=1e-8, set_zeroP=True,
                                                              pressure_precond="jacobi", final_multigrid_mesh=None))
    compute, timestep, nc, sn, h, nn, gd, Ud = gsim.setup(cfg)
    return timestep.solver, nn


def _flux(name, solver, bconn, nvec, U_full, nn):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    F = torch.full((nn,), float("nan"), dtype=torch.float64, device="cuda")
    _lib.call(name, solver.ctx.handle, ptr(bconn), ptr(nvec), int(bconn.shape[0]), int(bconn.shape[1]),
              ptr(U_full), ptr(F), stream())
    return F


def _rel(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)


@pytest.mark.parametrize("order", [1, 2])
def test_noalloc_flux_matches_two_calls_in_a_row(order):
    solver, nn = _channel_solver(order)
    g = torch.Generator().manual_seed(7 + order)
    # call 1: every Dirichlet face, a random boundary velocity
    U1 = torch.randn(solver.ndim * nn, generator=g, dtype=torch.float64).cuda()
    ref1 = _flux("fem_boundary_flux", solver, solver.bconn, solver.nvec, U1, nn)
    got1 = _flux("fem_boundary_flux_noalloc", solver, solver.bconn, solver.nvec, U1, nn)
    # call 2: half the faces and another velocity; the shared scratch still
    # holds call 1's values past the new faces' range
    half = solver.bconn.shape[0] // 2
    b2 = solver.bconn[:half].contiguous()
    n2 = solver.nvec.view(solver.bconn.shape[0], -1)[:half].reshape(-1).contiguous()
    U2 = torch.randn(solver.ndim * nn, generator=g, dtype=torch.float64).cuda()
    ref2 = _flux("fem_boundary_flux", solver, b2, n2, U2, nn)
    got2 = _flux("fem_boundary_flux_noalloc", solver, b2, n2, U2, nn)
    torch.cuda.synchronize()
    assert torch.isfinite(got1).all() and torch.isfinite(got2).all()
    assert _rel(got1, ref1) < TOL, _rel(got1, ref1)
    assert _rel(got2, ref2) < TOL, _rel(got2, ref2)
    assert _rel(ref1, ref2) > 1e-3  # the two calls really differ


def test_noalloc_flux_rejects_more_faces_than_its_scratch():
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    solver, nn = _channel_solver(1)
    lib = _lib.load()
    F = torch.zeros(nn, dtype=torch.float64, device="cuda")
    U = torch.zeros(solver.ndim * nn, dtype=torch.float64, device="cuda")
    nb = _face_limit() // 2 + 1  # lin2 faces: nb * 2 values, one face past the limit
    # the size check runs on the host before anything is launched, so the
    # (smaller) face arrays passed here are never read
    rc = lib.fem_boundary_flux_noalloc(solver.ctx.handle, ptr(solver.bconn), ptr(solver.nvec), nb, 2, ptr(U),
                                       ptr(F), stream())
    assert rc == -1
    assert b"exceeds the fixed scratch" in lib.fem_last_error()
    torch.cuda.synchronize()
    assert float(F.abs().max()) == 0.0


def test_noalloc_calls_allocate_no_device_memory():
    solver, nn = _channel_solver(1)
    g = torch.Generator().manual_seed(11)
    U = torch.randn(solver.ndim * nn, generator=g, dtype=torch.float64).cuda()
    ref = _flux("fem_boundary_flux", solver, solver.bconn, solver.nvec, U, nn)
    F = torch.empty(nn, dtype=torch.float64, device="cuda")
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream

    def call():
        _lib.call("fem_boundary_flux_noalloc", solver.ctx.handle, ptr(solver.bconn), ptr(solver.nvec),
                  int(solver.bconn.shape[0]), int(solver.bconn.shape[1]), ptr(U), ptr(F), stream())

    call()  # the first call on the device looks up the library's scratch
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        call()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, (free0, free1)
    assert _rel(F, ref) < TOL


def test_bad_node_index_is_skipped_and_reported_by_both_entry_points():
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    solver, nn = _channel_solver(2)
    lib = _lib.load()
    g = torch.Generator().manual_seed(5)
    U = torch.randn(solver.ndim * nn, generator=g, dtype=torch.float64).cuda()
    nb = solver.bconn.shape[0]
    bad = solver.bconn.clone()
    bad[3, 1] = nn + 5  # one node id past the mesh
    nv = solver.nvec.view(nb, -1)
    keep = [f for f in range(nb) if f != 3]
    b_ok = solver.bconn[keep].contiguous()
    n_ok = nv[keep].reshape(-1).contiguous()
    ref = _flux("fem_boundary_flux", solver, b_ok, n_ok, U, nn)
    for name in ("fem_boundary_flux", "fem_boundary_flux_noalloc"):
        got = _flux(name, solver, bad, solver.nvec, U, nn)
        cnt = ctypes.c_int(-1)
        assert lib.fem_boundary_flux_skipped(solver.ctx.handle, ctypes.byref(cnt), stream()) == 0
        assert cnt.value == 1, (name, cnt.value)
        assert torch.equal(got, ref), name
    _flux("fem_boundary_flux_noalloc", solver, solver.bconn, solver.nvec, U, nn)
    cnt = ctypes.c_int(-1)
    assert lib.fem_boundary_flux_skipped(solver.ctx.handle, ctypes.byref(cnt), stream()) == 0
    assert cnt.value == 0
