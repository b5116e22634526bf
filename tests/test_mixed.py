"""Mixed-precision pressure-Poisson solve (FP64 refinement around an FP32
MG-PCG): its solution agrees with the FP64 MG-PCG solve and with the oracle
to 1e-6 (the mixed path's stated bound), its FP64 residual reaches the
tolerance, and it is deterministic; pinned quad4, and the graph-driven form
for quad9 / mean-zero pressure, also inside the NS step."""
import ctypes

import numpy as np
import pytest
import torch

from tests.test_gpu_parity import rel


def _poisson(n, seed=5):
    from jax_fem_cfd_b200.context import Context, Mesh, make_mask
    from jax_fem_cfd_b200.core import multigrid as gmg
    ctx = Context(Mesh(0, False, n, n, 1, 1.0, 1.0))
    ctx.set_bc(None, make_mask(np.array([0]), ctx.nn), True)
    nlev = int(np.log2(n // 4)) + 1
    gmg.Hierarchy(ctx, nlev, [np.array([0])] * nlev, 1e-8)
    b = np.random.default_rng(seed).standard_normal(ctx.nn)
    b[0] = 0.0
    return ctx, b


def _mixed(ctx, b, tol=1e-10, inner=6):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    bg = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bg)
    cyc, res = ctypes.c_int(0), ctypes.c_double(0.0)
    _lib.call("fem_pressure_solve_mixed", ctx.handle, ptr(bg), ptr(x), tol, inner, 20, ctypes.byref(cyc),
              ctypes.byref(res), stream())
    torch.cuda.synchronize()
    return x.cpu().numpy(), cyc.value, res.value


def _fp64(ctx, b):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    bg = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bg)
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("fem_pressure_solve", ctx.handle, ptr(bg), ptr(x), 1e-10, 0.0, 1000, _lib.PREC["multigrid"], 0, 1,
              ptr(it), ptr(st), stream())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return x.cpu().numpy()


@pytest.fixture(scope="module")
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [32, 128, 256])
def test_mixed_matches_fp64_and_is_deterministic(_cuda, n):
    ctx, b = _poisson(n)
    xm, cycles, res = _mixed(ctx, b)
    assert res <= 1e-10 and 1 <= cycles <= 6, (res, cycles)
    x64 = _fp64(ctx, b)
    assert rel(xm, x64) < 1e-6, rel(xm, x64)
    assert xm[0] == 0.0
    xm2, _, _ = _mixed(ctx, b)
    np.testing.assert_array_equal(xm, xm2)


@pytest.mark.gpu
def test_mixed_matches_the_oracle(_cuda):
    from oracle import element as oel, emult as oem, mesh as om, multigrid as omg, shape as osh, solvers as osv
    n = 64
    ctx, b = _poisson(n, seed=8)
    xm, _, _ = _mixed(ctx, b)
    nc, nconn, *_ = om.create_mesh_2d(n, n, 1.0, 1.0)
    wq, N, Nd = osh.quad4_shape_functions(nc[nconn[0]])
    Le = oel.laplacian_element_calc(wq, Nd)
    data = omg.multigrid_setup([n, n], [4, 4], [1.0, 1.0], [], om.create_mesh_2d, osh.quad4_shape_functions, 1, None)

    def lhs(v):
        y = oem.laplacian_element_mult(v, Le, nconn, nc.shape[0])
        y[0] = 0.0
        return y

    xo, _ = osv.cg(lhs, b, x0=np.zeros_like(b), tol=1e-10, maxiter=1000,
                   M=lambda r: omg.v_cycle(r, *data, 1e-8, False, True))
    xo = xo.copy()
    xo[0] = 0.0
    assert rel(xm, xo) < 1e-6, rel(xm, xo)


def _poisson_q2_periodic(n, seed=6):
    """Q2 periodic lattice on [0, 2 pi]^2 with mean-zero pressure, hierarchy down to 4 x 4 elements."""
    from jax_fem_cfd_b200.context import Context, Mesh, make_mask
    from jax_fem_cfd_b200.core import multigrid as gmg
    ctx = Context(Mesh(1, True, n, n, 1, 2 * np.pi, 2 * np.pi))
    ctx.set_bc(None, make_mask(np.array([0]), ctx.nn), False)
    nlev = int(np.log2(n // 4)) + 1
    gmg.Hierarchy(ctx, nlev, [np.array([0])] * nlev, 1e-8)
    b = np.random.default_rng(seed).standard_normal(ctx.nn)
    return ctx, b - b.mean()


def _fp64_mean_zero(ctx, b):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    bg = torch.as_tensor(b, device="cuda")
    x = torch.zeros_like(bg)
    it = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("fem_pressure_solve", ctx.handle, ptr(bg), ptr(x), 1e-10, 0.0, 1000, _lib.PREC["multigrid"], 1, 1,
              ptr(it), ptr(st), stream())
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return x.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 64])
def test_mixed_q2_periodic_mean_zero_matches_fp64(_cuda, n):
    """quad9 on a periodic lattice with mean-zero pressure (the Taylor-Green
    pressure problem): the graph-driven solve (FP32 Chebyshev multigrid-PCG
    inside FP64 refinement, solution centred) agrees with the FP64 solve."""
    ctx, b = _poisson_q2_periodic(n)
    xm, cycles, res = _mixed(ctx, b, tol=1e-10, inner=4)
    assert res <= 1e-10 and 1 <= cycles <= 8, (res, cycles)
    x64 = _fp64_mean_zero(ctx, b)
    assert abs(xm.mean()) <= 1e-12 * np.abs(xm).max()
    assert rel(xm, x64) < 1e-6, rel(xm, x64)
    xm2, _, _ = _mixed(ctx, b, tol=1e-10, inner=4)
    np.testing.assert_array_equal(xm, xm2)


def _tg_mixed_cfg(mod, n, precision=None, tol=None):
    from bench import tg_config
    cfg = tg_config(mod, n)
    if precision:
        cfg.solver_config.precision = precision
    if tol is not None:
        cfg.solver_config.solver_tol = tol
    return cfg


@pytest.mark.gpu
def test_taylor_green_mixed_steps_match_the_oracle(_cuda):
    """Ten 4-step projection steps of the periodic quad9 Taylor-Green vortex
    (32 x 32 elements, nu 0.01, dt 1e-3) with the mixed-precision solves
    (FP64 refinement to 1e-10), against the oracle's FP64 steps solved to
    1e-12: velocity and pressure within 1e-6. (Two solves that both stop at a
    relative residual of 1e-8 differ by up to the pressure operator's condition
    number times 1e-8, a few 1e-6 here, whatever their precision.)"""
    import oracle.simulation as osim
    import jax_fem_cfd_b200.setup.simulation as gsim
    from bench import tg_initial
    res = []
    for mod, prec in ((gsim, "mixed"), (osim, None)):
        compute, timestep, nc, *_ = mod.setup(_tg_mixed_cfg(mod, 32, prec, 1e-10 if prec else 1e-12))
        ncn = nc.cpu().numpy() if isinstance(nc, torch.Tensor) else np.asarray(nc)
        U, P = tg_initial(ncn)
        U, P = np.asarray(U), np.asarray(P)
        for _ in range(10):
            U, P, ui, pi = timestep(U, P, 1e-3, 1.0, 0.01, None, 0.0, 0.0)
        res.append((np.asarray(U.cpu() if isinstance(U, torch.Tensor) else U),
                    np.asarray(P.cpu() if isinstance(P, torch.Tensor) else P)))
    (Um, Pm), (Uo, Po) = res
    assert rel(Um, Uo) < 1e-6 and rel(Pm, Po) < 1e-6, (rel(Um, Uo), rel(Pm, Po))


@pytest.mark.gpu
def test_cavity_mixed_steps_match_fp64(_cuda):
    """The 64 x 64 quad4 lid-driven cavity (Dirichlet walls: the momentum
    solve's identity rows) over 20 steps with both solves in mixed precision
    (FP64 refinement to 1e-10), against the FP64 steps solved to 1e-12: within
    1e-6, a few refinement cycles per solve."""
    import jax_fem_cfd_b200.setup.simulation as gsim
    from jax_fem_cfd_b200.serving import cavity_config
    out = []
    for prec in ("fp64", "mixed"):
        cfg = cavity_config(64, prec)
        cfg.solver_config.solver_tol = 1e-12 if prec == "fp64" else 1e-10
        compute, timestep, nc, sn, h, nn, gd, Ud = gsim.setup(cfg)
        Ud = gsim.set_face_velocity(Ud, sn[2], gd, 1.0, nn, var=1)
        U = torch.zeros(2 * nn, dtype=torch.float64, device="cuda")
        P = torch.zeros(nn, dtype=torch.float64, device="cuda")
        its = []
        for s in range(20):
            Fp, F = compute(Ud, None, s * 0.01, (s + 1) * 0.01)
            U, P, ui, pi = timestep(U, P, 0.01, 1.0, 0.01, Ud, Fp, F)
            its.append((int(ui), int(pi)))
        assert int(timestep.solver.status.max()) == 0
        out.append((U.cpu().numpy(), P.cpu().numpy(), its))
    (Uf, Pf, _), (Um, Pm, im) = out
    assert all(1 <= u <= 8 and 1 <= p <= 8 for u, p in im), im
    assert rel(Um, Uf) < 1e-6 and rel(Pm, Pf) < 1e-6, (rel(Um, Uf), rel(Pm, Pf))


@pytest.mark.gpu
def test_taylor_green_mixed_500_steps_match_the_oracle(_cuda):
    """The Taylor-Green vortex over the config's 500 steps (quad9 16 x 16,
    nu 0.01, dt 1e-3) with both solves in mixed precision (FP64 refinement to
    1e-10), against the oracle's FP64 steps solved to 1e-12: within 1e-6."""
    import oracle.simulation as osim
    import jax_fem_cfd_b200.setup.simulation as gsim
    from bench import tg_initial
    res = []
    for mod, prec in ((gsim, "mixed"), (osim, None)):
        compute, timestep, nc, *_ = mod.setup(_tg_mixed_cfg(mod, 16, prec, 1e-10 if prec else 1e-12))
        ncn = nc.cpu().numpy() if isinstance(nc, torch.Tensor) else np.asarray(nc)
        U, P = tg_initial(ncn)
        U, P = np.asarray(U), np.asarray(P)
        for _ in range(500):
            U, P, ui, pi = timestep(U, P, 1e-3, 1.0, 0.01, None, 0.0, 0.0)
        res.append((np.asarray(U.cpu() if isinstance(U, torch.Tensor) else U),
                    np.asarray(P.cpu() if isinstance(P, torch.Tensor) else P)))
    (Um, Pm), (Uo, Po) = res
    assert rel(Um, Uo) < 1e-6 and rel(Pm, Po) < 1e-6, (rel(Um, Uo), rel(Pm, Po))
