"""hex8 geometric multigrid (the 3D extension of core/multigrid.py) through the
C ABI against the oracle (oracle/multigrid3d.py), FP64 unless stated.

Tolerances: one V-cycle 1e-12 relative (summation order, the tensor-product
operator and the device Gauss-Jordan inverse differ from the oracle's sparse
products and LAPACK inverse only by rounding); multigrid-PCG solves and NS
steps 1e-10 with equal iteration counts (the FP64 bar); the mixed-precision
solve (FP32 inner, FP64 refinement) 1e-6 against the FP64 solve."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

VCYCLE_TOL = 1e-12
SOLVE_TOL = 1e-10
MIXED_TOL = 1e-6

BOXES = [([16, 8, 8], [4, 2, 2]), ([32, 16, 16], [4, 2, 2])]


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)


def _gpu_hierarchy(ne, nef, outlet):
    from jax_fem_cfd_b200.context import Context, Mesh, KIND_HEX
    from jax_fem_cfd_b200.core import multigrid as mg
    mesh = Mesh(KIND_HEX, False, *ne, 4.0, 1.0, 1.0)
    ctx = Context(mesh)
    nlev = int(np.log2(ne[0] // nef[0])) + 1
    pins = mg.level_pin_sets(mesh, nlev, outlet, None, 1)
    from jax_fem_cfd_b200.context import make_mask
    ctx.set_bc(None, make_mask(pins[0], ctx.nn), True)
    H = mg.Hierarchy(ctx, nlev, pins, 1e-8)
    return ctx, H, pins


def _rhs(levels, seed):
    L0 = levels[0]
    b = np.random.default_rng(seed).standard_normal(L0.nn)
    b[L0.gp] = 0.0
    return b


@pytest.mark.parametrize("ne,nef", BOXES)
@pytest.mark.parametrize("outlet", [[1], []])
def test_vcycle_matches_oracle(ne, nef, outlet):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    from oracle import multigrid3d as m3
    levels = m3.multigrid3d_setup(ne, nef, [4.0, 1.0, 1.0], outlet)
    ctx, H, _ = _gpu_hierarchy(ne, nef, outlet)
    r = _rhs(levels, 3)
    z = torch.empty(ctx.nn, dtype=torch.float64, device="cuda")
    _lib.call("fem_mg_vcycle", ctx.handle, ptr(torch.as_tensor(r).cuda()), ptr(z), stream())
    zo = m3.v_cycle3d(r, levels)
    assert rel(z, zo) < VCYCLE_TOL, rel(z, zo)


@pytest.mark.parametrize("ne,nef", BOXES)
def test_mgpcg_matches_oracle(ne, nef):
    """The reference's CG (stop rule r.r <= tol^2 b.b, maxiter 1000) with the
    hex8 V-cycle as M: equal iteration counts, solutions to 1e-10."""
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    from oracle import multigrid3d as m3
    from oracle.solvers import cg
    levels = m3.multigrid3d_setup(ne, nef, [4.0, 1.0, 1.0], [1])
    ctx, H, _ = _gpu_hierarchy(ne, nef, [1])
    L0 = levels[0]
    b = _rhs(levels, 4)
    x0 = np.random.default_rng(5).standard_normal(L0.nn) * 1e-2
    x0[L0.gp] = 0.0
    xo, ito = cg(lambda v: m3.apply_A(L0, v), b, x0=x0, tol=1e-8, maxiter=1000, M=lambda v: m3.v_cycle3d(v, levels))
    x = torch.as_tensor(x0).cuda()
    iters = torch.zeros(1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # the second call replays the cached graph
        x = torch.as_tensor(x0).cuda()
        _lib.call("fem_pressure_solve", ctx.handle, ptr(torch.as_tensor(b).cuda()), ptr(x), 1e-8, 0.0, 1000,
                  _lib.PREC["multigrid"], 0, 1, ptr(iters), ptr(status), stream())
        torch.cuda.synchronize()
        assert int(status) == 0
        assert int(iters) == ito, (int(iters), ito)
        assert rel(x, xo) < SOLVE_TOL, rel(x, xo)
    assert 3 <= ito <= 12


@pytest.mark.parametrize("ne,nef", BOXES)
def test_mixed_solve_matches_fp64(ne, nef):
    """FP64 refinement around FP32 multigrid-PCG: within 1e-6 of the FP64 solve,
    relative residual below the tolerance, in a few cycles."""
    import ctypes
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    from oracle import multigrid3d as m3
    from oracle.solvers import cg
    levels = m3.multigrid3d_setup(ne, nef, [4.0, 1.0, 1.0], [1])
    L0 = levels[0]
    b = _rhs(levels, 6)
    xo, _ = cg(lambda v: m3.apply_A(L0, v), b, x0=np.zeros(L0.nn), tol=1e-12, maxiter=1000,
               M=lambda v: m3.v_cycle3d(v, levels))
    ctx, H, _ = _gpu_hierarchy(ne, nef, [1])
    lib = _lib.load()
    for inner in (4, 6):
        x = torch.zeros(ctx.nn, dtype=torch.float64, device="cuda")
        cycles, relres = ctypes.c_int(), ctypes.c_double()
        rc = lib.fem_pressure_solve_mixed(ctx.handle, ptr(torch.as_tensor(b).cuda()), ptr(x), 1e-8, inner, 10,
                                          ctypes.byref(cycles), ctypes.byref(relres), stream())
        assert rc == 0, lib.fem_last_error()
        assert relres.value <= 1e-8 and 1 <= cycles.value <= 4, (cycles.value, relres.value)
        assert rel(x, xo) < MIXED_TOL, rel(x, xo)


def _channel_cfg(mod, precond, nel, fm=None, precision=None):
    kw = {} if precision is None else {"precision": precision}
    return mod.Config(mesh="simple", solver="standard",
                      mesh_config=mod.SimpleMeshConfig(num_elem=nel, domain_size=[4.0, 1.0, 1.0], shape_func_ord=1,
                                                       periodic=False),
                      solver_config=mod.StandardSolverConfig(dirichlet_faces=[0, 2, 3, 4, 5], symmetry_faces=[],
                                                             outlet_faces=[1], streamline_diff=False, solver_tol=1e-8,
                                                             set_zeroP=True, pressure_precond=precond,
                                                             final_multigrid_mesh=fm, **kw))


def _run_channel(mod, cfg, steps):
    compute, timestep, nc, sn, h, nn, gd, Ud = mod.setup(cfg)
    ncn = nc.cpu().numpy() if isinstance(nc, torch.Tensor) else nc
    face = sn[3].cpu().numpy() if isinstance(sn[3], torch.Tensor) else sn[3]
    y, z = ncn[face, 1], ncn[face, 2]
    vals = 16 * y * (1 - y) * z * (1 - z)
    Ud = mod.set_face_velocity(Ud, sn[3], gd, torch.as_tensor(vals) if isinstance(nc, torch.Tensor) else vals, nn,
                               var=1)
    U, P = np.zeros(3 * nn), np.zeros(nn)
    its = []
    for s in range(steps):
        Fp, F = compute(Ud, None, s * 2e-3, (s + 1) * 2e-3)
        U, P, ui, pi = timestep(U, P, 2e-3, 1.0, 1.0 / 200, Ud, Fp, F)
        its.append((int(ui), int(pi)))
    return U, P, its


def test_channel_step_with_multigrid_matches_oracle():
    """The 3D channel (hex8 16 x 8 x 8, parabolic inflow, outlet, walls, Re 200,
    dt 2e-3) with the multigrid pressure solve: 3 fem_step4 steps vs the oracle."""
    import oracle.simulation as osim
    import jax_fem_cfd_b200.setup.simulation as gsim
    Ug, Pg, ig = _run_channel(gsim, _channel_cfg(gsim, "multigrid", [16, 8, 8], [4, 2, 2]), 3)
    Uo, Po, io = _run_channel(osim, _channel_cfg(osim, "multigrid", [16, 8, 8], [4, 2, 2]), 3)
    assert ig == io, (ig, io)
    assert rel(Ug, Uo) < SOLVE_TOL and rel(Pg, Po) < SOLVE_TOL, (rel(Ug, Uo), rel(Pg, Po))


def test_channel_step_mixed_matches_fp64():
    """The same channel with the mixed-precision pressure solve: 5 steps within
    1e-6 of the FP64 multigrid steps."""
    import jax_fem_cfd_b200.setup.simulation as gsim
    Uf, Pf, _ = _run_channel(gsim, _channel_cfg(gsim, "multigrid", [32, 8, 8], [8, 2, 2]), 5)
    Um, Pm, im = _run_channel(gsim, _channel_cfg(gsim, "multigrid", [32, 8, 8], [8, 2, 2], "mixed"), 5)
    assert all(1 <= p <= 4 for _, p in im), im
    assert rel(Um, Uf) < MIXED_TOL and rel(Pm, Pf) < MIXED_TOL, (rel(Um, Uf), rel(Pm, Pf))
