"""Adjoint of the projection stage (jax_fem_cfd_b200.solvers.adjoint.Projection)
against central finite differences of the forward stage on a wall-bounded
cavity: the stage is affine in U*, so the difference quotient is exact up to
the pressure solve's tolerance."""
import numpy as np
import pytest
import torch


@pytest.fixture(scope="module")
def cavity():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from jax_fem_cfd_b200.serving import cavity_config
    from jax_fem_cfd_b200.setup import simulation as sim
    _, timestep, *rest = sim.setup(cavity_config(16))
    solver = timestep.solver
    return solver, solver.u_full(rest[-1])


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_projection_vjp_matches_finite_differences(cavity, seed):
    from jax_fem_cfd_b200.solvers.adjoint import Projection
    solver, ud = cavity
    n2, n = solver.ndim * solver.nn, solver.nn
    rng = np.random.default_rng(seed)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Us, gU, gP, dlt = t(rng.standard_normal(n2)), t(rng.standard_normal(n2)), t(rng.standard_normal(n)), \
        t(rng.standard_normal(n2))
    dt, rho = 0.01, 1.0

    def loss(u):
        U, P = Projection.apply(u, solver, dt, rho, ud, None, 1e-13)
        return float((gU * U).sum() + (gP * P).sum())

    x = Us.clone().requires_grad_(True)
    U, P = Projection.apply(x, solver, dt, rho, ud, None, 1e-13)
    ((gU * U).sum() + (gP * P).sum()).backward()
    g = x.grad.clone()
    eps = 1e-2
    fd = (loss(Us + eps * dlt) - loss(Us - eps * dlt)) / (2 * eps)
    vjp = float((g * dlt).sum())
    assert abs(vjp - fd) <= 1e-7 * max(abs(fd), 1.0), (vjp, fd)
    # U is U_d on the Dirichlet rows whatever U* is: an output gradient carried
    # only there pulls back to zero
    dm = solver.dmask.to(torch.bool)
    x2 = Us.clone().requires_grad_(True)
    U2, P2 = Projection.apply(x2, solver, dt, rho, ud, None, 1e-13)
    (torch.where(dm, gU, torch.zeros_like(gU)) * U2).sum().backward()
    assert float(x2.grad.abs().max()) == 0.0


@pytest.mark.gpu
def test_projection_refuses_mean_zero_pressure():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bench import tg_config
    from jax_fem_cfd_b200.setup import simulation as sim
    from jax_fem_cfd_b200.solvers.adjoint import Projection
    _, timestep, *rest = sim.setup(tg_config(sim, 8))
    solver = timestep.solver
    u = torch.zeros(solver.ndim * solver.nn, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        Projection.apply(u, solver, 0.01, 1.0, None, None)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_momentum_solve_vjp_matches_finite_differences(cavity, seed):
    """The adjoint BiCGSTAB solve (transposed, non-symmetric Ce, Dirichlet
    identity rows turned into columns) against central differences."""
    from jax_fem_cfd_b200.core import element_calc as ec
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import MomentumSolve
    solver, _ = cavity
    n2 = solver.ndim * solver.nn
    rng = np.random.default_rng(10 + seed)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    wq, N, Nd = solver.ctx.element_data()[:3]
    Un = t(rng.standard_normal(n2))
    Ce = ec.conservative_convec_elem_calc(nconn, Un, wq, N, Nd, solver.nn, solver.ndim, 0.5)
    rhs, g, dlt = t(rng.standard_normal(n2)), t(rng.standard_normal(n2)), t(rng.standard_normal(n2))
    args = (solver, Ce, 1.0, 0.05, 0.01)

    def loss(r):
        return float((g * MomentumSolve.apply(r, *args)).sum())

    x = rhs.clone().requires_grad_(True)
    (g * MomentumSolve.apply(x, *args)).sum().backward()
    eps = 1e-2
    fd = (loss(rhs + eps * dlt) - loss(rhs - eps * dlt)) / (2 * eps)
    vjp = float((x.grad * dlt).sum())
    assert abs(vjp - fd) <= 1e-7 * max(abs(fd), 1.0), (vjp, fd)


@pytest.mark.gpu
def test_step_forward_matches_the_product_step(cavity):
    """Step's composed forward (explicit Ce, separate solves) reproduces fem_step4."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import Step
    from jax_fem_cfd_b200.serving import cavity_config
    from jax_fem_cfd_b200.setup import simulation as sim
    compute, timestep, *rest = sim.setup(cavity_config(16))
    solver, Ud = timestep.solver, rest[-1]
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    rng = np.random.default_rng(4)
    U0 = torch.as_tensor(rng.standard_normal(solver.ndim * solver.nn), device="cuda")
    P0 = torch.zeros(solver.nn, dtype=torch.float64, device="cuda")
    Fp, F = compute(Ud, None, 0.0, 0.01)
    U1, P1, _, _ = timestep(U0, P0, 0.01, 1.0, 0.05, Ud, Fp, F)
    U2, P2 = Step.apply(U0, P0, solver, nconn, 0.01, 1.0, 0.05, solver.u_full(Ud))
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    # the product step solves to its configured 1e-8 (Step to 1e-13): agreement to 1e-6
    assert rel(U2, U1) < 1e-6 and rel(P2, P1) < 1e-6, (rel(U2, U1), rel(P2, P1))


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["U", "P"])
def test_step_vjp_matches_finite_differences(cavity, which):
    """The adjoint of a whole time step (projection, adjoint momentum solve, rhs
    and operator dependence on U_n through Ce(U_n)) against central differences."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import Step
    solver, ud = cavity
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    n2, n = solver.ndim * solver.nn, solver.nn
    rng = np.random.default_rng(21)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    U0, P0 = t(0.5 * rng.standard_normal(n2)), t(rng.standard_normal(n))
    gU, gP = t(rng.standard_normal(n2)), t(rng.standard_normal(n))
    args = (solver, nconn, 0.01, 1.0, 0.05, ud)

    def loss(u, p):
        U, P = Step.apply(u, p, *args)
        return float((gU * U).sum() + (gP * P).sum())

    u, p = U0.clone().requires_grad_(True), P0.clone().requires_grad_(True)
    U, P = Step.apply(u, p, *args)
    ((gU * U).sum() + (gP * P).sum()).backward()
    eps = 1e-4
    if which == "U":
        d = t(rng.standard_normal(n2))
        fd = (loss(U0 + eps * d, P0) - loss(U0 - eps * d, P0)) / (2 * eps)
        vjp = float((u.grad * d).sum())
    else:
        d = t(rng.standard_normal(n))
        fd = (loss(U0, P0 + eps * d) - loss(U0, P0 - eps * d)) / (2 * eps)
        vjp = float((p.grad * d).sum())
    assert abs(vjp - fd) <= 1e-6 * max(abs(fd), 1.0), (vjp, fd)


@pytest.mark.gpu
def test_checkpointed_rollout_gradient(cavity):
    """A 4-step rollout with a checkpoint every 2 steps gives the gradient of the
    plain rollout, and that gradient matches central differences."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import rollout
    solver, ud = cavity
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    n2, n = solver.ndim * solver.nn, solver.nn
    rng = np.random.default_rng(33)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    U0, P0, gU = t(0.5 * rng.standard_normal(n2)), t(np.zeros(n)), t(rng.standard_normal(n2))
    def grad(ckpt):
        u = U0.clone().requires_grad_(True)
        U, _ = rollout(solver, nconn, u, P0, 4, 0.01, 1.0, 0.05, ud, ckpt=ckpt)
        (gU * U).sum().backward()
        return u.grad

    g_plain, g_ckpt = grad(0), grad(2)
    assert float(torch.linalg.norm(g_ckpt - g_plain) / torch.linalg.norm(g_plain)) < 1e-12
    d, eps = t(rng.standard_normal(n2)), 1e-4
    with torch.no_grad():
        lp = float((gU * rollout(solver, nconn, U0 + eps * d, P0, 4, 0.01, 1.0, 0.05, ud)[0]).sum())
        lm = float((gU * rollout(solver, nconn, U0 - eps * d, P0, 4, 0.01, 1.0, 0.05, ud)[0]).sum())
    fd = (lp - lm) / (2 * eps)
    vjp = float((g_plain * d).sum())
    assert abs(vjp - fd) <= 1e-6 * max(abs(fd), 1.0), (vjp, fd)
