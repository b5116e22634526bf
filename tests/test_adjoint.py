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
def test_projection_vjp_mean_zero_pressure():
    """The projection of a periodic problem (mean-zero pressure: rhs and P
    centred around the solve on the mean-zero subspace) against central
    differences; the adjoint solve is the same centred solve."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from bench import tg_config
    from jax_fem_cfd_b200.setup import simulation as sim
    from jax_fem_cfd_b200.solvers.adjoint import Projection
    _, timestep, *rest = sim.setup(tg_config(sim, 8))
    solver = timestep.solver
    n2, n = solver.ndim * solver.nn, solver.nn
    rng = np.random.default_rng(3)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Us, gU, gP, dlt = t(rng.standard_normal(n2)), t(rng.standard_normal(n2)), t(rng.standard_normal(n)), \
        t(rng.standard_normal(n2))

    def loss(u):
        U, P = Projection.apply(u, solver, 0.01, 1.0, None, None, 1e-13)
        return float((gU * U).sum() + (gP * P).sum())

    x = Us.clone().requires_grad_(True)
    U, P = Projection.apply(x, solver, 0.01, 1.0, None, None, 1e-13)
    assert abs(float(P.mean())) < 1e-12 * float(P.abs().max())
    ((gU * U).sum() + (gP * P).sum()).backward()
    eps = 1e-2
    fd = (loss(Us + eps * dlt) - loss(Us - eps * dlt)) / (2 * eps)
    vjp = float((x.grad * dlt).sum())
    assert abs(vjp - fd) <= 1e-7 * max(abs(fd), 1.0), (vjp, fd)


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


def _transport_case(solver, supg, seed=40):
    from jax_fem_cfd_b200.context import make_mask
    n2, n = solver.ndim * solver.nn, solver.nn
    rng = np.random.default_rng(seed)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Un = t(0.5 * rng.standard_normal(n2))
    U = Un + t(0.1 * rng.standard_normal(n2))
    phin = t(rng.standard_normal(n))
    bottom = np.arange(17)  # the y = 0 row of the 17 x 17 node lattice
    mask = make_mask(bottom, n)
    phid = torch.zeros(n, dtype=torch.float64, device="cuda")
    phid[bottom] = t(rng.standard_normal(bottom.size))
    return Un, U, phin, phid, mask, rng


@pytest.mark.gpu
@pytest.mark.parametrize("supg", [False, True])
def test_transport_elements_reproduce_the_product_step(cavity, supg):
    """fem_transport_elements (the element matrices the adjoint solves with)
    equals the torch restatement, transposed too, and describes the system
    fem_transport_phi solves: the product's phi leaves a relative residual at
    the solver's tolerance in that system."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import Transport, transport_elements
    from torch_restatement import transport_element_matrices
    solver, _ = cavity
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    Un, U, phin, phid, mask, _ = _transport_case(solver, supg)
    dt, D = 0.01, 1e-3
    phi = Transport.apply(Un, U, phin, phid, solver, nconn, dt, D, supg, mask)
    Ek, Bk = transport_elements(solver, Un, U, dt, D, supg)
    EkT, BkT = transport_elements(solver, Un, U, dt, D, supg, transpose=True)
    wq, N, Nd = solver.ctx.element_data()[:3]
    Er, Br = transport_element_matrices(wq, N, Nd, 2, solver.nn, nconn, Un, U, dt, D, supg)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    assert rel(Ek, Er) < 1e-13 and rel(Bk, Br) < 1e-13
    assert torch.equal(EkT, Ek.transpose(1, 2)) and torch.equal(BkT, Bk.transpose(1, 2))
    Me, Le = solver.ctx.element_data()[3], solver.ctx.element_data()[4]
    n = solver.nn

    def apply(Kel, x):
        y = torch.zeros(n, dtype=torch.float64, device="cuda")
        y.index_add_(0, nconn.reshape(-1), torch.einsum("eab,eb->ea", Kel, x[nconn]).reshape(-1))
        return y

    m = mask.to(torch.bool)
    r = apply(Me / dt - 0.5 * D * Le + Bk, phin)
    r[m] = phid[m]
    Aphi = apply(Me / dt + 0.5 * D * Le + Ek, phi)
    Aphi[m] = phi[m]
    rel = float(torch.linalg.norm(Aphi - r) / torch.linalg.norm(r))
    assert rel < 1e-11, rel


@pytest.mark.gpu
@pytest.mark.parametrize("supg", [False, True])
@pytest.mark.parametrize("which", ["phi_n", "U_n", "U", "phi_d"])
def test_transport_vjp_matches_finite_differences(cavity, supg, which):
    """The transport adjoint (masked transposed BiCGSTAB, B^T, and the velocity
    dependence of Ce, Ctau, Mtau and tau) against central differences."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import Transport
    solver, _ = cavity
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    Un, U, phin, phid, mask, rng = _transport_case(solver, supg)
    dt, D = 0.01, 1e-3
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    g = t(rng.standard_normal(solver.nn))
    xs = dict(U_n=Un, U=U, phi_n=phin, phi_d=phid)
    d = t(rng.standard_normal(xs[which].numel()))
    if which == "phi_d":
        d = torch.where(mask.to(torch.bool), d, torch.zeros_like(d))

    def loss(**kw):
        a = {**xs, **kw}
        return float((g * Transport.apply(a["U_n"], a["U"], a["phi_n"], a["phi_d"], solver, nconn, dt, D, supg,
                                          mask)).sum())

    leaves = {k: v.clone().requires_grad_(True) for k, v in xs.items()}
    phi = Transport.apply(leaves["U_n"], leaves["U"], leaves["phi_n"], leaves["phi_d"], solver, nconn, dt, D, supg,
                          mask)
    (g * phi).sum().backward()
    eps = 1e-5
    fd = (loss(**{which: xs[which] + eps * d}) - loss(**{which: xs[which] - eps * d})) / (2 * eps)
    vjp = float((leaves[which].grad * d).sum())
    assert abs(vjp - fd) <= 1e-6 * max(abs(fd), 1.0), (vjp, fd)


@pytest.mark.gpu
def test_transport_rollout_gradient(cavity):
    """Flow and SUPG passive scalar over 4 steps: the checkpointed gradient in
    (U0, phi0) equals the plain one and matches central differences."""
    from jax_fem_cfd_b200.setup import regular_mesh as rm
    from jax_fem_cfd_b200.solvers.adjoint import rollout
    solver, ud = cavity
    _, nconn, *_ = rm.create_mesh_2d(16, 16, 1.0, 1.0)
    Un, _, phin, phid, mask, rng = _transport_case(solver, True, seed=41)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    P0 = torch.zeros(solver.nn, dtype=torch.float64, device="cuda")
    gphi = t(rng.standard_normal(solver.nn))
    kw = dict(phi_mask=mask, phid_full=phid, D=1e-3, supg=True)

    def run(u, phi, ckpt):
        return rollout(solver, nconn, u, P0, 4, 0.01, 1.0, 0.05, ud, ckpt=ckpt, phi0=phi, **kw)[2]

    def grads(ckpt):
        u, phi = Un.clone().requires_grad_(True), phin.clone().requires_grad_(True)
        (gphi * run(u, phi, ckpt)).sum().backward()
        return u.grad, phi.grad

    (gu0, gp0), (gu2, gp2) = grads(0), grads(2)
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    assert rel(gu2, gu0) < 1e-12 and rel(gp2, gp0) < 1e-12
    du, dp, eps = t(rng.standard_normal(Un.numel())), t(rng.standard_normal(phin.numel())), 1e-5
    with torch.no_grad():
        lp = float((gphi * run(Un + eps * du, phin + eps * dp, 0)).sum())
        lm = float((gphi * run(Un - eps * du, phin - eps * dp, 0)).sum())
    fd = (lp - lm) / (2 * eps)
    vjp = float((gu0 * du).sum() + (gp0 * dp).sum())
    assert abs(vjp - fd) <= 1e-6 * max(abs(fd), 1.0), (vjp, fd)


@pytest.mark.gpu
def test_deferred_status_raises_when_the_block_ends(cavity):
    """A solve that fails inside deferred_status (here: a non-finite U*, which
    the pressure solve reports in its status word) raises FemError when the
    block ends; outside a block the same call raises at once."""
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.solvers.adjoint import Projection, deferred_status
    solver, ud = cavity
    bad = torch.full((solver.ndim * solver.nn,), float("nan"), dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.FemError, match="deferred"):
        with deferred_status():
            Projection.apply(bad, solver, 0.01, 1.0, ud, None, 1e-13)
    with pytest.raises(_lib.FemError, match="pressure solve status 2"):
        Projection.apply(bad, solver, 0.01, 1.0, ud, None, 1e-13)
    good = torch.zeros(solver.ndim * solver.nn, dtype=torch.float64, device="cuda")
    with deferred_status():
        U, P = Projection.apply(good, solver, 0.01, 1.0, ud, None, 1e-13)
    assert torch.isfinite(U).all() and torch.isfinite(P).all()


@pytest.mark.gpu
@pytest.mark.parametrize("supg", [False, True])
@pytest.mark.parametrize("kind", ["q1", "q2_periodic"])
def test_transport_vjp_kernel_matches_torch_autograd(kind, supg):
    """fem_transport_vjp (d/dU_n and d/dU of <lam, B_k phi_n - E_k phi>
    summed over elements) against torch autograd of the torch restatement of
    E_k and B_k, which tests/test_adjoint_elements.py pins to the oracle."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jax_fem_cfd_b200.context import Context, Mesh
    from jax_fem_cfd_b200.solvers.adjoint import transport_vjp
    from torch_restatement import transport_element_matrices
    from oracle import mesh as om
    if kind == "q1":
        mesh, nconn = Mesh(0, False, 7, 5, 1, 1.4, 1.0), om.create_mesh_2d(7, 5, 1.4, 1.0)[1]
    else:
        mesh, nconn = (Mesh(1, True, 6, 4, 1, 2 * np.pi, 2 * np.pi),
                       om.create_periodic_mesh_2d_quad9(6, 4, 2 * np.pi, 2 * np.pi)[1])
    ctx = Context(mesh)
    nn = ctx.nn
    solver = type("S", (), {"ctx": ctx})()
    rng = np.random.default_rng(23 + int(supg))
    t = lambda a_: torch.as_tensor(a_, dtype=torch.float64, device="cuda")
    Un = t(0.5 * rng.standard_normal(2 * nn))
    U = Un + t(0.1 * rng.standard_normal(2 * nn))
    lam, phin, phi = (t(rng.standard_normal(nn)) for _ in range(3))
    dt, D = 0.01, 1e-3
    gUn, gU = transport_vjp(solver, Un, U, lam, phin, phi, dt, D, supg)
    wq, N, Nd = ctx.element_data()[:3]
    nc = torch.as_tensor(nconn).cuda()
    un, u = Un.clone().requires_grad_(True), U.clone().requires_grad_(True)
    Ek, Bk = transport_element_matrices(wq, N, Nd, 2, nn, nc, un, u, dt, D, supg)
    le, pe, fe = lam[nc], phin[nc], phi[nc]
    s = torch.einsum("ea,eab,eb->", le, Bk, pe) - torch.einsum("ea,eab,eb->", le, Ek, fe)
    rn, ru = torch.autograd.grad(s, (un, u))
    rel = lambda a, b: float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    assert rel(gUn, rn) < 1e-12 and rel(gU, ru) < 1e-12, (rel(gUn, rn), rel(gU, ru))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["q1", "q2_periodic", "hex8"])
def test_conv_vjp_kernel_matches_its_torch_restatement(kind):
    """fem_conv_vjp (d/dU <a, Ce(U) b>, the velocity side of the step adjoint)
    against conv_vjp_u_elements, the torch restatement pinned to the oracle's
    Ce on the CPU (tests/test_adjoint_elements.py)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import Context, Mesh, ptr, stream
    from torch_restatement import conv_vjp_u_elements
    from oracle import mesh as om
    if kind == "q1":
        mesh, nconn = Mesh(0, False, 7, 5, 1, 1.4, 1.0), om.create_mesh_2d(7, 5, 1.4, 1.0)[1]
    elif kind == "q2_periodic":
        mesh, nconn = (Mesh(1, True, 6, 4, 1, 2 * np.pi, 2 * np.pi),
                       om.create_periodic_mesh_2d_quad9(6, 4, 2 * np.pi, 2 * np.pi)[1])
    else:
        mesh, nconn = Mesh(2, False, 4, 3, 3, 1.0, 0.75, 0.75), om.create_mesh_3d(4, 3, 3, 1.0, 0.75, 0.75)[1]
    ctx = Context(mesh)
    nd, nn = ctx.ndim, ctx.nn
    rng = np.random.default_rng(17)
    t = lambda a_: torch.as_tensor(a_, dtype=torch.float64, device="cuda")
    a, b = t(rng.standard_normal(nd * nn)), t(rng.standard_normal(nd * nn))
    y = torch.empty(nd * nn, dtype=torch.float64, device="cuda")
    _lib.call("fem_conv_vjp", ctx.handle, nd, ptr(a), ptr(b), 0.5, ptr(y), stream())
    wq, N, Nd = ctx.element_data()[:3]
    ref = conv_vjp_u_elements(wq, N, Nd, nd, nn, torch.as_tensor(nconn).cuda(), a, b, 0.5)
    err = float(torch.linalg.norm(y - ref) / torch.linalg.norm(ref))
    assert err < 1e-13, err
