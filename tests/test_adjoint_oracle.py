"""Hand-written adjoint gradients against central differences of the ORACLE's
forward step (oracle/standard.py, oracle/transport.py), which the golden
fixtures pin to the reference's own source. The reference's gradient is
jax.grad of its time loop (utils/jax_iterative_solvers.py:209-211 under
setup/simulation.py:362-374); jax is not installed, so the check is its
finite-difference counterpart: the GPU adjoint of a step (or a 4-step rollout)
against (L(x + e d) - L(x - e d)) / 2e of the oracle's FP64 step, solved to
1e-13, for a random loss L = <g, output> and direction d. Tolerance 1e-6
relative (the finite-difference error at e = 1e-4 is far below it)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-6
EPS = 1e-4


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)


def _cavity_cfg(mod, n, tol):
    return mod.Config(mesh="simple", solver="standard",
                      mesh_config=mod.SimpleMeshConfig(num_elem=[n, n], domain_size=[1.0, 1.0], shape_func_ord=1,
                                                       periodic=False),
                      solver_config=mod.StandardSolverConfig(dirichlet_faces=[0, 1, 2, 3], symmetry_faces=[],
                                                             outlet_faces=[], streamline_diff=False, solver_tol=tol,
                                                             set_zeroP=True, pressure_precond="multigrid",
                                                             final_multigrid_mesh=[4, 4]))


def _tg_cfg(mod, n, tol):
    from bench import tg_config
    cfg = tg_config(mod, n)
    cfg.solver_config.solver_tol = tol
    return cfg


def _pair(cfg_fn, n):
    """(GPU solver, nconn, U_d full, oracle timestep, nn, ndim) of one problem."""
    import oracle.simulation as osim
    import jax_fem_cfd_b200.setup.simulation as gsim
    _, ts_g, nc, sn, h, nn, gd, Ud = gsim.setup(cfg_fn(gsim, n, 1e-8))
    _, ts_o, *_ = osim.setup(cfg_fn(osim, n, 1e-13))
    solver = ts_g.solver
    nconn = torch.as_tensor(_nconn(solver)).cuda()
    return solver, nconn, solver.u_full(Ud), ts_o, nn, solver.ndim


def _nconn(solver):
    from oracle import mesh as om
    m = solver.mesh
    if m.kind == 1:
        fn = om.create_periodic_mesh_2d_quad9 if m.periodic else om.create_mesh_2d_quad9
    else:
        fn = om.create_periodic_mesh_2d if m.periodic else om.create_mesh_2d
    return fn(m.nex, m.ney, m.lx, m.ly)[1]


@pytest.mark.parametrize("problem", ["cavity16_q1_pinned", "taylor_green8_q2_mean_zero"])
@pytest.mark.parametrize("which", ["U", "P"])
def test_step_gradient_matches_oracle_differences(problem, which):
    from jax_fem_cfd_b200.solvers.adjoint import Step
    cfg_fn, n = (_cavity_cfg, 16) if problem.startswith("cavity") else (_tg_cfg, 8)
    solver, nconn, ud, ts_o, nn, nd = _pair(cfg_fn, n)
    rng = np.random.default_rng(7 if which == "U" else 8)
    dt, rho, mu = 0.01, 1.0, 0.05
    U0, P0 = 0.5 * rng.standard_normal(nd * nn), rng.standard_normal(nn)
    if problem.startswith("taylor"):
        P0 -= P0.mean()
    gU, gP = rng.standard_normal(nd * nn), rng.standard_normal(nn)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    u, p = t(U0).requires_grad_(True), t(P0).requires_grad_(True)
    U, P = Step.apply(u, p, solver, nconn, dt, rho, mu, ud)
    ((t(gU) * U).sum() + (t(gP) * P).sum()).backward()

    def L(Ux, Px):
        Uo, Po, _, _ = ts_o(Ux, Px, dt, rho, mu, 0.0, 0.0, 0.0)
        return float(np.dot(gU, Uo) + np.dot(gP, Po))

    if which == "U":
        d = rng.standard_normal(nd * nn)
        fd = (L(U0 + EPS * d, P0) - L(U0 - EPS * d, P0)) / (2 * EPS)
        vjp = float((u.grad.cpu().numpy() * d).sum())
    else:
        d = rng.standard_normal(nn)
        fd = (L(U0, P0 + EPS * d) - L(U0, P0 - EPS * d)) / (2 * EPS)
        vjp = float((p.grad.cpu().numpy() * d).sum())
    assert abs(vjp - fd) <= GRAD_TOL * max(abs(fd), 1.0), (vjp, fd)


def test_rollout_gradient_matches_oracle_differences():
    """4 steps with a checkpoint every 2 (recomputed in the backward pass)."""
    from jax_fem_cfd_b200.solvers.adjoint import rollout
    solver, nconn, ud, ts_o, nn, nd = _pair(_cavity_cfg, 16)
    rng = np.random.default_rng(11)
    dt, rho, mu = 0.01, 1.0, 0.05
    U0, gU = 0.5 * rng.standard_normal(nd * nn), rng.standard_normal(nd * nn)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    u = t(U0).requires_grad_(True)
    U, _ = rollout(solver, nconn, u, t(np.zeros(nn)), 4, dt, rho, mu, ud, ckpt=2)
    (t(gU) * U).sum().backward()

    def L(Ux):
        Ux, Px = Ux, np.zeros(nn)
        for _ in range(4):
            Ux, Px, _, _ = ts_o(Ux, Px, dt, rho, mu, 0.0, 0.0, 0.0)
        return float(np.dot(gU, Ux))

    d = rng.standard_normal(nd * nn)
    fd = (L(U0 + EPS * d) - L(U0 - EPS * d)) / (2 * EPS)
    vjp = float((u.grad.cpu().numpy() * d).sum())
    assert abs(vjp - fd) <= GRAD_TOL * max(abs(fd), 1.0), (vjp, fd)


def _oracle_phi(Un, U, phin, gdphi, phid, nconn, nn, dt, D, supg):
    """The scalar update of solvers/passive_transport.py:80-95 for given U_n and U."""
    from oracle import element as ec, shape as osh, transport as otr
    from oracle import mesh as om
    nc, _, *_ = om.create_mesh_2d(16, 16, 1.0, 1.0)
    wq, N, Nd = osh.quad4_shape_functions(nc[nconn[0]])
    _, Me = ec.lumped_mass_matrix(nconn, wq, N, nn, 2)
    Le = ec.laplacian_element_calc(wq, Nd)
    Ce1_n = ec.conservative_convec_elem_calc(nconn, Un, wq, N, Nd, nn, 2, 1)
    Ce1 = ec.conservative_convec_elem_calc(nconn, U, wq, N, Nd, nn, 2, 1)
    if supg:
        Ct_n = ec.Ctau_tilde_elem_calc(nconn, Un, wq, N, Nd, nn, 2)
        tau = ec.calculate_tau(nconn, Un, Ce1, Ct_n, N, nn, 2, D, dt, r=2)
        Ctau, Mtau = tau[:, None, None] * Ct_n, tau[:, None, None] * Ce1_n.transpose(0, 2, 1)
        phi, _ = otr.update_phi_SUPG(phin, nconn, Mtau, Ctau, Me, Ce1, Ce1_n, Le, D, dt, nn, gdphi, phid, 1e-13)
    else:
        phi, _ = otr.update_phi(phin, nconn, Me, Ce1, Ce1_n, Le, D, dt, nn, gdphi, phid, 1e-13)
    return phi


@pytest.mark.parametrize("supg", [False, True])
@pytest.mark.parametrize("which", ["U_n", "U", "phi_n"])
def test_transport_gradient_matches_oracle_differences(supg, which):
    from jax_fem_cfd_b200.context import make_mask
    from jax_fem_cfd_b200.solvers.adjoint import Transport
    solver, nconn, _, _, nn, nd = _pair(_cavity_cfg, 16)
    nconn_np = nconn.cpu().numpy()
    rng = np.random.default_rng(50 + int(supg))
    dt, D = 0.01, 1e-3
    Un = 0.5 * rng.standard_normal(nd * nn)
    U = Un + 0.1 * rng.standard_normal(nd * nn)
    phin = rng.standard_normal(nn)
    bottom = np.arange(17)
    phid_vals = rng.standard_normal(bottom.size)
    phid_full = np.zeros(nn)
    phid_full[bottom] = phid_vals
    g = rng.standard_normal(nn)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    mask = make_mask(bottom, nn)
    leaves = {"U_n": t(Un).requires_grad_(True), "U": t(U).requires_grad_(True), "phi_n": t(phin).requires_grad_(True)}
    phi = Transport.apply(leaves["U_n"], leaves["U"], leaves["phi_n"], t(phid_full), solver, nconn, dt, D, supg, mask)
    (t(g) * phi).sum().backward()
    xs = {"U_n": Un, "U": U, "phi_n": phin}

    def L(**kw):
        a = {**xs, **kw}
        return float(np.dot(g, _oracle_phi(a["U_n"], a["U"], a["phi_n"], bottom, phid_vals, nconn_np, nn, dt, D,
                                           supg)))

    d = rng.standard_normal(xs[which].size)
    fd = (L(**{which: xs[which] + EPS * d}) - L(**{which: xs[which] - EPS * d})) / (2 * EPS)
    vjp = float((leaves[which].grad.cpu().numpy() * d).sum())
    assert abs(vjp - fd) <= GRAD_TOL * max(abs(fd), 1.0), (vjp, fd)
