"""The inverse transport problem (learnable initial velocity, scalar loss after
a rollout of flow and SUPG transport steps): its adjoint gradient against
central differences, checkpointing, and one descent step."""
import pytest
import torch


@pytest.fixture(scope="module")
def problem():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from jax_fem_cfd_b200.solvers.inverse_transport import InverseTransport
    return InverseTransport(n=32, steps=12, ckpt=5, tol=1e-12)


@pytest.mark.gpu
def test_problem_data(problem):
    # phi_0 covers [0.4, 0.6] x [0.2, 0.4] of the 33 x 33 lattice (spacing 1/32): x nodes 13-19,
    # y nodes 7-12
    assert int(problem.phi0.sum()) == 42
    assert float(problem.target.max()) > 0.9 and float(problem.mass.sum()) == pytest.approx(1.0, rel=1e-12)
    u0 = problem.initial_velocity()
    assert u0.dtype == torch.float32 and abs(float(u0.std()) - 0.1) < 0.005


@pytest.mark.gpu
def test_gradient_matches_finite_differences(problem):
    u0 = problem.initial_velocity().to(torch.float64)
    L, g = problem.value_and_grad(u0)
    L_plain, g_plain = problem.value_and_grad(u0, ckpt=0)
    assert L == L_plain
    assert float(torch.linalg.norm(g - g_plain) / torch.linalg.norm(g_plain)) < 1e-12
    gen = torch.Generator(device="cpu").manual_seed(7)
    d = torch.randn(u0.numel(), generator=gen, dtype=torch.float64).to(u0.device)
    eps = 1e-4
    with torch.no_grad():
        fd = (float(problem.loss(u0 + eps * d)) - float(problem.loss(u0 - eps * d))) / (2 * eps)
    vjp = float((g * d).sum())
    assert abs(vjp - fd) <= 1e-6 * max(abs(fd), abs(L)), (vjp, fd)


@pytest.mark.gpu
def test_descent_step_lowers_the_loss(problem):
    u0 = problem.initial_velocity()
    L0, g = problem.value_and_grad(u0)
    assert g.dtype == torch.float32 and torch.isfinite(g).all()
    step = 0.01 * float(u0.norm()) / float(g.norm())
    with torch.no_grad():
        L1 = float(problem.loss(u0 - step * g))
    assert L1 < L0, (L0, L1)
