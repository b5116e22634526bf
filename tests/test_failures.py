"""Failure detection on the GPU without a GPU fault: the solver status word
(non-finite input, iteration cap) and the grid barrier's time limit. After
each failure the same context solves a normal problem and reproduces the
result it gave before the failure bit for bit (the context stays usable). The
barrier test waits for a party that never arrives; the barrier's own 2 s limit
ends the wait and the kernel returns an error status."""
import numpy as np
import pytest
import torch

STATUS_BARRIER_TIMEOUT, STATUS_NONFINITE, STATUS_MAXITER = 1, 2, 4


@pytest.fixture(scope="module")
def poisson():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import Context, Mesh, make_mask, ptr, stream
    from jax_fem_cfd_b200.core import multigrid as gmg
    n = 64
    ctx = Context(Mesh(0, False, n, n, 1, 1.0, 1.0))
    ctx.set_bc(None, make_mask(np.array([0]), ctx.nn), True)
    nlev = int(np.log2(n // 4)) + 1
    gmg.Hierarchy(ctx, nlev, [np.array([0])] * nlev, 1e-8)

    def solve(b, maxiter=1000):
        bg = torch.as_tensor(b, device="cuda")
        x = torch.zeros_like(bg)
        it = torch.zeros(1, dtype=torch.int32, device="cuda")
        st = torch.zeros(1, dtype=torch.int32, device="cuda")
        _lib.call("fem_pressure_solve", ctx.handle, ptr(bg), ptr(x), 1e-8, 0.0, int(maxiter), _lib.PREC["multigrid"],
                  0, 1, ptr(it), ptr(st), stream())
        torch.cuda.synchronize()
        return x.cpu().numpy(), int(it.item()), int(st.item())

    b = np.random.default_rng(3).standard_normal(ctx.nn)
    b[0] = 0.0
    x_ref, it_ref, st_ref = solve(b)
    assert st_ref == 0 and 0 < it_ref < 30
    return ctx, solve, b, x_ref, it_ref


def _recovers(poisson):
    _, solve, b, x_ref, it_ref = poisson
    x, it, st = solve(b)
    assert st == 0 and it == it_ref
    np.testing.assert_array_equal(x, x_ref)


@pytest.mark.gpu
def test_nonfinite_input_is_reported(poisson):
    _, solve, b, _, _ = poisson
    bad = b.copy()
    bad[17] = np.nan
    _, it, st = solve(bad)
    assert st & STATUS_NONFINITE and it == 0
    _recovers(poisson)


@pytest.mark.gpu
def test_iteration_cap_is_reported(poisson):
    _, solve, b, _, it_ref = poisson
    _, it, st = solve(b, maxiter=2)
    assert st == STATUS_MAXITER and it == 2 < it_ref
    _recovers(poisson)


@pytest.mark.gpu
def test_barrier_time_limit_ends_the_wait(poisson):
    from jax_fem_cfd_b200 import _lib
    from jax_fem_cfd_b200.context import ptr, stream
    ctx = poisson[0]
    st = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    _lib.call("fem_selftest_barrier_timeout", ctx.handle, ptr(st), stream())
    torch.cuda.synchronize()
    assert int(st.item()) == STATUS_BARRIER_TIMEOUT
    _recovers(poisson)
