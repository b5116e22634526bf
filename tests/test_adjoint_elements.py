"""The torch restatements in tests/torch_restatement.py (the references for
the fem_transport_elements, fem_transport_vjp and fem_conv_vjp kernels) against
the oracle's element functions (core/element_calc.py:165-229 via
oracle/element.py), on CPU tensors."""
import numpy as np
import pytest
import torch


@pytest.mark.parametrize("supg", [True, False])
def test_transport_element_matrices_match_the_oracle(supg):
    from oracle import element as oe
    from oracle import mesh as om
    from oracle import shape as osh
    from torch_restatement import transport_element_matrices
    coords, nconn, *_ = om.create_mesh_2d(6, 5, 1.2, 1.0)
    wq, N, Nd = osh.quad4_shape_functions(coords[nconn[0]])
    nn, nd, dt, D = coords.shape[0], 2, 0.01, 1e-3
    rng = np.random.default_rng(3)
    Un = 0.5 * rng.standard_normal(nd * nn)
    U = Un + 0.1 * rng.standard_normal(nd * nn)
    Ce1 = oe.conservative_convec_elem_calc(nconn, U, wq, N, Nd, nn, nd, 1)
    Ce1_n = oe.conservative_convec_elem_calc(nconn, Un, wq, N, Nd, nn, nd, 1)
    if supg:
        Ct = oe.Ctau_tilde_elem_calc(nconn, Un, wq, N, Nd, nn, nd)
        tau = oe.calculate_tau(nconn, Un, Ce1, Ct, N, nn, nd, D, dt, r=2)
        Mtau, Ctau = tau[:, None, None] * Ce1_n.transpose(0, 2, 1), tau[:, None, None] * Ct
        Ek_ref, Bk_ref = Mtau / dt + 0.5 * (Ce1 + Ctau), Mtau / dt - 0.5 * (Ce1_n + Ctau)
    else:
        Ek_ref, Bk_ref = 0.5 * Ce1, -0.5 * Ce1_n
    t = torch.as_tensor
    Ek, Bk = transport_element_matrices(t(wq), t(N), t(Nd), nd, nn, t(nconn), t(Un), t(U), dt, D, supg)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    assert rel(Ek.numpy(), Ek_ref) < 1e-13 and rel(Bk.numpy(), Bk_ref) < 1e-13


def test_transport_element_matrices_are_differentiable_in_both_velocities():
    """torch.autograd.gradcheck of <a, E_k(U_n, U) b> + <c, B_k(U_n, U) d> in
    (U_n, U) with SUPG (tau, norms and Ce through autograd)."""
    from oracle import mesh as om
    from oracle import shape as osh
    from torch_restatement import transport_element_matrices
    coords, nconn, *_ = om.create_mesh_2d(3, 2, 1.0, 1.0)
    wq, N, Nd = osh.quad4_shape_functions(coords[nconn[0]])
    nn = coords.shape[0]
    rng = np.random.default_rng(5)
    t = lambda a: torch.as_tensor(a, dtype=torch.float64)
    W = [t(rng.standard_normal((nconn.shape[0], 4, 4))) for _ in range(2)]

    def f(un, u):
        Ek, Bk = transport_element_matrices(t(wq), t(N), t(Nd), 2, nn, torch.as_tensor(nconn), un, u, 0.01, 1e-3,
                                            True)
        return (W[0] * Ek).sum() + (W[1] * Bk).sum()

    un = t(0.5 * rng.standard_normal(2 * nn)).requires_grad_(True)
    u = t(0.5 * rng.standard_normal(2 * nn)).requires_grad_(True)
    assert torch.autograd.gradcheck(f, (un, u), eps=1e-6, atol=1e-7, rtol=1e-6)


@pytest.mark.parametrize("beta", [0.5, 1.0])
def test_convection_vjp_matches_the_oracle(beta):
    """Ce(U) is linear in U, so <a, Ce(d) b> = conv_vjp_u(a, b) . d exactly,
    with Ce from the oracle (core/element_calc.py:165-185) acting on each
    velocity component."""
    from oracle import element as oe
    from oracle import mesh as om
    from oracle import shape as osh
    from torch_restatement import conv_vjp_u_elements
    coords, nconn, *_ = om.create_mesh_2d(5, 4, 1.0, 0.8)
    wq, N, Nd = osh.quad4_shape_functions(coords[nconn[0]])
    nn, nd = coords.shape[0], 2
    rng = np.random.default_rng(11)
    a, b, d = (rng.standard_normal(nd * nn) for _ in range(3))
    Ce = oe.conservative_convec_elem_calc(nconn, d, wq, N, Nd, nn, nd, beta)
    ref = sum(np.einsum("ea,eab,eb->", a[c * nn:(c + 1) * nn][nconn], Ce, b[c * nn:(c + 1) * nn][nconn])
              for c in range(nd))
    t = torch.as_tensor
    g = conv_vjp_u_elements(t(wq), t(N), t(Nd), nd, nn, t(nconn), t(a), t(b), beta)
    assert abs(float(g @ t(d)) - ref) <= 1e-13 * abs(ref), (float(g @ t(d)), ref)
