"""Plain-PyTorch FP64 restatements of element-level functions whose CUDA
kernels the adjoint uses, for the tests only: the kernels are checked against
these, and these against the oracle's element functions
(core/element_calc.py:165-229 via oracle/element.py). Differentiable, so
torch.autograd gives the reference vector-Jacobian products."""
import torch


def conv_vjp_u_elements(wq, N, Nd, nd, nn, nconn, a, b, beta):
    """d/dU <a, Ce(U) b> (what fem_conv_vjp computes) on explicit element data
    (wq (nq[, 1]), N (nq, nen), Nd
    (nq, nd, nen) of a uniform mesh, nconn (ne, nen) int64)."""
    w = wq.reshape(-1)
    ae = a.view(nd, nn)[:, nconn]  # (c, e, i)
    be = b.view(nd, nn)[:, nconn]
    A = torch.einsum("qi,cei->ceq", N, ae)
    B = torch.einsum("qi,cei->ceq", N, be)
    dB = torch.einsum("qdi,cei->ceqd", Nd, be)
    s_ = torch.einsum("ceq,ceqd->eqd", A, dB)
    t_ = torch.einsum("ceq,ceq->eq", A, B)
    ge = torch.einsum("q,qk,eqd->edk", w, N, s_) + beta * torch.einsum("q,qdk,eq->edk", w, Nd, t_)
    out = torch.zeros(nd, nn, dtype=torch.float64, device=a.device)
    idx = nconn.reshape(-1)
    for d in range(nd):
        out[d].index_add_(0, idx, ge[:, d, :].reshape(-1))
    return out.reshape(-1)


def transport_element_matrices(wq, N, Nd, nd, nn, nconn, Un, U, dt, D, supg):
    """(E_k, B_k) of the transport step on explicit element data (the matrices
    fem_transport_elements builds; solvers/passive_transport.py:80-88 feeding
    :14-62, core/element_calc.py:165-229): wq (nq[, 1]), N (nq, nen),
    Nd (nq, nd, nen) of a uniform mesh, nconn (ne, nen) int64, U_n and U
    (nd * nn, component-major); torch tensors on any device."""
    w = wq.reshape(-1)

    def interp(V):
        return torch.einsum("qi,dei->eqd", N, V.view(nd, nn)[:, nconn])

    def conv(V):
        Ve = V.view(nd, nn)[:, nconn]
        adv = torch.einsum("q,qa,eqd,qdb->eab", w, N, interp(V), Nd)
        div = torch.einsum("qdi,dei->eq", Nd, Ve)
        return adv + torch.einsum("q,qa,eq,qb->eab", w, N, div, N)

    Ce_new, Ce_n = conv(U), conv(Un)
    if not supg:
        return 0.5 * Ce_new, -0.5 * Ce_n
    Uq = interp(Un)
    Ct = torch.einsum("q,qda,eqd,eqk,qkb->eab", w, Nd, Uq, Uq, Nd)
    ce = torch.sqrt((Ce_new ** 2).sum((1, 2)))
    kt = torch.sqrt((Ct ** 2).sum((1, 2)))
    un2 = (Uq ** 2).sum(2).mean(1)
    tau1 = ce / kt
    tau3 = tau1 * (un2 * ce) / ((D + 1e-6) * kt)
    tau = (tau1 ** -2 + (dt / 2) ** -2 + tau3 ** -2) ** -0.5
    Ctau = tau[:, None, None] * Ct
    Mtau = tau[:, None, None] * Ce_n.transpose(1, 2)
    return Mtau / dt + 0.5 * (Ce_new + Ctau), Mtau / dt - 0.5 * (Ce_n + Ctau)
