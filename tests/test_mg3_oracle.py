"""The oracle's hex8 multigrid (oracle/multigrid3d.py, a build-defined
extension: the reference refuses 3D multigrid) checked on the CPU, and the
tensor-product form of the hex8 Laplacian that the CUDA kernels apply checked
against the assembled element matrices."""
import numpy as np
import pytest

from oracle import multigrid3d as m3
from oracle.solvers import cg


def _levels(ne=(16, 8, 8), nef=(4, 2, 2), outlet=(1,)):
    return m3.multigrid3d_setup(list(ne), list(nef), [4.0, 1.0, 1.0], list(outlet))


def _axis_rows(h):
    ki, mi = 1.0 / h, h / 6.0
    K = np.array([[0.0, ki, -ki], [-ki, 2 * ki, -ki], [-ki, ki, 0.0]])
    M = np.array([[0.0, 2 * mi, mi], [mi, 4 * mi, mi], [mi, 2 * mi, 0.0]])
    return K, M


def _tensor_apply(v, dims, h):
    """A v with A = Kx My Mz + Mx Ky Mz + Mx My Kz from the 1D rows (the kernels' form)."""
    nx, ny, nz = dims
    V = v.reshape(nz, ny, nx)
    (Kx, Mx), (Ky, My), (Kz, Mz) = (_axis_rows(hh) for hh in h)

    def op1(A, U, axis, n):
        U = np.moveaxis(U, axis, -1)
        out = np.zeros_like(U)
        cls = np.ones(n, dtype=int)
        cls[0], cls[-1] = 0, 2
        Up = np.concatenate([U[..., :1], U, U[..., -1:]], axis=-1)
        for d in range(3):
            out += A[cls, d] * Up[..., d:d + n]
        return np.moveaxis(out, -1, axis)

    t1 = op1(Mz, op1(My, op1(Kx, V, 2, nx), 1, ny), 0, nz)
    t2 = op1(Mz, op1(Ky, op1(Mx, V, 2, nx), 1, ny), 0, nz)
    t3 = op1(Kz, op1(My, op1(Mx, V, 2, nx), 1, ny), 0, nz)
    return (t1 + t2 + t3).ravel()


def test_tensor_form_equals_assembled_laplacian():
    ne = (6, 5, 4)
    L = _levels(ne, (3, 5, 4), ())[0]
    v = np.random.default_rng(0).standard_normal(L.nn)
    h = (4.0 / ne[0], 1.0 / ne[1], 1.0 / ne[2])
    y = _tensor_apply(v, L.dims, h)
    ya = L.A @ v
    assert np.linalg.norm(y - ya) / np.linalg.norm(ya) < 1e-13


def test_restriction_is_prolongation_transpose():
    L = _levels()
    fine, coarse = L[0].dims, L[1].dims
    rng = np.random.default_rng(1)
    f = rng.standard_normal(np.prod(fine))
    c = rng.standard_normal(np.prod(coarse))
    a = np.dot(m3.restrict3d(f, fine), c)
    b = np.dot(f, m3.prolong3d(c, coarse, fine))
    assert abs(a - b) < 1e-12 * abs(b)


@pytest.mark.parametrize("outlet", [(1,), ()])
def test_vcycle_is_symmetric_and_pcg_converges(outlet):
    levels = _levels(outlet=outlet)
    L0 = levels[0]
    rng = np.random.default_rng(2)
    a, b = rng.standard_normal(L0.nn), rng.standard_normal(L0.nn)
    a[L0.gp] = 0.0
    b[L0.gp] = 0.0
    ma, mb = m3.v_cycle3d(a, levels), m3.v_cycle3d(b, levels)
    assert abs(np.dot(ma, b) - np.dot(a, mb)) < 1e-12 * abs(np.dot(ma, b))
    assert np.dot(ma, a) > 0
    x, it = cg(lambda v: m3.apply_A(L0, v), b, x0=np.zeros(L0.nn), tol=1e-8, maxiter=1000,
               M=lambda v: m3.v_cycle3d(v, levels))
    r = b - m3.apply_A(L0, x)
    assert it <= 10 and np.linalg.norm(r) <= 1e-8 * np.linalg.norm(b)


def test_power_estimate_bounds_the_spectrum():
    """The Chebyshev interval's top, 1.1 x the power estimate, lies above the
    largest eigenvalue of D^-1 A (dense check on a small level)."""
    L = _levels((8, 4, 4), (2, 1, 1), (1,))[0]
    f = L.free
    A = L.A.toarray()[np.ix_(f, f)]
    d = np.sqrt(L.invDm[f])
    lam = np.linalg.eigvalsh(d[:, None] * A * d[None, :]).max()
    assert L.bounds[1] >= lam > L.lam * 0.8
