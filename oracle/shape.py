"""Reference-element shape functions at Gauss points (oracle restatement of
core/shape_functions.py). Convention: wq (q, 1), N (q, I), Nderiv (q, dim, I).
Test infrastructure only."""
import numpy as np

_S3 = 1.0 / np.sqrt(3)


def lin2_shape_functions(coords):
    """core/shape_functions.py:11-25."""
    xi = np.array([-1, 1]) * _S3
    N = np.stack([(1 - xi) / 2, (1 + xi) / 2], axis=1)
    dNdxi = np.array([[-0.5, 0.5], [-0.5, 0.5]])
    h = np.sqrt((coords[1, 0] - coords[0, 0]) ** 2 + (coords[1, 1] - coords[0, 1]) ** 2)
    Nderiv = (dNdxi * (2 / h))[:, None, :]
    wq = (np.array([1, 1]) * (h / 2))[:, None]
    return wq, N, Nderiv


def quad4_shape_functions(coords):
    """core/shape_functions.py:27-45 (2x2 Gauss, unit weights folded into det J)."""
    xi = np.array([-1, 1, 1, -1]) * _S3
    eta = np.array([-1, -1, 1, 1]) * _S3
    N = np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta),
                  (1 - xi) * (1 + eta)], axis=1) / 4
    dNdxi = np.stack([-(1 - eta), 1 - eta, 1 + eta, -(1 + eta)], axis=1) / 4
    dNdeta = np.stack([-(1 - xi), -(1 + xi), 1 + xi, 1 - xi], axis=1) / 4
    J = np.stack([dNdxi @ coords, dNdeta @ coords], axis=1)
    wq = np.linalg.det(J)[:, None]
    Nderiv = np.linalg.inv(J) @ np.stack([dNdxi, dNdeta], axis=1)
    return wq, N, Nderiv


def hex8_shape_functions(coords):
    """core/shape_functions.py:47-87 (2x2x2 Gauss)."""
    xi = np.array([-1, 1, 1, -1, -1, 1, 1, -1]) * _S3
    eta = np.array([-1, -1, 1, 1, -1, -1, 1, 1]) * _S3
    ze = np.array([-1, -1, -1, -1, 1, 1, 1, 1]) * _S3
    sx = np.array([-1, 1, 1, -1, -1, 1, 1, -1])
    sy = np.array([-1, -1, 1, 1, -1, -1, 1, 1])
    sz = np.array([-1, -1, -1, -1, 1, 1, 1, 1])
    N = np.stack([(1 + sx[a] * xi) * (1 + sy[a] * eta) * (1 + sz[a] * ze) for a in range(8)], axis=1) / 8
    dNdxi = np.stack([sx[a] * (1 + sy[a] * eta) * (1 + sz[a] * ze) for a in range(8)], axis=1) / 8
    dNdeta = np.stack([sy[a] * (1 + sx[a] * xi) * (1 + sz[a] * ze) for a in range(8)], axis=1) / 8
    dNdze = np.stack([sz[a] * (1 + sx[a] * xi) * (1 + sy[a] * eta) for a in range(8)], axis=1) / 8
    J = np.stack([dNdxi @ coords, dNdeta @ coords, dNdze @ coords], axis=1)
    wq = np.linalg.det(J)[:, None]
    Nderiv = np.linalg.inv(J) @ np.stack([dNdxi, dNdeta, dNdze], axis=1)
    return wq, N, Nderiv


def lin3_shape_functions(coords):
    """core/shape_functions.py:89-106 (3-point Gauss on a quadratic edge)."""
    xi = np.array([-np.sqrt(3 / 5), 0.0, np.sqrt(3 / 5)])
    w = np.array([5 / 9, 8 / 9, 5 / 9])
    N = np.stack([xi * (xi - 1) / 2, 1 - xi ** 2, xi * (xi + 1) / 2], axis=1)
    dNdxi = np.stack([(2 * xi - 1) / 2, -2 * xi, (2 * xi + 1) / 2], axis=1)
    J = np.sqrt((dNdxi @ coords[:, 0]) ** 2 + (dNdxi @ coords[:, 1]) ** 2)
    Nderiv = (dNdxi / J[:, None])[:, None, :]
    wq = (w * J)[:, None]
    return wq, N, Nderiv


def quad9_shape_functions(coords):
    """core/shape_functions.py:108-159 (3x3 Gauss, eta-major point order)."""
    g = np.array([-np.sqrt(3 / 5), 0.0, np.sqrt(3 / 5)])
    xi, eta = np.meshgrid(g, g)
    xi, eta = xi.ravel(), eta.ravel()
    w1 = np.array([5 / 9, 8 / 9, 5 / 9])
    w = np.outer(w1, w1).ravel()
    N = np.stack([xi * eta * (xi - 1) * (eta - 1) / 4, (1 - xi ** 2) * eta * (eta - 1) / 2,
                  xi * eta * (xi + 1) * (eta - 1) / 4, xi * (xi + 1) * (1 - eta ** 2) / 2,
                  xi * eta * (xi + 1) * (eta + 1) / 4, (1 - xi ** 2) * eta * (eta + 1) / 2,
                  xi * eta * (xi - 1) * (eta + 1) / 4, xi * (xi - 1) * (1 - eta ** 2) / 2,
                  (1 - xi ** 2) * (1 - eta ** 2)], axis=1)
    dNdxi = np.stack([eta * (2 * xi - 1) * (eta - 1) / 4, -2 * xi * eta * (eta - 1) / 2,
                      eta * (2 * xi + 1) * (eta - 1) / 4, (2 * xi + 1) * (1 - eta ** 2) / 2,
                      eta * (2 * xi + 1) * (eta + 1) / 4, -2 * xi * eta * (eta + 1) / 2,
                      eta * (2 * xi - 1) * (eta + 1) / 4, (2 * xi - 1) * (1 - eta ** 2) / 2,
                      -2 * xi * (1 - eta ** 2)], axis=1)
    dNdeta = np.stack([xi * (xi - 1) * (2 * eta - 1) / 4, (1 - xi ** 2) * (2 * eta - 1) / 2,
                       xi * (xi + 1) * (2 * eta - 1) / 4, xi * (xi + 1) * (-2 * eta) / 2,
                       xi * (xi + 1) * (2 * eta + 1) / 4, (1 - xi ** 2) * (2 * eta + 1) / 2,
                       xi * (xi - 1) * (2 * eta + 1) / 4, xi * (xi - 1) * (-2 * eta) / 2,
                       -2 * eta * (1 - xi ** 2)], axis=1)
    J = np.stack([dNdxi @ coords, dNdeta @ coords], axis=1)
    wq = (w * np.linalg.det(J))[:, None]
    Nderiv = np.linalg.inv(J) @ np.stack([dNdxi, dNdeta], axis=1)
    return wq, N, Nderiv
