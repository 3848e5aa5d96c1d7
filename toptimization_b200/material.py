"""Element stiffness for unit-size Q4 (plane stress) and H8 elements.

The matrices are the reference's (`src/toptimization/material.py:20-179`):
2x2 (2x2x2) Gauss quadrature of B^T D B on the unit square (cube), DOFs
ordered [x,y] per corner, corners counter-clockwise from bottom-left. Computed
here with the strain-displacement matrices of all Gauss points stacked and
contracted at once.

`regularized_inverse` is the element-block preconditioner's matrix
(reference `src/toptimization/fem/fields.py:133-143`):
    alpha = 0.1 * mean(|diag Ke|),  Ke_inv = (Ke + alpha*I)^-1   (FP64).
"""

from __future__ import annotations

import numpy as np

_GP = 1.0 / np.sqrt(3.0)


def _gauss_points(dim: int) -> np.ndarray:
    """Quadrature points in reference-loop order (first axis outermost)."""
    g = np.array([-_GP, _GP])
    grids = np.meshgrid(*([g] * dim), indexing="ij")
    return np.stack([x.reshape(-1) for x in grids], axis=1)


def compute_Ke_2d(E: float = 1.0, nu: float = 0.3) -> np.ndarray:
    """8x8 Q4 plane-stress stiffness of a unit element, FP64."""
    D = (E / (1.0 - nu ** 2)) * np.array([[1.0, nu, 0.0],
                                          [nu, 1.0, 0.0],
                                          [0.0, 0.0, (1.0 - nu) / 2.0]])
    sx = np.array([-1.0, 1.0, 1.0, -1.0])   # corner signs in xi
    sy = np.array([-1.0, -1.0, 1.0, 1.0])   # corner signs in eta
    Ke = np.zeros((8, 8))
    for xi, eta in _gauss_points(2):
        # dN/dx = 2 dN/dxi on the unit square (J = I/2, det J = 1/4)
        dx = 2.0 * sx * (1.0 + sy * eta) / 4.0
        dy = 2.0 * sy * (1.0 + sx * xi) / 4.0
        B = np.zeros((3, 8))
        B[0, 0::2] = dx
        B[1, 1::2] = dy
        B[2, 0::2] = dy
        B[2, 1::2] = dx
        Ke += 0.25 * (B.T @ D @ B)
    return Ke


def compute_Ke_3d(E: float = 1.0, nu: float = 0.3) -> np.ndarray:
    """24x24 H8 stiffness of a unit cube element, FP64."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] = lam + 2.0 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    s = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                  [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=float)
    Ke = np.zeros((24, 24))
    for xi, eta, zeta in _gauss_points(3):
        a, b, c = s[:, 0], s[:, 1], s[:, 2]
        dx = 2.0 * a * (1 + b * eta) * (1 + c * zeta) / 8.0
        dy = 2.0 * b * (1 + a * xi) * (1 + c * zeta) / 8.0
        dz = 2.0 * c * (1 + a * xi) * (1 + b * eta) / 8.0
        B = np.zeros((6, 24))
        B[0, 0::3], B[1, 1::3], B[2, 2::3] = dx, dy, dz
        B[3, 0::3], B[3, 1::3] = dy, dx
        B[4, 1::3], B[4, 2::3] = dz, dy
        B[5, 0::3], B[5, 2::3] = dz, dx
        Ke += 0.125 * (B.T @ D @ B)
    return Ke


def compute_Ke(E: float, nu: float, dim: int) -> np.ndarray:
    return compute_Ke_2d(E, nu) if dim == 2 else compute_Ke_3d(E, nu)


def regularized_inverse(Ke: np.ndarray) -> tuple[np.ndarray, float]:
    """(Ke + alpha I)^-1 and alpha = 0.1 mean|diag Ke|, both FP64."""
    Ke = np.asarray(Ke, dtype=np.float64)
    alpha = 0.1 * float(np.mean(np.abs(np.diag(Ke))))
    return np.linalg.inv(Ke + alpha * np.eye(Ke.shape[0])), alpha
