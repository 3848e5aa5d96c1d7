"""The structured H8 element operator of the 3D stiffness kernels
(csrc/hex3d.cuh h8_forces) restated in NumPy, step for step:
* forward Walsh-Hadamard transforms onto the trilinear monomials;
* the constant, linear and bilinear gradient groups with the constants
  4 lam, 8 mu, 4 mu, 4 lam / 3, 4 mu / 3, 4 (lam + 4 mu) / 9 over 64;
* the transposed transform back to the corners.
It must equal w Ke u with the unit-cube H8 stiffness built like the
reference's (src/toptimization/material.py, 2x2x2 Gauss), for any u and
weight, and for other Poisson ratios."""

import numpy as np
import pytest

from toptimization_b200.material import compute_Ke_3d

# reference corner order (mesh.py) as bits (dx, dy, dz)
REF = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def _forward(v):
    """v[dx][dy][dz] -> c[mx][my][mz]: sums, and + at the corner whose bit is 1."""
    v = v.copy()
    for ax in range(3):
        lo, hi = np.take(v, 0, axis=ax), np.take(v, 1, axis=ax)
        v = np.stack([lo + hi, hi - lo], axis=ax)
    return v


def _back(f):
    """F[mx][my][mz] -> f[dx][dy][dz] = sum_m m(corner) F_m."""
    f = f.copy()
    for ax in range(3):
        lo, hi = np.take(f, 0, axis=ax), np.take(f, 1, axis=ax)
        f = np.stack([lo - hi, lo + hi], axis=ax)
    return f


def structured(u, w, E, nu):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    q = w / 64.0
    L4, M8, M4 = 4 * lam * q, 8 * mu * q, 4 * mu * q
    A, Cc, K2 = (4 / 3) * lam * q, (4 / 3) * mu * q, (4 / 9) * (lam + 4 * mu) * q
    V = np.zeros((2, 2, 2, 3))
    for i, (x, y, z) in enumerate(REF):
        V[x, y, z] = u.reshape(8, 3)[i]
    C = np.stack([_forward(V[..., k]) for k in range(3)], axis=-1)
    a, b, d = C[1, 0, 0], C[0, 1, 0], C[0, 0, 1]
    p, qq, r, t = C[1, 1, 0], C[0, 1, 1], C[1, 0, 1], C[1, 1, 1]
    ltr = L4 * (a[0] + b[1] + d[2])
    nx, ny, nz = ltr + M8 * a[0], ltr + M8 * b[1], ltr + M8 * d[2]
    sxy, sxz, syz = M4 * (a[1] + b[0]), M4 * (a[2] + d[0]), M4 * (b[2] + d[1])
    Te, Tx, Tz = A * (p[0] + qq[2]), A * (p[1] + r[2]), A * (r[0] + qq[1])
    W = p[2] + r[1] + qq[0]
    F = np.zeros((2, 2, 2, 3))
    F[1, 0, 0] = (nx, sxy, sxz)
    F[0, 1, 0] = (sxy, ny, syz)
    F[0, 0, 1] = (sxz, syz, nz)
    F[1, 1, 0] = (Te + M4 * p[0], Tx + M4 * p[1], Cc * (W + p[2]))
    F[0, 1, 1] = (Cc * (W + qq[0]), Tz + M4 * qq[1], Te + M4 * qq[2])
    F[1, 0, 1] = (Tz + M4 * r[0], Cc * (W + r[1]), Tx + M4 * r[2])
    F[1, 1, 1] = K2 * t
    f = np.stack([_back(F[..., k]) for k in range(3)], axis=-1)
    return np.array([f[x, y, z] for (x, y, z) in REF]).reshape(-1)


@pytest.mark.parametrize("E,nu", [(1.0, 0.3), (2.5, 0.2), (1.0, 0.45)])
def test_structured_operator_equals_dense_ke(E, nu):
    Ke = compute_Ke_3d(E, nu)
    rng = np.random.default_rng(3)
    for _ in range(10):
        u = rng.standard_normal(24)
        w = rng.uniform(1e-3, 1.0)
        ref = w * (Ke @ u)
        assert np.max(np.abs(structured(u, w, E, nu) - ref)) <= 1e-14 * np.max(np.abs(ref))


def test_rigid_body_modes_give_no_force():
    u = np.tile([0.3, -1.2, 0.7], 8)  # a translation
    assert np.max(np.abs(structured(u, 1.0, 1.0, 0.3))) < 1e-15
