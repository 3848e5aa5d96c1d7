"""Structured-grid indexing: element-to-DOF table, element centres, and the
compact per-node arrays the device kernels read.

Conventions are the reference's (`src/toptimization/mesh.py:1-24`):
  node (ix, iy)  -> ix*(nely+1) + iy        (column-major, iy fastest)
  element (ex,ey)-> ex*nely + ey
  element DOFs   -> [x,y] of its corners counter-clockwise from bottom-left:
                    (ex,ey), (ex+1,ey), (ex+1,ey+1), (ex,ey+1)

The device never reads `edof`: the kernels derive neighbours from (ix, iy).
`edof` is still built (vectorised, not a Python double loop) because it is part
of the public API and the oracle uses it.
"""

from __future__ import annotations

import numpy as np

# Corner offsets (dx, dy) of the four element nodes, local order 0..3.
Q4_CORNERS = ((0, 0), (1, 0), (1, 1), (0, 1))
# H8 corner offsets (dx, dy, dz), local order 0..7 (reference mesh.py:87-96).
H8_CORNERS = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
              (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))

FIXED_X = 1  # bit in the per-node fixed mask
FIXED_Y = 2
FIXED_Z = 4


def build_edof_2d(problem) -> np.ndarray:
    """(n_elem, 8) int32 element-to-DOF table (reference `mesh.py:33-65`)."""
    nelx, nely = problem.nelx, problem.nely
    ex, ey = np.meshgrid(np.arange(nelx), np.arange(nely), indexing="ij")
    ex, ey = ex.reshape(-1), ey.reshape(-1)          # element e = ex*nely+ey
    cols = []
    for dx, dy in Q4_CORNERS:
        node = (ex + dx) * (nely + 1) + (ey + dy)
        cols += [2 * node, 2 * node + 1]
    return np.stack(cols, axis=1).astype(np.int32)


def build_edof_3d(problem) -> np.ndarray:
    """(n_elem, 24) int32 element-to-DOF table (reference `mesh.py:68-112`)."""
    nelx, nely, nelz = problem.nelx, problem.nely, problem.nelz
    ex, ey, ez = np.meshgrid(np.arange(nelx), np.arange(nely), np.arange(nelz),
                             indexing="ij")
    ex, ey, ez = ex.reshape(-1), ey.reshape(-1), ez.reshape(-1)
    cols = []
    for dx, dy, dz in H8_CORNERS:
        node = ((ex + dx) * (nely + 1) + (ey + dy)) * (nelz + 1) + (ez + dz)
        cols += [3 * node, 3 * node + 1, 3 * node + 2]
    return np.stack(cols, axis=1).astype(np.int32)


def build_edof(problem) -> np.ndarray:
    return build_edof_2d(problem) if problem.dim == 2 else build_edof_3d(problem)


def element_centers_2d(problem) -> np.ndarray:
    """(n_elem, 2) float32 centres in element units (reference `mesh.py:123-136`)."""
    e = np.arange(problem.nelx * problem.nely)
    return np.stack([e // problem.nely + 0.5, e % problem.nely + 0.5],
                    axis=1).astype(np.float32)


def element_centers_3d(problem) -> np.ndarray:
    """(n_elem, 3) float32 centres (reference `mesh.py:139-154`)."""
    nyz = problem.nely * problem.nelz
    e = np.arange(problem.nelx * nyz)
    return np.stack([e // nyz + 0.5, (e // problem.nelz) % problem.nely + 0.5,
                     e % problem.nelz + 0.5], axis=1).astype(np.float32)


def element_centers(problem) -> np.ndarray:
    return element_centers_2d(problem) if problem.dim == 2 else element_centers_3d(problem)


# --------------------------------------------------------------------------
# Per-node arrays the device reads (2D and 3D)
# --------------------------------------------------------------------------

def fixed_node_mask(problem) -> np.ndarray:
    """uint8 per node: bit0 = x DOF fixed, bit1 = y DOF fixed (3D: bit2 = z).

    Replaces the reference's int32-per-DOF `is_fixed` field
    (`src/toptimization/fem/fields.py:146-148`) with one byte per node.
    """
    mask = np.zeros(problem.n_nodes, dtype=np.uint8)
    dofs = np.asarray(problem.fixed_dofs, dtype=np.int64)
    if dofs.size:
        dim = problem.dim
        np.bitwise_or.at(mask, dofs // dim, (1 << (dofs % dim)).astype(np.uint8))
    return mask


def force_vector(problem, dtype=np.float64) -> np.ndarray:
    """Assembled load vector: repeated DOFs add up, fixed DOFs are zeroed
    (reference `src/toptimization/fem/fields.py:150-156`, here in FP64)."""
    f = np.zeros(problem.n_dofs, dtype=dtype)
    np.add.at(f, np.asarray(problem.force_dofs, dtype=np.int64),
              np.asarray(problem.force_values, dtype=dtype))
    if len(problem.fixed_dofs):
        f[np.asarray(problem.fixed_dofs, dtype=np.int64)] = 0.0
    return f
