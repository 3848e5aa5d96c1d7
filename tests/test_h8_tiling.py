"""The tiling scheme of the 3D element-centric kernel (csrc/hex3d.cuh
k_hex_elem), modelled in NumPy on the CPU:
* tiles of EY x EZ elements with origins (y0 - 1 + ey, z0 - 1 + ez) that
  finish (EY-1) x (EZ-1) nodes;
* chunks of node planes along x, each starting with element plane xa-1;
* the dx = 1 corners carried to the next plane, and the three handover
  corners (0,1), (1,0), (0,0) taken from the neighbouring element threads,
  added in the kernel's order.
Every node must be written exactly once, and the result must equal the dense
K p assembled from the reference-built Ke. The element forces come from the
structured operator of test_h8_structured."""

import numpy as np
import pytest

from test_h8_structured import REF, structured
from toptimization_b200.material import compute_Ke_3d


def dense(nx, ny, nz, w, p):
    Ke = compute_Ke_3d(1.0, 0.3)
    out = np.zeros_like(p)
    for ex in range(nx):
        for ey in range(ny):
            for ez in range(nz):
                nodes = [((ex + dx) * (ny + 1) + ey + dy) * (nz + 1) + ez + dz for dx, dy, dz in REF]
                dofs = np.array([[3 * n + c for c in range(3)] for n in nodes]).reshape(-1)
                out[dofs] += w[(ex * ny + ey) * nz + ez] * (Ke @ p[dofs])
    return out


def tiled(nx, ny, nz, w, p, EY, EZ, xc):
    ny1, nz1 = ny + 1, nz + 1
    tzc = -(-(nz + 1) // (EZ - 1))
    tyc = -(-(ny + 1) // (EY - 1))
    out = np.full_like(p, np.nan)

    def node(x, y, z):
        if 0 <= x <= nx and 0 <= y <= ny and 0 <= z <= nz:
            n = (x * ny1 + y) * nz1 + z
            return p[3 * n:3 * n + 3]
        return np.zeros(3)

    def forces(ex, Y, Z):  # [bits dx + 2 dy + 4 dz][3]
        inside = 0 <= ex < nx and 0 <= Y < ny and 0 <= Z < nz
        wt = w[(ex * ny + Y) * nz + Z] if inside else 0.0
        u = np.array([node(ex + dx, Y + dy, Z + dz) for dx, dy, dz in REF]).reshape(-1)
        f = structured(u, wt, 1.0, 0.3).reshape(8, 3)
        fb = np.zeros((8, 3))
        for r, (dx, dy, dz) in enumerate(REF):
            fb[dx + 2 * dy + 4 * dz] = f[r]
        return fb

    def sums(F, ey, ez, dx):  # own (1,1), then (0,1), (1,0), (0,0) from the neighbours
        return ((F[ey, ez][dx + 6] + F[ey + 1, ez][dx + 4]) + F[ey, ez + 1][dx + 2]) + \
            F[ey + 1, ez + 1][dx]

    for tile in range(tyc * tzc):
        ty, tz = divmod(tile, tzc)
        y0, z0 = ty * (EY - 1), tz * (EZ - 1)
        for xa in range(0, nx + 1, xc):
            xb = min(xa + xc, nx + 1)

            def plane(ex):
                return {(ey, ez): forces(ex, y0 - 1 + ey, z0 - 1 + ez)
                        for ey in range(EY) for ez in range(EZ)}

            F = plane(xa - 1)
            carry = {(ey, ez): sums(F, ey, ez, 1) for ey in range(EY - 1) for ez in range(EZ - 1)}
            for x in range(xa, xb):
                F = plane(x)
                for ey in range(EY - 1):
                    for ez in range(EZ - 1):
                        oy, oz = y0 + ey, z0 + ez
                        if oy <= ny and oz <= nz:
                            n = (x * ny1 + oy) * nz1 + oz
                            assert np.isnan(out[3 * n]), "a node written twice"
                            out[3 * n:3 * n + 3] = carry[ey, ez] + sums(F, ey, ez, 0)
                        carry[ey, ez] = sums(F, ey, ez, 1)
    assert not np.isnan(out).any(), "a node never written"
    return out


@pytest.mark.parametrize("nx,ny,nz,EY,EZ,xc", [
    (5, 4, 3, 4, 3, 2), (3, 6, 7, 3, 5, 4), (4, 3, 5, 5, 4, 1), (6, 5, 4, 18, 14, 3)])
def test_tiled_element_march_equals_dense_matvec(nx, ny, nz, EY, EZ, xc):
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz)
    w = rng.uniform(0.1, 1.0, nx * ny * nz)
    p = rng.standard_normal(3 * (nx + 1) * (ny + 1) * (nz + 1))
    ref = dense(nx, ny, nz, w, p)
    got = tiled(nx, ny, nz, w, p, EY, EZ, xc)
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
