"""FP64 CPU oracle for the SIMP compliance-minimisation loop.

TEST INFRASTRUCTURE ONLY. This module is the checker: only `tests/`,
`__graft_entry__.smoke()` and `bench.py`'s CPU-baseline leg may import it. The
product path (`toptimization_b200`) never imports it and has no CPU fallback.

It restates, in vectorised NumPy/SciPy and in FP64, the reference's algorithm
(tomohiron907/toptimization, `src/toptimization/...`); every function cites the
lines it follows. Parity of this restatement is pinned against golden vectors
produced by running the reference's own kernels and `simp.run` in FP64 (see
`tests/golden/make_golden.py`, checked by `tests/test_oracle.py`).

Sparse assembly replaces the reference's matrix-free atomic scatter: the same
sums, in a different (and deterministic) order.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from toptimization_b200.material import compute_Ke, compute_Ke_2d, regularized_inverse
from toptimization_b200.mesh import build_edof_2d, build_edof_3d


@dataclass
class Mesh2D:
    """Structured Q4 mesh (`mesh.py:33-65`); with `nelz` set, the H8 mesh
    (`mesh.py:68-112`, node (ix,iy,iz) -> (ix(nely+1)+iy)(nelz+1)+iz, 24 DOFs
    per element). Every function below works on either through `edof`."""
    nelx: int
    nely: int
    Ke: np.ndarray
    fixed_dofs: np.ndarray
    nelz: int = 0
    edof: np.ndarray = field(init=False)

    def __post_init__(self):
        self.dim = 3 if self.nelz else 2
        if self.dim == 2:
            self.edof = build_edof_2d(self).astype(np.int64)
            self.n_elem = self.nelx * self.nely
            self.n_nodes = (self.nelx + 1) * (self.nely + 1)
        else:
            self.edof = build_edof_3d(self).astype(np.int64)
            self.n_elem = self.nelx * self.nely * self.nelz
            self.n_nodes = (self.nelx + 1) * (self.nely + 1) * (self.nelz + 1)
        self.n_dofs = self.dim * self.n_nodes
        self.is_fixed = np.zeros(self.n_dofs, dtype=bool)
        self.is_fixed[np.asarray(self.fixed_dofs, dtype=np.int64)] = True

    # COO index arrays of the assembled matrices, built on first use (E*dpe^2
    # entries: too large to keep for big 3D grids, which use matvec_free)
    @property
    def _rows(self):
        if not hasattr(self, "_rows_c"):
            dpe = self.edof.shape[1]
            self._rows_c = np.repeat(self.edof, dpe, axis=1).reshape(-1)
        return self._rows_c

    @property
    def _cols(self):
        if not hasattr(self, "_cols_c"):
            self._cols_c = np.tile(self.edof, (1, self.edof.shape[1])).reshape(-1)
        return self._cols_c


def Mesh3D(nelx, nely, nelz, Ke, fixed_dofs) -> Mesh2D:
    """The H8 mesh (see Mesh2D)."""
    return Mesh2D(nelx, nely, Ke, fixed_dofs, nelz=nelz)


def simp_scale(rho, E_min, penalty):
    """E_min + rho^p (1 - E_min)  (reference `fem/kernels.py:92,160`)."""
    return E_min + np.power(rho, penalty) * (1.0 - E_min)


def assemble_K(mesh: Mesh2D, scale: np.ndarray) -> sp.csr_matrix:
    """K(rho) with identity rows at fixed DOFs.

    Follows `fem/kernels.py:143-176`: Ap = sum_e scale_e Ke p_e, then
    Ap[i] = p[i] for fixed i (rows replaced, columns kept)."""
    vals = (scale[:, None, None] * mesh.Ke[None]).reshape(-1)
    keep = ~mesh.is_fixed[mesh._rows]
    fx = np.flatnonzero(mesh.is_fixed)
    rows = np.concatenate([mesh._rows[keep], fx])
    cols = np.concatenate([mesh._cols[keep], fx])
    v = np.concatenate([vals[keep], np.ones(fx.size)])
    return sp.csr_matrix((v, (rows, cols)), shape=(mesh.n_dofs, mesh.n_dofs))


def matvec(mesh, rho, p, E_min, penalty):
    """K(rho) p  (`fem/kernels.py:143-176`)."""
    return assemble_K(mesh, simp_scale(rho, E_min, penalty)) @ p


def matvec_free(mesh, scale, p):
    """K(rho) p element by element, without assembling K: the reference's
    matrix-free form (`fem/kernels.py:143-212`: gather p_e, Ke p_e, scale,
    scatter-add; fixed rows Ap = p), with the scatter as one bincount."""
    ke = (p[mesh.edof] @ mesh.Ke.T) * scale[:, None]
    ap = np.bincount(mesh.edof.reshape(-1), weights=ke.reshape(-1), minlength=mesh.n_dofs)
    ap[mesh.is_fixed] = p[mesh.is_fixed]
    return ap


class FreeOperator:
    """`K @ p` through matvec_free (for grids too large to assemble)."""

    def __init__(self, mesh, scale):
        self.mesh, self.scale = mesh, scale

    def __matmul__(self, p):
        return matvec_free(self.mesh, self.scale, p)


def jacobi_diag(mesh, scale):
    """diag_i = sum_e scale_e Ke_ii; fixed -> 1; floor 1e-20
    (`fem/kernels.py:76-101`)."""
    d = np.zeros(mesh.n_dofs)
    np.add.at(d, mesh.edof.reshape(-1), (scale[:, None] * np.diag(mesh.Ke)[None]).reshape(-1))
    d[mesh.is_fixed] = 1.0
    return np.where((~mesh.is_fixed) & (d < 1e-20), 1e-20, d)


def diag_count(mesh):
    """Elements sharing each DOF (`fem/preconditioner.py:19-30`)."""
    c = np.zeros(mesh.n_dofs, dtype=np.int64)
    np.add.at(c, mesh.edof.reshape(-1), 1)
    return c


def block_jacobi_matrix(mesh, scale):
    """The element-block preconditioner as a matrix
    (`fem/preconditioner.py:47-108`, `fem/fields.py:133-143`):
        M = C^-1/2 [sum_e w_e Ke_inv] C^-1/2,  w_e = s_e / max(s_e, alpha)^2,
    rows of fixed DOFs zeroed (z[fixed] = 0)."""
    Ke_inv, alpha = regularized_inverse(mesh.Ke)
    sc = np.maximum(scale, alpha)
    w = scale / (sc * sc)
    vals = (w[:, None, None] * Ke_inv[None]).reshape(-1)
    A = sp.csr_matrix((vals, (mesh._rows, mesh._cols)), shape=(mesh.n_dofs, mesh.n_dofs))
    cinv = 1.0 / np.sqrt(diag_count(mesh).astype(np.float64))
    cinv_rows = np.where(mesh.is_fixed, 0.0, cinv)
    return sp.diags(cinv_rows) @ A @ sp.diags(cinv)


def nodal_blocks(mesh, scale):
    """2x2 nodal block-Jacobi blocks B_n = sum_{e at n} s_e Ke[2a:2a+2, 2a:2a+2]
    (no reference counterpart); fixed DOFs get identity rows and columns."""
    B = np.zeros((mesh.n_nodes, 2, 2))
    for a in range(4):
        node = mesh.edof[:, 2 * a] // 2
        blk = mesh.Ke[2 * a:2 * a + 2, 2 * a:2 * a + 2]
        np.add.at(B, node, scale[:, None, None] * blk[None])
    fx = mesh.is_fixed.reshape(-1, 2)
    for d in range(2):
        B[fx[:, d], d, :] = 0.0
        B[fx[:, d], :, d] = 0.0
        B[fx[:, d], d, d] = 1.0
    return B


class Preconditioner:
    """z = M r for the four preconditioners (`fem/solver.py:79-102,127-145`)."""

    def __init__(self, kind, mesh, scale):
        self.kind = kind
        if kind == "jacobi":
            self.inv = 1.0 / jacobi_diag(mesh, scale)
        elif kind == "block_jacobi":
            self.M = block_jacobi_matrix(mesh, scale)
        elif kind == "nodal_block_jacobi":
            self.Binv = np.linalg.inv(nodal_blocks(mesh, scale))
        elif kind != "none":
            raise ValueError(kind)

    def __call__(self, r):
        if self.kind == "jacobi":
            return r * self.inv
        if self.kind == "block_jacobi":
            return self.M @ r
        if self.kind == "nodal_block_jacobi":
            return np.einsum("nij,nj->ni", self.Binv, r.reshape(-1, 2)).reshape(-1)
        return r.copy()


@dataclass
class SolveResult:
    u: np.ndarray
    iters: int
    status: str        # converged | max_iter | breakdown | zero_rhs
    rr: float


def _dot(a, b):
    return float(a @ b)


def pcg(mesh, scale, f, u0, tol, max_iter, precond="jacobi",
        assemble: bool = True, dot=_dot) -> SolveResult:
    """PCG exactly as the reference drives it (`fem/solver.py:27-159`):
    warm start with fixed DOFs zeroed, true initial residual, breakdown when
    |p.Ap| < 1e-30, recursive-residual stop ||r||^2 < (tol ||f||)^2 tested
    before the direction update, beta = rz_new/(rz_old + 1e-60). Returns the
    reference's count (it+1 on convergence, max_iter otherwise -- also after a
    breakdown). `dot` computes the iteration's dot products (a test swaps in
    other roundings of the same sums)."""
    f_norm = math.sqrt(float(f @ f))
    if f_norm < 1e-30:
        return SolveResult(np.zeros_like(f), 0, "zero_rhs", 0.0)
    tol_sq = (tol * f_norm) ** 2
    K = assemble_K(mesh, scale) if assemble else FreeOperator(mesh, scale)
    M = Preconditioner(precond, mesh, scale)
    u = u0.copy()
    u[mesh.is_fixed] = 0.0
    r = f - K @ u
    z = M(r)
    p = z.copy()
    rz_old = dot(r, z)
    rr = dot(r, r)
    for it in range(max_iter):
        Ap = K @ p
        pAp = dot(p, Ap)
        if abs(pAp) < 1e-30:
            return SolveResult(u, max_iter, "breakdown", rr)
        alpha = rz_old / pAp
        u += alpha * p
        r -= alpha * Ap
        z = M(r)
        rz_new = dot(r, z)
        rr = dot(r, r)
        if rr < tol_sq:
            return SolveResult(u, it + 1, "converged", rr)
        beta = rz_new / (rz_old + 1e-60)
        p = z + beta * p
        rz_old = rz_new
    return SolveResult(u, max_iter, "max_iter", rr)


def sensitivity(mesh, u, rho, E_min, penalty):
    """(dc, compliance): uKu_e = u_e^T Ke u_e, dc_e = -p rho^(p-1)(1-E_min) uKu_e,
    c = sum_e scale_e uKu_e  (`fem/kernels.py:234-272`)."""
    ue = u[mesh.edof]
    uKu = np.einsum("ei,ei->e", ue, ue @ mesh.Ke.T)
    dc = -penalty * np.power(rho, penalty - 1.0) * (1.0 - E_min) * uKu
    return dc, float(np.sum(simp_scale(rho, E_min, penalty) * uKu))


def filter_matrix(nelx, nely, rmin, nelz=0) -> tuple[sp.csr_matrix, np.ndarray]:
    """Hat-weight neighbour matrix H and row sums Hs
    (`optimizer/filter.py:22-103`): w = max(0, rmin - |c_e - c_j|) over the box
    |dx|,|dy| <= ceil(rmin) clipped to the domain, kept where w > 0; columns in
    the reference's (jx outer, jy inner) order. With nelz, the 3D box
    (`filter.py:75-97`, element (ex,ey,ez) -> (ex nely + ey) nelz + ez)."""
    if nelz:
        return _filter_matrix_3d(nelx, nely, nelz, rmin)
    R = math.ceil(rmin)
    ex, ey = np.divmod(np.arange(nelx * nely), nely)
    rows, cols, vals = [], [], []
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            w = rmin - math.sqrt(float(dx * dx + dy * dy))
            if not w > 0.0:
                continue
            jx, jy = ex + dx, ey + dy
            ok = (jx >= 0) & (jx < nelx) & (jy >= 0) & (jy < nely)
            rows.append(np.flatnonzero(ok))
            cols.append((jx * nely + jy)[ok])
            vals.append(np.full(ok.sum(), w))
    H = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nelx * nely, nelx * nely))
    H.sort_indices()
    return H, H @ np.ones(nelx * nely)


def _filter_matrix_3d(nelx, nely, nelz, rmin):
    R = math.ceil(rmin)
    n = nelx * nely * nelz
    e = np.arange(n)
    ex, ey, ez = e // (nely * nelz), (e // nelz) % nely, e % nelz
    rows, cols, vals = [], [], []
    for dx in range(-R, R + 1):
        for dy in range(-R, R + 1):
            for dz in range(-R, R + 1):
                w = rmin - math.sqrt(float(dx * dx + dy * dy + dz * dz))
                if not w > 0.0:
                    continue
                jx, jy, jz = ex + dx, ey + dy, ez + dz
                ok = ((jx >= 0) & (jx < nelx) & (jy >= 0) & (jy < nely)
                      & (jz >= 0) & (jz < nelz))
                rows.append(np.flatnonzero(ok))
                cols.append(((jx * nely + jy) * nelz + jz)[ok])
                vals.append(np.full(ok.sum(), w))
    H = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(n, n))
    H.sort_indices()
    return H, H @ np.ones(n)


def density_filter(H, Hs, x):
    """sum_j w_ej x_j / (sum_j w_ej + 1e-20)  (`optimizer/filter.py:106-149`)."""
    return (H @ x) / (Hs + 1e-20)


def sensitivity_filter(H, Hs, rho, dc):
    """sum_j w rho_j dc_j / (rho_e sum_j w + 1e-20)  (`optimizer/filter.py:152-171`)."""
    return (H @ (rho * dc)) / (rho * Hs + 1e-20)


def oc_update(rho, dc, volfrac, move, dv=None):
    """Bisection on lambda in [0, 1e9], at most 50 steps, stop when
    (hi-lo)/(hi+lo+1e-30) < 1e-4; the result and max change are those of the
    last midpoint evaluated (`optimizer/oc.py:21-93`)."""
    dv = np.ones_like(rho) if dv is None else dv
    lo, hi = 0.0, 1e9
    new, change = rho, 0.0
    lo_b = np.maximum(0.001, rho - move)
    hi_b = np.minimum(1.0, rho + move)
    for _ in range(50):
        mid = 0.5 * (lo + hi)
        be = np.maximum(-dc / (mid * dv + 1e-20), 0.0)
        new = np.maximum(lo_b, np.minimum(hi_b, rho * np.sqrt(be)))
        change = float(np.max(np.abs(new - rho)))
        vol = float(np.sum(new)) / rho.size
        if vol > volfrac:
            lo = mid
        else:
            hi = mid
        if (hi - lo) / (hi + lo + 1e-30) < 1e-4:
            break
    return new, change


@dataclass
class RunResult:
    rho: np.ndarray
    compliance: list
    volume: list
    change: list
    cg_iters: list
    status: list


def run(problem, max_iter=None, callback=None, dot=_dot) -> RunResult:
    """The SIMP loop of `optimizer/simp.py:108-109,141-219` (2D or 3D): density filter ->
    PCG on the physical density (warm start from it > 1) -> sensitivity ->
    dc projection -> OC on the design density -> volume; early stop when
    it > 5 and change < tol. The sensitivity-filter branch (:174-189) too.
    `dot` is passed to the PCG."""
    pr = problem
    Ke = compute_Ke(pr.E, pr.nu, pr.dim)
    nelz = pr.nelz if pr.dim == 3 else 0
    mesh = Mesh2D(pr.nelx, pr.nely, Ke, pr.fixed_dofs, nelz=nelz)
    f = np.zeros(mesh.n_dofs)
    np.add.at(f, np.asarray(pr.force_dofs, dtype=np.int64), np.asarray(pr.force_values, float))
    f[mesh.is_fixed] = 0.0
    H, Hs = filter_matrix(pr.nelx, pr.nely, pr.rmin, nelz)
    rho = np.full(mesh.n_elem, float(pr.volfrac))
    u_prev = np.zeros(mesh.n_dofs)
    out = RunResult(rho, [], [], [], [], [])
    n_it = pr.max_iter if max_iter is None else max_iter
    for it in range(1, n_it + 1):
        phys = density_filter(H, Hs, rho) if pr.filter_type == "density" else rho
        scale = simp_scale(phys, pr.E_min, pr.penalty)
        res = pcg(mesh, scale, f, u_prev if it > 1 else np.zeros(mesh.n_dofs),
                  pr.cg_tol, pr.max_cg_iter, pr.preconditioner, dot=dot)
        if res.status != "zero_rhs":
            u_prev = res.u
        dc, c = sensitivity(mesh, res.u, phys, pr.E_min, pr.penalty)
        if pr.filter_type == "density":
            dcf = density_filter(H, Hs, dc)
        else:
            dcf = sensitivity_filter(H, Hs, rho, dc)
        rho, change = oc_update(rho, dcf, pr.volfrac, pr.move_limit)
        out.compliance.append(c)
        out.volume.append(float(np.sum(rho)) / rho.size)
        out.change.append(change)
        out.cg_iters.append(res.iters)
        out.status.append(res.status)
        if callback is not None:
            callback(it, rho, c)
        if it > 5 and change < pr.tol:
            break
    out.rho = rho
    return out
