"""GPU parity of each libtpo kernel, called through the C ABI.

Checked against (a) golden vectors produced by the reference's own kernels
executed in FP64 (tests/golden/ref_kernels.npz) and (b) the FP64 oracle
(oracle/simp64.py) on seeded inputs, at small sizes and at the 2048x1024
bridge size. Tolerances are stated per test.
"""

import math

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import simp64 as O  # noqa: E402
from toptimization_b200 import _lib  # noqa: E402
from toptimization_b200.fem import kernels as K  # noqa: E402
from toptimization_b200.fem.solver import PCGSolver  # noqa: E402
from toptimization_b200.material import compute_Ke_2d, regularized_inverse  # noqa: E402
from toptimization_b200.optimizer import filter as F  # noqa: E402
from toptimization_b200.optimizer import oc as OCm  # noqa: E402

KE = compute_Ke_2d(1.0, 0.3)
G = golden("ref_kernels")
DEV = "cuda"


@pytest.fixture(scope="module", autouse=True)
def _stiffness(tpo_built):
    inv, alpha = regularized_inverse(KE)
    _lib.ensure_stiffness(KE, inv, alpha)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device=DEV, dtype=dtype)


def mask_from_dofs(nn, fixed):
    m = np.zeros(nn, dtype=np.uint8)
    fixed = np.asarray(fixed, dtype=np.int64)
    np.bitwise_or.at(m, fixed // 2, np.where(fixed % 2 == 0, 1, 2).astype(np.uint8))
    return m


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def left_clamped(nx, ny):
    return np.arange(0, 2 * (ny + 1))


# ---------------------------------------------------------------- matvec
def test_matvec_matches_reference_kernel():
    nx, ny = int(G["nelx"]), int(G["nely"])
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    m = dev(mask_from_dofs((nx + 1) * (ny + 1), G["fixed"]), torch.uint8)
    ap, pap = K.matvec(g, dev(G["rho"]), m, dev(G["p"]), with_dot=True)
    assert rel(ap.cpu().numpy(), G["Ap"]) < 1e-13
    assert abs(pap.item() - float(G["pAp"])) <= 1e-12 * abs(float(G["pAp"]))


@pytest.mark.parametrize("nx,ny", [(1, 1), (1, 7), (9, 1), (2, 2), (31, 29), (60, 20),
                                   (33, 61), (257, 130)])
def test_matvec_vs_oracle_sizes(nx, ny):
    rng = np.random.default_rng(nx * 1000 + ny)
    fixed = np.unique(rng.choice(2 * (nx + 1) * (ny + 1), size=max(1, nx), replace=True))
    mesh = O.Mesh2D(nx, ny, KE, fixed)
    rho = rng.uniform(0.001, 1.0, nx * ny)
    p = rng.standard_normal(mesh.n_dofs)
    ref = O.matvec(mesh, rho, p, 1e-9, 3.0)
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    m = dev(mask_from_dofs(mesh.n_nodes, fixed), torch.uint8)
    ap = K.matvec(g, dev(rho), m, dev(p)).cpu().numpy()
    assert rel(ap, ref) < 1e-13
    ap32 = K.matvec(g, dev(rho, torch.float32), m, dev(p, torch.float32)).cpu().numpy()
    assert rel(ap32, ref) < 5e-6


def test_matvec_bridge_full_size():
    """2048x1024 (4.2M DOFs): FP64 parity with the assembled oracle matrix,
    symmetry x.Ky == y.Kx, and identity rows at the pinned corners."""
    nx, ny = 2048, 1024
    fixed = np.array([0, 1, 2 * nx * (ny + 1), 2 * nx * (ny + 1) + 1])
    mesh = O.Mesh2D(nx, ny, KE, fixed)
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.001, 1.0, nx * ny)
    x = rng.standard_normal(mesh.n_dofs)
    y = rng.standard_normal(mesh.n_dofs)
    Kmat = O.assemble_K(mesh, O.simp_scale(rho, 1e-9, 3.0))
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    m = dev(mask_from_dofs(mesh.n_nodes, fixed), torch.uint8)
    kx = K.matvec(g, dev(rho), m, dev(x)).cpu().numpy()
    assert rel(kx, Kmat @ x) < 1e-12
    ky = K.matvec(g, dev(rho), m, dev(y)).cpu().numpy()
    free = ~mesh.is_fixed
    # symmetric on the free block (fixed rows are identity, columns are kept)
    xf, yf = np.where(free, x, 0.0), np.where(free, y, 0.0)
    kxf = K.matvec(g, dev(rho), m, dev(xf)).cpu().numpy()
    kyf = K.matvec(g, dev(rho), m, dev(yf)).cpu().numpy()
    assert abs(yf @ kxf - xf @ kyf) <= 1e-10 * abs(yf @ kxf)
    np.testing.assert_array_equal(kx[fixed], x[fixed])
    assert np.isfinite(ky).all()


def test_matvec_rigid_translation_is_free_of_stress():
    nx, ny = 40, 17
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    nn = (nx + 1) * (ny + 1)
    u = np.tile([0.3, -1.2], nn)
    ap = K.matvec(g, dev(np.full(nx * ny, 0.7)), dev(np.zeros(nn), torch.uint8), dev(u))
    assert float(ap.abs().max()) < 1e-13


# ---------------------------------------------------------------- filters
@pytest.mark.parametrize("rmin", [1.5, 2.5, 4.0])
def test_filters_match_reference_kernels(rmin):
    nx, ny = int(G["nelx"]), int(G["nely"])
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    out = torch.empty(nx * ny, dtype=torch.float64, device=DEV)
    F.density_filter(g, rmin, dev(G["rho"]), out)
    assert rel(out.cpu().numpy(), G[f"filt_rho_r{rmin}"]) < 1e-14
    F.density_filter(g, rmin, dev(G["dc_in"]), out)
    assert rel(out.cpu().numpy(), G[f"filt_dc_r{rmin}"]) < 1e-14
    F.sensitivity_filter(g, rmin, dev(G["rho"]), dev(G["dc_in"]), out)
    assert rel(out.cpu().numpy(), G[f"filt_sens_r{rmin}"]) < 1e-13


@pytest.mark.parametrize("nx,ny,rmin", [(1, 1, 1.5), (3, 50, 4.0), (64, 33, 1.0),
                                        (100, 70, 3.0), (70, 100, 16.0), (513, 200, 2.7)])
def test_filter_vs_oracle(nx, ny, rmin):
    rng = np.random.default_rng(int(rmin * 10) + nx)
    x = rng.uniform(0.0, 1.0, nx * ny)
    H, Hs = O.filter_matrix(nx, ny, rmin)
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    out = torch.empty(nx * ny, dtype=torch.float64, device=DEV)
    s64 = torch.empty_like(out)
    s32 = torch.empty(nx * ny, dtype=torch.float32, device=DEV)
    F.density_filter(g, rmin, dev(x), out, s64, s32)
    ref = O.density_filter(H, Hs, x)
    assert rel(out.cpu().numpy(), ref) < 1e-14
    np.testing.assert_allclose(s64.cpu().numpy(), O.simp_scale(ref, 1e-9, 3.0), rtol=1e-14)
    np.testing.assert_array_equal(s32.cpu().numpy(), s64.cpu().numpy().astype(np.float32))


def test_filter_bridge_full_size_preserves_constants():
    nx, ny = 2048, 1024
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    x = torch.full((nx * ny,), 0.3, dtype=torch.float64, device=DEV)
    out = torch.empty_like(x)
    F.density_filter(g, 4.0, x, out)
    assert float((out - 0.3).abs().max()) < 1e-15   # normalised weights
    rng = np.random.default_rng(3)
    xs = rng.uniform(size=nx * ny)
    F.density_filter(g, 4.0, dev(xs), out)
    H, Hs = O.filter_matrix(nx, ny, 4.0)
    assert rel(out.cpu().numpy(), O.density_filter(H, Hs, xs)) < 1e-14


# ---------------------------------------------------------------- sensitivity
def test_sensitivity_matches_reference_kernel():
    nx, ny = int(G["nelx"]), int(G["nely"])
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    dc = torch.empty(nx * ny, dtype=torch.float64, device=DEV)
    c = torch.empty(1, dtype=torch.float64, device=DEV)
    K.sensitivity(g, dev(G["rho"]), dev(G["p"]), dc, c, K.sensitivity_workspace(g, DEV))
    assert rel(dc.cpu().numpy(), G["sens_dc"]) < 1e-13
    assert c.item() == pytest.approx(float(G["sens_c"]), rel=1e-13)


@pytest.mark.parametrize("nx,ny", [(1, 1), (17, 3), (400, 200), (2048, 1024)])
def test_sensitivity_vs_oracle(nx, ny):
    rng = np.random.default_rng(nx + ny)
    mesh = O.Mesh2D(nx, ny, KE, np.array([0]))
    rho = rng.uniform(0.001, 1.0, nx * ny)
    u = rng.standard_normal(mesh.n_dofs)
    dc_ref, c_ref = O.sensitivity(mesh, u, rho, 1e-9, 3.0)
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    dc = torch.empty(nx * ny, dtype=torch.float64, device=DEV)
    c = torch.empty(1, dtype=torch.float64, device=DEV)
    K.sensitivity(g, dev(rho), dev(u), dc, c, K.sensitivity_workspace(g, DEV))
    assert rel(dc.cpu().numpy(), dc_ref) < 1e-13
    assert c.item() == pytest.approx(c_ref, rel=1e-12)


# ---------------------------------------------------------------- OC
@pytest.mark.parametrize("vf", [0.2, 0.4, 0.7])
def test_oc_matches_reference(vf):
    nx, ny = int(G["nelx"]), int(G["nely"])
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    rho = dev(G["rho"])
    out = torch.empty_like(rho)
    res = torch.empty(4, dtype=torch.float64, device=DEV)
    OCm.oc_update(g, vf, 0.2, rho, dev(G["dc_in"]), out, res, OCm.oc_workspace(g, DEV))
    assert np.abs(out.cpu().numpy() - G[f"oc_rho_vf{vf}"]).max() < 1e-15
    assert res[0].item() == pytest.approx(float(G[f"oc_change_vf{vf}"]), abs=1e-15)


@pytest.mark.parametrize("n,vf", [(1200, 0.5), (80000, 0.4), (2097152, 0.3)])
def test_oc_vs_oracle_in_place(n, vf):
    rng = np.random.default_rng(n)
    rho = rng.uniform(0.001, 1.0, n)
    dc = -rng.exponential(1.0, n) * 10.0 ** rng.uniform(-6, 2, n)
    ref, ch = O.oc_update(rho, dc, vf, 0.2)
    g = _lib.grid(n, 1, 1e-9, 3.0)
    r = dev(rho)
    res = torch.empty(4, dtype=torch.float64, device=DEV)
    OCm.oc_update(g, vf, 0.2, r, dev(dc), r, res, OCm.oc_workspace(g, DEV))   # in place
    assert np.abs(r.cpu().numpy() - ref).max() < 1e-12
    assert res[0].item() == pytest.approx(ch, abs=1e-12)
    assert res[1].item() == pytest.approx(ref.mean(), rel=1e-12)
    assert 1 <= res[3].item() <= 50


# ---------------------------------------------------------------- PCG
def _pcg_setup(nx, ny, fixed, loads, rho):
    mesh = O.Mesh2D(nx, ny, KE, fixed)
    f = np.zeros(mesh.n_dofs)
    for d, v in loads:
        f[d] += v
    f[mesh.is_fixed] = 0.0
    return mesh, f, dev(mask_from_dofs(mesh.n_nodes, fixed), torch.uint8)


def _iter_band(ref_iters) -> int:
    return max(3, int(np.ceil(0.02 * int(ref_iters))))


@pytest.mark.parametrize("pre", ["jacobi", "block_jacobi", "none"])
def test_pcg_matches_reference_solver(pre):
    """Cold then warm solve at tol 1e-10, as the reference's solver.solve ran them."""
    nx, ny = int(G["nelx"]), int(G["nely"])
    loads = list(zip(G["force_dofs"], G["force_values"]))
    mesh, f, m = _pcg_setup(nx, ny, G["fixed"], loads, None)
    s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), preconditioner=pre, max_iter=500, tol=1e-10)
    u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(G["rho"]), dev(f), m, u, warm_start=False)
    assert info.status == "converged"
    # Iteration counts at tol 1e-10 depend on rounding order (the reference's
    # own scatter uses float atomics, so its count is not rounding-stable
    # either): allow 3 iterations or 2 %, whichever is larger.
    assert abs(info.iters - int(G[f"pcg_{pre}_iters"])) <= _iter_band(G[f"pcg_{pre}_iters"])
    assert rel(u.cpu().numpy(), G[f"pcg_{pre}_u"]) < 1e-9
    rho2 = np.clip(G["rho"] * 0.9 + 0.05, 0.001, 1.0)
    info2 = s.solve(dev(rho2), dev(f), m, u, warm_start=True)
    assert abs(info2.iters - int(G[f"pcg_{pre}_warm_iters"])) <= _iter_band(
        G[f"pcg_{pre}_warm_iters"])
    assert rel(u.cpu().numpy(), G[f"pcg_{pre}_warm_u"]) < 1e-9


@pytest.mark.parametrize("pre", ["jacobi", "block_jacobi", "nodal_block_jacobi", "none"])
@pytest.mark.parametrize("nx,ny", [(60, 20), (97, 41)])
def test_pcg_vs_oracle(pre, nx, ny):
    rng = np.random.default_rng(nx * 7 + len(pre))
    fixed = left_clamped(nx, ny)
    loads = [(2 * (nx * (ny + 1) + ny // 2) + 1, -1.0)]
    mesh, f, m = _pcg_setup(nx, ny, fixed, loads, None)
    rho = rng.uniform(0.05, 1.0, nx * ny)
    ref = O.pcg(mesh, O.simp_scale(rho, 1e-9, 3.0), f, np.zeros(mesh.n_dofs), 1e-8, 5000, pre)
    s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), preconditioner=pre, max_iter=5000, tol=1e-8)
    u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(rho), dev(f), m, u, warm_start=False)
    assert info.status == ref.status == "converged"
    assert abs(info.iters - ref.iters) <= max(3, ref.iters // 100)
    uu = u.cpu().numpy()
    # both stopped at ||r|| < 1e-8 ||f||: solutions agree to the solve tolerance
    assert rel(uu, ref.u) < 1e-6
    # compliance f.u is quadratic in the error: much tighter
    assert float(f @ uu) == pytest.approx(float(f @ ref.u), rel=1e-9)


@pytest.mark.parametrize("pre", ["jacobi", "nodal_block_jacobi", "none"])
def test_one_launch_recurrence_matches_standard(pre):
    """The one-launch iteration (Chronopoulos-Gear form, one reduction) and the
    reference's two-step recurrence solve the same system: counts within the
    rounding band, solutions within the solve tolerance, f.u within 1e-9, and
    the one-launch kernel is what ran (profile counters)."""
    nx, ny = 150, 70
    rng = np.random.default_rng(11)
    fixed = left_clamped(nx, ny)
    loads = [(2 * (nx * (ny + 1) + ny // 2) + 1, -1.0)]
    mesh, f, m = _pcg_setup(nx, ny, fixed, loads, None)
    rho = rng.uniform(0.01, 1.0, nx * ny)
    lib = _lib.load()
    out = {}
    for rec in ("standard", "single"):
        s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), preconditioner=pre,
                      max_iter=20000, tol=1e-8, recurrence=rec)
        u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
        _lib.check(lib.tpo_profile_enable(1))
        _lib.check(lib.tpo_profile_reset())
        info = s.solve(dev(rho), dev(f), m, u, warm_start=False)
        prof = _lib.profile_read()
        _lib.check(lib.tpo_profile_enable(0))
        assert info.status == "converged", (rec, info)
        if rec == "single":
            assert prof["step_launches"] == info.updates and prof["dir_launches"] == 0
        else:
            assert prof["step_launches"] == 0 and prof["dir_launches"] == info.updates
        out[rec] = (info, u.cpu().numpy())
    (i0, u0), (i1, u1) = out["standard"], out["single"]
    assert abs(i0.iters - i1.iters) <= _iter_band(i0.iters)
    assert rel(u1, u0) < 1e-6
    assert float(f @ u1) == pytest.approx(float(f @ u0), rel=1e-9)
    K64 = O.assemble_K(mesh, O.simp_scale(rho, 1e-9, 3.0))
    r = f - K64 @ u1
    # the recursive residual met the tolerance; the true one follows it to round-off
    assert np.linalg.norm(r) < 1.01e-8 * np.linalg.norm(f)


def test_one_launch_recurrence_rejects_mixed_and_block():
    with pytest.raises(ValueError):
        PCGSolver(10, 5, 1e-9, 3.0, 1.0, precision="mixed", recurrence="single")
    with pytest.raises(ValueError):
        PCGSolver(10, 5, 1e-9, 3.0, 1.0, preconditioner="block_jacobi", recurrence="single")
    g = _lib.grid(10, 5, 1e-9, 3.0)
    cfg = _lib.TpoSolveCfg(precond=_lib.PRECOND["jacobi"], precision=_lib.PRECISION["mixed"],
                           max_iter=10, warm_start=0, tol=1e-8, f_norm_sq=1.0, inner_tol=1e-3,
                           max_outer=5, poll_every=0, recurrence=2)
    lib = _lib.load()
    nb = lib.tpo_pcg_workspace_bytes(g, cfg)
    ws = torch.empty(max(nb, 256), dtype=torch.uint8, device=DEV)
    z = torch.zeros(2 * 11 * 6, dtype=torch.float64, device=DEV)
    rho = torch.full((50,), 0.5, dtype=torch.float64, device=DEV)
    m = torch.zeros(66, dtype=torch.uint8, device=DEV)
    res = _lib.TpoSolveResult()
    rc = lib.tpo_pcg_solve(g, cfg, _lib.ptr(rho), _lib.ptr(z), _lib.ptr(m), _lib.ptr(z),
                           _lib.ptr(ws), ws.numel(), res, _lib.stream_handle())
    assert rc == 1  # TPO_ERR_ARGS
    assert b"one-launch" in lib.tpo_last_error_string()


@pytest.mark.parametrize("pre", ["jacobi", "block_jacobi", "nodal_block_jacobi"])
def test_pcg_mixed_precision(pre):
    nx, ny = 120, 60
    rng = np.random.default_rng(5)
    fixed = left_clamped(nx, ny)
    loads = [(2 * (nx * (ny + 1) + ny // 2) + 1, -1.0)]
    mesh, f, m = _pcg_setup(nx, ny, fixed, loads, None)
    rho = rng.uniform(0.001, 1.0, nx * ny)
    K64 = O.assemble_K(mesh, O.simp_scale(rho, 1e-9, 3.0))
    s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), preconditioner=pre, precision="mixed",
                  max_iter=20000, tol=1e-8, inner_tol=1e-3, max_outer=60)
    u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(rho), dev(f), m, u, warm_start=False)
    assert info.status == "converged", info
    uu = u.cpu().numpy()
    r = f - K64 @ uu                          # true FP64 residual
    assert np.linalg.norm(r) < 1e-8 * np.linalg.norm(f) * 1.0001
    assert info.rr == pytest.approx(float(r @ r), rel=1e-6)
    ref = O.pcg(mesh, O.simp_scale(rho, 1e-9, 3.0), f, np.zeros(mesh.n_dofs), 1e-10, 20000, pre)
    assert float(f @ uu) == pytest.approx(float(f @ ref.u), rel=1e-6)
    assert info.outer_iters >= 1


def test_pcg_zero_rhs_and_max_iter():
    nx, ny = 10, 6
    mesh, f, m = _pcg_setup(nx, ny, left_clamped(nx, ny), [(0, 5.0)], None)  # load on a fixed DOF
    assert not f.any()
    s = PCGSolver(nx, ny, 1e-9, 3.0, 0.0, max_iter=50, tol=1e-8)
    u = torch.ones(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(np.full(nx * ny, 0.5)), dev(f), m, u)
    assert info.status == "zero_rhs" and info.iters == 0 and float(u.abs().max()) == 0.0
    mesh, f, m = _pcg_setup(nx, ny, left_clamped(nx, ny), [(2 * 70 + 1, -1.0)], None)
    s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), max_iter=3, tol=1e-12)
    info = s.solve(dev(np.full(nx * ny, 0.5)), dev(f), m, u, warm_start=False)
    ref = O.pcg(mesh, O.simp_scale(np.full(nx * ny, 0.5), 1e-9, 3.0), f, np.zeros(mesh.n_dofs),
                1e-12, 3, "jacobi")
    assert info.status == "max_iter" and info.iters == 3 and info.updates == 3
    assert rel(u.cpu().numpy(), ref.u) < 1e-12


def test_pcg_breakdown_reports_max_iter_like_the_reference():
    """|p.Ap| < 1e-30 stops the solve; the reference then returns max_iter."""
    nx, ny = 8, 4
    mesh, f, m = _pcg_setup(nx, ny, left_clamped(nx, ny), [(2 * 40 + 1, -1e-3)], None)
    s = PCGSolver(nx, ny, 1e-30, 3.0, float(f @ f), preconditioner="none", max_iter=40,
                  tol=1e-8)
    u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(np.full(nx * ny, 1e-12)), dev(f), m, u, warm_start=False)
    ref = O.pcg(mesh, O.simp_scale(np.full(nx * ny, 1e-12), 1e-30, 3.0), f,
                np.zeros(mesh.n_dofs), 1e-8, 40, "none")
    assert ref.status == "breakdown"
    assert info.status == "breakdown" and info.iters == 40 and info.updates == 0


def test_pcg_bridge_full_size_few_iterations():
    """2048x1024: 25 Jacobi iterations from zero agree with the oracle's."""
    nx, ny = 2048, 1024
    fixed = np.array([0, 1, 2 * nx * (ny + 1), 2 * nx * (ny + 1) + 1])
    top = [(2 * (ix * (ny + 1) + ny) + 1, -1.0 / (nx + 1)) for ix in range(nx + 1)]
    mesh, f, m = _pcg_setup(nx, ny, fixed, top, None)
    rho = np.full(nx * ny, 0.3)
    ref = O.pcg(mesh, O.simp_scale(rho, 1e-9, 3.0), f, np.zeros(mesh.n_dofs), 1e-8, 25, "jacobi")
    s = PCGSolver(nx, ny, 1e-9, 3.0, float(f @ f), max_iter=25, tol=1e-8)
    u = torch.zeros(mesh.n_dofs, dtype=torch.float64, device=DEV)
    info = s.solve(dev(rho), dev(f), m, u, warm_start=False)
    assert info.updates == 25 and ref.iters == 25
    assert rel(u.cpu().numpy(), ref.u) < 1e-10
    assert math.isclose(info.rr, ref.rr, rel_tol=1e-8)
