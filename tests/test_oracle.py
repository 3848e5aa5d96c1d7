"""Pin the FP64 oracle to the reference.

The golden vectors were produced by running the reference's own kernels and
`simp.run` in FP64 (tests/golden/make_golden.py). The NumPy oracle and the
C/OpenMP oracle must reproduce them; tolerances are the measured spread of two
FP64 implementations of the same algorithm (summation order differs), as
documented per test.
"""

import copy

import numpy as np
import pytest

from conftest import REPO, golden
from oracle import simp64 as O
from toptimization_b200.material import compute_Ke_2d
from toptimization_b200.problem import load_problem, problem_from_dict

KE = compute_Ke_2d(1.0, 0.3)
G = golden("ref_kernels")

SMALL = dict(
    domain={"nelx": 20, "nely": 10}, material={"E": 1.0, "nu": 0.3, "E_min": 1e-9},
    boundary_conditions={"fixed": [{"nodes": {"type": "edge", "edge": "left"},
                                    "dofs": ["x", "y"]}]},
    loads=[{"nodes": {"type": "point", "location": [20, 5]}, "force": [0.0, -1.0]}],
    optimization={"volume_fraction": 0.5, "penalty": 3.0, "filter_radius": 1.5,
                  "filter_type": "density", "max_iterations": 50, "tolerance": 0.01,
                  "move_limit": 0.2},
    solver={"max_cg_iterations": 500, "cg_tolerance": 1e-8, "preconditioner": "jacobi"})


def small(**ov):
    """The reference's 20x10 cantilever example, with overrides as in the fixtures."""
    pr = problem_from_dict(copy.deepcopy(SMALL))
    for k, v in ov.items():
        setattr(pr, k, v)
    return pr


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


# ---------------------------------------------------------------- kernels
def _mesh():
    return O.Mesh2D(int(G["nelx"]), int(G["nely"]), KE, G["fixed"])


def test_matvec_and_diag():
    mesh = _mesh()
    s = O.simp_scale(G["rho"], 1e-9, 3.0)
    Ap = O.assemble_K(mesh, s) @ G["p"]
    assert rel(Ap, G["Ap"]) < 1e-15
    assert float(G["p"] @ Ap) == pytest.approx(float(G["pAp"]), rel=1e-14)
    assert rel(O.jacobi_diag(mesh, s), G["diag"]) < 1e-15
    np.testing.assert_array_equal(O.diag_count(mesh), G["diag_count"])


def test_element_block_preconditioner():
    mesh = _mesh()
    z = O.block_jacobi_matrix(mesh, O.simp_scale(G["rho"], 1e-9, 3.0)) @ G["p2"]
    assert rel(z, G["bj_z"]) < 1e-15
    assert float(G["p2"] @ z) == pytest.approx(float(G["bj_rz"]), rel=1e-14)


def test_sensitivity_and_volume():
    dc, c = O.sensitivity(_mesh(), G["p"], G["rho"], 1e-9, 3.0)
    assert rel(dc, G["sens_dc"]) < 1e-15
    assert c == pytest.approx(float(G["sens_c"]), rel=1e-14)
    assert G["rho"].mean() == pytest.approx(float(G["volume"]), rel=1e-14)


@pytest.mark.parametrize("rmin", [1.5, 2.5, 4.0])
def test_filters(rmin):
    H, Hs = O.filter_matrix(int(G["nelx"]), int(G["nely"]), rmin)
    np.testing.assert_array_equal(O.density_filter(H, Hs, G["rho"]), G[f"filt_rho_r{rmin}"])
    np.testing.assert_array_equal(O.density_filter(H, Hs, G["dc_in"]), G[f"filt_dc_r{rmin}"])
    assert rel(O.sensitivity_filter(H, Hs, G["rho"], G["dc_in"]), G[f"filt_sens_r{rmin}"]) < 1e-15


@pytest.mark.parametrize("vf", [0.2, 0.4, 0.7])
def test_oc(vf):
    new, ch = O.oc_update(G["rho"], G["dc_in"], vf, 0.2)
    np.testing.assert_array_equal(new, G[f"oc_rho_vf{vf}"])
    assert ch == float(G[f"oc_change_vf{vf}"])


@pytest.mark.parametrize("pre", ["jacobi", "block_jacobi", "none"])
def test_pcg(pre):
    mesh = _mesh()
    f = np.zeros(mesh.n_dofs)
    f[G["force_dofs"]] = G["force_values"]
    res = O.pcg(mesh, O.simp_scale(G["rho"], 1e-9, 3.0), f, np.zeros(mesh.n_dofs), 1e-10,
                500, pre)
    assert abs(res.iters - int(G[f"pcg_{pre}_iters"])) <= 2
    assert rel(res.u, G[f"pcg_{pre}_u"]) < 1e-11


# ---------------------------------------------------------------- whole runs
def _compare_run(res, g, comp_tol, rho_tol, cg_tol_iters):
    c = np.array(res.compliance)
    assert len(c) == len(g["compliance"])
    assert np.max(np.abs(c - g["compliance"]) / np.abs(g["compliance"])) < comp_tol
    assert np.abs(np.array(res.volume) - g["volume"]).max() < comp_tol
    assert np.abs(res.rho - g["rho_final"]).max() < rho_tol
    assert np.abs(np.array(res.cg_iters) - g["cg_iters"]).max() <= cg_tol_iters


def test_run_mbb_60x20_100_iterations():
    """Config 0. Measured spread vs the reference: compliance 1.7e-11,
    density 1.7e-8 (PCG stop points differ by one iteration now and then)."""
    res = O.run(load_problem(REPO / "examples" / "mbb_60x20.yaml"))
    _compare_run(res, golden("ref_run_mbb_60x20"), 1e-9, 5e-8, 1)


def test_config0_density_floor_is_rounding_noise():
    """The density after config 0's 100 OC iterations is not reproducible to
    1e-8 by any implementation that rounds differently from the reference.
    The same oracle with only its PCG dot products rounded exactly
    (math.fsum) lands 4.7e-8 away from the reference and 5.2e-8 away from the
    oracle as shipped, while the compliance history still agrees to ~2e-10.
    At cg_tol 1e-8 a solve is only determined to its tolerance: a rounding
    change moves a stop point by an iteration, and the OC iterations carry
    the difference on. The GPU's density bound on config 0 rests on this."""
    import math

    def exact_dot(a, b):
        return math.fsum((a * b).tolist())

    g = golden("ref_run_mbb_60x20")
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    base = O.run(pr)
    exact = O.run(load_problem(REPO / "examples" / "mbb_60x20.yaml"), dot=exact_dot)
    c_ref = g["compliance"]
    assert np.max(np.abs(np.array(exact.compliance) - c_ref) / np.abs(c_ref)) < 1e-9
    assert np.abs(exact.rho - g["rho_final"]).max() > 2e-8
    assert np.abs(exact.rho - base.rho).max() > 2e-8


@pytest.mark.parametrize("name,ov", [
    ("small_jacobi", dict(max_iter=30, tol=0.0)),
    ("small_sensitivity", dict(max_iter=30, tol=0.0, filter_type="sensitivity")),
    ("small_earlystop", dict(max_iter=200)),
])
def test_run_small_converged_solves(name, ov):
    _compare_run(O.run(small(**ov)), golden(f"ref_run_{name}"), 1e-9, 5e-9, 1)


@pytest.mark.parametrize("name,ov", [
    ("small_block_jacobi", dict(max_iter=30, tol=0.0, preconditioner="block_jacobi")),
    ("small_none", dict(max_iter=30, tol=0.0, preconditioner="none")),
])
def test_run_small_capped_solves(name, ov):
    """From OC iteration 5 on these PCG solves stop at max_cg_iterations=500
    without converging; the iterate after a fixed number of unconverged
    steps depends on rounding, so only the converged prefix is tight."""
    g = golden(f"ref_run_{name}")
    res = O.run(small(**ov))
    c = np.array(res.compliance)
    conv = int(np.argmax(g["cg_iters"] == 500))
    assert conv >= 3
    assert np.max(np.abs(c[:conv] - g["compliance"][:conv]) / g["compliance"][:conv]) < 1e-8
    assert np.max(np.abs(c - g["compliance"]) / g["compliance"]) < 1e-3
    assert np.abs(res.rho - g["rho_final"]).max() < 5e-3


BRIDGE_100x50 = dict(
    domain={"nelx": 100, "nely": 50}, material={"E": 1.0, "nu": 0.3, "E_min": 1e-9},
    boundary_conditions={"fixed": [
        {"nodes": {"type": "point", "corner": "bottom-left"}, "dofs": ["x", "y"]},
        {"nodes": {"type": "point", "corner": "bottom-right"}, "dofs": ["x", "y"]}]},
    loads=[{"nodes": {"type": "point", "location": [50, 50]}, "force": [0.0, -1.0]}],
    optimization={"volume_fraction": 0.4, "penalty": 3.0, "filter_radius": 2.0,
                  "filter_type": "density", "max_iterations": 12, "tolerance": 0.0,
                  "move_limit": 0.2},
    solver={"max_cg_iterations": 2000, "cg_tolerance": 1e-8, "preconditioner": "jacobi"})


def bridge_100x50():
    """The reference's bridge example problem (12 OC iterations, fixed count)."""
    return problem_from_dict(copy.deepcopy(BRIDGE_100x50))


def test_run_bridge_100x50():
    _compare_run(O.run(bridge_100x50()), golden("ref_run_bridge_100x50"), 1e-9, 5e-8, 2)


def test_c_oracle_matches_numpy_oracle():
    from oracle import simp_cpu
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    pr.max_iter = 8
    ref = O.run(pr)
    cpu = simp_cpu.CpuSimp(pr)
    out = [cpu.iteration() for _ in range(8)]
    c = np.array([o["compliance"] for o in out])
    assert np.max(np.abs(c - ref.compliance) / np.abs(ref.compliance)) < 1e-9
    assert np.abs(cpu.rho() - ref.rho).max() < 1e-8
    assert [o["cg_iters"] for o in out] == pytest.approx(ref.cg_iters, abs=1)
