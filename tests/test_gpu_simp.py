"""GPU parity of whole SIMP optimisations, through the public API
(`toptimization_b200.optimizer.simp.run`), against the reference executed in
FP64 (tests/golden/ref_run_*.npz) and against the oracles.

Tolerances: compliance history 1e-9 relative (every iteration); density
max-abs 2.5e-8 after 100 OC iterations of the MBB 60x20 (measured on B200:
1.65e-8). Two FP64 CPU implementations of the same algorithm (the reference's
own code and oracle/simp64.py) already differ by 1.7e-8 in density there:
single CG stop points move by one iteration and the OC dynamics amplify
rounding; the bound is that spread with a margin of 1.5. At cg_tol 1e-12
(no stop point moves) the GPU is within 3.9e-9 (bound 1e-8); on the shorter
runs (12-53 OC iterations) within 4e-9 (bounds 5e-9 and 1e-8).
"""

import copy

import numpy as np
import pytest

from conftest import REPO, golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from oracle import simp64 as O  # noqa: E402
from toptimization_b200.optimizer.simp import RunHistory, SimpDesign, run  # noqa: E402
from toptimization_b200.problem import load_problem, problem_from_dict  # noqa: E402
from test_oracle import SMALL, bridge_100x50, small  # noqa: E402


def gpu_run(pr, **kw):
    hist = RunHistory()
    rho = run(pr, backend="cuda", live_viz=False, verbose=False, save=False, history=hist, **kw)
    return rho.reshape(-1), hist


def errors(rho, hist, g):
    c = np.array(hist.compliance)
    return dict(
        comp=float(np.max(np.abs(c - g["compliance"]) / np.abs(g["compliance"]))),
        vol=float(np.abs(np.array(hist.volume) - g["volume"]).max()),
        rho=float(np.abs(rho - g["rho_final"]).max()),
        cg=int(np.abs(np.array(hist.cg_iters) - g["cg_iters"]).max()),
        n=len(c), n_ref=len(g["compliance"]))


def test_mbb_60x20_100_iterations_vs_reference(tpo_built):
    """Config 0: plain FP64, Jacobi PCG at 1e-8, 100 OC iterations."""
    g = golden("ref_run_mbb_60x20")
    rho, hist = gpu_run(load_problem(REPO / "examples" / "mbb_60x20.yaml"))
    e = errors(rho, hist, g)
    print("mbb_60x20 vs reference:", e)
    assert e["n"] == e["n_ref"] == 100
    assert e["comp"] < 1e-9
    assert e["vol"] < 1e-9
    assert e["rho"] < 2.5e-8
    # stop points move where the residual crawls along the threshold
    assert e["cg"] <= 10


def test_mbb_60x20_tight_tolerance_vs_reference(tpo_built):
    g = golden("ref_run_mbb_60x20_tight")
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    pr.cg_tol, pr.max_cg_iter, pr.max_iter = 1e-12, 5000, 60
    rho, hist = gpu_run(pr)
    e = errors(rho, hist, g)
    print("mbb_60x20 cg_tol 1e-12 vs reference:", e)
    assert e["comp"] < 1e-10 and e["rho"] < 1e-8 and e["cg"] <= 1


@pytest.mark.parametrize("name,ov", [
    ("small_jacobi", dict(max_iter=30, tol=0.0)),
    ("small_sensitivity", dict(max_iter=30, tol=0.0, filter_type="sensitivity")),
    ("small_earlystop", dict(max_iter=200)),
])
def test_small_runs_vs_reference(tpo_built, name, ov):
    g = golden(f"ref_run_{name}")
    rho, hist = gpu_run(small(**ov))
    e = errors(rho, hist, g)
    print(name, e)
    assert e["n"] == e["n_ref"]       # same early-stop iteration
    assert e["comp"] < 1e-9 and e["rho"] < 5e-9 and e["cg"] <= 1


@pytest.mark.parametrize("name,pre", [("small_block_jacobi", "block_jacobi"),
                                      ("small_none", "none")])
def test_small_capped_runs_vs_reference(tpo_built, name, pre):
    """These solves hit max_cg_iterations=500 from OC iteration 5 on; the
    converged prefix is tight, the rest agrees to the rounding-dependent
    spread (see tests/test_oracle.py)."""
    g = golden(f"ref_run_{name}")
    rho, hist = gpu_run(small(max_iter=30, tol=0.0, preconditioner=pre))
    c = np.array(hist.compliance)
    conv = int(np.argmax(g["cg_iters"] == 500))
    assert np.max(np.abs(c[:conv] - g["compliance"][:conv]) / g["compliance"][:conv]) < 1e-8
    assert np.max(np.abs(c - g["compliance"]) / g["compliance"]) < 1e-3
    assert np.abs(rho - g["rho_final"]).max() < 5e-3


def test_bridge_100x50_vs_reference(tpo_built):
    g = golden("ref_run_bridge_100x50")
    rho, hist = gpu_run(bridge_100x50())
    e = errors(rho, hist, g)
    print("bridge_100x50", e)
    assert e["comp"] < 1e-9 and e["rho"] < 1e-8 and e["cg"] <= 2


def test_nodal_block_jacobi_vs_oracle(tpo_built):
    """The 2x2 nodal block-Jacobi option has no reference counterpart: checked
    against the oracle's restatement."""
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    pr.preconditioner = "nodal_block_jacobi"
    ref = O.run(pr)
    rho, hist = gpu_run(pr)
    c = np.array(hist.compliance)
    # the 2x2 inverse is formed differently (explicit formula vs LAPACK) and
    # the solve runs the one-launch recurrence (the oracle: the reference's
    # two-step one): rounding-level differences that the OC dynamics amplify
    # over 100 steps. Compliance stays within 5e-9; the density spread is of
    # the size the oracle itself shows against the reference's own FP64 run
    # (1.7e-8 on the Jacobi MBB) times the amplification of this trajectory.
    assert np.max(np.abs(c - ref.compliance) / np.abs(ref.compliance)) < 5e-9
    assert np.abs(rho - ref.rho).max() < 2e-7
    assert np.abs(np.array(hist.cg_iters) - ref.cg_iters).max() <= 10


@pytest.mark.parametrize("pre", ["jacobi", "nodal_block_jacobi"])
def test_mixed_precision_mbb_vs_reference(tpo_built, pre):
    """Mixed form (FP32-stored PCG with FP64 residual replacement, stop rule
    on the FP64 residual at 1e-8):
    compliance history within 1e-6 of the FP64 reference."""
    g = golden("ref_run_mbb_60x20")
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    pr.preconditioner = pre
    rho, hist = gpu_run(pr, precision="mixed")
    e = errors(rho, hist, g)
    print("mixed", pre, e, "outer", hist.outer_iters[:5])
    assert all(s == "converged" for s in hist.solve_status)
    assert e["comp"] < 1e-6
    assert e["rho"] < 1e-3


def test_cantilever_400x200_vs_c_oracle(tpo_built):
    """Config 1 (nodal block-Jacobi), first 8 OC iterations, plain FP64 and
    mixed, against the C/OpenMP oracle."""
    from oracle import simp_cpu
    pr = load_problem(REPO / "examples" / "cantilever_400x200.yaml")
    pr.max_iter = 8
    cpu = simp_cpu.CpuSimp(pr)
    ref = [cpu.iteration() for _ in range(8)]
    c_ref = np.array([r["compliance"] for r in ref])
    rho, hist = gpu_run(pr)
    c = np.array(hist.compliance)
    assert np.max(np.abs(c - c_ref) / c_ref) < 1e-9
    assert np.abs(rho - cpu.rho()).max() < 1e-8
    assert np.abs(np.array(hist.cg_iters) - [r["cg_iters"] for r in ref]).max() <= 2
    rho_m, hist_m = gpu_run(pr, precision="mixed")
    cm = np.array(hist_m.compliance)
    # Same input densities: the mixed solve meets the same FP64 stop rule.
    assert abs(cm[0] - c_ref[0]) / c_ref[0] < 1e-7
    # Later iterations: the OC bisection stops at a relative gap of 1e-4, so
    # its multiplier is a discrete function of dc and round-off-level
    # differences in dc can move the design by a bisection step; the two
    # trajectories then agree to that scale, not to the solve tolerance.
    assert np.max(np.abs(cm - c_ref) / c_ref) < 1e-4


def test_bridge_2048x1024_first_iteration(tpo_built):
    """Config 2 at full size: the first OC iteration's FP64 solve meets the
    stop rule on the true FP64 residual (checked with the oracle's assembled
    K), compliance equals f.u, and the mixed form's compliance is within
    1e-6 of the plain FP64 one."""
    pr = load_problem(REPO / "examples" / "bridge_2048x1024.yaml")
    d64 = SimpDesign(pr, precision="fp64")
    rec = d64.step()
    assert rec.solve.status == "converged"
    u = d64.u.cpu().numpy()
    rho_phys = d64.rho_phys.cpu().numpy()
    mesh = O.Mesh2D(pr.nelx, pr.nely, O.compute_Ke_2d(1.0, 0.3), pr.fixed_dofs)
    f = d64.f.cpu().numpy()
    r = f - O.assemble_K(mesh, O.simp_scale(rho_phys, pr.E_min, pr.penalty)) @ u
    assert np.linalg.norm(r) < 1.05e-8 * np.linalg.norm(f)
    assert rec.compliance == pytest.approx(float(f @ u), rel=1e-7)
    dmx = SimpDesign(pr, precision="mixed")
    recm = dmx.step()
    assert recm.solve.status == "converged"
    assert recm.compliance == pytest.approx(rec.compliance, rel=1e-6)
    print("bridge first iteration: fp64 CG", rec.cg_iters, f"{rec.seconds:.3f}s; mixed inner",
          recm.cg_iters, "outer", recm.solve.outer_iters, f"{recm.seconds:.3f}s")
