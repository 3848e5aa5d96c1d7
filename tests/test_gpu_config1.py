"""The 400x200 cantilever as the benchmark configuration states it
(examples/cantilever_400x200.yaml: left edge clamped, unit downward load at
the mid-height node of the right edge, volfrac 0.4, rmin 3, PCG to 1e-8 with
at most 10000 iterations), 200 OC iterations, in the plain FP64 and the mixed
form, with the 2x2 nodal block-Jacobi preconditioner and with the reference's
element-block preconditioner (src/toptimization/fem/preconditioner.py:47-108).

Against the C/OpenMP oracle's FP64 trajectories
(tests/golden/oracle_cantilever_400x200_*.npz, tests/golden/make_config1.py).
Each test prints the compliance (relative, worst iteration) and the final
density (max-abs) errors of its form.

Bounds:
  * nodal, FP64: compliance 1e-9 relative at every iteration, final density
    5e-6 max-abs, CG counts within 3 %. The oracle itself, run with 8 instead
    of 4 OpenMP threads (its reductions round differently), moves by 6.6e-10
    in compliance, 2.6e-6 in density and up to 82 CG iterations (2.5 %) over
    these 200 OC iterations; the GPU measured 6.1e-10, 1.9e-6 and 76.
  * nodal, mixed (inner FP32-stored PCG, residual replaced in FP64 each time
    it has dropped by 1e-4, the file's inner_tolerance; stop on the FP64
    residual at 1e-8): compliance 1e-6 relative at every iteration, final
    density 1e-3 max-abs (the OC bisection stops at a relative gap of 1e-4,
    so its multiplier is a discrete function of dc).
  * element-block: its solves stop at the 10000-iteration cap from OC
    iteration 3 on, in the oracle as on the GPU. Up to there (two converged
    solves) the FP64 form is held to 1e-9 and the mixed form to 1e-6; after
    that a capped solve's iterate depends on rounding (the residual is still
    far above the tolerance), so the histories agree to the size of that
    effect.
"""

import numpy as np
import pytest

from conftest import REPO, golden

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from toptimization_b200.optimizer.simp import RunHistory, run  # noqa: E402
from toptimization_b200.problem import load_problem  # noqa: E402


def _run(pre, precision):
    pr = load_problem(REPO / "examples" / "cantilever_400x200.yaml")
    pr.preconditioner = pre
    hist = RunHistory()
    rho = run(pr, backend="cuda", live_viz=False, verbose=False, save=False, history=hist,
              precision=precision)
    return rho.reshape(-1), hist


def _errors(rho, hist, g):
    c = np.array(hist.compliance)
    rel = np.abs(c - g["compliance"]) / np.abs(g["compliance"])
    return dict(n=len(c), comp=float(rel.max()), comp_hist=rel,
                rho=float(np.abs(rho - g["rho_final"]).max()),
                vol=float(np.abs(np.array(hist.volume) - g["volume"]).max()),
                cg=np.array(hist.cg_iters) - g["cg_iters"])


def _report(tag, e):
    print(f"{tag}: iterations {e['n']}, compliance rel err max {e['comp']:.3e}, "
          f"density max-abs {e['rho']:.3e}, volume {e['vol']:.2e}, "
          f"CG count diff [{e['cg'].min()}, {e['cg'].max()}]")


def test_cantilever_400x200_nodal_fp64():
    g = golden("oracle_cantilever_400x200_nodal_block_jacobi")
    rho, hist = _run("nodal_block_jacobi", "fp64")
    e = _errors(rho, hist, g)
    _report("400x200 nodal fp64", e)
    assert e["n"] == 200
    assert all(s == "converged" for s in hist.solve_status)
    assert e["comp"] < 1e-9
    assert e["rho"] < 5e-6
    assert np.abs(e["cg"]).max() <= max(3, int(0.03 * g["cg_iters"].max()))


def test_cantilever_400x200_nodal_mixed():
    g = golden("oracle_cantilever_400x200_nodal_block_jacobi")
    rho, hist = _run("nodal_block_jacobi", "mixed")
    e = _errors(rho, hist, g)
    _report("400x200 nodal mixed", e)
    assert e["n"] == 200
    assert all(s == "converged" for s in hist.solve_status)
    assert e["comp"] < 1e-6
    assert e["rho"] < 1e-3


@pytest.mark.parametrize("precision,bound", [("fp64", 1e-9), ("mixed", 1e-6)])
def test_cantilever_400x200_element_block(precision, bound):
    g = golden("oracle_cantilever_400x200_block_jacobi")
    conv = int(np.argmax(g["cg_iters"] == 10000))  # first capped solve
    assert conv == 2
    rho, hist = _run("block_jacobi", precision)
    e = _errors(rho, hist, g)
    _report(f"400x200 element-block {precision}", e)
    print("  compliance rel err, first 6 iterations:", np.array2string(e["comp_hist"][:6],
                                                                      precision=2))
    assert e["n"] == 200
    assert e["comp_hist"][:conv].max() < bound
    # Capped solves: the iterate after 10000 steps depends on rounding, and
    # after 200 OC iterations on such solves the design has settled into a
    # different layout (measured: density max-abs 0.999); its compliance still
    # tracks the oracle's (measured worst 1.1e-2 FP64, 1.4e-2 mixed) and
    # ends within 2 %.
    assert e["comp"] < 3e-2
    assert e["comp_hist"][-1] < 2e-2
