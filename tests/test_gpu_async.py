"""The asynchronous solve (tpo_pcg_solve_async) and the CUDA-graph engine.

  * every form (plain FP64 in both recurrences, the element-block
    preconditioner, the mixed form with a point and with the element-block
    preconditioner) gives the same bits as the blocking solve, result record
    included, also when it stops at max_iter or has a zero right-hand side;
  * captured inside a caller's CUDA graph, replays give the same bits;
  * simp.run(engine="graph") (every OC iteration one graph, the PCG loop on
    the device) is bit-identical to the direct run, FP64 and mixed, with
    either filter.
"""

import copy

import numpy as np
import pytest

from conftest import REPO

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from toptimization_b200.fem.solver import PCGSolver  # noqa: E402
from toptimization_b200.material import compute_Ke_2d, regularized_inverse  # noqa: E402
from toptimization_b200.mesh import fixed_node_mask, force_vector  # noqa: E402
from toptimization_b200.optimizer.simp import RunHistory, run  # noqa: E402
from toptimization_b200.problem import load_problem  # noqa: E402
from toptimization_b200 import _lib  # noqa: E402

FORMS = [("jacobi", "fp64", "auto"), ("nodal_block_jacobi", "fp64", "standard"),
         ("block_jacobi", "fp64", "auto"), ("nodal_block_jacobi", "mixed", "auto"),
         ("jacobi", "mixed", "auto"), ("block_jacobi", "mixed", "auto"),
         ("none", "fp64", "auto")]


def _setup(max_iter=3000):
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    Ke = compute_Ke_2d(pr.E, pr.nu)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    dev = torch.device("cuda", 0)
    f_np = force_vector(pr)
    gen = torch.Generator(device=dev).manual_seed(7)
    rho = 0.05 + 0.95 * torch.rand(pr.n_elem, generator=gen, device=dev, dtype=torch.float64)
    return pr, dev, f_np, torch.from_numpy(f_np).to(dev), \
        torch.from_numpy(fixed_node_mask(pr)).to(dev), rho


def _solver(pr, f_np, pre, prec, rec, dev, max_iter=3000):
    return PCGSolver(pr.nelx, pr.nely, pr.E_min, pr.penalty, float(f_np @ f_np),
                     preconditioner=pre, precision=prec, recurrence=rec, max_iter=max_iter,
                     tol=1e-8, inner_tol=1e-3, device=dev)


def _same(a, b):
    return (a.status, a.iters, a.outer_iters, a.updates, a.rr) == \
        (b.status, b.iters, b.outer_iters, b.updates, b.rr)


@pytest.mark.parametrize("pre,prec,rec", FORMS)
@pytest.mark.parametrize("max_iter", [3000, 7])
def test_async_equals_blocking(tpo_built, pre, prec, rec, max_iter):
    pr, dev, f_np, f, fixed, rho = _setup()
    s1 = _solver(pr, f_np, pre, prec, rec, dev, max_iter)
    s2 = _solver(pr, f_np, pre, prec, rec, dev, max_iter)
    u1 = torch.zeros(pr.n_dofs, dtype=torch.float64, device=dev)
    u2 = torch.zeros_like(u1)
    info1 = s1.solve(rho, f, fixed, u1, warm_start=False)
    res = s2.result_buffer()
    s2.solve_async(rho, f, fixed, u2, res, warm_start=False)
    torch.cuda.synchronize()
    info2 = PCGSolver.decode(res)
    print(pre, prec, rec, max_iter, info1, info2)
    assert _same(info1, info2)
    assert torch.equal(u1, u2)
    if max_iter == 7:
        assert info2.status == "max_iter"
    elif pre != "block_jacobi" and pre != "none":
        assert info2.status == "converged"
    # a warm-started second solve on the same state
    info1 = s1.solve(rho * 0.9, f, fixed, u1, warm_start=True)
    s2.solve_async(rho * 0.9, f, fixed, u2, res, warm_start=True)
    torch.cuda.synchronize()
    assert _same(info1, PCGSolver.decode(res)) and torch.equal(u1, u2)


def test_async_zero_rhs(tpo_built):
    pr, dev, f_np, f, fixed, rho = _setup()
    s = _solver(pr, np.zeros_like(f_np), "jacobi", "fp64", "auto", dev)
    u = torch.ones(pr.n_dofs, dtype=torch.float64, device=dev)
    res = s.result_buffer()
    s.solve_async(rho, torch.zeros_like(f), fixed, u, res, warm_start=True)
    torch.cuda.synchronize()
    assert PCGSolver.decode(res).status == "zero_rhs"
    assert torch.count_nonzero(u) == 0


@pytest.mark.parametrize("pre,prec", [("jacobi", "fp64"), ("nodal_block_jacobi", "mixed"),
                                      ("block_jacobi", "fp64")])
def test_async_inside_a_callers_graph(tpo_built, pre, prec):
    pr, dev, f_np, f, fixed, rho = _setup()
    ref_s = _solver(pr, f_np, pre, prec, "auto", dev)
    u_ref = torch.zeros(pr.n_dofs, dtype=torch.float64, device=dev)
    info_ref = ref_s.solve(rho, f, fixed, u_ref, warm_start=False)
    s = _solver(pr, f_np, pre, prec, "auto", dev)
    u = torch.zeros_like(u_ref)
    res = s.result_buffer()
    s.solve_async(rho, f, fixed, u, res, warm_start=False)  # first call outside capture
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side, capture_error_mode="thread_local"):
        s.solve_async(rho, f, fixed, u, res, warm_start=False)
    for _ in range(2):
        u.fill_(0.25)
        res.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert _same(info_ref, PCGSolver.decode(res))
        assert torch.equal(u, u_ref)


@pytest.mark.parametrize("pre,prec,filt,iters", [
    ("jacobi", "fp64", "density", 100), ("nodal_block_jacobi", "mixed", "density", 40),
    ("block_jacobi", "fp64", "density", 15), ("jacobi", "fp64", "sensitivity", 30)])
def test_graph_engine_bit_identical_to_direct(tpo_built, pre, prec, filt, iters):
    pr = load_problem(REPO / "examples" / "mbb_60x20.yaml")
    pr.preconditioner, pr.filter_type, pr.max_iter = pre, filt, iters
    hd, hg = RunHistory(), RunHistory()
    rd = run(copy.deepcopy(pr), verbose=False, save=False, history=hd, precision=prec)
    rg = run(copy.deepcopy(pr), verbose=False, save=False, history=hg, precision=prec,
             engine="graph")
    assert np.array_equal(rd, rg)
    for k in ("compliance", "volume", "change", "cg_iters", "solve_status", "outer_iters"):
        assert getattr(hd, k) == getattr(hg, k), k
