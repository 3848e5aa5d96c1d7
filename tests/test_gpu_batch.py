"""Batched designs on the GPU (tpo_batch_* through the C ABI).

  * a design's results are bit-identical alone and inside a mix of uneven
    designs (its launch geometry and reduction order do not depend on the
    other designs), in a different slot;
  * the CUDA-graph OC iteration gives the same bits as the host-polled one;
  * against the single-design mixed solver: the first OC iteration (same
    input density) agrees to the PCG tolerance, the 8-iteration history to
    the OC-bisection scale;
  * slots are released and reused; the stop rule ends designs.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from toptimization_b200.batch import Batch, autotune, random_designs  # noqa: E402
from toptimization_b200.optimizer.simp import SimpDesign  # noqa: E402


def _designs(n, seed, lo=64, hi=160, iters=6):
    return random_designs(n, seed=seed, nelx_range=(lo, hi), max_iter=iters)


def _run(problems, use_graph=True, order=None, tiles=None):
    b = Batch(len(problems) + 2, use_graph=use_graph, tiles=tiles)
    idx = order if order is not None else range(len(problems))
    slots = {i: b.add(problems[i]) for i in idx}
    b.run()
    out = {i: b.result(s) for i, s in slots.items()}
    b.close()
    return out


def test_alone_and_in_the_mix_are_identical(tpo_built):
    ps = _designs(5, seed=21)
    alone = _run([ps[2]])[0]
    mix = _run(ps, order=[4, 0, 3, 2, 1])[2]
    assert np.array_equal(alone[0], mix[0])
    for k in ("compliance", "volume", "change", "cg_iters"):
        assert np.array_equal(alone[1][k], mix[1][k]), k
    assert len(alone[1]["compliance"]) == 6


def test_graph_and_host_loop_agree(tpo_built):
    ps = _designs(3, seed=5)
    g = _run(ps, use_graph=True)
    h = _run(ps, use_graph=False)
    for i in range(3):
        assert np.array_equal(g[i][0], h[i][0])
        assert np.array_equal(g[i][1]["compliance"], h[i][1]["compliance"])


def test_batch_matches_single_design_solver(tpo_built):
    ps = _designs(3, seed=9, lo=80, hi=140, iters=8)
    res = _run(ps)
    for i, pr in enumerate(ps):
        d = SimpDesign(pr, precision="mixed", preconditioner=pr.preconditioner)
        comp = np.array([d.step().compliance for _ in range(pr.max_iter)])
        cb = res[i][1]["compliance"]
        assert len(cb) == pr.max_iter
        assert abs(cb[0] - comp[0]) / comp[0] < 1e-7
        assert np.max(np.abs(cb - comp) / comp) < 1e-4
        assert np.all(res[i][1]["pcg_status"] == 1)  # every solve converged
        rho = res[i][0]
        assert abs(rho.mean() - pr.volfrac) < 1e-3


def test_batch_matches_oracle(tpo_built):
    """Batched (mixed-form) designs against the FP64 oracle's own run of the
    same problems (oracle/simp64.py, the reference's loop
    src/toptimization/optimizer/simp.py:141-219): the first OC iteration
    (same input density) to the PCG tolerance, the 5-iteration compliance and
    volume histories and the final density to the OC-bisection scale (its
    multiplier is a discrete function of dc)."""
    from oracle import simp64 as O
    ps = _designs(3, seed=17, lo=64, hi=110, iters=5)
    res = _run(ps)
    for i, pr in enumerate(ps):
        ref = O.run(pr)
        rho, h = res[i]
        cb = np.asarray(h["compliance"])
        assert len(cb) == len(ref.compliance) == pr.max_iter
        e_first = abs(cb[0] - ref.compliance[0]) / ref.compliance[0]
        e_all = float(np.max(np.abs(cb - ref.compliance) / ref.compliance))
        e_rho = float(np.abs(np.asarray(rho).reshape(-1) - ref.rho).max())
        e_vol = float(np.abs(np.asarray(h["volume"]) - ref.volume).max())
        print(f"design {i} ({pr.nelx}x{pr.nely}): compliance first {e_first:.2e}, "
              f"worst {e_all:.2e}; density max-abs {e_rho:.2e}; volume {e_vol:.2e}")
        assert e_first < 1e-7
        assert e_all < 1e-4
        assert e_vol < 1e-4
        assert e_rho < 1e-2


def test_slots_release_and_stop_rule(tpo_built):
    ps = _designs(3, seed=13, iters=4)
    b = Batch(2)
    s0 = b.add(ps[0], max_iter=2)
    s1 = b.add(ps[1], max_iter=4)
    assert b.step()
    it, act = b.states()
    assert it[s0] == 1 and it[s1] == 1
    assert b.step()
    it, act = b.states()
    assert act[s0] == 0 and act[s1] == 1 and it[s0] == 2
    b.remove(s0)
    s2 = b.add(ps[2], max_iter=1)
    assert s2 == s0
    b.run()
    it, act = b.states()
    assert it[s1] == 4 and it[s2] == 1 and not act.any()
    b.close()


def test_autotune_reports_every_candidate(tpo_built):
    ps = _designs(4, seed=2)
    res = autotune(ps, candidates=[(8, 4), (16, 8), (32, 16)], steps=16)
    assert set(res["ms"]) == {(8, 4), (16, 8), (32, 16)}
    assert res["best"] in res["ms"] and all(v > 0 for v in res["ms"].values())
    # other tiles change the rounding order of the FP32 Krylov vectors, so the
    # two solves take different paths; both meet the FP64 stop rule
    # ||f - K u|| < 1e-8 ||f||, which bounds the compliance gap by about
    # ||r|| ||K^-1 f|| / c, a few 1e-7 on these designs
    a = _run(ps[:2], tiles=(8, 4))
    c = _run(ps[:2], tiles=(32, 16))
    for i in range(2):
        ca, cc = a[i][1]["compliance"], c[i][1]["compliance"]
        assert abs(ca[0] - cc[0]) / ca[0] < 1e-6


def test_rounds_and_oc_iterations_agree(tpo_built):
    """Continuous-batching rounds (each design at its own pace) give the same
    bits as OC iterations in lock step."""
    ps = _designs(4, seed=31)
    a = Batch(4)
    sa = [a.add(p) for p in ps]
    a.run(rounds=False)
    b = Batch(4)
    sb = [b.add(p) for p in ps]
    b.run(rounds=True)
    for i in range(4):
        assert np.array_equal(a.density(sa[i]), b.density(sb[i]))
        assert np.array_equal(a.history(sa[i])["compliance"], b.history(sb[i])["compliance"])
    a.close()
    b.close()


@pytest.mark.parametrize("step_elems", [65536, 1500])
def test_served_results_equal_alone(tpo_built, step_elems):
    """Each request's result in the served stream (others arriving and
    leaving around it) is bit-identical to the same request run alone, with
    every step (alone) and, for step_elems 1500, served with step periods of
    2 to 16 (size-aware steps)."""
    from toptimization_b200.serve import Server, poisson_stream
    reqs = poisson_stream(6, rate=200.0, seed=3, nelx_range=(64, 160), max_iter=4)
    srv = Server(max_slots=8, keep_density=True, size_steps=True, size_step_elems=step_elems)
    periods = [srv.step_period(r.problem) for r in reqs]
    rep = srv.serve(reqs)
    srv.close()
    assert len(rep.completions) == 6 and rep.peak_resident >= 2
    if step_elems < 65536:
        assert max(periods) >= 4
    for c in rep.completions:
        alone = Batch(1)
        s = alone.add(reqs[c.rid].problem)
        alone.run(rounds=True)
        assert np.array_equal(alone.density(s), c.density)
        assert alone.history(s)["compliance"][-1] == c.compliance
        alone.close()
    summ = rep.summary()
    assert summ["p50_s"] <= summ["p95_s"] <= summ["p99_s"]


def test_admission_respects_the_memory_budget(tpo_built):
    from toptimization_b200.batch import footprint_bytes
    from toptimization_b200.serve import Server, poisson_stream
    reqs = poisson_stream(5, rate=1000.0, seed=4, nelx_range=(64, 96), max_iter=2)
    fps = sorted(footprint_bytes(r.problem) for r in reqs)
    budget = fps[-1] + fps[-2]  # any two fit, never three
    srv = Server(hbm_budget=budget, max_slots=8)
    rep = srv.serve(reqs)
    srv.close()
    assert len(rep.completions) == 5
    assert rep.peak_resident <= 2 and rep.peak_bytes <= budget


def test_batch_engine_run_matches_direct(tpo_built):
    """simp.run(engine="batch"): the design through the batched engine, each
    OC iteration one CUDA graph launch, same OC rules; first-iteration
    compliance equal to the direct mixed run to the PCG tolerance, the history
    to the bisection scale."""
    from toptimization_b200.optimizer.simp import RunHistory, run
    pr = _designs(1, seed=17, lo=80, hi=120, iters=6)[0]
    hg, hd = RunHistory(), RunHistory()
    rg = run(pr, verbose=False, save=False, history=hg, engine="batch")
    rd = run(pr, verbose=False, save=False, history=hd, precision="mixed")
    assert rg.shape == rd.shape == (pr.nelx, pr.nely)
    cg, cd = np.array(hg.compliance), np.array(hd.compliance)
    assert len(cg) == len(cd) == pr.max_iter
    assert abs(cg[0] - cd[0]) / cd[0] < 1e-6
    assert np.max(np.abs(cg - cd) / cd) < 1e-4
    assert all(s == "converged" for s in hg.solve_status)
