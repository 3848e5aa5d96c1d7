"""Host logic of the serving loop on CPU: admission by HBM footprint and free
slot, release on completion, latency bookkeeping. The batched engine is
replaced by a fake whose designs finish after a fixed number of rounds."""

import numpy as np
import pytest

from toptimization_b200 import serve
from toptimization_b200.batch import footprint_bytes


class FakeBatch:
    def __init__(self, max_designs, **kw):
        self.max = max_designs
        self.progress = {}
        self.need = {}
        self.closed = False

    def set_step_period(self, slot, period):
        assert slot in self.progress and period >= 1

    def add(self, pr, max_iter=None, tag=None):
        slot = next(i for i in range(self.max) if i not in self.progress)
        self.progress[slot] = 0
        self.need[slot] = 2 + pr.nelx % 3   # rounds until the design is done
        return slot

    def round(self, rounds=1):
        for s in self.progress:
            self.progress[s] += rounds

    def states(self):
        it = np.full(self.max, -1, np.int32)
        act = np.zeros(self.max, np.int32)
        for s, p in self.progress.items():
            it[s] = min(p, self.need[s])
            act[s] = int(p < self.need[s])
        return it, act

    def history(self, slot):
        return {"compliance": np.array([1.0 + slot])}

    def density(self, slot):
        return np.zeros((2, 2))

    def remove(self, slot):
        del self.progress[slot], self.need[slot]

    def close(self):
        self.closed = True


@pytest.fixture
def fake_batch(monkeypatch, tpo_built):
    monkeypatch.setattr(serve, "Batch", FakeBatch)


def test_admission_by_footprint_and_slots(fake_batch):
    reqs = serve.poisson_stream(7, rate=1e6, seed=2, nelx_range=(64, 96), max_iter=2)
    fps = sorted(footprint_bytes(r.problem) for r in reqs)
    srv = serve.Server(hbm_budget=fps[-1] + fps[-2], max_slots=8, rounds_per_check=1)
    rep = srv.serve(reqs)
    srv.close()
    assert [c.rid for c in rep.completions] == list(range(7))
    assert rep.peak_resident <= 2 and rep.peak_bytes <= fps[-1] + fps[-2]
    assert all(c.done >= c.admitted >= 0 and c.latency >= 0 for c in rep.completions)
    s = rep.summary()
    assert s["requests"] == 7 and s["p50_s"] <= s["p95_s"] <= s["p99_s"]


def test_slot_limit_binds_before_memory(fake_batch):
    reqs = serve.poisson_stream(5, rate=1e6, seed=3, nelx_range=(64, 80), max_iter=2)
    srv = serve.Server(hbm_budget=1e12, max_slots=3, rounds_per_check=1)
    rep = srv.serve(reqs)
    assert len(rep.completions) == 5 and rep.peak_resident == 3


def test_summary_percentiles():
    cs = [serve.Completion(i, 0.0, 0.0, float(i + 1), 1, 1.0) for i in range(100)]
    s = serve.ServeReport(cs).summary()
    assert s["designs_per_s"] == pytest.approx(100 / 100.0)
    assert s["p50_s"] == pytest.approx(50.5) and s["p99_s"] == pytest.approx(99.01)


def test_step_period_is_a_power_of_two_bounded_by_the_round():
    from toptimization_b200.serve import step_period
    assert step_period(1000, 32, 65536) == 1
    assert step_period(65536, 32, 65536) == 1
    assert step_period(2 * 65536, 32, 65536) == 2
    assert step_period(3 * 65536, 32, 65536) == 2
    assert step_period(1024 * 1024, 32, 65536) == 16
    assert step_period(1 << 30, 32, 65536) == 32
    assert step_period(1 << 30, 4, 65536) == 4
    for n in (1, 7000, 130000, 500000, 4000000):
        p = step_period(n, 32, 65536)
        assert p & (p - 1) == 0 and 1 <= p <= 32
