"""Serving design requests with continuous batching on one GPU.

Requests (mesh size, boundary conditions, load, volfrac, rmin, OC iteration
count) arrive over time. The server admits a request as soon as it has
arrived and its HBM footprint (density, displacement, PCG vectors, filter
buffers: its design workspace) fits the memory budget and a slot is free;
its state then stays resident on the device until its last OC iteration.
Every round advances all resident designs together (`Batch.round`), each at
its own OC iteration, warm-starting every PCG from the design's previous
displacement. Requests that arrive while others are on the GPU join at the
next round.

Size-aware steps (size_steps=True; off by default, since they trade
throughput for the small designs' latency): a design of E elements takes
every p-th PCG step of a
round, p the largest power of two <= E / E_ref (at most the round's steps),
E_ref the larger of size_step_elems and the smallest resident design. Each
resident design then costs about the same GPU time per step, so small
designs are not paced by the largest ones; when the small ones have left,
the large ones return to every step. A design's iterates, and so its
result, do not depend on p. No reference counterpart: the reference solves one problem per
process (`src/toptimization/cli.py:22-144`).

The one-at-a-time baseline serves the same stream with plain FP64 solves
through the single-design API, one request after another.
"""

from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np
import torch

from .batch import Batch, footprint_bytes, random_designs
from .problem import Problem


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the stream starts
    problem: Problem


@dataclass
class Completion:
    rid: int
    arrival: float
    admitted: float
    done: float
    oc_iters: int
    compliance: float
    density: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeReport:
    completions: list[Completion]
    rounds: int = 0
    peak_resident: int = 0
    peak_bytes: int = 0
    wall: float = 0.0
    extra: dict = field(default_factory=dict)

    def summary(self) -> dict:
        lat = np.array([c.latency for c in self.completions])
        first = min(c.arrival for c in self.completions)
        last = max(c.done for c in self.completions)
        out = {"requests": len(self.completions),
               "designs_per_s": round(len(self.completions) / (last - first), 4),
               "p50_s": round(float(np.percentile(lat, 50)), 4),
               "p95_s": round(float(np.percentile(lat, 95)), 4),
               "p99_s": round(float(np.percentile(lat, 99)), 4),
               "mean_s": round(float(lat.mean()), 4),
               "makespan_s": round(last - first, 3)}
        if self.rounds:
            out.update(rounds=self.rounds, peak_resident=self.peak_resident,
                       peak_gb=round(self.peak_bytes / 1e9, 3))
        out.update(self.extra)
        return out


def poisson_stream(n: int, rate: float, seed: int = 0, nelx_range=(64, 1024),
                   max_iter: int = 50) -> list[Request]:
    """`n` requests with exponential inter-arrival gaps of mean 1/rate
    (numpy.random.default_rng(seed)); designs drawn by `random_designs`
    (seed + 1) with nelx in `nelx_range`, mixed precision."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    ps = random_designs(n, seed=seed + 1, nelx_range=nelx_range, max_iter=max_iter)
    return [Request(i, float(t[i]), ps[i]) for i in range(n)]


def step_period(n_elem: int, round_steps: int, elems: int) -> int:
    """Largest power of two p <= n_elem / elems, 1 <= p <= round_steps."""
    p = 1
    while 2 * p <= round_steps and 2 * p * elems <= n_elem:
        p *= 2
    return p


class Server:
    """Continuous-batching server over one `Batch`."""

    def __init__(self, hbm_budget: float = 150e9, max_slots: int = 256, *,
                 preconditioner: str = "nodal_block_jacobi", use_graph: bool = True,
                 tiles: tuple[int, int] | None = None, round_steps: int = 32,
                 rounds_per_check: int = 4, keep_density: bool = False,
                 size_steps: bool = False, size_step_elems: int = 65536, device=None):
        self.budget = float(hbm_budget)
        self.round_steps = int(round_steps)
        self.size_steps = bool(size_steps)
        self.size_step_elems = int(size_step_elems)
        self.batch = Batch(max_slots, preconditioner=preconditioner, use_graph=use_graph,
                           tiles=tiles, round_steps=round_steps, device=device)
        self.rounds_per_check = int(rounds_per_check)
        self.max_slots = max_slots
        self.keep_density = keep_density

    def serve(self, requests: list[Request]) -> ServeReport:
        b = self.batch
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        resident: dict[int, tuple[Request, float, int]] = {}
        periods: dict[int, int] = {}
        used = 0
        rep = ServeReport([])
        t0 = time.perf_counter()
        while pending or resident:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                fp = footprint_bytes(pending[0].problem)
                if len(resident) >= self.max_slots or used + fp > self.budget:
                    break
                req = pending.popleft()
                slot = b.add(req.problem)
                resident[slot] = (req, time.perf_counter() - t0, fp)
                used += fp
            if not resident:
                time.sleep(max(0.0, pending[0].arrival - now))
                continue
            if self.size_steps:
                self._set_periods(resident, periods)
            rep.peak_resident = max(rep.peak_resident, len(resident))
            rep.peak_bytes = max(rep.peak_bytes, used)
            # admission and completions are checked between groups of rounds;
            # a request that arrives meanwhile waits at most one group
            b.round(self.rounds_per_check)
            rep.rounds += self.rounds_per_check
            it, act = b.states()
            t = time.perf_counter() - t0
            for slot in [s for s in resident if not act[s]]:
                req, adm, fp = resident.pop(slot)
                hist = b.history(slot)
                rho = b.density(slot) if self.keep_density else None
                rep.completions.append(Completion(req.rid, req.arrival, adm, t, int(it[slot]),
                                                  float(hist["compliance"][-1]), rho))
                b.remove(slot)
                periods.pop(slot, None)
                used -= fp
        rep.wall = time.perf_counter() - t0
        rep.completions.sort(key=lambda c: c.rid)
        return rep

    def step_period(self, pr: Problem, ref: int | None = None) -> int:
        return step_period(pr.n_elem, self.round_steps,
                           max(self.size_step_elems, ref or 0))

    def _set_periods(self, resident: dict, periods: dict) -> None:
        """Step periods relative to the smallest resident design."""
        ref = min(req.problem.n_elem for req, _, _ in resident.values())
        for slot, (req, _, _) in resident.items():
            p = self.step_period(req.problem, ref)
            if periods.get(slot, 1) != p:
                self.batch.set_step_period(slot, p)
            periods[slot] = p

    def close(self) -> None:
        self.batch.close()


def serve_one_at_a_time(requests: list[Request], precision: str = "fp64",
                        keep_density: bool = False, device=None) -> ServeReport:
    """The same stream served one request at a time with the single-design
    solver (plain FP64 by default), in arrival order."""
    from .optimizer.simp import SimpDesign
    rep = ServeReport([])
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = time.perf_counter() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        adm = time.perf_counter() - t0
        d = SimpDesign(req.problem, device=device, precision=precision,
                       preconditioner=req.problem.preconditioner)
        c = 0.0
        for _ in range(req.problem.max_iter):
            c = d.step().compliance
        torch.cuda.synchronize()
        rho = d.density().reshape(req.problem.nelx, req.problem.nely) if keep_density else None
        rep.completions.append(Completion(req.rid, req.arrival, adm, time.perf_counter() - t0,
                                          req.problem.max_iter, c, rho))
        del d
    rep.wall = time.perf_counter() - t0
    return rep


__all__ = ["Request", "Completion", "ServeReport", "Server", "poisson_stream",
           "serve_one_at_a_time", "step_period"]
