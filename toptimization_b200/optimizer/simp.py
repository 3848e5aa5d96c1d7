"""SIMP compliance minimisation: the optimisation loop on the device.

Drop-in for the reference's `src/toptimization/optimizer/simp.py:19-231`
(`run(problem, backend, live_viz, viz_callback) -> ndarray (nelx, nely)`).
Per OC iteration (`simp.py:141-219`):

    density filter rho -> rho_phys          (filter.py:106-124)
    PCG  K(rho_phys) u = f, warm from it>1  (solver.py:27-159)
    sensitivity on rho_phys -> dc, c        (kernels.py:234-272)
    dc projection  H dc / Hs                (filter.py:174-180)
    OC bisection on the design rho          (oc.py:52-93)
    volume = mean(rho)                      (kernels.py:330-336)
    stop when it > 5 and change < tol       (simp.py:217-219)

(or, with filter_type "sensitivity", the solve on rho and Sigmund's filter,
simp.py:174-189). Every field lives in one `SimpDesign` as CUDA tensors; the
host reads five scalars per iteration.

3D problems (dim 3, H8 elements) run the same loop through the tpo3_* entry
points: FP64 PCG with "jacobi", "block_jacobi" or "none", the 3D filter box,
and the result shaped (nelx, nely, nelz) (`simp.py:309-312`).

Not reproduced: Taichi backend selection (CUDA only), matplotlib live
windows and PNG output (headless; `density_final.npy` and the histories are
written as in `simp.py:294-306`).
"""

from __future__ import annotations

import json
import math
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Callable

import numpy as np
import torch

from .. import _lib
from ..fem import kernels as K
from ..fem.solver import PCGSolver, SolveInfo
from ..material import compute_Ke_2d, compute_Ke_3d, regularized_inverse
from ..mesh import fixed_node_mask, force_vector
from . import filter as filt
from . import oc as oc_mod


@dataclass
class IterationRecord:
    it: int
    compliance: float
    volume: float
    change: float
    cg_iters: int
    solve: SolveInfo
    seconds: float
    launches: int = 0  # this library's kernels the OC iteration ran (CapturedDesign)


@dataclass
class RunHistory:
    compliance: list = field(default_factory=list)
    volume: list = field(default_factory=list)
    change: list = field(default_factory=list)
    cg_iters: list = field(default_factory=list)
    solve_status: list = field(default_factory=list)
    outer_iters: list = field(default_factory=list)
    seconds: list = field(default_factory=list)

    def append(self, r: IterationRecord) -> None:
        self.compliance.append(r.compliance)
        self.volume.append(r.volume)
        self.change.append(r.change)
        self.cg_iters.append(r.cg_iters)
        self.solve_status.append(r.solve.status)
        self.outer_iters.append(r.solve.outer_iters)
        self.seconds.append(r.seconds)


class SimpDesign:
    """Device-resident state of one design and one OC iteration at a time."""

    def __init__(self, problem, device=None, precision: str | None = None,
                 preconditioner: str | None = None, poll_every: int = 0):
        self.problem = pr = problem
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise ValueError("SimpDesign needs a CUDA device")
        self.precision = precision or getattr(pr, "precision", "fp64")
        self.preconditioner = preconditioner or pr.preconditioner
        nelz = pr.nelz if pr.dim == 3 else 0
        if nelz and self.precision != "fp64":
            raise ValueError("3D designs run the FP64 solve")
        with torch.cuda.device(self.device):
            if nelz:
                Ke = compute_Ke_3d(pr.E, pr.nu)
                Ke_inv, alpha = regularized_inverse(Ke)
                _lib.ensure_stiffness3(Ke, Ke_inv, alpha)
            else:
                Ke = compute_Ke_2d(pr.E, pr.nu)
                Ke_inv, alpha = regularized_inverse(Ke)
                _lib.ensure_stiffness(Ke, Ke_inv, alpha)
        self.grid = (_lib.grid3(pr.nelx, pr.nely, nelz, pr.E_min, pr.penalty) if nelz
                     else _lib.grid(pr.nelx, pr.nely, pr.E_min, pr.penalty))
        dev = self.device
        f_np = force_vector(pr)
        self.f_norm_sq = float(np.dot(f_np, f_np))
        self.fixed = torch.from_numpy(fixed_node_mask(pr)).to(dev)
        self.f = torch.from_numpy(f_np).to(dev)
        E, N = pr.n_elem, pr.n_dofs
        self.rho = torch.full((E,), float(pr.volfrac), dtype=torch.float64, device=dev)
        self.rho_phys = torch.empty(E, dtype=torch.float64, device=dev)
        self.dc = torch.empty(E, dtype=torch.float64, device=dev)
        self.dc_filt = torch.empty(E, dtype=torch.float64, device=dev)
        self.u = torch.zeros(N, dtype=torch.float64, device=dev)
        # [compliance, change, volume, lambda, bisection steps]
        self.scalars = torch.zeros(5, dtype=torch.float64, device=dev)
        self.solver = PCGSolver(pr.nelx, pr.nely, pr.E_min, pr.penalty, self.f_norm_sq,
                                preconditioner=self.preconditioner, precision=self.precision,
                                max_iter=pr.max_cg_iter, tol=pr.cg_tol,
                                inner_tol=getattr(pr, "inner_tol", 1e-3),
                                max_outer=getattr(pr, "max_outer_iter", 50),
                                recurrence=getattr(pr, "recurrence", "auto"),
                                poll_every=poll_every, device=dev, nelz=nelz)
        self.sens_ws = K.sensitivity_workspace(self.grid, dev)
        self.oc_ws = oc_mod.oc_workspace(self.grid, dev)
        self.it = 0

    def step(self) -> IterationRecord:
        """One OC iteration; returns its record (reads 5 scalars)."""
        pr = self.problem
        t0 = time.perf_counter()
        self.it += 1
        warm = self.it > 1
        with torch.cuda.device(self.device):
            if pr.filter_type == "density":
                filt.density_filter(self.grid, pr.rmin, self.rho, self.rho_phys)
                info = self.solver.solve(self.rho_phys, self.f, self.fixed, self.u, warm)
                K.sensitivity(self.grid, self.rho_phys, self.u, self.dc, self.scalars[0:1],
                              self.sens_ws)
                filt.density_filter(self.grid, pr.rmin, self.dc, self.dc_filt)
            else:
                info = self.solver.solve(self.rho, self.f, self.fixed, self.u, warm)
                K.sensitivity(self.grid, self.rho, self.u, self.dc, self.scalars[0:1],
                              self.sens_ws)
                filt.sensitivity_filter(self.grid, pr.rmin, self.rho, self.dc, self.dc_filt)
            oc_mod.oc_update(self.grid, pr.volfrac, pr.move_limit, self.rho, self.dc_filt,
                             self.rho, self.scalars[1:5], self.oc_ws)
            c, change, vol, _lam, _steps = self.scalars.cpu().tolist()
        return IterationRecord(self.it, c, vol, change, info.iters, info,
                               time.perf_counter() - t0)

    def density(self) -> np.ndarray:
        return self.rho.cpu().numpy()


class CapturedDesign(SimpDesign):
    """A SimpDesign whose OC iteration is one CUDA graph: the filters, the
    asynchronous PCG solve (its loop a device-side while node,
    `PCGSolver.solve_async`), the sensitivity and the OC update are captured
    once and replayed every iteration; the host reads the five scalars and the
    solve result after each replay. The same kernels in the same order as
    `SimpDesign.step`, so the same results, for every 2D form (FP64 and mixed,
    every preconditioner, both filter types). The first OC iteration (the cold
    start) runs uncaptured; it also sets up the launch plans."""

    def __init__(self, problem, device=None, precision: str | None = None,
                 preconditioner: str | None = None):
        if problem.dim != 2:
            raise ValueError("engine='graph' runs 2D designs")
        super().__init__(problem, device=device, precision=precision,
                         preconditioner=preconditioner)
        self.result = self.solver.result_buffer()
        self.graph = None

    def _enqueue(self, warm: bool) -> None:
        pr = self.problem
        c0 = _lib.launch_count()
        if pr.filter_type == "density":
            filt.density_filter(self.grid, pr.rmin, self.rho, self.rho_phys)
            c1 = _lib.launch_count()
            self.solver.solve_async(self.rho_phys, self.f, self.fixed, self.u, self.result, warm)
            c2 = _lib.launch_count()
            K.sensitivity(self.grid, self.rho_phys, self.u, self.dc, self.scalars[0:1],
                          self.sens_ws)
            filt.density_filter(self.grid, pr.rmin, self.dc, self.dc_filt)
        else:
            c1 = _lib.launch_count()
            self.solver.solve_async(self.rho, self.f, self.fixed, self.u, self.result, warm)
            c2 = _lib.launch_count()
            K.sensitivity(self.grid, self.rho, self.u, self.dc, self.scalars[0:1], self.sens_ws)
            filt.sensitivity_filter(self.grid, pr.rmin, self.rho, self.dc, self.dc_filt)
        oc_mod.oc_update(self.grid, pr.volfrac, pr.move_limit, self.rho, self.dc_filt,
                         self.rho, self.scalars[1:5], self.oc_ws)
        # kernels of the iteration outside the solve (the solve reports its own)
        self.outside_launches = (c1 - c0) + (_lib.launch_count() - c2)

    def step(self) -> IterationRecord:
        t0 = time.perf_counter()
        self.it += 1
        with torch.cuda.device(self.device):
            if self.it == 1:
                self._enqueue(False)
            else:
                if self.graph is None:
                    side = torch.cuda.Stream(self.device)
                    side.wait_stream(torch.cuda.current_stream(self.device))
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=side, capture_error_mode="thread_local"):
                        self._enqueue(True)
                    self.graph = g
                self.graph.replay()
            c, change, vol, _lam, _steps = self.scalars.cpu().tolist()
            info = PCGSolver.decode(self.result)
        return IterationRecord(self.it, c, vol, change, info.iters, info,
                               time.perf_counter() - t0, self.outside_launches + info.launches)


class GraphDesign:
    """One design run through the batched engine (`toptimization_b200.batch`)
    as a batch of one: each OC iteration is a single CUDA graph launch in which
    a conditional while node runs the PCG loop on the device (no host round
    trip inside the iteration). Mixed precision, density filter and a point
    preconditioner only. Same `step()` / `density()` interface as
    `SimpDesign`."""

    def __init__(self, problem, device=None, preconditioner: str | None = None):
        from ..batch import Batch
        pr = problem
        pre = preconditioner or pr.preconditioner
        if pr.filter_type != "density":
            raise ValueError("engine='graph' runs the density filter only")
        if pre not in ("jacobi", "nodal_block_jacobi", "none"):
            raise ValueError("engine='graph' takes a point preconditioner")
        self.problem = pr
        self.precision = "mixed"
        self.preconditioner = pre
        self.batch = Batch(1, preconditioner=pre, use_graph=True, device=device)
        self.slot = self.batch.add(pr)
        self.it = 0

    def step(self) -> IterationRecord:
        t0 = time.perf_counter()
        self.batch.step()
        h = self.batch.history(self.slot)
        self.it = len(h["compliance"])
        i = self.it - 1
        status = _lib.SOLVE_STATUS.get(int(h["pcg_status"][i]), str(int(h["pcg_status"][i])))
        info = SolveInfo(status, int(h["cg_iters"][i]), int(h["outer_iters"][i]),
                         int(h["cg_iters"][i]), float("nan"))
        return IterationRecord(self.it, float(h["compliance"][i]), float(h["volume"][i]),
                               float(h["change"][i]), int(h["cg_iters"][i]), info,
                               time.perf_counter() - t0)

    def density(self) -> np.ndarray:
        return self.batch.density(self.slot).reshape(-1)


def _check_backend(backend: str) -> None:
    if backend not in ("auto", "cuda"):
        raise ValueError(f"Unknown backend '{backend}': toptimization_b200 runs on CUDA only")
    if not torch.cuda.is_available():
        raise RuntimeError("no CUDA device available (toptimization_b200 has no CPU path)")


def run(problem, backend: str = "auto", live_viz: bool = True,
        viz_callback: Callable | None = None, *, precision: str | None = None,
        preconditioner: str | None = None, device=None, verbose: bool = True,
        save: bool = True, history: RunHistory | None = None,
        engine: str = "direct") -> np.ndarray:
    """Run SIMP topology optimisation; returns the final design density as an
    array of shape (nelx, nely) -- (nelx, nely, nelz) in 3D -- FP64 (reference
    simp.py:19-41,309-312).

    `viz_callback(rho_np, it, compliance, volume)` is called every iteration
    (simp.py:213-214). `live_viz` is accepted for compatibility; there is no
    window (headless). `precision` overrides `problem.precision`
    ("fp64" | "mixed"); `history` (optional) receives every per-iteration record.
    `engine="graph"` runs each OC iteration as one CUDA graph with the PCG
    loop on the device, any 2D form (`CapturedDesign`); `engine="batch"` runs
    the design through the batched engine as a batch of one (mixed precision,
    density filter, point preconditioner; `GraphDesign`).
    """
    _check_backend(backend)
    pr = problem
    if engine == "graph":
        if pr.dim != 2:
            raise ValueError("engine='graph' runs 2D designs")
        design = CapturedDesign(pr, device=device, precision=precision,
                                preconditioner=preconditioner)
    elif engine == "batch":
        if pr.dim != 2:
            raise ValueError("engine='batch' runs 2D designs")
        if (precision or pr.precision) != "mixed":
            raise ValueError("engine='batch' runs the mixed-precision form")
        design = GraphDesign(pr, device=device, preconditioner=preconditioner)
    elif engine == "direct":
        design = SimpDesign(pr, device=device, precision=precision,
                            preconditioner=preconditioner)
    else:
        raise ValueError(f"unknown engine {engine!r}")
    hist = history if history is not None else RunHistory()
    if verbose:
        size = f"{pr.nelx}x{pr.nely}" + (f"x{pr.nelz}" if pr.dim == 3 else "")
        print(f"[toptimization_b200] {pr.name}: {size}, n_dofs={pr.n_dofs:,}, "
              f"precision={design.precision}, preconditioner={design.preconditioner}")
        print(f"{'Iter':>5} {'Compliance':>14} {'Volume':>8} {'Change':>9} {'CG':>6} {'s/iter':>7}")
        print("-" * 55)
    for _ in range(pr.max_iter):
        rec = design.step()
        hist.append(rec)
        if verbose:
            print(f"{rec.it:>5d} {rec.compliance:>14.6f} {rec.volume:>8.4f} {rec.change:>9.4f} "
                  f"{rec.cg_iters:>6d} {rec.seconds:>7.2f}")
        if viz_callback is not None:
            viz_callback(design.density(), rec.it, rec.compliance, rec.volume)
        if rec.it > 5 and rec.change < pr.tol:
            if verbose:
                print(f"\n[toptimization_b200] Converged at iter {rec.it} (change={rec.change:.6f})")
            break
    rho = design.density()
    if save:
        _save_final(pr, rho, hist)
    if pr.dim == 3:
        return rho.reshape(pr.nelx, pr.nely, pr.nelz)
    return rho.reshape(pr.nelx, pr.nely)


def _save_final(pr, rho: np.ndarray, hist: RunHistory) -> None:
    out = Path(pr.output_dir)
    out.mkdir(parents=True, exist_ok=True)
    np.save(out / "density_final.npy", rho)
    with open(out / "history.json", "w") as fh:
        json.dump({"compliance": hist.compliance, "volume": hist.volume,
                   "change": hist.change, "cg_iters": hist.cg_iters,
                   "solve_status": hist.solve_status}, fh)
