"""Batched designs: many independent SIMP problems of uneven size advance
together, one kernel launch per step for the whole batch (`tpo_batch_*`).

The reference runs one problem per process with module-global fields
(`src/toptimization/optimizer/simp.py:19-312`, `fem/fields.py:53-63`); this
module has no reference counterpart. Each design runs the reference's OC
iteration (density filter, PCG solve warm-started from its previous
displacement, sensitivity, dc filter, OC bisection; `simp.py:141-219`) with
the mixed-precision PCG. A design's results do not depend on which other
designs share the batch: its launch geometry depends only on its own size and
the batch's strip lengths.

    batch = Batch(max_designs=64)
    slots = [batch.add(problem) for problem in problems]
    while batch.step():          # one OC iteration of every active design
        pass
    rho, hist = batch.result(slots[0])

`random_designs` draws the uneven-size workload (MBB, cantilever and bridge
families with a point load in the middle 80 % of the loaded edge);
`autotune` picks the strip lengths (columns per CTA) of the batched PCG
kernels by timing them on a scratch copy of the batch.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .material import compute_Ke_2d, regularized_inverse
from .mesh import fixed_node_mask, force_vector
from .problem import Problem, problem_from_dict

HIST_FIELDS = ("compliance", "volume", "change", "cg_iters", "outer_iters", "pcg_status")
DEFAULT_TILES = (16, 8)  # (stencil columns per CTA, update columns per CTA)


def design_struct(pr: Problem, max_iter: int | None = None) -> _lib.TpoBatchDesign:
    f = force_vector(pr)
    return _lib.TpoBatchDesign(
        nelx=pr.nelx, nely=pr.nely, e_min=pr.E_min, penalty=pr.penalty, volfrac=pr.volfrac,
        move=pr.move_limit, rmin=pr.rmin, tol=pr.tol, cg_tol=pr.cg_tol,
        inner_tol=pr.inner_tol, f_norm_sq=float(f @ f), rho0=pr.volfrac,
        max_oc_iter=int(max_iter if max_iter is not None else pr.max_iter),
        max_cg_iter=pr.max_cg_iter, max_outer=pr.max_outer_iter, pad=0)


def footprint_bytes(pr: Problem, max_iter: int | None = None) -> int:
    """Device bytes one design holds while it is resident (its workspace)."""
    layout = _lib.TpoBatchLayout()
    n = _lib.load().tpo_batch_design_workspace_bytes(design_struct(pr, max_iter), layout)
    if n == 0:
        raise ValueError(_lib.load().tpo_last_error_string().decode())
    return int(n)


@dataclass
class _Slot:
    problem: Problem
    ws: torch.Tensor
    layout: _lib.TpoBatchLayout
    max_iter: int
    tag: object = None


class Batch:
    """A set of resident designs advanced together on one GPU."""

    def __init__(self, max_designs: int, *, preconditioner: str = "nodal_block_jacobi",
                 use_graph: bool = True, tiles: tuple[int, int] | None = None,
                 round_steps: int = 32, device=None):
        if preconditioner not in ("jacobi", "nodal_block_jacobi", "none"):
            raise ValueError("batched designs take a point preconditioner")
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.lib = _lib.load()
        with torch.cuda.device(self.device):
            Ke = compute_Ke_2d(1.0, 0.3)
            inv, alpha = regularized_inverse(Ke)
            _lib.ensure_stiffness(Ke, inv, alpha)
            ls, lu = tiles if tiles is not None else DEFAULT_TILES
            self.cfg = _lib.TpoBatchCfg(
                precond=_lib.PRECOND[preconditioner], precision=_lib.PRECISION["mixed"],
                use_graph=1 if use_graph else 0, stencil_cols=int(ls), update_cols=int(lu),
                round_steps=int(round_steps))
            nb = self.lib.tpo_batch_workspace_bytes(int(max_designs))
            self.ws = torch.empty(nb, dtype=torch.uint8, device=self.device)
            h = ctypes.c_void_p()
            _lib.check(self.lib.tpo_batch_create(int(max_designs), self.cfg, _lib.ptr(self.ws),
                                                 nb, ctypes.byref(h)))
        self.handle = h
        self.max_designs = int(max_designs)
        self.preconditioner = preconditioner
        self.slots: dict[int, _Slot] = {}

    # -- membership
    def add(self, pr: Problem, max_iter: int | None = None, tag=None) -> int:
        """Admit a design; returns its slot. Its state stays on the device
        until `remove`."""
        if pr.dim != 2 or pr.filter_type != "density":
            raise ValueError("batched designs are 2D with the density filter")
        d = design_struct(pr, max_iter)
        layout = _lib.TpoBatchLayout()
        nbytes = self.lib.tpo_batch_design_workspace_bytes(d, layout)
        if nbytes == 0:
            raise ValueError(self.lib.tpo_last_error_string().decode())
        with torch.cuda.device(self.device):
            ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            f = torch.from_numpy(force_vector(pr)).to(self.device)
            fixed = torch.from_numpy(fixed_node_mask(pr)).to(self.device)
            slot = ctypes.c_int32(-1)
            _lib.check(self.lib.tpo_batch_add(self.handle, d, _lib.ptr(f), _lib.ptr(fixed),
                                              _lib.ptr(ws), nbytes, _lib.stream_handle(),
                                              ctypes.byref(slot)))
        self.slots[slot.value] = _Slot(pr, ws, layout, int(d.max_oc_iter), tag)
        return slot.value

    def remove(self, slot: int) -> None:
        _lib.check(self.lib.tpo_batch_remove(self.handle, int(slot)))
        del self.slots[slot]

    def set_step_period(self, slot: int, period: int) -> None:
        """The design takes every `period`-th PCG step of a loop body (1: all):
        the same iterates, spread over more bodies."""
        _lib.check(self.lib.tpo_batch_set_step_period(self.handle, int(slot), int(period)))

    def set_tiles(self, stencil_cols: int, update_cols: int) -> None:
        _lib.check(self.lib.tpo_batch_set_tiles(self.handle, int(stencil_cols), int(update_cols)))

    # -- execution
    def step(self) -> bool:
        """One OC iteration of every active design. Returns whether any
        design still has OC iterations left."""
        with torch.cuda.device(self.device):
            _lib.check(self.lib.tpo_batch_oc_iteration(self.handle, _lib.stream_handle()))
        it, active = self.states()
        return bool(active.any())

    def round(self, rounds: int = 1) -> None:
        """`rounds` rounds of continuous batching (`tpo_batch_round`), then one
        status read: every design advances by one PCG loop body or one
        OC-iteration stage per round, whatever the OC iteration it is at."""
        with torch.cuda.device(self.device):
            _lib.check(self.lib.tpo_batch_round(self.handle, int(rounds), _lib.stream_handle()))

    def states(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.max_designs
        it = (ctypes.c_int32 * n)()
        act = (ctypes.c_int32 * n)()
        _lib.check(self.lib.tpo_batch_states(self.handle, n, it, act))
        return np.frombuffer(it, dtype=np.int32).copy(), np.frombuffer(act, dtype=np.int32).copy()

    def run(self, rounds: bool = False) -> None:
        """Run every design to its end, by OC iterations (all designs step
        together) or by rounds (each design at its own pace)."""
        if not rounds:
            while self.step():
                pass
            return
        while True:
            self.round()
            if not self.states()[1].any():
                return

    # -- results
    def _view(self, slot: int, off: int, count: int) -> torch.Tensor:
        s = self.slots[slot]
        return s.ws[off:off + 8 * count].view(torch.float64)

    def density(self, slot: int) -> np.ndarray:
        s = self.slots[slot]
        pr = s.problem
        return self._view(slot, s.layout.rho, pr.n_elem).cpu().numpy().reshape(pr.nelx, pr.nely)

    def displacement(self, slot: int) -> np.ndarray:
        s = self.slots[slot]
        return self._view(slot, s.layout.u, s.problem.n_dofs).cpu().numpy()

    def history(self, slot: int) -> dict:
        s = self.slots[slot]
        it, _ = self.states()
        n = int(it[slot])
        h = self._view(slot, s.layout.hist, 6 * s.max_iter).cpu().numpy().reshape(-1, 6)[:n]
        return {k: h[:, i].copy() for i, k in enumerate(HIST_FIELDS)}

    def result(self, slot: int) -> tuple[np.ndarray, dict]:
        return self.density(slot), self.history(slot)

    def time_steps(self, steps: int) -> float:
        ms = ctypes.c_float()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.tpo_batch_time_steps(self.handle, int(steps),
                                                     _lib.stream_handle(), ctypes.byref(ms)))
        return float(ms.value)

    def close(self) -> None:
        if self.handle is not None:
            self.lib.tpo_batch_destroy(self.handle)
            self.handle = None
            self.slots.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# Workload: designs of uneven size from a seed
# --------------------------------------------------------------------------

def _family_dict(family: str, nelx: int, nely: int, frac: float, volfrac: float, rmin: float,
                 max_iter: int, precision: str = "mixed",
                 preconditioner: str = "nodal_block_jacobi") -> dict:
    """YAML mapping of one design. The point load sits at fraction `frac` of
    the loaded edge (top edge for MBB and bridge, right edge for the
    cantilever); the boundary conditions follow the MBB half-beam (left-edge
    x DOFs and the bottom-right y DOF fixed), the cantilever (left edge
    clamped) and the bridge (bottom corners pinned)."""
    if family == "mbb":
        ix = int(round(frac * nelx))
        fixed = [{"nodes": {"type": "edge", "edge": "left"}, "dofs": ["x"]},
                 {"nodes": {"type": "point", "location": [nelx, 0]}, "dofs": ["y"]}]
        load = [ix, nely]
    elif family == "cantilever":
        iy = int(round(frac * nely))
        fixed = [{"nodes": {"type": "edge", "edge": "left"}, "dofs": ["x", "y"]}]
        load = [nelx, iy]
    elif family == "bridge":
        ix = int(round(frac * nelx))
        fixed = [{"nodes": {"type": "point", "location": [0, 0]}, "dofs": ["x", "y"]},
                 {"nodes": {"type": "point", "location": [nelx, 0]}, "dofs": ["x", "y"]}]
        load = [ix, nely]
    else:
        raise ValueError(family)
    return {
        "problem": {"name": f"{family} {nelx}x{nely}", "dimension": 2},
        "domain": {"nelx": nelx, "nely": nely},
        "material": {"E": 1.0, "nu": 0.3, "E_min": 1e-9},
        "boundary_conditions": {"fixed": fixed},
        "loads": [{"nodes": {"type": "point", "location": load}, "force": [0.0, -1.0]}],
        "optimization": {"volume_fraction": volfrac, "penalty": 3.0, "filter_radius": rmin,
                         "filter_type": "density", "max_iterations": max_iter,
                         "tolerance": 0.0, "move_limit": 0.2},
        "solver": {"max_cg_iterations": 20000, "cg_tolerance": 1e-8,
                   "preconditioner": preconditioner, "precision": precision,
                   "inner_tolerance": 1e-3, "max_outer_iterations": 100},
        "output": {"directory": "results/batch", "save_interval": 1000, "format": "png"},
    }


def random_designs(n: int, seed: int = 0, nelx_range: tuple[int, int] = (64, 512),
                   max_iter: int = 50, precision: str = "mixed") -> list[Problem]:
    """`n` designs drawn from `numpy.random.default_rng(seed)`:
    nelx ~ U{lo..hi}; aspect nelx/nely ~ U{1, 2, 3}, nely = max(1, round(nelx /
    aspect)); family ~ U{MBB, cantilever, bridge}; load position ~ U over the
    middle 80 % of the loaded edge; volfrac ~ U[0.3, 0.6]; rmin ~ U[1.5, 4.0];
    E0 = 1, Emin = 1e-9, nu = 0.3, p = 3."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nelx = int(rng.integers(nelx_range[0], nelx_range[1] + 1))
        aspect = int(rng.choice([1, 2, 3]))
        nely = max(1, int(round(nelx / aspect)))
        family = str(rng.choice(["mbb", "cantilever", "bridge"]))
        frac = float(rng.uniform(0.1, 0.9))
        volfrac = float(rng.uniform(0.3, 0.6))
        rmin = float(rng.uniform(1.5, 4.0))
        out.append(problem_from_dict(_family_dict(family, nelx, nely, frac, volfrac, rmin,
                                                  max_iter, precision)))
    return out


# --------------------------------------------------------------------------
# Autotuner
# --------------------------------------------------------------------------

TILE_CANDIDATES = [(ls, lu) for ls in (8, 12, 16, 24, 32, 48) for lu in (4, 8, 16)]


def autotune(problems: list[Problem], candidates=None, steps: int = 64,
             preconditioner: str = "nodal_block_jacobi", device=None) -> dict:
    """Choose the strip lengths of the batched PCG kernels for this set of
    designs: build a scratch batch holding all of them, time `steps` PCG steps
    of the whole batch for each candidate (CUDA events, after one untimed
    warm-up pass) and return {"best": (ls, lu), "ms": {candidate: ms}}.
    The scratch batch is discarded, so the timed steps do not disturb any
    batch whose results are wanted."""
    cands = list(candidates) if candidates is not None else TILE_CANDIDATES
    scratch = Batch(len(problems), preconditioner=preconditioner, use_graph=False,
                    device=device)
    try:
        for pr in problems:
            scratch.add(pr, max_iter=1)
        timings = {}
        for ls, lu in cands:
            scratch.set_tiles(ls, lu)
            scratch.time_steps(8)  # warm-up: first launches with these tiles
            timings[(ls, lu)] = scratch.time_steps(steps)
        best = min(timings, key=timings.get)
    finally:
        scratch.close()
    return {"best": best, "ms": timings, "steps": steps}


def run_serial_mixed(problems: list[Problem], device=None) -> list[tuple[np.ndarray, list]]:
    """The same designs one at a time through the single-design API (the
    per-design reference for the batch's results)."""
    from .optimizer.simp import SimpDesign
    out = []
    for pr in problems:
        d = SimpDesign(pr, device=device, precision="mixed", preconditioner=pr.preconditioner)
        comp = []
        for _ in range(pr.max_iter):
            comp.append(d.step().compliance)
        out.append((d.density().reshape(pr.nelx, pr.nely), comp))
    return out


__all__ = ["Batch", "random_designs", "autotune", "footprint_bytes", "HIST_FIELDS",
           "TILE_CANDIDATES", "run_serial_mixed"]
