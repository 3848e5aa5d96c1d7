"""PCG solve of K(rho) u = f on the device.

Counterpart of the reference's `src/toptimization/fem/solver.py:27-159`. The
reference drives CG from a Python loop with two host syncs per iteration; here
`tpo_pcg_solve` keeps alpha, beta and the stop test on the GPU and the host only
polls a status word every `poll_every` iterations; `solve_async`
(`tpo_pcg_solve_async`) runs the whole loop on the device with no host wait,
so that it can be captured in a CUDA graph. The stopping rule, warm
start, breakdown test and returned iteration count are the reference's:

  * ||f|| < 1e-30             -> u = 0, 0 iterations
  * tol_sq = (tol ||f||)^2,   stop when the recursive ||r||^2 < tol_sq,
    tested after the update and before the direction update
  * |p.Ap| < 1e-30            -> stop (the reference then reports max_iter)
  * beta = rz_new / (rz_old + 1e-60)
  * returns it+1 on convergence, max_iter otherwise

Preconditioners: "jacobi", "block_jacobi" (the reference's element-block
form), "nodal_block_jacobi" (2x2 nodal blocks, new) and "none".
Recurrence: "auto" (one kernel launch per iteration, in the Chronopoulos-Gear
form with a single global reduction, for the plain FP64 solve with a point
preconditioner; the element-block preconditioner and the mixed form keep two),
"standard" (the reference's own recurrence, two launches per iteration) or
"single" (force the one-launch form). The two recurrences produce the same
iterates in exact arithmetic.
3D (H8) grids (`nelz` > 0) solve in FP64 with "jacobi", "block_jacobi" or
"none" and the standard recurrence (`tpo3_pcg_solve`), the same rules.
Precisions: "fp64" (plain) and "mixed" (Krylov vectors r, p, Ap stored in
FP32, FP64 arithmetic, dot products, alpha/beta and solution u; the recursive
residual is replaced by the FP64 residual f - K u whenever it has dropped by
`inner_tol`, and convergence to `tol` is decided on that FP64 residual).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import torch

from .. import _lib


RECURRENCE = {"auto": 0, "standard": 1, "single": 2}  # TPO_RECURRENCE_*


@dataclass
class SolveInfo:
    status: str
    iters: int         # the reference's count (mixed: total inner iterations)
    outer_iters: int
    updates: int
    rr: float
    launches: int = 0  # kernels the solve ran
    bodies: int = 0    # device loop bodies (asynchronous solve)

    @property
    def converged(self) -> bool:
        return self.status in ("converged", "zero_rhs")


class PCGSolver:
    """Reusable solver for one grid: holds the workspace and the config."""

    def __init__(self, nelx: int, nely: int, e_min: float, penalty: float,
                 f_norm_sq: float, *, preconditioner: str = "jacobi",
                 precision: str = "fp64", max_iter: int = 2000, tol: float = 1e-8,
                 inner_tol: float = 1e-3, max_outer: int = 50, poll_every: int = 0,
                 recurrence: str = "auto", device=None, nelz: int = 0):
        if preconditioner not in _lib.PRECOND:
            raise ValueError(f"unknown preconditioner {preconditioner!r}")
        if precision not in _lib.PRECISION:
            raise ValueError(f"unknown precision {precision!r}")
        if recurrence not in RECURRENCE:
            raise ValueError(f"unknown recurrence {recurrence!r}")
        if recurrence == "single" and (preconditioner == "block_jacobi" or precision != "fp64"):
            raise ValueError("the one-launch recurrence serves the FP64 solve with a point "
                             "preconditioner only")
        if nelz and (preconditioner == "nodal_block_jacobi" or precision != "fp64"
                     or recurrence == "single"):
            raise ValueError("3D solves are FP64 with jacobi, block_jacobi or none and the "
                             "standard recurrence")
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.grid = (_lib.grid3(nelx, nely, nelz, e_min, penalty) if nelz
                     else _lib.grid(nelx, nely, e_min, penalty))
        self.cfg = _lib.TpoSolveCfg(
            precond=_lib.PRECOND[preconditioner], precision=_lib.PRECISION[precision],
            max_iter=int(max_iter), warm_start=1, tol=float(tol), f_norm_sq=float(f_norm_sq),
            inner_tol=float(inner_tol), max_outer=int(max_outer), poll_every=int(poll_every),
            recurrence=RECURRENCE[recurrence])
        lib = _lib.load()
        self._solve = lib.tpo3_pcg_solve if nelz else lib.tpo_pcg_solve
        self.nelz = nelz
        nbytes = (lib.tpo3_pcg_workspace_bytes(self.grid, self.cfg) if nelz
                  else lib.tpo_pcg_workspace_bytes(self.grid, self.cfg))
        self.workspace = torch.empty(nbytes, dtype=torch.uint8, device=self.device)

    def solve(self, rho_phys: torch.Tensor, f: torch.Tensor, fixed: torch.Tensor,
              u: torch.Tensor, warm_start: bool = True) -> SolveInfo:
        """Solve in place: u holds the warm start on entry (ignored if
        warm_start is False) and the solution on exit. Blocks until done."""
        for t in (rho_phys, f, u):
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
                raise ValueError("rho_phys, f and u must be contiguous float64 CUDA tensors")
        if fixed.dtype != torch.uint8:
            raise ValueError("fixed must be a uint8 per-node mask")
        self.cfg.warm_start = 1 if warm_start else 0
        res = _lib.TpoSolveResult()
        _lib.check(self._solve(
            self.grid, self.cfg, _lib.ptr(rho_phys), _lib.ptr(f), _lib.ptr(fixed), _lib.ptr(u),
            _lib.ptr(self.workspace), self.workspace.numel(), res, _lib.stream_handle()))
        return SolveInfo(_lib.SOLVE_STATUS.get(res.status, str(res.status)), res.iters,
                         res.outer_iters, res.updates, res.rr, res.launches, res.bodies)

    RESULT_BYTES = ctypes.sizeof(_lib.TpoSolveResult)

    def result_buffer(self) -> torch.Tensor:
        """Device memory for one solve result (written by `solve_async`)."""
        return torch.zeros(self.RESULT_BYTES, dtype=torch.uint8, device=self.device)

    def solve_async(self, rho_phys: torch.Tensor, f: torch.Tensor, fixed: torch.Tensor,
                    u: torch.Tensor, result: torch.Tensor, warm_start: bool = True) -> None:
        """`solve`, enqueued on the current stream with no host wait: the PCG
        loop runs on the device (tpo_pcg_solve_async) and its outcome lands in
        `result` (a `result_buffer()`; read it with `decode`). Inside a CUDA
        graph capture the solve becomes part of the graph. 2D grids."""
        if self.nelz:
            raise ValueError("3D solves are blocking only (tpo3_pcg_solve)")
        for t in (rho_phys, f, u):
            if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
                raise ValueError("rho_phys, f and u must be contiguous float64 CUDA tensors")
        if fixed.dtype != torch.uint8:
            raise ValueError("fixed must be a uint8 per-node mask")
        if result.numel() * result.element_size() < self.RESULT_BYTES or not result.is_cuda:
            raise ValueError("result must be a CUDA buffer of at least RESULT_BYTES bytes")
        self.cfg.warm_start = 1 if warm_start else 0
        _lib.check(_lib.load().tpo_pcg_solve_async(
            self.grid, self.cfg, _lib.ptr(rho_phys), _lib.ptr(f), _lib.ptr(fixed), _lib.ptr(u),
            _lib.ptr(self.workspace), self.workspace.numel(), _lib.ptr(result),
            _lib.stream_handle()))

    @classmethod
    def decode(cls, result: torch.Tensor) -> SolveInfo:
        """The SolveInfo held in a result buffer (copies it to the host)."""
        raw = bytes(result.reshape(-1)[: cls.RESULT_BYTES].cpu().numpy().tobytes())
        res = _lib.TpoSolveResult.from_buffer_copy(raw)
        return SolveInfo(_lib.SOLVE_STATUS.get(res.status, str(res.status)), res.iters,
                         res.outer_iters, res.updates, res.rr, res.launches, res.bodies)
