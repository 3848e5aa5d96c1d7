"""Thin wrappers over the libtpo kernels that act on FE fields.

Counterparts of the reference's `src/toptimization/fem/kernels.py`:
  matvec        -> compute_matvec_2d / matvec_and_dot_2d   (kernels.py:143-176,
                   fused_kernels.py:21-56)
  sensitivity   -> compute_sensitivity_2d                   (kernels.py:234-272)
With a `TpoGrid3` (3D, H8) the same calls run compute_matvec_3d /
matvec_and_dot_3d (kernels.py:179-212, fused_kernels.py:59-94) and
compute_sensitivity_3d (kernels.py:275-308), FP64 only; the reference
dispatches on `dim` the same way.
All arguments are CUDA tensors; calls are asynchronous on the current stream.
"""

from __future__ import annotations

import torch

from .. import _lib


def _require_cuda(*ts):
    for t in ts:
        if t is not None and (not t.is_cuda or not t.is_contiguous()):
            raise ValueError("libtpo expects contiguous CUDA tensors")


def matvec(grid: _lib.TpoGrid, rho: torch.Tensor, fixed: torch.Tensor, p: torch.Tensor,
           ap: torch.Tensor | None = None, workspace: torch.Tensor | None = None,
           with_dot: bool = False):
    """ap = K(rho) p (identity rows at fixed DOFs); optionally also p.ap.

    `rho` and `p` share a dtype (float64 or float32). Returns ap, or
    (ap, pap) where pap is a 1-element float64 device tensor."""
    _require_cuda(rho, fixed, p, ap)
    lib = _lib.load()
    if ap is None:
        ap = torch.empty_like(p)
    if workspace is None:
        workspace = matvec_workspace(grid, p.device)
    pap = torch.empty(1, dtype=torch.float64, device=p.device) if with_dot else None
    if _lib.is3d(grid):
        if p.dtype != torch.float64:
            raise ValueError("the 3D matvec is FP64 only")
        fn = lib.tpo3_matvec_f64
    else:
        fn = lib.tpo_matvec_f64 if p.dtype == torch.float64 else lib.tpo_matvec_f32
    if rho.dtype != p.dtype:
        raise ValueError("rho and p must share a dtype")
    _lib.check(fn(grid, _lib.ptr(rho), _lib.ptr(fixed), _lib.ptr(p), _lib.ptr(ap),
                  _lib.ptr(pap), _lib.ptr(workspace), workspace.numel(), _lib.stream_handle()))
    return (ap, pap) if with_dot else ap


def apply_stiffness(grid: _lib.TpoGrid, scale: torch.Tensor, fixed: torch.Tensor,
                    p: torch.Tensor, ap: torch.Tensor, workspace: torch.Tensor,
                    pap: torch.Tensor | None = None) -> None:
    """ap = K p with precomputed element scales (the PCG's operator)."""
    lib = _lib.load()
    fn = lib.tpo_apply_stiffness_f64 if p.dtype == torch.float64 else lib.tpo_apply_stiffness_f32
    if scale.dtype != p.dtype:
        raise ValueError("scale and p must share a dtype")
    _lib.check(fn(grid, _lib.ptr(scale), _lib.ptr(fixed), _lib.ptr(p), _lib.ptr(ap),
                  _lib.ptr(pap), _lib.ptr(workspace), workspace.numel(), _lib.stream_handle()))


def matvec_workspace(grid, device) -> torch.Tensor:
    lib = _lib.load()
    n = (lib.tpo3_matvec_workspace_bytes(grid) if _lib.is3d(grid)
         else lib.tpo_matvec_workspace_bytes(grid))
    return torch.empty(n, dtype=torch.uint8, device=device)


def sensitivity(grid: _lib.TpoGrid, rho_phys: torch.Tensor, u: torch.Tensor,
                dc: torch.Tensor, compliance: torch.Tensor, workspace: torch.Tensor) -> None:
    """dc = d(compliance)/d(rho_phys); compliance[0] = sum_e scale_e u_e^T Ke u_e."""
    _require_cuda(rho_phys, u, dc, compliance, workspace)
    lib = _lib.load()
    fn = lib.tpo3_sensitivity if _lib.is3d(grid) else lib.tpo_sensitivity
    _lib.check(fn(grid, _lib.ptr(rho_phys), _lib.ptr(u), _lib.ptr(dc),
                                   _lib.ptr(compliance), _lib.ptr(workspace), workspace.numel(),
                                   _lib.stream_handle()))


def sensitivity_workspace(grid, device) -> torch.Tensor:
    lib = _lib.load()
    n = (lib.tpo3_sensitivity_workspace_bytes(grid) if _lib.is3d(grid)
         else lib.tpo_sensitivity_workspace_bytes(grid))
    return torch.empty(n, dtype=torch.uint8, device=device)
