"""Optimality-criteria update with the bisection on the device.

Counterpart of the reference's `src/toptimization/optimizer/oc.py:52-93`,
which bisects lambda from the host with one kernel launch and one sync per
step. `tpo_oc_update` runs every step on the GPU (the volume reduction, the
lo/hi move and the stop test happen in the last CTA of each step), with the
reference's rules: lambda in [0, 1e9], at most 50 steps, stop when
(hi-lo)/(hi+lo+1e-30) < 1e-4, result and max change from the last midpoint.
Pointwise over elements, so 2D and 3D (`TpoGrid3`) designs share it.
"""

from __future__ import annotations

import torch

from .. import _lib


def oc_workspace(grid, device) -> torch.Tensor:
    lib = _lib.load()
    n = (lib.tpo3_oc_workspace_bytes(grid) if _lib.is3d(grid)
         else lib.tpo_oc_workspace_bytes(grid))
    return torch.empty(n, dtype=torch.uint8, device=device)


def oc_update(grid: _lib.TpoGrid, volfrac: float, move: float, rho: torch.Tensor,
              dc: torch.Tensor, rho_out: torch.Tensor, result: torch.Tensor,
              workspace: torch.Tensor, dv: torch.Tensor | None = None) -> None:
    """rho_out = OC(rho, dc); result[:4] = (max change, mean(rho_out),
    last lambda, bisection steps) on the device. rho_out may be rho."""
    lib = _lib.load()
    fn = lib.tpo3_oc_update if _lib.is3d(grid) else lib.tpo_oc_update
    _lib.check(fn(
        grid, float(volfrac), float(move), _lib.ptr(rho), _lib.ptr(dc), _lib.ptr(dv),
        _lib.ptr(rho_out), _lib.ptr(result), _lib.ptr(workspace), workspace.numel(),
        _lib.stream_handle()))
