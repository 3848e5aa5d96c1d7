"""Hat-weight filters on the device.

Counterpart of the reference's `src/toptimization/optimizer/filter.py`. The
reference builds a neighbour list on the host (a Python loop over every
element, `filter.py:22-103`) and gathers from it; libtpo derives the weights
w = max(0, rmin - dist) analytically inside each CTA, so there is no
precompute and no list in memory. Same box, same w > 0 rule, same
neighbour order, same 1e-20 in the denominators. A `TpoGrid3` runs the 3D
box (`filter.py:75-97`).
"""

from __future__ import annotations

import torch

from .. import _lib


def density_filter(grid: _lib.TpoGrid, rmin: float, x: torch.Tensor, out: torch.Tensor,
                   scale_out: torch.Tensor | None = None,
                   scale32_out: torch.Tensor | None = None) -> None:
    """out = H x / (H 1 + 1e-20): the density filter (`filter.py:106-124`) and
    the chain-rule dc projection (`filter.py:127-149,174-180`). Optionally
    also writes the SIMP scale of `out` in FP64 / FP32 (2D only)."""
    if _lib.is3d(grid):
        if scale_out is not None or scale32_out is not None:
            raise ValueError("the 3D filter writes no scales")
        _lib.check(_lib.load().tpo3_density_filter(grid, float(rmin), _lib.ptr(x),
                                                   _lib.ptr(out), _lib.stream_handle()))
        return
    _lib.check(_lib.load().tpo_density_filter(
        grid, float(rmin), _lib.ptr(x), _lib.ptr(out), _lib.ptr(scale_out),
        _lib.ptr(scale32_out), _lib.stream_handle()))


def sensitivity_filter(grid: _lib.TpoGrid, rmin: float, rho: torch.Tensor, dc: torch.Tensor,
                       out: torch.Tensor) -> None:
    """Sigmund's filter: out = H(rho dc) / (rho H 1 + 1e-20) (`filter.py:152-171`)."""
    lib = _lib.load()
    fn = lib.tpo3_sensitivity_filter if _lib.is3d(grid) else lib.tpo_sensitivity_filter
    _lib.check(fn(
        grid, float(rmin), _lib.ptr(rho), _lib.ptr(dc), _lib.ptr(out), _lib.stream_handle()))
