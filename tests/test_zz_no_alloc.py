"""tpo_sensitivity_noalloc: the compliance/sensitivity entry point for callers
that cannot allocate device memory (a framework that owns the whole memory
budget in its own pool, or a binding that only receives finished buffers).

It takes no workspace: its scratch is a fixed device array inside libtpo.
Checked through the C ABI against tpo_sensitivity, the entry point with a
caller workspace, on two calls in a row (the scratch keeps the first call's
contents, so the second call checks that the ticket is cleared), plus the
size limit. Collected last so that a run stopping at the first failure has
already run everything else; it also passes alone in a fresh process.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

from toptimization_b200 import _lib  # noqa: E402
from toptimization_b200.material import compute_Ke_2d, regularized_inverse  # noqa: E402


def _call_noalloc(g, rho, u, dc, c):
    return _lib.load().tpo_sensitivity_noalloc(g, _lib.ptr(rho), _lib.ptr(u), _lib.ptr(dc),
                                               _lib.ptr(c), _lib.stream_handle())


def _call_workspace(g, rho, u, dc, c):
    L = _lib.load()
    ws = torch.empty(L.tpo_sensitivity_workspace_bytes(g), dtype=torch.uint8, device="cuda")
    return L.tpo_sensitivity(g, _lib.ptr(rho), _lib.ptr(u), _lib.ptr(dc), _lib.ptr(c),
                             _lib.ptr(ws), ws.numel(), _lib.stream_handle())


@pytest.mark.parametrize("nx,ny", [(60, 20), (2048, 1024)])
def test_noalloc_matches_workspace_entry_point(tpo_built, nx, ny):
    Ke = compute_Ke_2d(1.0, 0.3)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    rng = np.random.default_rng(nx)
    for call in range(2):          # two calls in a row, different inputs
        rho = torch.from_numpy(rng.uniform(0.001, 1.0, nx * ny)).cuda()
        u = torch.from_numpy(rng.standard_normal(2 * (nx + 1) * (ny + 1))).cuda()
        dc_a, dc_b = torch.empty_like(rho), torch.empty_like(rho)
        c_a = torch.empty(1, dtype=torch.float64, device="cuda")
        c_b = torch.empty(1, dtype=torch.float64, device="cuda")
        _lib.check(_call_workspace(g, rho, u, dc_a, c_a))
        _lib.check(_call_noalloc(g, rho, u, dc_b, c_b))
        torch.cuda.synchronize()
        a, b = dc_a.cpu().numpy(), dc_b.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max(), f"call {call}"
        assert c_b.item() == pytest.approx(c_a.item(), rel=1e-13), f"call {call}"


def test_noalloc_second_call_on_another_stream(tpo_built):
    """A call on a new stream, after the first call (on the default stream)
    has finished: the scratch's ticket starts at zero again, so the result
    still equals the workspace entry point's."""
    Ke = compute_Ke_2d(1.0, 0.3)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    nx, ny = 256, 96
    g = _lib.grid(nx, ny, 1e-9, 3.0)
    rng = np.random.default_rng(5)
    rho = torch.from_numpy(rng.uniform(0.001, 1.0, nx * ny)).cuda()
    u = torch.from_numpy(rng.standard_normal(2 * (nx + 1) * (ny + 1))).cuda()
    dc_a, dc_b = torch.empty_like(rho), torch.empty_like(rho)
    c_a = torch.empty(1, dtype=torch.float64, device="cuda")
    c_b = torch.empty(1, dtype=torch.float64, device="cuda")
    _lib.check(_call_workspace(g, rho, u, dc_a, c_a))
    _lib.check(_call_noalloc(g, rho, u, dc_b, c_b))
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        dc_b.zero_()
        _lib.check(_call_noalloc(g, rho, u, dc_b, c_b))
    s.synchronize()
    a, b = dc_a.cpu().numpy(), dc_b.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    assert c_b.item() == pytest.approx(c_a.item(), rel=1e-13)


def test_noalloc_rejects_grids_beyond_the_scratch(tpo_built):
    Ke = compute_Ke_2d(1.0, 0.3)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    g = _lib.grid(16 * 32737, 128, 1e-9, 3.0)   # 32737 partial sums > 32736
    dummy = torch.empty(2, dtype=torch.float64, device="cuda")
    rc = _call_noalloc(g, dummy, dummy, dummy, dummy)
    assert rc == 1
    assert b"32736" in _lib.load().tpo_last_error_string()
