"""The C-ABI library: it builds, loads without a GPU, exports every function
include/tpo.h declares, and rejects bad arguments before touching CUDA."""

import ctypes
import re

import pytest

from conftest import REPO
from toptimization_b200 import _lib
from toptimization_b200.csrc import build

HEADER = REPO / "include" / "tpo.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tpo3?_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return ctypes.CDLL(str(build.OUT))


def test_header_declares_the_binding_table():
    assert declared_functions() == sorted(_lib.exported_symbols())


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_python_binding_loads(lib):
    L = _lib.load()
    assert L.tpo_version() == 1


def test_workspace_queries_are_host_only():
    L = _lib.load()
    g = _lib.grid(2048, 1024, 1e-9, 3.0)
    for pre in _lib.PRECOND.values():
        for prec in _lib.PRECISION.values():
            cfg = _lib.TpoSolveCfg(precond=pre, precision=prec, max_iter=10)
            n = L.tpo_pcg_workspace_bytes(g, cfg)
            word = 8 if prec == _lib.PRECISION["fp64"] else 4
            assert n > 4 * word * 2 * 2049 * 1025  # at least r, p (x2), Ap
    assert L.tpo_matvec_workspace_bytes(g) >= 8 * 2048 * 1024
    assert L.tpo_oc_workspace_bytes(g) > 0
    assert L.tpo_sensitivity_workspace_bytes(g) > 0
    assert L.tpo_pcg_workspace_bytes(_lib.grid(0, 5, 1e-9, 3.0), cfg) == 0


def test_argument_errors_before_cuda():
    L = _lib.load()
    bad = _lib.grid(0, 4, 1e-9, 3.0)
    assert L.tpo_density_filter(bad, 1.5, 1, 1, 0, 0, 0) == 1          # TPO_ERR_ARGS
    assert b"nelx" in L.tpo_last_error_string()
    g = _lib.grid(8, 4, 1e-9, 3.0)
    assert L.tpo_density_filter(g, 17.0, 1, 1, 0, 0, 0) == 1          # R > 16
    assert L.tpo_density_filter(g, 0.0, 1, 1, 0, 0, 0) == 1
    assert L.tpo_sensitivity_filter(g, 1.5, 0, 1, 1, 0) == 1          # NULL rho
    with pytest.raises(_lib.TpoError):
        _lib.check(L.tpo_oc_update(g, 0.5, 0.2, 0, 0, 0, 0, 0, 0, 0, 0))


def test_3d_workspace_queries_and_argument_errors():
    """The tpo3_* entry points size their workspaces on the host and check
    their arguments before any CUDA call."""
    L = _lib.load()
    g = _lib.grid3(128, 64, 64, 1e-9, 3.0)
    nd = 3 * 129 * 65 * 65
    for pre in ("none", "jacobi", "block_jacobi"):
        cfg = _lib.TpoSolveCfg(precond=_lib.PRECOND[pre], precision=0, max_iter=10)
        assert L.tpo3_pcg_workspace_bytes(g, cfg) > 8 * 4 * nd    # r, p (x2), Ap
    assert L.tpo3_matvec_workspace_bytes(g) >= 8 * 128 * 64 * 64
    assert L.tpo3_sensitivity_workspace_bytes(g) > 0
    assert L.tpo3_oc_workspace_bytes(g) > 0
    bad = _lib.grid3(4, 0, 3, 1e-9, 3.0)
    assert L.tpo3_matvec_workspace_bytes(bad) == 0
    assert L.tpo3_density_filter(bad, 1.5, 1, 1, 0) == 1            # TPO_ERR_ARGS
    assert b"nelz" in L.tpo_last_error_string()
    small = _lib.grid3(4, 4, 4, 1e-9, 3.0)
    assert L.tpo3_density_filter(small, 8.5, 1, 1, 0) == 1          # R > 8
    assert L.tpo3_sensitivity_filter(small, 1.5, 0, 1, 1, 0) == 1   # NULL rho
    with pytest.raises(_lib.TpoError):
        _lib.check(L.tpo3_oc_update(bad, 0.5, 0.2, 0, 0, 0, 0, 0, 0, 0, 0))
