"""ctypes wrapper of the C/OpenMP oracle (oracle/csrc/simp_cpu.c).

TEST AND BASELINE INFRASTRUCTURE ONLY (see that file's header). Only tests/,
`__graft_entry__.smoke()` and bench.py's CPU legs use it.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_int, c_long, c_void_p

import numpy as np

from . import build_c
from toptimization_b200.material import compute_Ke, regularized_inverse
from toptimization_b200.mesh import force_vector

PRECOND = {"none": 0, "jacobi": 1, "block_jacobi": 2, "nodal_block_jacobi": 3}
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(str(build_c.build()))
        PD = POINTER(c_double)
        L.ocpu_create.restype = c_void_p
        L.ocpu_create.argtypes = [c_int, c_int, c_int, PD, PD, c_double,
                                  POINTER(ctypes.c_int64), c_long,
                                  PD, c_double, c_double, c_double, c_double, c_double, c_int,
                                  c_double, c_int, c_int]
        L.ocpu_destroy.argtypes = [c_void_p]
        L.ocpu_iteration.argtypes = [c_void_p, c_int, PD]
        L.ocpu_get_rho.argtypes = [c_void_p, PD]
        L.ocpu_set_rho.argtypes = [c_void_p, PD]
        L.ocpu_get_u.argtypes = [c_void_p, PD]
        L.ocpu_matvec.argtypes = [c_void_p, PD, PD, PD]
        L.ocpu_threads.restype = c_int
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(POINTER(c_double))


class CpuSimp:
    """One design on the CPU (2D or 3D); `iteration()` runs one OC iteration."""

    def __init__(self, problem, preconditioner=None):
        pr = problem
        self.problem = pr
        nz = pr.nelz if pr.dim == 3 else 0
        Ke = np.ascontiguousarray(compute_Ke(pr.E, pr.nu, pr.dim))
        Kinv, alpha = regularized_inverse(Ke)
        Kinv = np.ascontiguousarray(Kinv)
        fixed = np.ascontiguousarray(np.asarray(pr.fixed_dofs, dtype=np.int64))
        f = np.ascontiguousarray(force_vector(pr))
        pre = PRECOND[preconditioner or pr.preconditioner]
        self.h = lib().ocpu_create(pr.nelx, pr.nely, nz, _pd(Ke), _pd(Kinv), alpha,
                                   fixed.ctypes.data_as(POINTER(ctypes.c_int64)), fixed.size,
                                   _pd(f), pr.E_min, pr.penalty, pr.rmin, pr.volfrac,
                                   pr.move_limit, pre, pr.cg_tol, pr.max_cg_iter,
                                   1 if pr.filter_type == "sensitivity" else 0)
        if not self.h:
            raise ValueError("ocpu_create failed (out of memory, or the nodal block "
                             "preconditioner on a 3D grid)")

    def iteration(self, max_cg: int = 0) -> dict:
        out = np.zeros(7)
        lib().ocpu_iteration(self.h, int(max_cg), _pd(out))
        return dict(compliance=out[0], volume=out[1], change=out[2], cg_iters=int(out[3]),
                    status=int(out[4]), pcg_seconds=out[5], other_seconds=out[6])

    def rho(self) -> np.ndarray:
        out = np.empty(self.problem.n_elem)
        lib().ocpu_get_rho(self.h, _pd(out))
        return out

    def set_rho(self, rho) -> None:
        a = np.ascontiguousarray(rho, dtype=np.float64)
        lib().ocpu_set_rho(self.h, _pd(a))

    def u(self) -> np.ndarray:
        out = np.empty(self.problem.n_dofs)
        lib().ocpu_get_u(self.h, _pd(out))
        return out

    def matvec(self, rho_phys, p) -> np.ndarray:
        r = np.ascontiguousarray(rho_phys, dtype=np.float64)
        pp = np.ascontiguousarray(p, dtype=np.float64)
        out = np.empty_like(pp)
        lib().ocpu_matvec(self.h, _pd(r), _pd(pp), _pd(out))
        return out

    def close(self):
        if self.h:
            lib().ocpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def threads() -> int:
    return lib().ocpu_threads()
