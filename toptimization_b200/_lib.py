"""ctypes binding of libtpo (the C ABI in include/tpo.h).

The library is built in-tree (`toptimization_b200/libtpo.so`, see
`toptimization_b200/csrc/build.py`). There is no fallback: if the library is
missing or no CUDA device is usable, every device entry point raises.
"""

from __future__ import annotations

import ctypes
import os
import threading
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_size_t, c_uint8, c_void_p
from pathlib import Path

LIB_PATH = Path(os.environ.get("TPO_LIBRARY", Path(__file__).with_name("libtpo.so")))

TPO_OK = 0
SOLVE_STATUS = {0: "running", 1: "converged", 2: "max_iter", 3: "breakdown",
                4: "nonfinite", 5: "zero_rhs", 7: "timeout", 8: "loop_limit"}
PRECOND = {"none": 0, "jacobi": 1, "block_jacobi": 2, "nodal_block_jacobi": 3}
PRECISION = {"fp64": 0, "mixed": 1}


class TpoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libtpo error {code}: {msg}")
        self.code = code


class TpoGrid(ctypes.Structure):
    _fields_ = [("nelx", c_int32), ("nely", c_int32), ("e_min", c_double),
                ("penalty", c_double)]


class TpoGrid3(ctypes.Structure):
    """3D (H8) grid: nelx x nely x nelz unit cubes."""
    _fields_ = [("nelx", c_int32), ("nely", c_int32), ("nelz", c_int32), ("pad", c_int32),
                ("e_min", c_double), ("penalty", c_double)]


class TpoSolveCfg(ctypes.Structure):
    _fields_ = [("precond", c_int32), ("precision", c_int32), ("max_iter", c_int32),
                ("warm_start", c_int32), ("tol", c_double), ("f_norm_sq", c_double),
                ("inner_tol", c_double), ("max_outer", c_int32), ("poll_every", c_int32),
                ("recurrence", c_int32)]


class TpoSolveResult(ctypes.Structure):
    _fields_ = [("status", c_int32), ("iters", c_int32), ("outer_iters", c_int32),
                ("updates", c_int32), ("rr", c_double), ("launches", c_int32),
                ("bodies", c_int32)]


class TpoProfile(ctypes.Structure):
    _fields_ = [("dir_launches", ctypes.c_int64), ("dir_ms", c_double),
                ("update_launches", ctypes.c_int64), ("update_ms", c_double),
                ("dir_bytes", ctypes.c_int64), ("update_bytes", ctypes.c_int64),
                ("launches", ctypes.c_int64), ("apply_launches", ctypes.c_int64),
                ("apply_ms", c_double), ("apply_bytes", ctypes.c_int64),
                ("step_launches", ctypes.c_int64), ("step_ms", c_double),
                ("step_bytes", ctypes.c_int64)]


class TpoBatchCfg(ctypes.Structure):
    _fields_ = [("precond", c_int32), ("precision", c_int32), ("use_graph", c_int32),
                ("stencil_cols", c_int32), ("update_cols", c_int32), ("round_steps", c_int32)]


class TpoBatchDesign(ctypes.Structure):
    _fields_ = [("nelx", c_int32), ("nely", c_int32), ("e_min", c_double),
                ("penalty", c_double), ("volfrac", c_double), ("move", c_double),
                ("rmin", c_double), ("tol", c_double), ("cg_tol", c_double),
                ("inner_tol", c_double), ("f_norm_sq", c_double), ("rho0", c_double),
                ("max_oc_iter", c_int32), ("max_cg_iter", c_int32), ("max_outer", c_int32),
                ("pad", c_int32)]


class TpoBatchLayout(ctypes.Structure):
    _fields_ = [("rho", c_size_t), ("rho_phys", c_size_t), ("u", c_size_t), ("hist", c_size_t)]


_PD = POINTER(c_double)
_PI = POINTER(c_int32)
_SIGS = {
    "tpo_version": (c_int, []),
    "tpo_last_error_string": (ctypes.c_char_p, []),
    "tpo_set_stiffness": (c_int, [_PD, _PD, c_double]),
    "tpo_matvec_workspace_bytes": (c_size_t, [POINTER(TpoGrid)]),
    "tpo_matvec_f64": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_matvec_f32": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_apply_stiffness_f64": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_apply_stiffness_f32": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_pcg_workspace_bytes": (c_size_t, [POINTER(TpoGrid), POINTER(TpoSolveCfg)]),
    "tpo_pcg_solve": (c_int, [POINTER(TpoGrid), POINTER(TpoSolveCfg), c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_size_t, POINTER(TpoSolveResult),
                              c_void_p]),
    "tpo_test_withhold_stage": (c_int, [c_int32]),
    "tpo_pcg_solve_async": (c_int, [POINTER(TpoGrid), POINTER(TpoSolveCfg), c_void_p,
                                    c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p,
                                    c_void_p]),
    "tpo_sensitivity_workspace_bytes": (c_size_t, [POINTER(TpoGrid)]),
    "tpo_sensitivity": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_size_t, c_void_p]),
    "tpo_sensitivity_noalloc": (c_int, [POINTER(TpoGrid), c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "tpo_density_filter": (c_int, [POINTER(TpoGrid), c_double, c_void_p, c_void_p, c_void_p,
                                   c_void_p, c_void_p]),
    "tpo_sensitivity_filter": (c_int, [POINTER(TpoGrid), c_double, c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    "tpo_oc_workspace_bytes": (c_size_t, [POINTER(TpoGrid)]),
    "tpo_oc_update": (c_int, [POINTER(TpoGrid), c_double, c_double, c_void_p, c_void_p,
                              c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_profile_enable": (c_int, [c_int]),
    "tpo_profile_reset": (c_int, []),
    "tpo_profile_read": (c_int, [POINTER(TpoProfile)]),
    "tpo_set_stiffness3": (c_int, [_PD, _PD, c_double]),
    "tpo3_matvec_workspace_bytes": (c_size_t, [POINTER(TpoGrid3)]),
    "tpo3_matvec_f64": (c_int, [POINTER(TpoGrid3), c_void_p, c_void_p, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo3_pcg_workspace_bytes": (c_size_t, [POINTER(TpoGrid3), POINTER(TpoSolveCfg)]),
    "tpo3_pcg_solve": (c_int, [POINTER(TpoGrid3), POINTER(TpoSolveCfg), c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_size_t, POINTER(TpoSolveResult),
                               c_void_p]),
    "tpo3_sensitivity_workspace_bytes": (c_size_t, [POINTER(TpoGrid3)]),
    "tpo3_sensitivity": (c_int, [POINTER(TpoGrid3), c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_void_p, c_size_t, c_void_p]),
    "tpo3_density_filter": (c_int, [POINTER(TpoGrid3), c_double, c_void_p, c_void_p,
                                    c_void_p]),
    "tpo3_sensitivity_filter": (c_int, [POINTER(TpoGrid3), c_double, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "tpo3_oc_workspace_bytes": (c_size_t, [POINTER(TpoGrid3)]),
    "tpo3_oc_update": (c_int, [POINTER(TpoGrid3), c_double, c_double, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "tpo_batch_workspace_bytes": (c_size_t, [c_int32]),
    "tpo_batch_design_workspace_bytes": (c_size_t, [POINTER(TpoBatchDesign),
                                                    POINTER(TpoBatchLayout)]),
    "tpo_batch_create": (c_int, [c_int32, POINTER(TpoBatchCfg), c_void_p, c_size_t,
                                 POINTER(c_void_p)]),
    "tpo_batch_destroy": (c_int, [c_void_p]),
    "tpo_batch_add": (c_int, [c_void_p, POINTER(TpoBatchDesign), c_void_p, c_void_p, c_void_p,
                              c_size_t, c_void_p, _PI]),
    "tpo_batch_remove": (c_int, [c_void_p, c_int32]),
    "tpo_batch_set_tiles": (c_int, [c_void_p, c_int32, c_int32]),
    "tpo_batch_set_step_period": (c_int, [c_void_p, c_int32, c_int32]),
    "tpo_batch_oc_iteration": (c_int, [c_void_p, c_void_p]),
    "tpo_batch_round": (c_int, [c_void_p, c_int32, c_void_p]),
    "tpo_batch_states": (c_int, [c_void_p, c_int32, _PI, _PI]),
    "tpo_batch_time_steps": (c_int, [c_void_p, c_int32, c_void_p, POINTER(ctypes.c_float)]),
}

_lock = threading.Lock()
_lib = None


def exported_symbols() -> list[str]:
    return list(_SIGS)


def load() -> ctypes.CDLL:
    """Load libtpo once; raise if it is not built."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"libtpo not found at {LIB_PATH}; build it with "
                    "`python -m toptimization_b200.csrc.build` (no CPU fallback exists)")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in _SIGS.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def check(rc: int) -> None:
    if rc != TPO_OK:
        msg = load().tpo_last_error_string()
        raise TpoError(rc, msg.decode() if msg else "")


def grid(nelx: int, nely: int, e_min: float, penalty: float) -> TpoGrid:
    return TpoGrid(int(nelx), int(nely), float(e_min), float(penalty))


def grid3(nelx: int, nely: int, nelz: int, e_min: float, penalty: float) -> TpoGrid3:
    return TpoGrid3(int(nelx), int(nely), int(nelz), 0, float(e_min), float(penalty))


def is3d(g) -> bool:
    return isinstance(g, TpoGrid3)


def launch_count() -> int:
    """Kernel launches this library has enqueued since the last
    tpo_profile_reset (a counter on the host; graph replays do not add)."""
    out = TpoProfile()
    check(load().tpo_profile_read(ctypes.byref(out)))
    return int(out.launches)


def ptr(t) -> int:
    """Device pointer of a torch tensor (0 for None)."""
    return 0 if t is None else int(t.data_ptr())


def stream_handle(stream=None) -> int:
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


_stiffness_set: dict[int, bytes] = {}


def ensure_stiffness(Ke, Ke_inv, alpha_reg: float) -> None:
    """Upload Ke (and the element-block inverse) to the current device's
    constant memory, once per device and matrix."""
    import numpy as np
    import torch
    dev = torch.cuda.current_device()
    ke = np.ascontiguousarray(Ke, dtype=np.float64).reshape(64)
    ki = np.ascontiguousarray(Ke_inv, dtype=np.float64).reshape(64)
    key = ke.tobytes() + ki.tobytes() + np.float64(alpha_reg).tobytes()
    if _stiffness_set.get(dev) == key:
        return
    check(load().tpo_set_stiffness(ke.ctypes.data_as(_PD), ki.ctypes.data_as(_PD),
                                   c_double(alpha_reg)))
    _stiffness_set[dev] = key


def ensure_stiffness3(Ke, Ke_inv, alpha_reg: float) -> None:
    """Upload the 24x24 H8 Ke and its regularised inverse, once per device
    and matrix."""
    import numpy as np
    import torch
    dev = torch.cuda.current_device()
    ke = np.ascontiguousarray(Ke, dtype=np.float64).reshape(576)
    ki = np.ascontiguousarray(Ke_inv, dtype=np.float64).reshape(576)
    key = ke.tobytes() + ki.tobytes() + np.float64(alpha_reg).tobytes()
    if _stiffness3_set.get(dev) == key:
        return
    check(load().tpo_set_stiffness3(ke.ctypes.data_as(_PD), ki.ctypes.data_as(_PD),
                                    c_double(alpha_reg)))
    _stiffness3_set[dev] = key


_stiffness3_set: dict[int, bytes] = {}


def profile_read() -> dict:
    p = TpoProfile()
    check(load().tpo_profile_read(p))
    return {k: getattr(p, k) for k, _ in TpoProfile._fields_}


__all__ = ["load", "check", "grid", "grid3", "is3d", "ptr", "stream_handle",
           "ensure_stiffness", "ensure_stiffness3", "TpoGrid", "TpoGrid3",
           "TpoSolveCfg", "TpoSolveResult", "TpoBatchCfg", "TpoBatchDesign", "TpoBatchLayout",
           "TpoError", "PRECOND", "PRECISION", "SOLVE_STATUS",
           "exported_symbols", "c_float", "c_uint8"]
