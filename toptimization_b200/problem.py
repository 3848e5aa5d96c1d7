"""Problem definition: the YAML schema and the `Problem` record.

Same schema, defaults, validation errors and DOF numbering as the reference's
parser (`src/toptimization/problem.py:18-164`), so existing problem files load
unchanged and give bit-identical fixed-DOF and load arrays.

Numbering conventions (reference `src/toptimization/problem.py:167-173,314-315`):
  2D node (ix, iy)      -> ix*(nely+1) + iy
  3D node (ix, iy, iz)  -> ix*(nely+1)*(nelz+1) + iy*(nelz+1) + iz
  DOF of node n, axis d -> dim*n + d      (d: x=0, y=1, z=2)

Three solver options have no counterpart in the reference and are accepted on
top of its schema: `solver.preconditioner: nodal_block_jacobi` (2x2 nodal
block-Jacobi), `solver.precision: fp64|mixed` (plain FP64 PCG, or a PCG on
FP32-stored vectors with FP64 residual replacement, with
`solver.inner_tolerance` and `solver.max_outer_iterations`) and
`solver.recurrence: auto|standard|single` (one kernel launch per PCG
iteration, or the reference's own two-step recurrence).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path
from typing import Literal

import numpy as np
import yaml

PRECONDITIONERS = ("jacobi", "block_jacobi", "nodal_block_jacobi", "none")
PRECISIONS = ("fp64", "mixed")
RECURRENCES = ("auto", "standard", "single")
_AXIS = {"x": 0, "y": 1, "z": 2}


@dataclass
class Problem:
    """Every number a topology-optimisation run needs.

    Field-for-field the reference's dataclass (`src/toptimization/problem.py:18-78`)
    plus the optional mixed-precision settings at the end (defaulted, so
    positional construction as in the reference's tests still works).
    """

    name: str
    dim: Literal[2, 3]
    nelx: int
    nely: int
    nelz: int
    E: float
    nu: float
    E_min: float
    fixed_dofs: np.ndarray
    force_dofs: np.ndarray
    force_values: np.ndarray
    volfrac: float
    penalty: float
    rmin: float
    filter_type: Literal["density", "sensitivity"]
    max_iter: int
    tol: float
    move_limit: float
    max_cg_iter: int
    cg_tol: float
    preconditioner: str
    output_dir: Path
    save_interval: int
    output_format: Literal["png", "vtk"]
    precision: str = "fp64"
    inner_tol: float = 1e-3
    max_outer_iter: int = 50
    recurrence: str = "auto"

    n_nodes: int = field(init=False)
    n_dofs: int = field(init=False)
    n_elem: int = field(init=False)
    free_dofs: np.ndarray = field(init=False)
    dofs_per_node: int = field(init=False)

    def __post_init__(self) -> None:
        # Derived sizes, as in reference problem.py:68-78.
        self.dofs_per_node = self.dim
        if self.dim == 2:
            self.n_nodes = (self.nelx + 1) * (self.nely + 1)
            self.n_elem = self.nelx * self.nely
        else:
            self.n_nodes = (self.nelx + 1) * (self.nely + 1) * (self.nelz + 1)
            self.n_elem = self.nelx * self.nely * self.nelz
        self.n_dofs = self.dim * self.n_nodes
        self.free_dofs = np.setdiff1d(np.arange(self.n_dofs, dtype=int), self.fixed_dofs)


def load_problem(yaml_path: str | Path) -> Problem:
    """Parse and validate a YAML problem file (reference `problem.py:81-164`)."""
    with Path(yaml_path).open() as fh:
        raw = yaml.safe_load(fh)
    return problem_from_dict(raw)


def problem_from_dict(raw: dict) -> Problem:
    """Build a `Problem` from an already-parsed YAML mapping."""
    sec = {k: (raw.get(k) or {}) for k in
           ("problem", "domain", "material", "optimization", "solver", "output")}
    prob, dom, mat, opt, sol, out = (sec[k] for k in
                                     ("problem", "domain", "material", "optimization",
                                      "solver", "output"))

    dim = int(prob.get("dimension", 2))
    if dim not in (2, 3):
        raise ValueError(f"dimension must be 2 or 3, got {dim}")
    nelx, nely = int(dom["nelx"]), int(dom["nely"])
    nelz = int(dom.get("nelz", 1)) if dim == 3 else 1

    filter_type = opt.get("filter_type", "density")
    if filter_type not in ("density", "sensitivity"):
        raise ValueError(
            f"filter_type must be 'density' or 'sensitivity', got {filter_type}")
    preconditioner = sol.get("preconditioner", "jacobi")
    if preconditioner not in PRECONDITIONERS:
        raise ValueError(
            "preconditioner must be 'jacobi', 'block_jacobi', 'nodal_block_jacobi' "
            f"or 'none', got {preconditioner}")
    precision = sol.get("precision", "fp64")
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be 'fp64' or 'mixed', got {precision}")
    recurrence = sol.get("recurrence", "auto")
    if recurrence not in RECURRENCES:
        raise ValueError(
            f"recurrence must be 'auto', 'standard' or 'single', got {recurrence}")
    if recurrence == "single" and (preconditioner == "block_jacobi" or precision != "fp64"):
        raise ValueError("recurrence 'single' needs precision fp64 and a point "
                         "preconditioner (jacobi, nodal_block_jacobi or none)")
    output_format = out.get("format", "png")
    if output_format not in ("png", "vtk"):
        raise ValueError(f"output format must be 'png' or 'vtk', got {output_format}")

    bcs = raw.get("boundary_conditions") or {}
    fixed = _fixed_dofs(bcs.get("fixed", []), nelx, nely, nelz, dim)
    force_dofs, force_values = _loads(raw.get("loads") or [], nelx, nely, nelz, dim)

    return Problem(
        name=prob.get("name", "Topology Optimization"),
        dim=dim, nelx=nelx, nely=nely, nelz=nelz,
        E=float(mat.get("E", 1.0)),
        nu=float(mat.get("nu", 0.3)),
        E_min=float(mat.get("E_min", 1e-9)),
        fixed_dofs=fixed, force_dofs=force_dofs, force_values=force_values,
        volfrac=float(opt.get("volume_fraction", 0.5)),
        penalty=float(opt.get("penalty", 3.0)),
        rmin=float(opt.get("filter_radius", 1.5)),
        filter_type=filter_type,
        max_iter=int(opt.get("max_iterations", 200)),
        tol=float(opt.get("tolerance", 0.01)),
        move_limit=float(opt.get("move_limit", 0.2)),
        max_cg_iter=int(sol.get("max_cg_iterations", 2000)),
        cg_tol=float(sol.get("cg_tolerance", 1e-6)),
        preconditioner=preconditioner,
        output_dir=Path(out.get("directory", "results")),
        save_interval=int(out.get("save_interval", 10)),
        output_format=output_format,
        precision=precision,
        inner_tol=float(sol.get("inner_tolerance", 1e-3)),
        max_outer_iter=int(sol.get("max_outer_iterations", 50)),
        recurrence=recurrence,
    )


# --------------------------------------------------------------------------
# Node specifications -> node indices
# --------------------------------------------------------------------------

def node_index_2d(ix: int, iy: int, nely: int) -> int:
    return ix * (nely + 1) + iy


def node_index_3d(ix: int, iy: int, iz: int, nely: int, nelz: int) -> int:
    return (ix * (nely + 1) + iy) * (nelz + 1) + iz


def _axes(labels, dim: int) -> list[int]:
    """DOF labels -> axis offsets (reference `problem.py:231-241`)."""
    out = []
    for lab in labels:
        if lab not in _AXIS:
            raise ValueError(f"Unknown DOF label '{lab}'. Use 'x', 'y', or 'z'.")
        if _AXIS[lab] >= dim:
            raise ValueError(f"DOF '{lab}' not valid for {dim}D problem")
        out.append(_AXIS[lab])
    return out


def _fixed_dofs(entries, nelx, nely, nelz, dim) -> np.ndarray:
    """Union of all fixed DOFs, sorted ascending (reference `problem.py:176-198`)."""
    dofs: set[int] = set()
    for ent in entries:
        axes = _axes(ent.get("dofs", ["x", "y"]), dim)
        for n in resolve_nodes(ent["nodes"], nelx, nely, nelz, dim):
            dofs.update(dim * n + a for a in axes)
    return np.array(sorted(dofs), dtype=int)


def _loads(entries, nelx, nely, nelz, dim):
    """(force_dofs, force_values) in file order, zero components skipped
    (reference `problem.py:201-228`)."""
    dofs: list[int] = []
    vals: list[float] = []
    for ent in entries:
        vec = ent["force"]
        if len(vec) != dim:
            raise ValueError(f"force vector length {len(vec)} != dim {dim}")
        for n in resolve_nodes(ent["nodes"], nelx, nely, nelz, dim):
            for a, v in enumerate(vec):
                if v != 0.0:
                    dofs.append(dim * n + a)
                    vals.append(float(v))
    if not dofs:
        raise ValueError("No nonzero forces specified in problem definition")
    return np.array(dofs, dtype=int), np.array(vals, dtype=float)


def resolve_nodes(spec: dict, nelx: int, nely: int, nelz: int, dim: int) -> list[int]:
    """A node spec -> list of global node indices (reference `problem.py:244-263`)."""
    kind = spec["type"]
    if kind == "edge" and dim == 2:
        return _edge_2d(spec["edge"], nelx, nely)
    if kind == "face" and dim == 3:
        return _face_3d(spec["face"], nelx, nely, nelz)
    if kind == "point":
        return [_point(spec, nelx, nely, nelz, dim)]
    if kind == "region":
        return _region(spec, nelx, nely, nelz, dim)
    raise ValueError(f"Unknown node spec type '{kind}' for dim={dim}")


def _edge_2d(edge: str, nelx: int, nely: int) -> list[int]:
    # reference problem.py:266-278
    if edge == "left":
        pts = [(0, iy) for iy in range(nely + 1)]
    elif edge == "right":
        pts = [(nelx, iy) for iy in range(nely + 1)]
    elif edge == "bottom":
        pts = [(ix, 0) for ix in range(nelx + 1)]
    elif edge == "top":
        pts = [(ix, nely) for ix in range(nelx + 1)]
    else:
        raise ValueError(f"Unknown edge '{edge}'. Use 'left', 'right', 'top', 'bottom'.")
    return [node_index_2d(ix, iy, nely) for ix, iy in pts]


def _face_3d(face: str, nelx: int, nely: int, nelz: int) -> list[int]:
    # reference problem.py:281-311; enumeration order kept (outer, inner)
    rx, ry, rz = range(nelx + 1), range(nely + 1), range(nelz + 1)
    grids = {
        "left": [(0, a, b) for a in ry for b in rz],
        "right": [(nelx, a, b) for a in ry for b in rz],
        "bottom": [(a, 0, b) for a in rx for b in rz],
        "top": [(a, nely, b) for a in rx for b in rz],
        "front": [(a, b, 0) for a in rx for b in ry],
        "back": [(a, b, nelz) for a in rx for b in ry],
    }
    if face not in grids:
        raise ValueError(f"Unknown face '{face}'.")
    return [node_index_3d(x, y, z, nely, nelz) for x, y, z in grids[face]]


def _point(spec: dict, nelx: int, nely: int, nelz: int, dim: int) -> int:
    # reference problem.py:318-367: 2D locations are node coordinates clamped
    # to the grid; 3D locations are not clamped.
    if "location" in spec:
        loc = spec["location"]
        if dim == 2:
            return node_index_2d(min(int(loc[0]), nelx), min(int(loc[1]), nely), nely)
        return node_index_3d(int(loc[0]), int(loc[1]), int(loc[2]), nely, nelz)
    if "corner" in spec:
        name = spec["corner"]
        if dim == 2:
            table = {"bottom-left": (0, 0), "bottom-right": (nelx, 0),
                     "top-left": (0, nely), "top-right": (nelx, nely)}
            if name not in table:
                raise ValueError(f"Unknown 2D corner '{name}'")
            return node_index_2d(*table[name], nely)
        table = {"front-bottom-left": (0, 0, 0), "front-bottom-right": (nelx, 0, 0),
                 "back-bottom-left": (0, 0, nelz), "back-bottom-right": (nelx, 0, nelz)}
        if name not in table:
            raise ValueError(f"Unknown 3D corner '{name}'")
        return node_index_3d(*table[name], nely, nelz)
    raise ValueError("Point node spec requires 'location' or 'corner'")


def _region(spec: dict, nelx: int, nely: int, nelz: int, dim: int) -> list[int]:
    # reference problem.py:370-391: inclusive integer box, x outermost
    x0, x1 = spec.get("x", [0, nelx])
    y0, y1 = spec.get("y", [0, nely])
    xs, ys = range(int(x0), int(x1) + 1), range(int(y0), int(y1) + 1)
    if dim == 2:
        return [node_index_2d(ix, iy, nely) for ix in xs for iy in ys]
    z0, z1 = spec.get("z", [0, nelz])
    zs = range(int(z0), int(z1) + 1)
    return [node_index_3d(ix, iy, iz, nely, nelz) for ix in xs for iy in ys for iz in zs]
