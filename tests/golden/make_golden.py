"""Generate the golden vectors under tests/golden/ from the reference itself.

Run in a container that has the reference checkout (not on the GPU machines):

    python tests/golden/make_golden.py --reference <reference checkout>/src

(or set TPO_REFERENCE_SRC to that directory)

What is recorded, all from the reference's own code:
  boundary.npz        Ke (Q4, H8), Ke_inv/alpha, edof (4x3), the fixed-DOF and
                      load arrays of every reference example, of examples/ and
                      of the parser-coverage files in tests/golden/yaml/.
  ref_kernels.npz     single calls of the reference's kernels (matvec, diag,
                      element-block preconditioner, sensitivity, the three
                      filters, the OC update, a PCG solve per preconditioner)
                      on a seeded 12x5 cantilever.
  ref_kernels3d.npz   the same single calls through the reference's 3D (H8)
                      kernels on a seeded 5x3x2 cantilever;
  ref_kernels3d_rollers.npz  and on a 3x5x4 block on rollers (partial DOF
                      sets on three faces) with three point loads.
  ref_run_*.npz       whole `simp.run` optimisations: compliance, volume,
                      change and CG-count histories plus final densities
                      (ref_run_3d_*: the 3D loop on an 8x4x3 cantilever).

The kernels run under `taichi_fp64_shim` (Taichi is not installable here), with
every value in FP64; see that module's header for exactly what it implements.
"""

from __future__ import annotations

import argparse
import contextlib
import io
import multiprocessing as mp
import os
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def _import_reference(ref_src: str):
    sys.path.insert(0, str(HERE))
    import taichi_fp64_shim as shim
    shim.install()
    sys.path.insert(0, ref_src)
    import toptimization.fem.fields  # noqa: F401
    import toptimization.optimizer.filter  # noqa: F401
    shim.promote_reference_numpy()


def _boundary(ref_src: str, ref_examples: Path) -> dict:
    _import_reference(ref_src)
    from toptimization.material import compute_Ke_2d, compute_Ke_3d
    from toptimization.mesh import build_edof_2d, element_centers_2d
    from toptimization.problem import load_problem, Problem

    out = {"Ke2d": compute_Ke_2d(1.0, 0.3), "Ke3d": compute_Ke_3d(1.0, 0.3),
           "Ke2d_E2_nu025": compute_Ke_2d(2.0, 0.25)}
    Ke = out["Ke2d"]
    alpha = 0.1 * float(np.mean(np.abs(np.diag(Ke))))
    out["Ke2d_inv"] = np.linalg.inv(Ke + alpha * np.eye(8))
    out["Ke2d_alpha"] = np.float64(alpha)
    p = Problem(name="t", dim=2, nelx=4, nely=3, nelz=1, E=1.0, nu=0.3, E_min=1e-9,
                fixed_dofs=np.array([0, 1]), force_dofs=np.array([39]),
                force_values=np.array([-1.0]), volfrac=0.5, penalty=3.0, rmin=1.5,
                filter_type="density", max_iter=1, tol=0.01, move_limit=0.2,
                max_cg_iter=10, cg_tol=1e-8, preconditioner="jacobi",
                output_dir=Path("."), save_interval=1, output_format="png")
    out["edof_4x3"] = build_edof_2d(p)
    out["centers_4x3"] = element_centers_2d(p)
    yamls = (sorted(ref_examples.glob("*.yaml")) + sorted((REPO / "examples").glob("*.yaml"))
             + sorted((HERE / "yaml").glob("*.yaml")))
    names = []
    for y in yamls:
        prefix = {ref_examples: "ref_", REPO / "examples": "ex_", HERE / "yaml": "yaml_"}
        tag = prefix[y.parent] + y.stem
        pr = load_problem(_reference_compatible(y))
        names.append(tag)
        out[f"{tag}__fixed"] = pr.fixed_dofs
        out[f"{tag}__fdofs"] = pr.force_dofs
        out[f"{tag}__fvals"] = pr.force_values
        out[f"{tag}__sizes"] = np.array([pr.nelx, pr.nely, pr.n_nodes, pr.n_dofs, pr.n_elem])
    out["yaml_names"] = np.array(names)
    return out


def _reference_compatible(yaml_path: Path) -> Path:
    """The reference parser rejects the 2x2 nodal block-Jacobi option; the
    fixed-DOF and load arrays do not depend on it, so parse a copy naming
    'jacobi' instead."""
    import yaml
    raw = yaml.safe_load(yaml_path.read_text())
    if (raw.get("solver") or {}).get("preconditioner") == "nodal_block_jacobi":
        raw["solver"]["preconditioner"] = "jacobi"
        tmp = Path(tempfile.mkdtemp()) / yaml_path.name
        tmp.write_text(yaml.safe_dump(raw))
        return tmp
    return yaml_path


def _small_problem(nelx=12, nely=5, rmin=1.5, pre="jacobi"):
    from toptimization.problem import Problem
    nn = (nelx + 1) * (nely + 1)
    fixed = np.arange(0, 2 * (nely + 1))                   # left edge, x and y
    load = 2 * (nelx * (nely + 1) + nely // 2) + 1         # right edge mid, y
    return Problem(name="k", dim=2, nelx=nelx, nely=nely, nelz=1, E=1.0, nu=0.3,
                   E_min=1e-9, fixed_dofs=fixed, force_dofs=np.array([load]),
                   force_values=np.array([-1.0]), volfrac=0.4, penalty=3.0, rmin=rmin,
                   filter_type="density", max_iter=1, tol=0.0, move_limit=0.2,
                   max_cg_iter=500, cg_tol=1e-10, preconditioner=pre,
                   output_dir=Path(tempfile.mkdtemp()), save_interval=10 ** 6,
                   output_format="png"), nn


def _small_problem_3d(nelx=5, nely=3, nelz=2):
    """Left face clamped; y load on the right face's bottom edge."""
    from toptimization.problem import Problem
    ny1, nz1 = nely + 1, nelz + 1
    fixed = np.arange(0, 3 * ny1 * nz1)
    load = np.array([3 * ((nelx * ny1 + 0) * nz1 + iz) + 1 for iz in range(nz1)])
    return Problem(name="k3", dim=3, nelx=nelx, nely=nely, nelz=nelz, E=1.0, nu=0.3,
                   E_min=1e-9, fixed_dofs=fixed, force_dofs=load,
                   force_values=np.full(load.size, -1.0 / load.size), volfrac=0.4,
                   penalty=3.0, rmin=1.5, filter_type="density", max_iter=1, tol=0.0,
                   move_limit=0.2, max_cg_iter=500, cg_tol=1e-10, preconditioner="jacobi",
                   output_dir=Path(tempfile.mkdtemp()), save_interval=10 ** 6,
                   output_format="png")


def _small_problem_3d_rollers(nelx=3, nely=5, nelz=4):
    """Rollers: y fixed on the bottom face, x on the left face, z on the front
    face (partial DOF sets); three point loads of mixed direction."""
    from toptimization.problem import Problem
    ny1, nz1 = nely + 1, nelz + 1

    def node(ix, iy, iz):
        return (ix * ny1 + iy) * nz1 + iz
    fixed = set()
    for ix in range(nelx + 1):
        for iz in range(nz1):
            fixed.add(3 * node(ix, 0, iz) + 1)
    for iy in range(ny1):
        for iz in range(nz1):
            fixed.add(3 * node(0, iy, iz))
    for ix in range(nelx + 1):
        for iy in range(ny1):
            fixed.add(3 * node(ix, iy, 0) + 2)
    loads = [(3 * node(nelx, nely, nelz) + 1, -1.0), (3 * node(nelx, 2, 3), 0.5),
             (3 * node(1, nely, 2) + 2, -0.25)]
    return Problem(name="k3b", dim=3, nelx=nelx, nely=nely, nelz=nelz, E=1.0, nu=0.3,
                   E_min=1e-9, fixed_dofs=np.array(sorted(fixed)),
                   force_dofs=np.array([d for d, _ in loads]),
                   force_values=np.array([v for _, v in loads]), volfrac=0.4,
                   penalty=3.0, rmin=1.5, filter_type="density", max_iter=1, tol=0.0,
                   move_limit=0.2, max_cg_iter=500, cg_tol=1e-10, preconditioner="jacobi",
                   output_dir=Path(tempfile.mkdtemp()), save_interval=10 ** 6,
                   output_format="png")


def _kernels(ref_src: str) -> dict:
    _import_reference(ref_src)
    pr, _ = _small_problem()
    return _kernel_suite(ref_src, pr, 2, 20261203, (1.5, 2.5, 4.0))


def _kernels3d(ref_src: str) -> dict:
    _import_reference(ref_src)
    return _kernel_suite(ref_src, _small_problem_3d(), 3, 20261204, (1.5, 2.2))


def _kernels3d_rollers(ref_src: str) -> dict:
    _import_reference(ref_src)
    return _kernel_suite(ref_src, _small_problem_3d_rollers(), 3, 20261205, (1.2, 2.9))


def _kernel_suite(ref_src: str, pr, dim: int, seed: int, rmin_list) -> dict:
    _import_reference(ref_src)
    import math
    from toptimization.fem import fields as F, kernels as K, fused_kernels as FK
    from toptimization.fem import preconditioner as PC, solver
    from toptimization.optimizer import filter as filt, oc
    from toptimization.mesh import build_edof, element_centers
    from toptimization.material import compute_Ke

    rng = np.random.default_rng(seed)
    E, N = pr.n_elem, pr.n_dofs
    Ke = compute_Ke(1.0, 0.3, dim)
    edof = build_edof(pr)
    dpe = Ke.shape[0]

    def alloc(rmin):
        F.allocate(n_dofs=N, n_elem=E, dpe=dpe,
                   max_neighbors=(2 * math.ceil(rmin) + 1) ** dim,
                   Ke_np=Ke, edof_np=edof, fixed_dofs=pr.fixed_dofs,
                   force_dofs=pr.force_dofs, force_values=pr.force_values)

    out = {"nelx": np.int64(pr.nelx), "nely": np.int64(pr.nely),
           "nelz": np.int64(pr.nelz),
           "fixed": pr.fixed_dofs, "force_dofs": pr.force_dofs,
           "force_values": pr.force_values}
    rho = rng.uniform(0.001, 1.0, E)
    p = rng.standard_normal(N)
    p2 = rng.standard_normal(N)
    out.update(rho=rho, p=p, p2=p2)
    Emin, pen = pr.E_min, pr.penalty

    alloc(1.5)
    F.rho.from_numpy(rho)
    F.p.from_numpy(p)
    K.compute_matvec(F.p, F.Ap, F.rho, F.Ke, F.edof, F.is_fixed, Emin, pen, E, dim)
    out["Ap"] = F.Ap.to_numpy()
    out["pAp"] = np.float64(FK.matvec_and_dot(F.p, F.Ap, F.rho, F.Ke, F.edof, F.is_fixed,
                                              Emin, pen, E, dim))
    K.compute_diagonal(F.diag, F.rho, F.Ke, F.edof, F.is_fixed, Emin, pen, E, dim)
    out["diag"] = F.diag.to_numpy()
    PC.setup(F.edof, F.diag_count, E, dim)
    out["diag_count"] = F.diag_count.to_numpy()
    F.r.from_numpy(p2)
    rz = PC.apply_and_rz(F.r, F.z, F.rho, F.Ke_inv, F.edof, F.diag_count, F.is_fixed,
                         F._dot_result, Emin, pen, F.KE_ALPHA_REG, E, dim)
    out["bj_z"] = F.z.to_numpy()
    out["bj_rz"] = np.float64(rz)
    out["bj_rr"] = np.float64(F._dot_result[None])
    F.u.from_numpy(p)
    c = K.compute_sensitivity(F.u, F.rho, F.dc, F.dv, F.Ke, F.edof, Emin, pen, E, dim)
    out["sens_dc"] = F.dc.to_numpy()
    out["sens_c"] = np.float64(c)
    out["volume"] = np.float64(K.compute_volume(F.rho, E))

    dcs = -np.abs(rng.standard_normal(E)) * rng.uniform(0.1, 10.0, E)
    out["dc_in"] = dcs
    centers = element_centers(pr)
    for rmin in rmin_list:
        pr.rmin = rmin
        alloc(rmin)
        filt.precompute_filter(pr, centers)
        F.rho.from_numpy(rho)
        filt.apply_density_filter(F.rho, F.rho_filt, F.filt_neighbors, F.filt_weights,
                                  F.filt_n_nb, E)
        out[f"filt_rho_r{rmin}"] = F.rho_filt.to_numpy()
        F.dc.from_numpy(dcs)
        filt.apply_dc_filter_density_mode(E)
        out[f"filt_dc_r{rmin}"] = F.dc_filt.to_numpy()
        filt.apply_dc_filter_sensitivity_mode(E)
        out[f"filt_sens_r{rmin}"] = F.dc_filt.to_numpy()

    # OC update on the synthetic sensitivity, several volume targets
    for vf in (0.2, 0.4, 0.7):
        alloc(1.5)
        pr.volfrac = vf
        F.rho.from_numpy(rho)
        F.dc_filt.from_numpy(dcs)
        F.dv.fill(1.0)
        ch = oc.oc_update(pr)
        out[f"oc_rho_vf{vf}"] = F.rho.to_numpy()
        out[f"oc_change_vf{vf}"] = np.float64(ch)

    # One PCG solve from zero per preconditioner on the random density
    for pre in ("jacobi", "block_jacobi", "none"):
        alloc(1.5)
        F.rho.from_numpy(rho)
        if pre == "block_jacobi":
            PC.setup(F.edof, F.diag_count, E, dim)
        K.fill_scalar(F.u_prev, 0.0)
        n = solver.solve(E_min=Emin, penalty=pen, dim=dim, max_iter=500, tol=1e-10,
                         preconditioner=pre, warm_start=False)
        out[f"pcg_{pre}_u"] = F.u.to_numpy()
        out[f"pcg_{pre}_iters"] = np.int64(n)
        # a warm-started second solve at a perturbed density
        F.rho.from_numpy(np.clip(rho * 0.9 + 0.05, 0.001, 1.0))
        n2 = solver.solve(E_min=Emin, penalty=pen, dim=dim, max_iter=500, tol=1e-10,
                          preconditioner=pre, warm_start=True)
        out[f"pcg_{pre}_warm_u"] = F.u.to_numpy()
        out[f"pcg_{pre}_warm_iters"] = np.int64(n2)
    return out


def _run(args) -> dict:
    ref_src, yaml_path, overrides, snap_iters = args
    _import_reference(ref_src)
    from toptimization.problem import load_problem
    from toptimization.optimizer import simp, oc
    from toptimization.fem import solver

    pr = load_problem(yaml_path)
    for k, v in overrides.items():
        setattr(pr, k, v)
    pr.output_dir = Path(tempfile.mkdtemp())
    cg, change, snaps, comp, vol = [], [], {}, [], []
    orig_solve, orig_oc = solver.solve, oc.oc_update

    def solve(*a, **k):
        n = orig_solve(*a, **k)
        cg.append(n)
        return n

    def oc_update(problem):
        ch = orig_oc(problem)
        change.append(ch)
        return ch

    def cb(rho, it, c, v):
        comp.append(c)
        vol.append(v)
        if it in snap_iters:
            snaps[f"rho_it{it}"] = rho.copy()

    solver.solve, oc.oc_update = solve, oc_update
    with contextlib.redirect_stdout(io.StringIO()):
        rho = simp.run(pr, backend="cpu", live_viz=False, viz_callback=cb)
    return dict(compliance=np.array(comp), volume=np.array(vol), change=np.array(change),
                cg_iters=np.array(cg), rho_final=rho.reshape(-1), **snaps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TPO_REFERENCE_SRC"),
                    help="the src/ directory of a reference checkout")
    ap.add_argument("--only", default="")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set TPO_REFERENCE_SRC")
    ref_src = a.reference
    ref_examples = Path(ref_src).parent / "examples"
    ctx = mp.get_context("spawn")
    small = str(ref_examples / "cantilever_small.yaml")
    cant3d = str(HERE / "yaml" / "cantilever_3d_small.yaml")
    runs = {
        "ref_run_mbb_60x20": (str(REPO / "examples" / "mbb_60x20.yaml"), {}, (1, 10, 50)),
        "ref_run_mbb_60x20_tight": (str(REPO / "examples" / "mbb_60x20.yaml"),
                                    {"cg_tol": 1e-12, "max_cg_iter": 5000, "max_iter": 60},
                                    (1, 10, 30)),
        "ref_run_small_jacobi": (small, {"max_iter": 30, "tol": 0.0}, (1, 10)),
        "ref_run_small_block_jacobi": (small, {"max_iter": 30, "tol": 0.0,
                                               "preconditioner": "block_jacobi"}, (1, 10)),
        "ref_run_small_none": (small, {"max_iter": 30, "tol": 0.0,
                                       "preconditioner": "none"}, (1, 10)),
        "ref_run_small_sensitivity": (small, {"max_iter": 30, "tol": 0.0,
                                              "filter_type": "sensitivity"}, (1, 10)),
        "ref_run_small_earlystop": (small, {"max_iter": 200}, ()),
        "ref_run_bridge_100x50": (str(ref_examples / "bridge_2d.yaml"),
                                  {"max_iter": 12, "tol": 0.0}, (1,)),
        "ref_run_3d_jacobi": (cant3d, {}, (1, 10)),
        "ref_run_3d_block_jacobi": (cant3d, {"max_iter": 8,
                                             "preconditioner": "block_jacobi"}, (1,)),
        "ref_run_3d_sensitivity": (cant3d, {"max_iter": 8, "filter_type": "sensitivity",
                                            "preconditioner": "none"}, (1,)),
    }
    jobs = []
    with ctx.Pool(8) as pool:
        if not a.only or a.only == "boundary":
            jobs.append(("boundary", pool.apply_async(_boundary, (ref_src, ref_examples))))
        if not a.only or a.only == "ref_kernels":
            jobs.append(("ref_kernels", pool.apply_async(_kernels, (ref_src,))))
        if not a.only or a.only == "ref_kernels3d":
            jobs.append(("ref_kernels3d", pool.apply_async(_kernels3d, (ref_src,))))
        if not a.only or a.only == "ref_kernels3d_rollers":
            jobs.append(("ref_kernels3d_rollers",
                         pool.apply_async(_kernels3d_rollers, (ref_src,))))
        for name, (y, ov, snaps) in runs.items():
            if not a.only or a.only == name:
                jobs.append((name, pool.apply_async(_run, ((ref_src, y, ov, snaps),))))
        for name, job in jobs:
            res = job.get()
            np.savez_compressed(HERE / f"{name}.npz", **res)
            print("wrote", name, flush=True)


if __name__ == "__main__":
    main()
