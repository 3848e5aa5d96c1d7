"""Generate the 400x200 cantilever trajectories (tests/golden/oracle_cantilever_400x200_*.npz).

    python tests/golden/make_config1.py [--threads N] [--pre nodal_block_jacobi block_jacobi]

The cantilever of examples/cantilever_400x200.yaml (left edge clamped, unit
downward load at the mid-height node of the right edge, volfrac 0.4, rmin 3,
PCG to 1e-8, at most 10000 CG iterations) is run for 200 OC iterations, all in
FP64, by the C/OpenMP oracle (oracle/csrc/simp_cpu.c). One file per
preconditioner:
  nodal_block_jacobi  the 2x2 nodal block-Jacobi option (no reference
                      counterpart);
  block_jacobi        the reference's element-block preconditioner
                      (src/toptimization/fem/preconditioner.py:47-108); its
                      solves stop at the 10000-iteration cap from the first
                      OC iterations on.
Each file holds the compliance, volume, change and CG-count histories and the
final density. The oracle is pinned to the reference's own runs by
tests/test_oracle.py; this case is too large for the FP64 Taichi stand-in.
Needs no reference checkout; takes tens of minutes on 4 cores.
"""

from __future__ import annotations

import argparse
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def run(pre: str, iters: int = 200) -> dict:
    from oracle import simp_cpu
    from toptimization_b200.problem import load_problem

    pr = load_problem(REPO / "examples" / "cantilever_400x200.yaml")
    pr.preconditioner = pre
    cpu = simp_cpu.CpuSimp(pr)
    hist = {k: [] for k in ("compliance", "volume", "change", "cg_iters", "status")}
    t0 = time.time()
    for it in range(iters):
        r = cpu.iteration()
        for k in hist:
            hist[k].append(r[k])
        if (it + 1) % 10 == 0:
            print(f"  {pre} it {it + 1}: c={r['compliance']:.12g} cg={r['cg_iters']} "
                  f"({time.time() - t0:.0f} s)", flush=True)
    out = {k: np.array(v) for k, v in hist.items()}
    out["rho_final"] = cpu.rho()
    out["threads"] = np.array(simp_cpu.threads())
    cpu.close()
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--pre", nargs="+", default=["nodal_block_jacobi", "block_jacobi"])
    ap.add_argument("--iters", type=int, default=200)
    a = ap.parse_args()
    if a.threads:
        os.environ["OMP_NUM_THREADS"] = str(a.threads)
    sys.path.insert(0, str(REPO))
    for pre in a.pre:
        out = run(pre, a.iters)
        path = HERE / f"oracle_cantilever_400x200_{pre}.npz"
        np.savez_compressed(path, **out)
        print(f"wrote {path} ({path.stat().st_size} bytes)", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
