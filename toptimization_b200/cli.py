"""Command line: `python -m toptimization_b200 run|validate <problem.yaml>`.

Same subcommands, options and exit codes as the reference's CLI
(`src/toptimization/cli.py:22-144`). `--backend` accepts the reference's
choices so existing scripts keep working, but only `auto`/`cuda` run (the
others exit 1 with a message: this package has no CPU, Metal or Vulkan path).
Windows are never opened (headless); `--no-viz/--no-live/--show` are accepted.
`--precision` and `--preconditioner` override the file.
"""

from __future__ import annotations

import argparse
import sys
from pathlib import Path


def _parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="toptimization_b200",
                                description="B200 topology optimization (SIMP method)")
    sub = p.add_subparsers(dest="command")
    r = sub.add_parser("run", help="Run topology optimization")
    r.add_argument("problem", help="Path to YAML problem definition file")
    r.add_argument("--backend", choices=["auto", "metal", "cpu", "cuda", "vulkan"],
                   default="auto")
    r.add_argument("--no-viz", action="store_true", help="Disable all visualization")
    r.add_argument("--no-live", action="store_true", help="Disable live window")
    r.add_argument("--output", metavar="DIR", help="Override output directory")
    r.add_argument("--show", action="store_true", help="(accepted; headless)")
    r.add_argument("--precision", choices=["fp64", "mixed"], default=None)
    r.add_argument("--preconditioner",
                   choices=["jacobi", "block_jacobi", "nodal_block_jacobi", "none"], default=None)
    r.add_argument("--quiet", action="store_true")
    v = sub.add_parser("validate", help="Validate a problem file without running")
    v.add_argument("problem", help="Path to YAML problem definition file")
    return p


def _cmd_validate(args) -> int:
    from .problem import load_problem
    path = Path(args.problem)
    if not path.exists():
        print(f"Error: file not found: {path}", file=sys.stderr)
        return 1
    try:
        pr = load_problem(path)
    except Exception as e:  # reference cli.py:98-100
        print(f"Validation failed: {e}", file=sys.stderr)
        return 1
    mesh = f"{pr.nelx} x {pr.nely}" + (f" x {pr.nelz}" if pr.dim == 3 else "")
    print(f"Problem '{pr.name}' is valid.")
    for label, value in [("Dimension", f"{pr.dim}D"), ("Mesh", mesh),
                         ("Elements", f"{pr.n_elem:,}"), ("DOFs", f"{pr.n_dofs:,}"),
                         ("Fixed DOFs", f"{len(pr.fixed_dofs):,}"),
                         ("Force DOFs", f"{len(pr.force_dofs):,}"),
                         ("Volume frac", pr.volfrac),
                         ("Filter", f"{pr.filter_type} (rmin={pr.rmin})"),
                         ("Max iter", pr.max_iter), ("Solver", f"{pr.preconditioner}, "
                                                               f"{pr.precision}")]:
        print(f"  {label:<12}: {value}")
    return 0


def _cmd_run(args) -> int:
    from .problem import load_problem
    path = Path(args.problem)
    if not path.exists():
        print(f"Error: file not found: {path}", file=sys.stderr)
        return 1
    try:
        pr = load_problem(path)
    except Exception as e:
        print(f"Error loading problem: {e}", file=sys.stderr)
        return 1
    if args.output:
        pr.output_dir = Path(args.output)
    try:
        from .optimizer.simp import run
        run(pr, backend=args.backend, live_viz=False, precision=args.precision,
            preconditioner=args.preconditioner, verbose=not args.quiet)
    except Exception as e:
        print(f"Error during optimization: {e}", file=sys.stderr)
        return 1
    print(f"\nResults saved to: {pr.output_dir}/")
    return 0


def main(argv=None) -> int:
    args = _parser().parse_args(argv)
    if args.command == "run":
        return _cmd_run(args)
    if args.command == "validate":
        return _cmd_validate(args)
    _parser().print_help()
    return 0


if __name__ == "__main__":
    sys.exit(main())
