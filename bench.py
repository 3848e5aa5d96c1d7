#!/usr/bin/env python
"""Benchmark: OC iterations per second of the SIMP loop on the 2048x1024 bridge.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the bridge problem, examples/bridge_2048x1024.yaml): 2048x1024 Q4
grid (2,097,152 elements, 4,200,450 DOFs), corners pinned, -1/2049 on every
top node, volfrac 0.3, rmin 4, 2x2 nodal block-Jacobi PCG to 1e-8 warm-started
from the previous displacement. A step is one OC iteration (density filter,
PCG solve, sensitivity, dc filter, OC bisection). W untimed steps on one
design, then K timed steps -- OC iterations 1..K -- of a fresh design from the
initial density, each bracketed by CUDA events on the launching stream, with a
256 MiB write between steps to flush L2. The headline `value` is the mixed
form (FP32-stored inner PCG inside FP64 refinement) through the CUDA-graph
engine (simp.run(engine="graph"): each OC iteration one graph, the PCG loop
a device-side while node); the plain FP64 form is timed on the same OC
iterations and engine beside it, the host-polled engine ("direct") on the
same iterations too, and `e2e` runs the same OC iterations through
simp.run(engine="graph") with host buffers. Per-kernel device times come
from the host-polled path (the library brackets every PCG launch with
events), one OC iteration per form. The line also carries a
whole, measured (not extrapolated) comparison on the 400x200 cantilever:
GPU forms against the CPU port on the host cores.

--impl reference times the CPU port of the reference algorithm
(oracle/csrc/simp_cpu.c, OpenMP on all host cores) on one whole OC iteration
of the same workload (the first, uncapped PCG); the reference's own CPU path
is Taichi, which is not available in this image.

Multi-GPU (torchrun): every rank solves its own bridge replica (the loop does
not shard); value = all ranks' OC iterations / the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

WORKLOAD_YAML = REPO / "examples" / "bridge_2048x1024.yaml"
METRIC = "OC iter/s @2048x1024 mixed vs FP64 at 1e-6 compliance; designs/s, p99 latency"
UNIT = "OC iter/s"
PRECONDITIONER = "nodal_block_jacobi"
# The GPU arm's CPU baseline times the C/OpenMP port on a bounded sample (one
# OC iteration with the PCG capped at CPU_SAMPLE_CG iterations) and scales the
# PCG time to the CG count that the GPU's own FP64 solve measured over the
# same OC iterations in the same run (the port runs the same algorithm).
CPU_SAMPLE_CG = 48
CONFIG1_YAML = REPO / "examples" / "cantilever_400x200.yaml"
CONFIG1_STEPS = 4
L2_FLUSH_BYTES = 256 << 20


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-direct", action="store_true")
    ap.add_argument("--case", choices=["pcg", "matvec"], default=None,
                    help="profiling case: one PCG solve on the bridge capped at --cg-iters, "
                         "or 5 stiffness applications (FP64) on the bridge")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--cg-iters", type=int, default=30)
    ap.add_argument("--recurrence", choices=["auto", "standard", "single"], default="auto",
                    help="PCG iteration form: one launch per iteration (auto) or the "
                         "reference's two-step recurrence (standard)")
    ap.add_argument("--workload", choices=["bridge", "batch", "serve", "solid3d"],
                    default="bridge",
                    help="bridge: the 2048x1024 headline line; batch: uneven designs "
                         "advanced together; serve: a Poisson request stream; solid3d: "
                         "the 3D H8 cantilever (examples/cantilever3d_128x64x64.yaml)")
    ap.add_argument("--designs", type=int, default=64, help="batch: number of designs")
    ap.add_argument("--oc-iters", type=int, default=50, help="batch/serve: OC iterations")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--serial-sample", type=int, default=8,
                    help="batch/serve: designs timed one at a time for the baseline")
    ap.add_argument("--requests", type=int, default=48, help="serve: requests per rate")
    ap.add_argument("--rates", default="5,50,200", help="serve: arrival rates (req/s)")
    ap.add_argument("--nelx-max", type=int, default=1024, help="serve: largest nelx")
    ap.add_argument("--size-steps", action="store_true",
                    help="serve: size-aware step periods (large designs take every p-th PCG step)")
    return ap.parse_args()


_RECURRENCE = "auto"


def load_workload():
    from toptimization_b200.problem import load_problem
    pr = load_problem(WORKLOAD_YAML)
    pr.recurrence = _RECURRENCE
    return pr


def workload_config(pr, **extra):
    cfg = {"workload": f"bridge {pr.nelx}x{pr.nely} Q4 (examples/bridge_2048x1024.yaml)",
           "n_elem": pr.n_elem, "n_dofs": pr.n_dofs, "preconditioner": PRECONDITIONER,
           "cg_tol": pr.cg_tol, "inner_tol": pr.inner_tol, "volfrac": pr.volfrac,
           "rmin": pr.rmin, "recurrence": pr.recurrence,
           "step": "one OC iteration (filter, PCG, sensitivity, dc filter, OC)",
           "l2": "flushed between timed steps (256 MiB write)"}
    cfg.update(extra)
    return cfg


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling during the timed region (200 ms period)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        power = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "power_w_max": max(power) if power else None}


# ------------------------------------------------------------------ helpers
def measured_peak():
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
        return float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, bf16 copy)"
    except Exception:
        return 6650.0, "fallback (6.65 TB/s)"


def ncu_traffic(kernel_key: str):
    """dram bytes per launch of a kernel from the committed ncu summary."""
    try:
        data = json.loads((REPO / "profiles" / "traffic.json").read_text())
        return data.get(kernel_key)
    except Exception:
        return None


def time_steps(design, steps, warmup, flush_buf, torch):
    for _ in range(warmup):
        design.step()
    torch.cuda.synchronize()
    times, recs = [], []
    for _ in range(steps):
        flush_buf.fill_(1.0)                      # L2 flush, outside the timed interval
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        rec = design.step()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b))
        recs.append(rec)
    return times, recs


def profile_pass(design, lib, _lib, torch, steps=1):
    """Per-kernel device times of the PCG kernels over `steps` more OC
    iterations (CUDA events around every launch, recorded by the library)."""
    lib.tpo_profile_enable(1)
    lib.tpo_profile_reset()
    for _ in range(steps):
        design.step()
    torch.cuda.synchronize()
    prof = _lib.profile_read()
    lib.tpo_profile_enable(0)
    out = {}
    for k in ("dir", "update", "step"):
        if prof[f"{k}_launches"] == 0:
            continue
        n = max(prof[f"{k}_launches"], 1)
        us = prof[f"{k}_ms"] / n * 1e3
        bpl = prof[f"{k}_bytes"] / n
        out[k] = {"launches": prof[f"{k}_launches"], "avg_us": round(us, 2),
                  "bytes_per_launch": int(bpl),
                  "gbs": round(bpl / (us * 1e-6) / 1e9, 1) if us > 0 else None,
                  "total_ms": round(prof[f"{k}_ms"], 3)}
    return out


def time_matvec(pr, dtype, torch, reps=20):
    """The stiffness kernel alone (precomputed scales); the library brackets
    the kernel launch with CUDA events. Its inputs are packed into the padded
    layout just before the launch, so they start partly L2-resident."""
    import numpy as np
    from toptimization_b200 import _lib
    from toptimization_b200.fem import kernels as K
    from toptimization_b200.mesh import fixed_node_mask
    lib = _lib.load()
    g = _lib.grid(pr.nelx, pr.nely, pr.E_min, pr.penalty)
    dev = torch.device("cuda", torch.cuda.current_device())
    gen = torch.Generator(device=dev).manual_seed(1)
    scale = (torch.rand(pr.n_elem, device=dev, generator=gen, dtype=torch.float64) ** 3
             ).to(dtype)
    p = torch.randn(pr.n_dofs, device=dev, generator=gen, dtype=torch.float64).to(dtype)
    ap = torch.empty_like(p)
    fixed = torch.from_numpy(fixed_node_mask(pr)).to(dev)
    ws = K.matvec_workspace(g, dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(3):
        K.apply_stiffness(g, scale, fixed, p, ap, ws)
    lib.tpo_profile_enable(1)
    lib.tpo_profile_reset()
    for _ in range(reps):
        flush.fill_(2.0)
        K.apply_stiffness(g, scale, fixed, p, ap, ws)
    torch.cuda.synchronize()
    prof = _lib.profile_read()
    lib.tpo_profile_enable(0)
    us = prof["apply_ms"] / max(prof["apply_launches"], 1) * 1e3
    nbytes = prof["apply_bytes"] // max(prof["apply_launches"], 1)   # p, Ap, scales, mask
    return {"us": round(us, 2), "gbs": round(nbytes / (us * 1e-6) / 1e9, 1),
            "bytes_per_launch": int(nbytes), "launches": int(prof["apply_launches"]),
            "arith": "fp64" if dtype == torch.float64 else "fp32"}


def cpu_sample(pr, cg_per_oc, steps=1, warm_steps=0):
    """C/OpenMP port of the reference on the host cores: each sample is one
    OC iteration with the PCG capped at CPU_SAMPLE_CG iterations; the PCG time
    is scaled to `cg_per_oc` iterations."""
    from oracle import simp_cpu
    cpu = simp_cpu.CpuSimp(pr, preconditioner=PRECONDITIONER)
    for _ in range(warm_steps):
        cpu.iteration(max_cg=CPU_SAMPLE_CG)
    est = []
    for _ in range(steps):
        r = cpu.iteration(max_cg=CPU_SAMPLE_CG)
        per_cg = r["pcg_seconds"] / max(r["cg_iters"], 1)
        est.append(r["other_seconds"] + per_cg * cg_per_oc)
    cpu.close()
    t = sum(est) / len(est)
    return {"value": round(1.0 / t, 5), "unit": UNIT, "cores": simp_cpu.threads(),
            "kind": "port", "extrapolated": True,
            "sample": (f"C/OpenMP port of the reference loop (oracle/csrc/simp_cpu.c, FP64, "
                       f"{PRECONDITIONER}) on the full 2048x1024 bridge: {steps} OC "
                       f"iteration(s) with the PCG capped at {CPU_SAMPLE_CG} iterations, "
                       f"PCG time scaled to {cg_per_oc} iterations per OC iteration (the "
                       "mean CG count of this run's GPU FP64 solves over the timed OC "
                       "iterations)"),
            "seconds_per_oc_iter": round(t, 3)}


def config1_measured(dev, torch, flush, steps=CONFIG1_STEPS):
    """OC iterations 1..steps of the 400x200 cantilever (examples/
    cantilever_400x200.yaml, nodal block-Jacobi PCG to 1e-8, uncapped), whole
    and measured on both sides: the GPU forms through SimpDesign (CUDA
    events, warm-up on another design), the C/OpenMP port of the reference
    loop on all host cores (wall clock). Nothing is extrapolated."""
    from oracle import simp_cpu
    from toptimization_b200.optimizer.simp import SimpDesign
    from toptimization_b200.problem import load_problem
    pr = load_problem(CONFIG1_YAML)
    out = {"workload": "cantilever 400x200 Q4 (examples/cantilever_400x200.yaml)",
           "preconditioner": PRECONDITIONER, "oc_iterations": f"1..{steps}", "unit": UNIT}
    for prec in ("fp64", "mixed"):
        w = SimpDesign(pr, device=dev, precision=prec, preconditioner=PRECONDITIONER)
        w.step()
        del w
        d = SimpDesign(pr, device=dev, precision=prec, preconditioner=PRECONDITIONER)
        times, recs = time_steps(d, steps, 0, flush, torch)
        out[f"gpu_{prec}"] = round(steps / (sum(times) / 1e3), 3)
        out[f"gpu_{prec}_cg_iters"] = [r.cg_iters for r in recs]
        del d
    cpu = simp_cpu.CpuSimp(pr, preconditioner=PRECONDITIONER)
    cg = []
    t0 = time.perf_counter()
    for _ in range(steps):
        cg.append(cpu.iteration()["cg_iters"])
    t = time.perf_counter() - t0
    cpu.close()
    out.update({"cpu_port": round(steps / t, 4), "cpu_port_cg_iters": cg,
                "cores": simp_cpu.threads(), "kind": "port", "extrapolated": False})
    out["gpu_fp64_over_cpu"] = round(out["gpu_fp64"] / out["cpu_port"], 1)
    out["gpu_mixed_over_cpu"] = round(out["gpu_mixed"] / out["cpu_port"], 1)
    return out


# ------------------------------------------------------------------ reference arm
def run_reference(args):
    """The C/OpenMP port of the reference loop on all host cores: one whole
    OC iteration of the bridge, the first from the initial density, with the
    PCG uncapped, measured by the wall clock (about two minutes on 16 host
    threads). Nothing is extrapolated. The GPU arm's `value` covers OC
    iterations 1..K, whose later solves need more CG iterations than the
    first, so the ratio of the two understates the GPU's speed-up."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import simp_cpu
    pr = load_workload()
    t0 = time.perf_counter()
    cpu = simp_cpu.CpuSimp(pr, preconditioner=PRECONDITIONER)
    t1 = time.perf_counter()
    r = cpu.iteration()
    t = time.perf_counter() - t1
    cores = simp_cpu.threads()
    cpu.close()
    wall = time.perf_counter() - t0
    value = round(1.0 / t, 5)
    sample = (f"C/OpenMP port of the reference loop (oracle/csrc/simp_cpu.c, FP64, "
              f"{PRECONDITIONER}) on the full 2048x1024 bridge: OC iteration 1 from the "
              f"initial density, uncapped PCG ({r['cg_iters']} CG iterations to 1e-8), "
              "measured whole")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": 1, "steps_requested": args.steps,
            "warmup": 0, "ms_per_step": round(1e3 * t, 2), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(pr, precision="fp64 (CPU port)",
                                      cg_iters=int(r["cg_iters"]), oc_iterations_timed="1"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "extrapolated": False, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": round(wall, 1)}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm
def run_ours(args):
    import numpy as np
    import torch

    from toptimization_b200 import replicas
    rk = replicas.from_env()
    world, rank, local = rk.world, rk.rank, rk.local
    torch.cuda.set_device(local)
    replicas.init(rk, "nccl", 300, torch.device("cuda", local))

    from toptimization_b200 import _lib
    from toptimization_b200.csrc import build as csrc_build
    from toptimization_b200.optimizer.simp import CapturedDesign, SimpDesign, run
    if rank == 0:
        csrc_build.build()
    replicas.barrier(rk)  # the library is built once, by rank 0
    lib = _lib.load()
    dev = torch.device("cuda", local)
    pr = load_workload()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def barrier():
        replicas.barrier(rk)

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, rk, dev)

    def warm_then_fresh(precision, cls=SimpDesign):
        """W untimed OC iterations on a throwaway design (kernel load, launch
        plans, allocator), then a fresh design from the initial density: the
        timed steps are OC iterations 1..K, the window the e2e run covers."""
        if args.warmup:
            w = cls(pr, device=dev, precision=precision, preconditioner=PRECONDITIONER)
            for _ in range(args.warmup):
                w.step()
            torch.cuda.synchronize()
            del w
        return cls(pr, device=dev, precision=precision, preconditioner=PRECONDITIONER)

    # ---- mixed (headline), timed, through the CUDA-graph engine (each OC
    # iteration one graph, the PCG loop on the device: simp.run(engine="graph"))
    mixed = warm_then_fresh("mixed", CapturedDesign)
    barrier()
    with ClockSampler(local) as clocks:
        times_m, recs_m = time_steps(mixed, args.steps, 0, flush, torch)
    barrier()
    launches = sum(r.launches for r in recs_m)
    t_mixed = max_over_ranks(sum(times_m))
    clock_info = clocks.summary()
    rho_mixed = mixed.density()
    del mixed

    # ---- per-kernel device times (events around every PCG launch, recorded by
    # the library) on the host-polled path, same kernels: one OC iteration
    def kernel_pass(precision):
        d = SimpDesign(pr, device=dev, precision=precision, preconditioner=PRECONDITIONER)
        out = profile_pass(d, lib, _lib, torch)
        del d
        return out
    kern_mixed = kernel_pass("mixed")

    # ---- the host-polled path (simp.run(engine="direct")), same OC iterations
    direct = None
    if not args.no_direct:
        dd = warm_then_fresh("mixed")
        barrier()
        times_x, recs_x = time_steps(dd, args.steps, 0, flush, torch)
        barrier()
        t_x = max_over_ranks(sum(times_x))
        direct = {"value": round(world * args.steps / (t_x / 1e3), 4),
                  "ms_per_step": round(t_x / args.steps, 3),
                  "engine": "simp.run(engine='direct'): host polls the PCG status",
                  "same_results_as_graph": [r.compliance for r in recs_x] ==
                                           [r.compliance for r in recs_m]}
        del dd

    # ---- plain FP64, same OC iterations, same engine
    fp64 = None
    if not args.no_fp64:
        d64 = warm_then_fresh("fp64", CapturedDesign)
        barrier()
        times_d, recs_d = time_steps(d64, args.steps, 0, flush, torch)
        barrier()
        t_d = max_over_ranks(sum(times_d))
        rho_fp64 = d64.density()
        del d64
        kern_fp64 = kernel_pass("fp64")
        cd = np.array([r.compliance for r in recs_d])
        fp64 = {"value": round(world * args.steps / (t_d / 1e3), 4),
                "ms_per_step": round(t_d / args.steps, 3),
                "cg_iters_mean": float(np.mean([r.cg_iters for r in recs_d])),
                "cg_iters": [r.cg_iters for r in recs_d],
                "compliance": [float(x) for x in cd], "kernels": kern_fp64,
                "density_max_abs_mixed_vs_fp64": float(np.abs(rho_mixed - rho_fp64).max())}

    # ---- matvec roofline (FP64 and FP32 operator alone)
    mv64 = time_matvec(pr, torch.float64, torch)
    mv32 = time_matvec(pr, torch.float32, torch)

    # ---- e2e through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        pr_e = load_workload()
        pr_e.max_iter = args.steps  # OC iterations 1..K: the window of `value`
        pr_e.preconditioner = PRECONDITIONER
        got = []
        barrier()
        t0 = time.perf_counter()
        run(pr_e, backend="cuda", live_viz=False, precision="mixed", verbose=False, save=False,
            viz_callback=lambda rho, it, c, v: got.append(rho.nbytes), engine="graph")
        torch.cuda.synchronize()
        t_e = max_over_ranks(time.perf_counter() - t0)
        n_it = pr_e.max_iter
        h2d = 8 * pr.n_dofs + pr.n_nodes + 2 * 64 * 8       # f, fixed mask, Ke, Ke_inv
        e2e = {"value": round(world * n_it / t_e, 4), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d / n_it),
               "d2h_bytes_per_step": int(np.mean(got)) + 5 * 8,
               "note": (f"simp.run(engine='graph') from a host Problem to the host density: OC iterations "
                        f"1..{n_it} from the initial design, the same iterations as `value`, "
                        "plus setup, H2D of loads and BCs, per-iteration D2H of the density "
                        "to a viz_callback and of 5 scalars")}

    if rank != 0:
        replicas.finish(rk)
        return 0

    value = world * args.steps / (t_mixed / 1e3)
    peak, peak_kind = measured_peak()
    # dominant PCG kernel of the timed (mixed) step, by device time in the timing pass
    km = kern_mixed
    key = max(km, key=lambda k: km[k]["total_ms"])
    names = {"dir": "k_tstencil<float,double,DIR> (p = z + beta p, K p, p.Kp; TMA-staged)",
             "update": "k_update_flat<float,double,nodal,double> (u, r update, z = M r, r.z)",
             "step": "k_cgstep<float,double,nodal> (whole PCG iteration in one launch, "
                     "TMA-staged)"}
    kd = km[key]
    achieved = kd["gbs"]
    roofline = {"bound": "hbm", "kernel": names[key], "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 3) if achieved else None,
                "traffic": ncu_traffic("mixed_" + key), "bytes_per_launch": kd["bytes_per_launch"],
                "avg_launch_us": kd["avg_us"], "launches_timed": kd["launches"],
                "peak_kind": peak_kind, "kernels_mixed": km}
    mv = {"f64": dict(mv64, frac=round(mv64["gbs"] / peak, 3)),
          "f32": dict(mv32, frac=round(mv32["gbs"] / peak, 3))}

    line = {"metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(t_mixed / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (the bridge problem of examples/bridge_2048x1024.yaml)",
            "config": workload_config(pr, precision="mixed (FP32 inner PCG, FP64 refinement)",
                                      oc_iterations_timed=(
                                          f"1..{args.steps} of a fresh design (warm-up: "
                                          f"{args.warmup} OC iterations of another one)"),
                                      parallelism="replicas" if world > 1 else "single GPU"),
            "mixed": {"cg_iters": [r.cg_iters for r in recs_m],
                      "outer_iters": [r.solve.outer_iters for r in recs_m],
                      "compliance": [r.compliance for r in recs_m]},
            "gpu_launches": int(launches), "roofline": roofline, "matvec": mv,
            "clocks": clock_info}
    if fp64 is not None:
        line["plain_fp64"] = fp64
        line["mixed_over_fp64"] = round(value / fp64["value"], 3)
        rel = [abs(a - b) / abs(b) for a, b in zip(line["mixed"]["compliance"], fp64["compliance"])]
        line["compliance_rel_err_mixed_vs_fp64"] = max(rel)
        line["density_max_abs_mixed_vs_fp64"] = fp64["density_max_abs_mixed_vs_fp64"]
    if direct is not None:
        line["mixed_direct_engine"] = direct
    if e2e is not None:
        line["e2e"] = e2e
    if world == 1 and not args.no_cpu:
        if fp64 is not None:
            line["cpu_baseline"] = cpu_sample(pr, int(round(fp64["cg_iters_mean"])))
        line["cantilever_400x200_measured"] = config1_measured(dev, torch, flush)
    print(json.dumps(line), flush=True)
    replicas.finish(rk)
    return 0


def run_case(args):
    """A fixed amount of PCG work on the full bridge (uniform density 0.3), for
    ncu captures: the residual kernel, then --cg-iters iterations."""
    import numpy as np
    import torch
    from toptimization_b200.csrc import build as csrc_build
    from toptimization_b200.fem.solver import PCGSolver
    from toptimization_b200.material import compute_Ke_2d, regularized_inverse
    from toptimization_b200.mesh import fixed_node_mask, force_vector
    from toptimization_b200 import _lib
    csrc_build.build()
    pr = load_workload()
    Ke = compute_Ke_2d(pr.E, pr.nu)
    inv, alpha = regularized_inverse(Ke)
    _lib.ensure_stiffness(Ke, inv, alpha)
    f_np = force_vector(pr)
    dev = torch.device("cuda", 0)
    f = torch.from_numpy(f_np).to(dev)
    fixed = torch.from_numpy(fixed_node_mask(pr)).to(dev)
    rho = torch.full((pr.n_elem,), 0.3, dtype=torch.float64, device=dev)
    u = torch.zeros(pr.n_dofs, dtype=torch.float64, device=dev)
    s = PCGSolver(pr.nelx, pr.nely, pr.E_min, pr.penalty, float(np.dot(f_np, f_np)),
                  preconditioner=PRECONDITIONER, precision=args.precision,
                  recurrence=args.recurrence,
                  max_iter=args.cg_iters, tol=1e-12, device=dev)
    info = s.solve(rho, f, fixed, u, warm_start=False)
    torch.cuda.synchronize()
    print(json.dumps({"case": "pcg", "precision": args.precision, "status": info.status,
                      "updates": info.updates}))
    return 0


def run_batch(args):
    """Uneven designs (nelx in [64, 512], aspect 1-3, MBB/cantilever/bridge,
    seeded) advanced together, mixed precision, strip lengths from the
    autotuner, each OC iteration one CUDA graph launch; designs/s against the
    same designs solved one at a time (a timed sample, scaled to the batch)."""
    import numpy as np
    import torch
    from toptimization_b200.batch import Batch, autotune, random_designs
    from toptimization_b200.csrc import build as csrc_build
    from toptimization_b200.optimizer.simp import SimpDesign
    from toptimization_b200 import replicas
    rk = replicas.from_env()
    torch.cuda.set_device(rk.local)
    replicas.init(rk, "nccl", 600, torch.device("cuda", rk.local))
    if rk.rank == 0:
        csrc_build.build()
    replicas.barrier(rk)
    # every rank draws the same designs and runs its round-robin share
    ps = replicas.shard(random_designs(args.designs, seed=args.seed, nelx_range=(64, 512),
                                       max_iter=args.oc_iters), rk)
    t = time.perf_counter()
    tune = autotune(ps, steps=64)
    t_tune = time.perf_counter() - t
    out = {"metric": "designs/s (batched uneven designs, mixed, 1 GPU)",
           "unit": "designs/s", "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{len(ps)} designs, nelx U[64,512], aspect U{{1,2,3}}, "
                                  f"MBB/cantilever/bridge, {args.oc_iters} OC iterations, "
                                  f"seed {args.seed}",
                      "elements_total": int(sum(p.n_elem for p in ps)),
                      "tiles": list(tune["best"]), "autotune_s": round(t_tune, 2),
                      "autotune_ms": {f"{a}x{b}": round(v, 3)
                                      for (a, b), v in tune["ms"].items()}}}
    for mode in ("graph_oc_iterations", "rounds"):
        b = Batch(len(ps), use_graph=True, tiles=tune["best"])
        slots = [b.add(p) for p in ps]
        replicas.barrier(rk)
        t = time.perf_counter()
        b.run(rounds=(mode == "rounds"))
        replicas.barrier(rk)
        dt = replicas.max_over_ranks(time.perf_counter() - t, rk,
                                     torch.device("cuda", rk.local))
        cg = [float(b.history(s)["cg_iters"].sum()) for s in slots]
        out[mode] = {"seconds": round(dt, 3),
                     "designs_per_s": round(replicas.job_rate(len(ps), dt, rk), 4),
                     "oc_iters_per_s": round(replicas.job_rate(len(ps) * args.oc_iters, dt, rk),
                                             2),
                     "cg_iters_total_rank0": int(sum(cg))}
        b.close()
    out["n_gpus"] = rk.world
    out["scaling"] = "weak" if rk.multi else None
    k = min(args.serial_sample, len(ps))
    t = time.perf_counter()
    for p in ps[:k]:
        d = SimpDesign(p, precision="mixed", preconditioner=p.preconditioner)
        for _ in range(p.max_iter):
            d.step()
    torch.cuda.synchronize()
    per = (time.perf_counter() - t) / k
    frac = sum(p.n_elem for p in ps[:k]) / sum(p.n_elem for p in ps)
    serial_est = (time.perf_counter() - t) / frac
    out["one_at_a_time_mixed"] = {"sample_designs": k, "seconds_per_design": round(per, 3),
                                  "estimated_seconds_all": round(serial_est, 2),
                                  "scaling": "sample time scaled by the element count"}
    best = max(out["graph_oc_iterations"]["designs_per_s"], out["rounds"]["designs_per_s"])
    out["value"] = best
    out["speedup_vs_one_at_a_time"] = round(best / rk.world * serial_est / len(ps), 2)
    if rk.rank == 0:
        print(json.dumps(out), flush=True)
    replicas.finish(rk)
    return 0


def run_serve(args):
    """Poisson request streams (seeded) served with continuous batching under a
    150 GB HBM budget; p50/p95/p99 latency and designs/s per arrival rate,
    beside one-at-a-time plain FP64 solves of the same requests."""
    import torch
    from toptimization_b200.csrc import build as csrc_build
    from toptimization_b200.serve import Server, poisson_stream, serve_one_at_a_time
    import torch.distributed as dist
    from toptimization_b200 import replicas
    from toptimization_b200.serve import ServeReport
    rk = replicas.from_env()
    torch.cuda.set_device(rk.local)
    replicas.init(rk, "nccl", 1800, torch.device("cuda", rk.local))
    if rk.rank == 0:
        csrc_build.build()
    replicas.barrier(rk)
    rates = [float(r) for r in args.rates.split(",")]

    def served(reqs, server):
        """Each rank serves its round-robin share; completions of all ranks are
        gathered so the latency percentiles cover the whole stream."""
        rep = server(replicas.shard(reqs, rk))
        if rk.multi:
            parts = [None] * rk.world
            dist.all_gather_object(parts, [(c.rid, c.arrival, c.admitted, c.done, c.oc_iters,
                                            c.compliance) for c in rep.completions])
            from toptimization_b200.serve import Completion
            allc = [Completion(*t) for part in parts for t in part]
            rep = ServeReport(sorted(allc, key=lambda c: c.rid), rep.rounds, rep.peak_resident,
                              rep.peak_bytes, rep.wall)
        return rep

    def batched(reqs):
        srv = Server(hbm_budget=150e9, max_slots=256, size_steps=args.size_steps)
        try:
            return srv.serve(reqs)
        finally:
            srv.close()

    out = {"metric": "designs/s and latency (served stream, mixed, 1 GPU)",
           "unit": "designs/s", "higher_is_better": True, "n_gpus": 1, "data": "synthetic",
           "config": {"workload": f"{args.requests} requests per rate, nelx U[64,{args.nelx_max}], "
                                  f"aspect U{{1,2,3}}, MBB/cantilever/bridge, "
                                  f"{args.oc_iters} OC iterations, seed {args.seed}",
                      "hbm_budget_gb": 150, "rates": rates,
                      "size_steps": args.size_steps}, "per_rate": {}}
    for rate in rates:
        reqs = poisson_stream(args.requests, rate, seed=args.seed,
                              nelx_range=(64, args.nelx_max), max_iter=args.oc_iters)
        out["per_rate"][str(rate)] = served(reqs, batched).summary()
    reqs = poisson_stream(args.requests, rates[-1], seed=args.seed,
                          nelx_range=(64, args.nelx_max), max_iter=args.oc_iters)
    k = min(args.serial_sample, len(reqs))
    out["value"] = max(v["designs_per_s"] for v in out["per_rate"].values())
    if k > 0:
        ss = served(reqs[:k], lambda r: serve_one_at_a_time(r, precision="fp64")).summary()
        out["one_at_a_time_fp64"] = dict(ss, note=f"first {k} requests of the {rates[-1]}/s stream")
        # the batched server on exactly those requests, for a like-for-like ratio
        bs = served(reqs[:k], batched).summary()
        out["batched_same_sample"] = bs
        out["designs_per_s_ratio_same_sample"] = round(bs["designs_per_s"] / ss["designs_per_s"], 2)
    out["n_gpus"] = rk.world
    if rk.rank == 0:
        print(json.dumps(out), flush=True)
    replicas.finish(rk)
    return 0


SOLID3D_YAML = REPO / "examples" / "cantilever3d_128x64x64.yaml"
SOLID3D_UNIT = "OC iter/s"
SOLID3D_CPU_CG = 600
# FP64 flops of the structured H8 element operator (hex3d.cuh h8_forces):
# transforms 69 + 69, stresses and modal forces 41 operations, 12 of them FMAs
H8_FLOPS_PER_ELEMENT = 191
# FP64 FMA issue of the B200: 148 SMs x 64 FP64 FMA/clk x 2 flops x 1.965 GHz
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def cpu_sample_3d(pr, cg_per_oc):
    """C/OpenMP port of the reference loop (oracle/csrc/simp_cpu.c, FP64,
    Jacobi, 8-colour H8 element scatter) on the full 3D grid: one OC iteration
    with the PCG capped at SOLID3D_CPU_CG iterations, PCG time scaled to
    `cg_per_oc` iterations."""
    from oracle import simp_cpu
    cpu = simp_cpu.CpuSimp(pr, preconditioner="jacobi")
    r = cpu.iteration(max_cg=SOLID3D_CPU_CG)
    cpu.close()
    per_cg = r["pcg_seconds"] / max(r["cg_iters"], 1)
    t = r["other_seconds"] + per_cg * cg_per_oc
    return {"value": round(1.0 / t, 6), "unit": SOLID3D_UNIT, "cores": simp_cpu.threads(),
            "kind": "port",
            "sample": (f"C/OpenMP port of the reference loop (oracle/csrc/simp_cpu.c, FP64, "
                       f"jacobi, H8 element scatter in 8 colours) on the full "
                       f"{pr.nelx}x{pr.nely}x{pr.nelz} grid: one OC iteration with the PCG "
                       f"capped at {SOLID3D_CPU_CG} iterations, PCG time scaled to "
                       f"{cg_per_oc} iterations per OC iteration"),
            "seconds_per_oc_iter": round(t, 3)}


def run_solid3d(args):
    """OC iterations/s of the 3D (H8) loop: FP64 Jacobi PCG, density filter."""
    import numpy as np
    import torch
    from toptimization_b200 import _lib
    from toptimization_b200.csrc import build as csrc_build
    from toptimization_b200.optimizer.simp import SimpDesign, run
    from toptimization_b200.problem import load_problem
    csrc_build.build()
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    pr = load_problem(SOLID3D_YAML)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    d = SimpDesign(pr, device=dev, precision="fp64", preconditioner="jacobi")
    for _ in range(args.warmup):
        d.step()
    lib.tpo_profile_reset()
    with ClockSampler(0) as clocks:
        times, recs = time_steps(d, args.steps, 0, flush, torch)
    launches = _lib.profile_read()["launches"]
    kern = profile_pass(d, lib, _lib, torch)
    del d
    t = sum(times)
    value = args.steps / (t / 1e3)
    cg_mean = float(np.mean([r.cg_iters for r in recs]))
    peak, peak_kind = measured_peak()
    nn = pr.n_nodes
    names = {"dir": "k_hex_elem<DIR> (element-centric plane march: p = z + beta p from "
                    "cp.async-staged planes, structured H8 element forces, corners handed "
                    "over in shared memory, p.Kp)",
             "update": "k_hex_update<jacobi> (u, r update, z = r / diag, r.z, ||r||^2)"}
    key = max(kern, key=lambda k: kern[k]["total_ms"])
    kd = kern[key]
    # structured H8 operator: 191 FP64 flops per element (an FMA counts 2)
    flops = H8_FLOPS_PER_ELEMENT * pr.n_elem if key == "dir" else 8 * pr.n_dofs
    tflops = flops / (kd["avg_us"] * 1e-6) / 1e12
    roofline = {"bound": "hbm", "kernel": names[key], "achieved": kd["gbs"], "peak": peak,
                "unit": "GB/s", "frac": round(kd["gbs"] / peak, 3) if kd["gbs"] else None,
                "traffic": ncu_traffic("solid3d_" + key),
                "bytes_per_launch": kd["bytes_per_launch"], "avg_launch_us": kd["avg_us"],
                "launches_timed": kd["launches"], "peak_kind": peak_kind,
                "fp64": {"achieved_tflops": round(tflops, 2),
                         "nominal_tflops": round(FP64_NOMINAL_TFLOPS, 1),
                         "frac": round(tflops / FP64_NOMINAL_TFLOPS, 3),
                         "flops_per_launch": flops,
                         "note": "algorithmic flops of the structured operator; the kernel "
                                 "is bound by instruction issue at 16 warps per SM, neither "
                                 "by HBM nor by the FP64 pipe"},
                "kernels": kern}
    e2e = None
    if not args.no_e2e:
        pr_e = load_problem(SOLID3D_YAML)
        pr_e.max_iter = args.warmup + args.steps
        pr_e.tol = 0.0
        got = []
        t0 = time.perf_counter()
        run(pr_e, backend="cuda", live_viz=False, verbose=False, save=False,
            viz_callback=lambda rho, it, c, v: got.append(rho.nbytes))
        torch.cuda.synchronize()
        t_e = time.perf_counter() - t0
        h2d = 8 * pr.n_dofs + pr.n_nodes + 2 * 576 * 8
        e2e = {"value": round(pr_e.max_iter / t_e, 4), "unit": SOLID3D_UNIT,
               "h2d_bytes_per_step": int(h2d / pr_e.max_iter),
               "d2h_bytes_per_step": int(np.mean(got)) + 5 * 8,
               "note": (f"simp.run() from a host Problem to the host density, {pr_e.max_iter} "
                        "OC iterations from the initial design")}
    line = {"metric": f"OC iter/s @3D cantilever {pr.nelx}x{pr.nely}x{pr.nelz} H8 FP64",
            "value": round(value, 4), "unit": SOLID3D_UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(t / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": f"synthetic (the 3D cantilever of {SOLID3D_YAML.relative_to(REPO)})",
            "config": {"workload": f"3D cantilever {pr.nelx}x{pr.nely}x{pr.nelz} H8 "
                                   f"({SOLID3D_YAML.relative_to(REPO)})",
                       "n_elem": pr.n_elem, "n_dofs": pr.n_dofs, "preconditioner": "jacobi",
                       "cg_tol": pr.cg_tol, "rmin": pr.rmin, "volfrac": pr.volfrac,
                       "oc_iterations_timed": f"{args.warmup + 1}..{args.warmup + args.steps}",
                       "step": "one OC iteration (filter, PCG, sensitivity, dc filter, OC)",
                       "l2": "flushed between timed steps (256 MiB write)"},
            "cg_iters": [r.cg_iters for r in recs], "compliance": [r.compliance for r in recs],
            "gpu_launches": int(launches), "roofline": roofline, "clocks": clocks.summary()}
    if e2e is not None:
        line["e2e"] = e2e
    if not args.no_cpu:
        line["cpu_baseline"] = cpu_sample_3d(pr, int(round(cg_mean)))
    print(json.dumps(line), flush=True)
    return 0


def main():
    global _RECURRENCE
    args = parse_args()
    _RECURRENCE = args.recurrence
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "solid3d":
        return run_solid3d(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.case == "pcg":
        return run_case(args)
    if args.case == "matvec":
        import torch
        from toptimization_b200.csrc import build as csrc_build
        csrc_build.build()
        torch.cuda.set_device(0)
        from toptimization_b200 import _lib
        from toptimization_b200.material import compute_Ke_2d, regularized_inverse
        Ke = compute_Ke_2d(1.0, 0.3)
        inv, alpha = regularized_inverse(Ke)
        _lib.ensure_stiffness(Ke, inv, alpha)
        r = time_matvec(load_workload(), torch.float64, torch, reps=5)
        print(json.dumps({"case": "matvec", **r}))
        return 0
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
