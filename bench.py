"""Benchmark: multigrid solves/s to 1e-10 relative residual on the
1024x1024 stretched mapped grid (x = xi + 0.1 sin(2 pi xi) sin(2 pi eta),
y = (e^{beta eta} - 1)/(e^beta - 1) with a 64:1 first-cell aspect ratio; Dirichlet
x sides, Neumann y sides; seeded 16-mode Fourier rhs, J-weighted mean removed).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one full solve (until |r|/|r0| <= 1e-10) of that problem.  The
default solver is the V-cycle accelerated by restarted GMRES(128)
(MGP_FLAG_GMRES: one V-cycle per preconditioner application) with the
V-cycle's grid levels in FP32 inside the FP64 outer iteration
(MGP_FLAG_MIXED) and its bottom solved exactly on the 32 x 32 level
(MGP_FLAG_DIRECT_COARSE | MGP_FLAG_DIRECT_LARGE: the inverse built on the
device when the solver is created); --solver krylov selects
BiCGStab(V-cycle) (MGP_FLAG_KRYLOV), --coarse direct an exact bottom on the
8 x 8 level, and --solver vcycle, --precision fp64 and --coarse reference
the reference's stationary iteration, plain FP64 and the reference's bottom
solver.  The line also carries one timed solve of the same
solver in FP64 ("fp64_same_solver") and of the plain FP64 V-cycle iteration
("plain_vcycle"), and the headline solution's error against both.  Under
torchrun every rank solves its own copy (replicas; the solve does not shard)
and rank 0 prints one JSON line.

At N=1 the line also carries:
  * "batched" (512 independent problems, sides
    log-uniform in [64,1024]): the lockstep batch (MGP_FLAG_LOCKSTEP, every
    V-cycle phase of all unconverged problems in one launch per group, knobs
    chosen by the autotuner) in mixed precision and in FP64, each against
    the same problems one at a time, and the per-problem concurrent
    BiCGStab(V-cycle) path; "batched_headline" is the metric's own
    comparison, mixed against plain FP64 with the served p50/p99;
  * "served" (Poisson arrivals of solves drawn from 64 problems
    with sides log-uniform in [32,2048] rounded to 8, hierarchies resident,
    tolerance 1e-8 or 1e-10) at 10, 30 and 100 requests/s, stopping once p99
    diverges; --serve-sweep extends the rates to 3000/s;
  * "precision_study": mixed precision against FP64 and against the exact
    solution of a manufactured problem on the skewed, stretched grid at
    512..4096, for the BiCGStab(V-cycle) solve and the deferred-correction
    solve, with the observed order of the discretisation error, and the same
    solvers with BF16 values on the levels below the finest;
  * "roofline_4096": the level-0 FP32 sweep timed live at 4096^2, beside the
    headline's 1024^2 "roofline";
  * "identity128": the 128^2 identity-map Dirichlet problem (V-cycles, ms per
    solve, error) for the FP64 V-cycle, the headline solver and the oracle.

--impl reference times the CPU restatement of the reference algorithm (the
reference is Fortran and no Fortran compiler exists on these hosts) on all
host cores, on a bounded sample of V-cycles of the same solve.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_GRID = 1024
TOL = 1e-10
MAXITERS = 4000
NU = (8, 8, 8)            # smooth_down, smooth_up, smooth_bottom (the reference test setting, test.f90:2546-2548)
METRIC = "solves/s @1e-10 rel resid"
WORKLOAD = "wavy_stretched_1024"
# words moved per cell by one smoothing sweep: read phi, rhs, invdiag, 4 Jgup; write phi
SWEEP_WORDS = 8
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_GRID)
    p.add_argument("--cpu-vcycles", type=int, default=4,
                   help="V-cycles per core in each bounded sample of --impl reference")
    p.add_argument("--cpu-vcycles-1core", type=int, default=8, help="V-cycles in each cpu_baseline sample")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--solver", default="gmres", choices=["gmres", "krylov", "vcycle"])
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                   help="mixed: FP32 grid levels inside the FP64 outer iteration (MGP_FLAG_MIXED)")
    p.add_argument("--coarse", default="large", choices=["direct", "large", "reference"],
                   help="bottom of the Krylov solvers' V-cycle: exact on the first level of at most 64 cells "
                        "(MGP_FLAG_DIRECT_COARSE), of at most 1024 (with MGP_FLAG_DIRECT_LARGE), or the reference's")
    p.add_argument("--no-plain", action="store_true", help="skip the extra plain V-cycle solve")
    p.add_argument("--no-batch", action="store_true", help="skip the batched and served legs")
    p.add_argument("--batch", type=int, default=512, help="problems in the batched leg")
    p.add_argument("--streams", type=int, default=16, help="concurrent solves in the batched and served legs")
    p.add_argument("--no-study", action="store_true", help="skip the precision/convergence study leg")
    p.add_argument("--serve-sweep", action="store_true",
                   help="extend the served leg's arrival rates to 3000/s (several minutes)")
    p.add_argument("--study-sizes", default="512,1024,2048,4096",
                   help="grid sides of the precision/convergence study")
    return p.parse_args()


def workload(n):
    from mgpoisson2d_b200 import workloads as W
    return W.wavy_stretched(n)


# --------------------------------------------------------------------------- #
# clocks sampled during the timed region
# --------------------------------------------------------------------------- #
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        out.update(sm_mhz=sm[len(sm) // 2] if sm else None, sm_max_mhz=max(mx) if mx else None, reasons=reasons,
                   samples=len(rows))
        return out


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic():
    """DRAM bytes per smoothing sweep from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        d = json.load(open(path))
        return d
    except Exception:
        return None


# --------------------------------------------------------------------------- #
# CPU legs
# --------------------------------------------------------------------------- #
# The oracle (a C restatement of the reference's FP64 solve) is built with
# -march=native on the host that times it: the same arithmetic (no contraction,
# no reassociation), tuned for that CPU.
_CPU = {}


def _cpu_oracle():
    os.environ["MGP_ORACLE_NATIVE"] = "1"
    import ctypes
    from oracle import oracle as O
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(1)
    return O


def _cpu_init(n):
    """Per CPU worker: the workload's inputs and the time of the solve's
    set-up half (hierarchy, inverse diagonals, first residual: a call with no
    V-cycle)."""
    from mgpoisson2d_b200.types import BoxData
    O = _cpu_oracle()
    v, geo, rhs, bc, _ = workload(n)
    t0 = time.perf_counter()
    O.vcycle(BoxData(v, 1, 1), rhs, geo, bc, True, TOL, 0, smooth_down=NU[0], smooth_up=NU[1], smooth_bottom=NU[2],
             gs_order=0)
    _CPU.update(O=O, prob=(v, geo, rhs, bc), t_setup=time.perf_counter() - t0)


def _cpu_step(vcycles):
    """One bounded sample: a fresh solve of the workload on the oracle
    (lexicographic Gauss-Seidel, the reference's stationary V-cycle), stopped
    after `vcycles` V-cycles.  Returns (seconds, V-cycles run, set-up seconds)."""
    from mgpoisson2d_b200.types import BoxData
    O = _CPU["O"]
    v, geo, rhs, bc = _CPU["prob"]
    t0 = time.perf_counter()
    rep = O.vcycle(BoxData(v, 1, 1), rhs, geo, bc, True, TOL, vcycles, smooth_down=NU[0], smooth_up=NU[1],
                   smooth_bottom=NU[2], gs_order=0)
    return time.perf_counter() - t0, rep.iterations, _CPU["t_setup"]


def solve_fraction(sec, vcycles, t_setup, vsolve):
    """Fraction of a full solve (set-up + vsolve V-cycles) that a sample of
    `vcycles` V-cycles taking `sec` seconds (set-up included) completed."""
    tvc = max(sec - t_setup, 1e-12) / max(vcycles, 1)
    return sec / (t_setup + vsolve * tvc)


def oracle_vcycles_per_solve(n):
    """V-cycles of the oracle's full lexicographic solve of this workload: the
    committed fixture of that solve (tests/golden/make_fixtures.py) at 1024^2,
    else the count recorded in profiles/vcycles.json."""
    fx = os.path.join(ROOT, "tests", "golden", "wavy1024.npz")
    if n == 1024 and os.path.exists(fx):
        import numpy as np
        return int(np.load(fx)["iterations"]), "tests/golden/wavy1024.npz (full oracle solve, 1 core)"
    try:
        return int(json.load(open(os.path.join(ROOT, "profiles", "vcycles.json")))[str(n)]), "profiles/vcycles.json"
    except Exception:
        return 1000, "default"


def cpu_baseline_1core(n, vcycles, runs=3):
    """cpu_baseline: the native oracle on one core, `runs` bounded samples of
    `vcycles` V-cycles each (in a spawned process, so the timed work shares no
    interpreter with the GPU process); the median sample's solve fraction per
    second is the solves/s."""
    import multiprocessing as mp
    vsolve, src = oracle_vcycles_per_solve(n)
    _cpu_oracle().build(force=True)
    with mp.get_context("spawn").Pool(1, initializer=_cpu_init, initargs=(n,)) as pool:
        res = [pool.apply(_cpu_step, (vcycles,)) for _ in range(runs)]
    rates = sorted(solve_fraction(sec, vc, ts, vsolve) / sec for sec, vc, ts in res)
    med = rates[len(rates) // 2]
    sec, vc, ts = res[0]
    return {"value": med, "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"median of {runs} samples of {vcycles} V-cycles of a fresh {n}^2 solve (set-up included) on "
                      f"the oracle built with -march=native on this host (lexicographic Gauss-Seidel, the "
                      f"reference's stationary iteration, FP64); a solve = set-up + {vsolve} V-cycles ({src}); "
                      f"samples {', '.join(f'{r[0]:.2f}' for r in res)} s, set-up {ts:.3f} s",
            "vcycles_per_solve": vsolve, "s_per_vcycle": (sec - ts) / max(vc, 1)}


def _cpu_identity128(runs):
    """Full oracle solves of the 128^2 identity-map Dirichlet problem on one
    core (lexicographic Gauss-Seidel, FP64): median seconds and V-cycles."""
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    O = _cpu_oracle()
    v, geo, rhs, bc, u = W.identity_dirichlet(128)
    secs = []
    for _ in range(runs):
        phi = BoxData(v, 1, 1)
        t0 = time.perf_counter()
        rep = O.vcycle(phi, rhs, geo, bc, True, TOL, 100, smooth_down=NU[0], smooth_up=NU[1], smooth_bottom=NU[2],
                       gs_order=0)
        secs.append(time.perf_counter() - t0)
    return sorted(secs)[len(secs) // 2], rep.iterations, float(abs(phi.interior() - u).max())


def identity128_leg(M, cpu, runs=20):
    """The 128^2 identity-map Dirichlet problem (u = sin 2 pi x sin 3 pi y plus
    1e-3 noise in the rhs): V-cycles, ms per solve and the error against u for
    the reference's FP64 V-cycle and the headline solver, on the device (median
    of `runs` solves with device arrays) and, with `cpu`, on the oracle."""
    import torch
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    v, geo, rhs, bc, u = W.identity_dirichlet(128)
    rhs_d = rhs.to_device()
    stream = torch.cuda.current_stream()
    base = M.FLAG_DIRICHLET_COUPLED_DIAG
    out = {"workload": "identity_dirichlet_128", "tol": TOL, "nu": list(NU), "timing": f"median of {runs} solves"}
    for name, fl in (("fp64_vcycle", base),
                     ("mixed_gmres", base | M.FLAG_GMRES | M.FLAG_MIXED | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE)):
        with M.Solver(v, geo, bc, M.KIND_MG, fl) as s:
            phi = BoxData(v, 1, 1).to_device()
            ms = []
            for k in range(runs + 3):
                phi.data.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = s.vcycle(phi, rhs_d, bc, True, TOL, 200, 1, *NU)
                e1.record(stream)
                e1.synchronize()
                if k >= 3:
                    ms.append(e0.elapsed_time(e1))
        out[name] = {"vcycles": r.iterations, "final_relres": r.final_relres, "ms_per_solve": sorted(ms)[len(ms) // 2],
                     "err_max": float(abs(phi.to_host().interior() - u).max())}
    if cpu:
        import multiprocessing as mp
        _cpu_oracle().build(force=False)
        with mp.get_context("spawn").Pool(1) as pool:
            sec, its, e = pool.apply(_cpu_identity128, (5,))
        out["cpu_1core"] = {"vcycles": its, "ms_per_solve": sec * 1e3, "err_max": e, "kind": "port",
                            "sample": "median of 5 full oracle solves (-march=native, FP64, lexicographic GS)"}
    return out


def run_reference(args):
    """--impl reference: the reference's algorithm on the CPU, on every host
    core the process may use.  Each step is one bounded sample per core (a
    fresh solve stopped after --cpu-vcycles V-cycles, all cores at once); the
    step's work is the sum over cores of the solve fraction each sample
    completed, and value = that work over the steps' wall time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    vsolve, src = oracle_vcycles_per_solve(args.n)
    _cpu_oracle().build(force=True)
    ctx = mp.get_context("spawn")
    walls, work = [], []
    with ctx.Pool(cores, initializer=_cpu_init, initargs=(args.n,)) as pool:
        for step in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            res = pool.map(_cpu_step, [args.cpu_vcycles] * cores, chunksize=1)
            wall = time.perf_counter() - t0
            if step >= args.warmup:
                walls.append(wall)
                work.append(sum(solve_fraction(sec, vc, ts, vsolve) for sec, vc, ts in res))
    value = sum(work) / sum(walls)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(walls) / len(walls),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": args.n, "tol": TOL, "nu": list(NU)},
        "solver": "vcycle (the reference's stationary iteration, lexicographic Gauss-Seidel)",
        "solves_per_step": sum(work) / len(work), "vcycles_per_solve": vsolve, "vcycles_per_solve_source": src,
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"per step, {cores} processes each run a fresh {args.n}^2 solve on the oracle "
                                   f"(-march=native, FP64) for {args.cpu_vcycles} V-cycles at once; a solve = set-up "
                                   f"+ {vsolve} V-cycles ({src})"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------- #
# Batched and served legs (many independent problems)
# --------------------------------------------------------------------------- #
def batched_leg(M, args):
    """`args.batch` problems of the batched workload (sides log-uniform in
    [64, 1024], rounded to 16; random stretch and skew; Dirichlet), inputs and
    hierarchies resident, solved to 1e-10:
      * lockstep (MGP_FLAG_LOCKSTEP: every V-cycle phase of all unconverged
        problems in one launch per group; groups and two-sweep launches chosen
        by Batch.autotune, which changes no bit) in mixed precision and in
        FP64, the exact bottom on the coarse-cycle level;
      * the same problems one at a time (the same solver, one stream);
      * the per-problem concurrent path (BiCGStab(V-cycle), `args.streams`
        streams), the batched form without lockstep.
    Device-synchronised wall time around each batch call."""
    import numpy as np
    import torch
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    probs = [W.batch_problem_device(i) for i in range(args.batch)]   # geometry and rhs made on the device
    rhs_d = [p[2] for p in probs]
    bcs = [p[3] for p in probs]
    cells = sum(p[0].nx * p[0].ny for p in probs)
    base = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE
    legs = [("mixed", base | M.FLAG_LOCKSTEP | M.FLAG_MIXED, True),
            ("fp64", base | M.FLAG_LOCKSTEP, True),
            ("concurrent_bicgstab_mixed", base | M.FLAG_KRYLOV | M.FLAG_MIXED, False)]
    out = {"problems": args.batch, "cells": cells, "streams": args.streams,
           "workload": "sides log-uniform [64,1024] rounded to 16, stretch U[1,1.08] in a min(64,ny/4)-cell layer, "
                       "skew U[0,25] deg, 16-mode rhs, Dirichlet; seeds 4e6+i; geometry and rhs generated on the device",
           "timing": "device-synchronised wall time around one batch call, after an autotuning / warm-up call"}
    for name, fl, lock in legs:
        phis = [BoxData.device_zeros(p[0], 1, 1) for p in probs]
        with M.Batch([(v, g, bc) for v, g, _, bc in probs], M.KIND_MG, fl, nstreams=args.streams) as b:
            tune = None
            if lock:
                tune = b.autotune(phis, rhs_d, bcs, True, TOL, MAXITERS, groups=(1, 2, 4, 8, 16))
            else:
                b.vcycle(phis, rhs_d, bcs, True, TOL, MAXITERS)   # warm-up (graph capture)
            for p in phis:
                p.data.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            reps = b.vcycle(phis, rhs_d, bcs, True, TOL, MAXITERS)
            torch.cuda.synchronize()
            tb = time.perf_counter() - t0
        assert all(r.final_relres <= TOL for r in reps), "batched solve did not converge"
        row = {"solves_per_s": args.batch / tb, "seconds": tb,
               "vcycles_mean": float(np.mean([r.iterations for r in reps])),
               "vcycles_max": int(max(r.iterations for r in reps)),
               "solver": "stationary V-cycle, lockstep" if lock else "BiCGStab(V-cycle), a stream per problem"}
        if tune:
            row["tuning"] = {"groups": tune["groups"], "two_sweep_launches": tune["pairs"],
                             "searched_s": {k: round(v, 4) for k, v in tune["seconds"].items()}}
        if lock:   # the same problems one at a time, same solver
            solvers = [M.Solver(v, g, bc, M.KIND_MG, fl) for v, g, _, bc in probs]
            for s_, p, f, (v, g, _, bc) in zip(solvers, phis, rhs_d, probs):
                p.data.zero_()
                s_.vcycle(p, f, bc, True, TOL, MAXITERS)   # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for s_, p, f, (v, g, _, bc) in zip(solvers, phis, rhs_d, probs):
                p.data.zero_()
                s_.vcycle(p, f, bc, True, TOL, MAXITERS)
            torch.cuda.synchronize()
            ts = time.perf_counter() - t0
            for s_ in solvers:
                s_.close()
            row["sequential_solves_per_s"] = args.batch / ts
        out[name] = row
    out["mixed_over_fp64"] = out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]
    out["lockstep_over_concurrent"] = out["mixed"]["solves_per_s"] / out["concurrent_bicgstab_mixed"]["solves_per_s"]
    return out


def batched_multi(M, args, flags, rank, world):
    """The batched workload over `world` GPUs: each rank builds (on its device)
    and solves its share of the problems, balanced by estimated hierarchy
    bytes (mgpoisson2d_b200.partition); no collective touches the data.  The
    time is the max over ranks of each rank's device-timed batch."""
    import torch
    import torch.distributed as dist
    from mgpoisson2d_b200 import partition as P
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    costs = [float(P.estimated_bytes(*W.batch_problem_params(i)[:2], True)) for i in range(args.batch)]
    mine = P.my_share(costs, rank, world)
    probs = [W.batch_problem_device(i) for i in mine]
    stream = torch.cuda.current_stream()
    ms = 0.0
    b = M.Batch([(v, g, bc) for v, g, _, bc in probs], M.KIND_MG, flags, nstreams=args.streams) if probs else None
    phis = [BoxData.device_zeros(p[0], 1, 1) for p in probs]
    if b:
        b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, TOL, MAXITERS)   # warm-up
        for p in phis:
            p.data.zero_()
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if b:
        b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, TOL, MAXITERS)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    if b:
        b.close()
    t = torch.tensor([ms], device="cuda", dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"problems": args.batch, "ranks": world, "streams_per_rank": args.streams,
            "partition": "longest first, by estimated hierarchy bytes", "imbalance": P.imbalance(costs, world),
            "batched_solves_per_s": args.batch / (float(t.item()) * 1e-3), "precision": "mixed",
            "timing": "device events around each rank's batch, max over ranks"}


def served_leg(M, args, flags_list, pool=64, seed=5, rates=(10, 30, 100)):
    """The served workload swept over arrival rates: a pool of `pool` problems
    (sides log-uniform in [32, 2048] rounded to a multiple of 8, maps as the
    batched workload, seed 5), requests drawn from the pool with Poisson
    arrivals at each rate, tolerance 1e-8 or 1e-10 with probability 1/2,
    min(2000, 8 x rate) requests per rate (at least 100), hierarchies resident
    per problem; stops after the first rate whose p99 has diverged (above 10x
    the lowest rate's p99, or fewer than 0.7 of the offered solves/s).  The
    solver is the headline's, GMRES(V-cycle) with the exact bottom, mixed and
    FP64."""
    import numpy as np
    import torch
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    probs = [W.batch_problem_device(i, seed=seed, nmin=32, nmax=2048, round_to=8) for i in range(pool)]
    torch.cuda.synchronize()
    out = {"pool": pool, "sides": [32, 2048], "slots": args.streams, "tolerances": [1e-8, 1e-10],
           "cells_mean": float(np.mean([p[0].nx * p[0].ny for p in probs]))}
    for name, fl in flags_list:
        rows = []
        with M.Server(nworkers=args.streams, flags=fl) as srv:
            warm = [srv.submit(v, g, bc, BoxData.device_zeros(v, 1, 1), rhs, True, 1e-10, MAXITERS, key=k + 1)
                    for k, (v, g, rhs, bc) in enumerate(probs)]
            for t in warm:
                srv.wait(t)
            base_p99 = None
            for lam in rates:
                nreq = int(min(2000, max(100, 8 * lam)))
                rng = np.random.default_rng(seed * 1000 + lam)
                gaps = rng.exponential(1.0 / lam, nreq)
                which = rng.integers(0, pool, nreq)
                tols = np.where(rng.random(nreq) < 0.5, 1e-8, 1e-10)
                outs = [BoxData.device_zeros(probs[k][0], 1, 1) for k in which]
                tickets = []
                t0 = time.perf_counter()
                t_next = t0
                for n in range(nreq):
                    t_next += gaps[n]
                    while time.perf_counter() < t_next:
                        time.sleep(max(0.0, min(0.001, t_next - time.perf_counter())))
                    v, g, rhs, bc = probs[which[n]]
                    tickets.append(srv.submit(v, g, bc, outs[n], rhs, True, float(tols[n]), MAXITERS,
                                              key=int(which[n]) + 1))
                lats = np.sort(np.array([srv.wait(t)[1] for t in tickets])) * 1e3
                span = time.perf_counter() - t0
                p99 = float(lats[min(len(lats) - 1, int(math.ceil(0.99 * len(lats))) - 1)])
                row = {"offered_per_s": lam, "requests": nreq, "solves_per_s": nreq / span,
                       "p50_ms": float(lats[len(lats) // 2]), "p99_ms": p99}
                rows.append(row)
                base_p99 = base_p99 or p99
                if p99 > 10 * base_p99 or row["solves_per_s"] < 0.7 * lam:
                    break
        out[name] = rows
    return out


# --------------------------------------------------------------------------- #
# GPU arm
# --------------------------------------------------------------------------- #
def pinned(bd):
    """A copy of a host BoxData in page-locked memory (the e2e leg's inputs and
    output live there, so the call's host<->device copies are DMA transfers)."""
    import torch
    from mgpoisson2d_b200.types import BoxData
    buf = torch.empty(bd.data.size, dtype=torch.float64, pin_memory=True)
    arr = buf.numpy().reshape(bd.data.shape, order="F")
    arr[...] = bd.data
    out = BoxData(bd.valid, bd.ngx, bd.ngy, bd.offi, bd.offj, data=arr)
    out._pinned = buf   # keeps the page-locked buffer alive
    return out


def vcycle_bytes(M, v, mixed, direct, nu=NU, large=False):
    """Algorithmic bytes of one V-cycle: per level with N cells and word size
    w, N w [8 (nu1 + nu2) + 6 + rho + 2 + rho + 3] (sweeps; residual fused
    with restriction; prolongation; the coarse guess r invdiag; rho = coarse
    cells per fine cell), plus 11 FP64 words per finest cell for the outer
    residual, norm and update.  Levels of at most 1024 cells (the coarse CTA)
    are FP64; with FP32 grid levels the others take 4 B.  The bottom is the
    first level of at most 64 cells with `direct`, of at most 1024 with
    `large` as well; its solve is counted as time, except the large bottom's
    product with the inverse, 8 N (N + 2) bytes."""
    md = M.estimate_maxdepth(1000, v)
    rx, ry, md = M.create_mgschedule(md, v)
    nx, ny, levels = v.nx, v.ny, []
    for d in range(md + 1):
        levels.append((nx, ny))
        if d < md:
            nx, ny = nx // rx[d], ny // ry[d]
    bottom = len(levels) - 1
    total = 11 * 8 * v.nx * v.ny
    if direct and large:
        dc = next((d for d, (a, b) in enumerate(levels) if a * b <= 1024), bottom)
        if 64 < levels[dc][0] * levels[dc][1] <= 1024:
            bottom = dc
            nb = levels[dc][0] * levels[dc][1]
            total += 8 * nb * (nb + 2)
            direct = False
    if direct:
        bottom = next((d for d, (a, b) in enumerate(levels) if a * b <= 64), bottom)
    for d in range(bottom):
        n = levels[d][0] * levels[d][1]
        w = 4 if (mixed and n > 1024) else 8
        rho = 1.0 / (rx[d] * ry[d])
        total += n * w * (8 * (nu[0] + nu[1]) + 6 + rho + 2 + rho + 3)
    return total


def roofline_large(M, n=4096):
    """The level-0 FP32 sweep at n^2 (the skewed, stretched grid of the
    precision study), timed live as the bench's own roofline: one mixed
    BiCGStab(V-cycle) solve with the finest level's smoothing bracketed by
    CUDA events (MGP_FLAG_TIME_SMOOTHER), algorithmic bytes 8 words of 4 B a
    cell per sweep."""
    import torch
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    v, geo, rhs, bc, _ = W.skew_stretched_device(n)
    fl = (M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV | M.FLAG_MIXED | M.FLAG_DIRECT_COARSE |
          M.FLAG_TIME_SMOOTHER)
    with M.Solver(v, geo, bc, M.KIND_MG, fl) as s:
        phi = BoxData.device_zeros(v, 1, 1)
        s.vcycle(phi, rhs, bc, False, TOL, 4)   # warm-up
        phi.data.zero_()
        r = s.vcycle(phi, rhs, bc, False, TOL, MAXITERS)
    sweep_s = r.smooth0_seconds / max(r.smooth0_sweeps, 1)
    peak, kind = measured_peak()
    alg = SWEEP_WORDS * 4 * v.nx * v.ny
    del v, geo, rhs, bc, phi
    torch.cuda.empty_cache()
    return {"kernel": f"k_sweep9 level 0 (FP32 fields, TMA staging), {n}^2", "achieved": alg / sweep_s / 1e9,
            "peak": peak, "peak_kind": kind, "unit": "GB/s", "frac": alg / sweep_s / 1e9 / peak,
            "alg_bytes_per_sweep": alg, "sweep_us": sweep_s * 1e6, "sweeps": r.smooth0_sweeps}


def precision_study(M, sizes):
    """Mixed precision against FP64 and against the exact solution on the
    skewed, boundary-layer-stretched manufactured problem (u = e^x cos 4 pi y,
    Dirichlet data at the face centres, metric generated on the device), for
    two solvers: BiCGStab(V-cycle) with the exact bottom ("mixed", "fp64") and
    the deferred-correction solve, DD V-cycles inside the FP64 9-point
    residual loop, nu = 8/8/8 ("dc_mixed", "dc_fp64"), each also with BF16
    values on the levels below the finest ("bf16", "dc_bf16").  Per solve: V-cycles
    (DC iterations), time, relative max / L2 error against u; per pair the
    mixed solution's distance from the FP64 one; per size step the observed
    order log2(e_n / e_2n) of the discretisation error."""
    import torch
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData
    kry = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV | M.FLAG_DIRECT_COARSE
    solvers = (("mixed", M.KIND_MG, kry | M.FLAG_MIXED), ("fp64", M.KIND_MG, kry),
               ("bf16", M.KIND_MG, kry | M.FLAG_MIXED | M.FLAG_BF16_COARSE),
               ("dc_mixed", M.KIND_DD, M.FLAG_MIXED), ("dc_fp64", M.KIND_DD, 0),
               ("dc_bf16", M.KIND_DD, M.FLAG_MIXED | M.FLAG_BF16_COARSE))
    stream = torch.cuda.current_stream()
    rows = []
    for n in sizes:
        v, geo, rhs, bc, u = W.skew_stretched_device(n)
        f = BoxData.device_zeros(v)   # the DC solve takes f; rhs = J f
        f.data[:] = rhs.data / geo.J.data[1:-1, 1:-1]
        row = {"n": n}
        sol = {}
        for name, kind, fl in solvers:
            with M.Solver(v, geo, bc, kind, fl) as s:
                phi = BoxData.device_zeros(v, 1, 1)
                if kind == M.KIND_DD:
                    ff = BoxData.device_zeros(v)
                    ff.data[:] = f.data
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                if kind == M.KIND_DD:
                    r = s.dc_vcycle(phi, ff, bc, False, TOL, MAXITERS, 1, 8, 8, 8)
                else:
                    r = s.vcycle(phi, rhs, bc, False, TOL, MAXITERS)
                e1.record(stream)
                e1.synchronize()
            p = phi.data[1:-1, 1:-1]
            sol[name] = p
            row[name] = {"vcycles": r.iterations, "final_relres": r.final_relres, "ms": e0.elapsed_time(e1),
                         "err_max": float((p - u).abs().max() / u.abs().max()),
                         "err_l2": float(torch.linalg.norm(p - u) / torch.linalg.norm(u))}
        for a, b, key in (("mixed", "fp64", "mixed_vs_fp64"), ("dc_mixed", "dc_fp64", "dc_mixed_vs_fp64"),
                          ("bf16", "fp64", "bf16_vs_fp64"), ("dc_bf16", "dc_fp64", "dc_bf16_vs_fp64")):
            d = sol[a] - sol[b]
            row[key] = {"rel_l2": float(torch.linalg.norm(d) / torch.linalg.norm(sol[b])),
                        "rel_max": float(d.abs().max() / sol[b].abs().max())}
        rows.append(row)
        del v, geo, rhs, bc, u, f, sol
    for a, b in zip(rows, rows[1:]):
        for name, _, _ in solvers:
            b[name]["order_l2"] = math.log2(a[name]["err_l2"] / b[name]["err_l2"]) / math.log2(b["n"] / a["n"])
    torch.cuda.empty_cache()
    return {"workload": "skew_stretched (30 deg skew, 1.05 boundary-layer stretch, u = e^x cos 4 pi y)",
            "tol": TOL, "solvers": {"mixed / fp64": "bicgstab(vcycle), exact bottom",
                                    "dc_mixed / dc_fp64": "deferred correction (dc_vcycle), nu 8/8/8",
                                    "bf16 / dc_bf16": "the mixed solvers with the levels below the finest holding "
                                                      "BF16 values (MGP_FLAG_BF16_COARSE: a numerics study; the "
                                                      "storage stays FP32, so its times include the rounding "
                                                      "launches and no saved bytes)"},
            "rows": rows}


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import numpy as np
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    import mgpoisson2d_b200.api as M
    from mgpoisson2d_b200.types import BoxData

    v, geo, rhs, bc, _ = workload(args.n)
    base_flags = M.FLAG_DIRICHLET_COUPLED_DIAG
    fp64_flags = base_flags | {"krylov": M.FLAG_KRYLOV, "gmres": M.FLAG_GMRES, "vcycle": 0}[args.solver]
    if args.solver != "vcycle" and args.coarse != "reference":
        fp64_flags |= M.FLAG_DIRECT_COARSE | (M.FLAG_DIRECT_LARGE if args.coarse == "large" else 0)
    flags = fp64_flags | (M.FLAG_MIXED if args.precision == "mixed" else 0)
    solver = M.Solver(v, geo, bc, M.KIND_MG, flags)
    phi_d = BoxData(v, 1, 1).to_device()
    rhs_d = rhs.to_device()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def solve():
        phi_d.data.zero_()
        return solver.vcycle(phi_d, rhs_d, bc, True, TOL, MAXITERS, 1, *NU)

    reps = []
    for _ in range(args.warmup):
        reps.append(solve())
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = M.kernel_launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    step_ms = []
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1.0)   # L2 flush between steps; outside the per-step events
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rep = solve()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        reps.append(rep)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    launches = M.kernel_launch_count() - launches0
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms * 1e-3)
    last = reps[-1]
    assert last.relres[-1] <= TOL and not last.diverged, "solve did not converge"
    srt = sorted(step_ms)
    latency = {"p50": srt[len(srt) // 2], "p99": srt[min(len(srt) - 1, math.ceil(0.99 * len(srt)) - 1)],
               "unit": "ms", "samples": len(srt)}

    sol = phi_d.to_host().interior().copy()

    def one_solve(fl):
        """One timed solve with other flags; returns (summary, solution)."""
        ps = M.Solver(v, geo, bc, M.KIND_MG, fl)
        phi_d.data.zero_()
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = ps.vcycle(phi_d, rhs_d, bc, True, TOL, MAXITERS, 1, *NU)
        e1.record(stream)
        e1.synchronize()
        ps.close()
        ms = e0.elapsed_time(e1)
        return ({"solves_per_s": 1e3 / ms, "ms_per_solve": ms, "vcycles": r.iterations,
                 "final_relres": r.final_relres, "timed_solves": 1}, phi_d.to_host().interior().copy())

    def err(a, ref):
        return {"rel_l2": float(np.linalg.norm(a - ref) / np.linalg.norm(ref)),
                "rel_max": float(np.abs(a - ref).max() / np.abs(ref).max())}

    # the same solver in plain FP64, and the reference's stationary iteration
    # (FP64 V-cycles), for comparison; the error of the headline solution is
    # stated against both FP64 solutions
    fp64 = plain = None
    accuracy = {}
    if not args.no_plain:
        if args.precision == "mixed":
            fp64, sol64 = one_solve(fp64_flags)
            accuracy["vs_fp64_same_solver"] = err(sol, sol64)
        if args.solver == "vcycle" and args.precision == "fp64":
            plain = {"solves_per_s": value, "ms_per_solve": total_ms / args.steps, "vcycles": last.iterations}
        else:
            plain, solp = one_solve(base_flags)
            accuracy["vs_fp64_vcycle"] = err(sol, solp)

    # live roofline of the dominant kernel: one more solve with the finest
    # level's smoothing bracketed by events
    prof = M.Solver(v, geo, bc, M.KIND_MG, flags | M.FLAG_TIME_SMOOTHER)
    phi_d.data.zero_()
    flush.fill_(1.0)
    prep = prof.vcycle(phi_d, rhs_d, bc, True, TOL, MAXITERS, 1, *NU)
    prof.close()
    sweep_s = prep.smooth0_seconds / max(prep.smooth0_sweeps, 1)
    word = 4 if args.precision == "mixed" else 8
    alg_bytes = SWEEP_WORDS * word * v.nx * v.ny
    peak, peak_kind = measured_peak()
    achieved = alg_bytes / sweep_s / 1e9
    tr = (committed_traffic() or {}).get("fp32" if word == 4 else "fp64")
    roofline = {"bound": "hbm", "kernel": f"k_sweep9 level 0 ({'FP32' if word == 4 else 'FP64'} fields, TMA staging)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_kind": peak_kind, "traffic": (tr or {}).get("bytes_per_sweep"),
                "alg_bytes_per_sweep": alg_bytes, "sweep_us": sweep_s * 1e6}

    vb = vcycle_bytes(M, v, args.precision == "mixed", bool(fp64_flags & M.FLAG_DIRECT_COARSE),
                      large=bool(fp64_flags & M.FLAG_DIRECT_LARGE))
    vc_s = (total_ms / args.steps) * 1e-3 / max(last.iterations, 1)
    vcycle_roofline = {"bytes_per_vcycle": vb, "s_per_vcycle": vc_s, "achieved": vb / vc_s / 1e9, "peak": peak,
                       "unit": "GB/s", "frac": vb / vc_s / 1e9 / peak,
                       "note": "whole V-cycle, algorithmic bytes of every level (bottom solve as time, the large bottom's "
                               "product with its inverse as bytes); the time is "
                               "the solve's divided by its V-cycles, Krylov vector work included"}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "n": args.n, "tol": TOL, "nu": list(NU),
                   "l2": "flushed between steps (256 MiB write, outside step events)",
                   "parallelism": f"replicas{world}"},
        "solver": {"method": {"krylov": "bicgstab(vcycle)", "gmres": "gmres(vcycle)", "vcycle": "vcycle"}[args.solver],
                   "precision": ("FP32 grid levels, FP64 outer iteration / residual / update / coarse levels"
                                 if args.precision == "mixed" else "FP64"),
                   "flags": "dirichlet_coupled_diag" + ("" if args.solver == "vcycle" else "|" + args.solver) +
                            ("|mixed" if args.precision == "mixed" else "") +
                            ("|direct_coarse" if fp64_flags & M.FLAG_DIRECT_COARSE else "") +
                            ("|direct_large" if fp64_flags & M.FLAG_DIRECT_LARGE else ""),
                   "bottom": ("exact solve of the first level <= 1024 cells (inverse built on the device)"
                              if fp64_flags & M.FLAG_DIRECT_LARGE else
                              "exact solve of the first level <= 64 cells" if fp64_flags & M.FLAG_DIRECT_COARSE
                              else "relax + BiCGStab to 1e-6 (reference)"),
                   "vcycles_per_solve": last.iterations, "final_relres": last.final_relres,
                   "maxdepth": last.maxdepth},
        "latency_ms": latency, "fp64_same_solver": fp64, "plain_vcycle": plain, "accuracy": accuracy,
        "roofline": roofline, "vcycle_roofline": vcycle_roofline, "clocks": clocks, "gpu_launches": launches,
        "unknowns_vcycles_per_s": value * last.iterations * v.nx * v.ny,
        "wall_s": wall,
    }

    if rank == 0 and not args.no_e2e:
        # end to end through the reference-facing call: host arrays in pinned
        # memory, hierarchy built inside the call (mgp_vcycle has the Fortran
        # argument list); one untimed call, then the median of up to three
        # timed calls
        from mgpoisson2d_b200.types import GeoData
        geo_p = GeoData(pinned(geo.J), pinned(geo.Jgup_xx), pinned(geo.Jgup_xy), pinned(geo.Jgup_yx),
                        pinned(geo.Jgup_yy), geo.dx, geo.dy)
        rhs_p, phi_h = pinned(rhs), pinned(BoxData(v, 1, 1))
        M.set_flags(flags)
        times = []
        for k in range(1 + min(args.steps, 3)):
            phi_h.data[...] = 0.0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            erep = M.vcycle(phi_h, rhs_p, geo_p, bc, True, TOL, MAXITERS, -1, 1, *NU)
            if k:
                times.append(time.perf_counter() - t0)
        M.set_flags(0)
        e2e_s = sorted(times)[len(times) // 2]
        h2d = 8 * (phi_h.data.size + rhs.data.size + v.nx * v.ny + 4 * (v.nx + 1) * v.ny)
        line["e2e"] = {"value": 1.0 / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": 8 * phi_h.data.size,
                       "api": "mgp_vcycle (host arrays in pinned memory; hierarchy built inside the call)",
                       "vcycles": erep.iterations, "timed_calls": len(times), "stat": "median"}
    if world > 1 and not args.no_batch:   # every rank: its share of the batch
        batched_n = batched_multi(M, args, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV | M.FLAG_MIXED |
                                  M.FLAG_DIRECT_COARSE, rank, world)
        if rank == 0:
            line["batched"] = batched_n
    if rank == 0 and world == 1 and not args.no_batch:
        batched = batched_leg(M, args)
        line["batched"] = batched
        gm = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_GMRES | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE
        rates = (10, 30, 100, 300, 1000, 3000) if args.serve_sweep else (10, 30, 100)
        served = served_leg(M, args, [("mixed", gm | M.FLAG_MIXED), ("fp64", gm)], rates=rates)
        line["served"] = served
        # the metric's own comparison: mixed against plain FP64, batched and served
        line["batched_headline"] = {
            "mixed_solves_per_s": batched["mixed"]["solves_per_s"], "fp64_solves_per_s": batched["fp64"]["solves_per_s"],
            "mixed_over_fp64": batched["mixed_over_fp64"], "problems": batched["problems"],
            "served_mixed_p50_ms": served["mixed"][0]["p50_ms"], "served_mixed_p99_ms": served["mixed"][0]["p99_ms"],
            "served_fp64_p50_ms": served["fp64"][0]["p50_ms"], "served_fp64_p99_ms": served["fp64"][0]["p99_ms"],
            "served_rate_per_s": served["mixed"][0]["offered_per_s"]}
    if rank == 0 and world == 1 and not args.no_study:
        line["precision_study"] = precision_study(M, [int(x) for x in args.study_sizes.split(",") if x])
        line["roofline_4096"] = roofline_large(M)
        line["identity128"] = identity128_leg(M, not args.no_cpu)
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline_1core(args.n, args.cpu_vcycles_1core)
        line["cpu_baseline"] = cb
        if plain:   # the same algorithm on both sides: the stationary FP64 V-cycle
            line["same_algorithm"] = {"gpu_fp64_vcycle_solves_per_s": plain["solves_per_s"],
                                      "cpu_1core_solves_per_s": cb["value"],
                                      "ratio": plain["solves_per_s"] / cb["value"],
                                      "gpu_vcycles": plain["vcycles"], "cpu_vcycles": cb["vcycles_per_solve"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
