"""A short, fixed run of the benchmark workload for profilers:

    python -m mgpoisson2d_b200.profile [--n 1024] [--vcycles 2] [--warmup 1] [--mixed] [--krylov | --gmres]
                                       [--workload wavy|skew|served] [--served-index K] [--direct [--direct-large]]

Builds the resident solver for the stretched mapped grid (wavy: the bench
workload; skew: the skewed boundary-layer manufactured problem; served:
problem K of the served pool, sides log-uniform in [32, 2048] rounded to 8,
seed 5, e.g. K = 44, 1160 x 1720, whose coarse cycle starts at 145 x 215), runs `warmup` solves capped at `vcycles` V-cycles, then one more,
and prints the device time per V-cycle.  Under ncu, the kernels of the last
solve follow those of the warm-up solves in launch order.
"""
from __future__ import annotations

import argparse
import time


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--n", type=int, default=1024)
    p.add_argument("--vcycles", type=int, default=2)
    p.add_argument("--warmup", type=int, default=1)
    p.add_argument("--dd", action="store_true", help="deferred-correction driver")
    p.add_argument("--mixed", action="store_true", help="FP32 grid levels (MGP_FLAG_MIXED)")
    p.add_argument("--krylov", action="store_true", help="BiCGStab acceleration (MGP_FLAG_KRYLOV)")
    p.add_argument("--gmres", action="store_true", help="GMRES acceleration (MGP_FLAG_GMRES)")
    p.add_argument("--direct", action="store_true", help="exact bottom solve (MGP_FLAG_DIRECT_COARSE)")
    p.add_argument("--direct-large", action="store_true",
                   help="with --direct: the exact bottom on the first level of at most 1024 cells "
                        "(MGP_FLAG_DIRECT_LARGE)")
    p.add_argument("--workload", default="wavy", choices=["wavy", "skew", "served"])
    p.add_argument("--served-index", type=int, default=44, help="with --workload served: the pool problem")
    p.add_argument("--time-smoother", action="store_true", help="also report the finest level's time per sweep")
    p.add_argument("--batch", type=int, default=0,
                   help="instead: a lockstep batch of this many problems of the batched workload "
                        "(MGP_FLAG_LOCKSTEP, exact bottoms; --mixed for FP32 grid levels)")
    p.add_argument("--groups", type=int, default=8, help="with --batch: lockstep groups")
    a = p.parse_args()
    if a.batch:
        return run_batch(a)

    import torch

    import mgpoisson2d_b200.api as M
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData

    torch.cuda.set_device(0)
    if a.workload == "wavy":
        v, geo, rhs, bc, _ = W.wavy_stretched(a.n)
        homog = True
    elif a.workload == "served":
        v, geo, rhs, bc = W.batch_problem_device(a.served_index, seed=5, nmin=32, nmax=2048, round_to=8)
        homog = True
    else:
        v, geo, rhs, bc, _ = W.skew_stretched_device(a.n)
        homog = False
    kind = M.KIND_DD if a.dd else M.KIND_MG
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | (M.FLAG_MIXED if a.mixed else 0) | (M.FLAG_KRYLOV if a.krylov else 0)
    flags |= M.FLAG_TIME_SMOOTHER if a.time_smoother else 0
    flags |= M.FLAG_GMRES if a.gmres else 0
    flags |= M.FLAG_DIRECT_COARSE if a.direct else 0
    flags |= M.FLAG_DIRECT_LARGE if a.direct_large else 0
    s = M.Solver(v, geo, bc, kind, flags)
    phi, f = BoxData.device_zeros(v, 1, 1), (rhs.to_device() if a.workload == "wavy" else rhs)
    if a.workload == "served":
        a.n = f"{v.nx}x{v.ny}"
    if a.dd:
        f.data /= geo.J.to_device().data[1:-1, 1:-1]
    run = (lambda: s.dc_vcycle(phi, f, bc, homog, 1e-10, a.vcycles, 1, 8, 8, 8)) if a.dd else \
        (lambda: s.vcycle(phi, f, bc, homog, 1e-10, a.vcycles, 1, 8, 8, 8))
    for _ in range(a.warmup):
        phi.data.zero_()
        run()
    phi.data.zero_()
    torch.cuda.synchronize()
    l0 = M.kernel_launch_count()
    t0 = time.perf_counter()
    rep = run()
    dt = time.perf_counter() - t0
    print(f"n={a.n} vcycles={rep.iterations} device {rep.seconds * 1e3:.3f} ms "
          f"({rep.seconds / max(rep.iterations, 1) * 1e3:.3f} ms/V-cycle), wall {dt * 1e3:.3f} ms, "
          f"{M.kernel_launch_count() - l0} launches, relres {rep.relres[-1]:.3e}")
    if a.time_smoother:
        print(f"finest-level sweep {rep.smooth0_seconds / max(rep.smooth0_sweeps, 1) * 1e6:.2f} us "
              f"({rep.smooth0_sweeps} sweeps)")
    s.close()


def run_batch(a):
    """`warmup` + 1 lockstep solves of the first `batch` problems of the
    batched workload (sides log-uniform in [64, 1024]) to 1e-10."""
    import torch

    import mgpoisson2d_b200.api as M
    from mgpoisson2d_b200 import workloads as W
    from mgpoisson2d_b200.types import BoxData

    torch.cuda.set_device(0)
    probs = [W.batch_problem_device(i) for i in range(a.batch)]
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_LOCKSTEP | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE
    flags |= M.FLAG_MIXED if a.mixed else 0
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, flags, nstreams=max(1, a.groups)) as b:
        b.set_tuning(a.groups, 1)
        phis = [BoxData.device_zeros(p[0], 1, 1) for p in probs]
        for k in range(a.warmup + 1):
            for ph in phis:
                ph.data.zero_()
            torch.cuda.synchronize()
            l0 = M.kernel_launch_count()
            t0 = time.perf_counter()
            reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, 200)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
    print(f"batch={a.batch} wall {dt * 1e3:.1f} ms ({a.batch / dt:.1f} solves/s), "
          f"V-cycles mean {sum(r.iterations for r in reps) / len(reps):.2f} max {max(r.iterations for r in reps)}, "
          f"{M.kernel_launch_count() - l0} launches")


if __name__ == "__main__":
    main()
