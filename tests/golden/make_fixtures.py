"""Generate the golden fixtures of the benchmark workloads from the CPU
oracle (oracle/mgp_oracle.c, a restatement of the reference's FP64 solve).

The reference (Fortran 90) cannot be compiled where these fixtures are made
(no Fortran compiler), so the fixtures hold the oracle's own FP64 solutions at
the workloads' full sizes, solved in the reference's lexicographic
Gauss-Seidel order (MGPoisson2D.f90:596-640, poisson2d.f90:1702-1812) with the
reference settings nu = 8/8/8, numcycles = 1 and the coupled Dirichlet
diagonal (without it the reference iteration diverges on every problem with
two adjacent Dirichlet sides).  The GPU tests compare the device's solutions
with them; they never run this script.

    python tests/golden/make_fixtures.py [identity128] [wavy1024] [wavy1024_colour]

identity128  128^2 identity map, homogeneous Dirichlet (workloads.identity_dirichlet):
             the whole solution, the relres history.
wavy1024  1024^2 wavy map with 64:1 stretching, Dirichlet x / Neumann y
          (workloads.wavy_stretched): norms of the whole solution, every 8th
          cell in each direction (16384 values), 16384 cells at seeded random
          positions, the relres history.  About four minutes on one core.
wavy1024_colour  the same solve in the device's colour order.

Each fixture also records checksums of its inputs, so a test can tell an
input that drifted (a different libm) from a solver that did.
"""
from __future__ import annotations

import ctypes
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mgpoisson2d_b200 import workloads as W  # noqa: E402
from mgpoisson2d_b200.types import BoxData  # noqa: E402
from oracle import oracle as O  # noqa: E402

NU = 8
TOL = 1e-10


def input_sums(geo, rhs):
    return np.array([rhs.interior().sum(), np.abs(rhs.interior()).sum(), geo.J.interior().sum(),
                     geo.Jgup_xx.interior().sum(), geo.Jgup_xy.interior().sum(), geo.Jgup_yx.interior().sum(),
                     geo.Jgup_yy.interior().sum()])


def solve(v, geo, rhs, bc, homog, maxiters, gs_order):
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(1)
    try:
        phi = BoxData(v, 1, 1)
        t0 = time.time()
        rep = O.vcycle(phi, rhs, geo, bc, homog, TOL, maxiters, smooth_down=NU, smooth_up=NU, smooth_bottom=NU,
                       gs_order=gs_order)
        dt = time.time() - t0
    finally:
        O.lib().or_set_dirichlet_coupled_diagonal(0)
    return phi.interior().copy(), rep, dt


def identity128():
    v, geo, rhs, bc, u = W.identity_dirichlet(128)
    sol, rep, dt = solve(v, geo, rhs, bc, True, 100, 0)
    out = os.path.join(HERE, "identity128.npz")
    np.savez_compressed(out, solution=sol, relres=rep.relres, iterations=rep.iterations, maxdepth=rep.maxdepth,
                        diverged=rep.diverged, inputs=input_sums(geo, rhs), seconds=dt,
                        err_max=np.abs(sol - u).max())
    print(f"identity128: {rep.iterations} V-cycles, relres {rep.final_relres:.3e}, {dt:.1f} s -> {out}")


def sample_points(n, count=16384, seed=8):
    rng = np.random.default_rng(seed)
    return rng.integers(0, n, count), rng.integers(0, n, count)


def wavy1024(gs_order=0):
    n = 1024
    v, geo, rhs, bc, _ = W.wavy_stretched(n)
    sol, rep, dt = solve(v, geo, rhs, bc, True, 2000, gs_order)
    si, sj = sample_points(n)
    name = "wavy1024.npz" if gs_order == 0 else "wavy1024_colour.npz"
    out = os.path.join(HERE, name)
    np.savez_compressed(out, strided=sol[::8, ::8].copy(), sample_i=si, sample_j=sj, sample=sol[si, sj],
                        l2=np.linalg.norm(sol), maxabs=np.abs(sol).max(), total=sol.sum(), relres=rep.relres,
                        iterations=rep.iterations, maxdepth=rep.maxdepth, diverged=rep.diverged,
                        inputs=input_sums(geo, rhs), seconds=dt, gs_order=gs_order)
    print(f"wavy1024 (gs_order {gs_order}): {rep.iterations} V-cycles, relres {rep.final_relres:.3e}, "
          f"{dt:.1f} s -> {out}")


if __name__ == "__main__":
    O.build()
    which = sys.argv[1:] or ["identity128", "wavy1024"]
    for w in which:
        if w == "identity128":
            identity128()
        elif w == "wavy1024":
            wavy1024(0)
        elif w == "wavy1024_colour":
            wavy1024(1)
        else:
            raise SystemExit(f"unknown fixture {w}")
