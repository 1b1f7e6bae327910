"""Lockstep batches (MGP_FLAG_LOCKSTEP): every V-cycle phase of all unconverged
problems in one launch.  Each problem's solution must have the bits of its own
stationary V-cycle (the resident solver without the flag), whatever else is in
the batch and whenever the others converge; the V-cycle counts must be the
same; and the solutions must agree with the CPU oracle in both sweep orders
(problems of the batched workload, whose uneven sides give (2,1) and (1,2)
levels)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from mgpoisson2d_b200 import workloads as W
from mgpoisson2d_b200.types import BoxData
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# problems of the batched workload: 2, 5, 6, 8 coarsen (2,1) first, 7 and 13 (1,2); sides 64..1008
PROBS = [0, 1, 2, 5, 6, 7, 8, 13, 14, 20]


@pytest.fixture(scope="module")
def M():
    assert torch.cuda.is_available(), "needs a CUDA device"
    import mgpoisson2d_b200.api as api
    return api


@pytest.fixture(scope="module")
def probs():
    return [W.batch_problem(i) for i in PROBS]


def _alone(M, prob, flags, maxiters=60):
    v, geo, rhs, bc = prob
    with M.Solver(v, geo, bc, M.KIND_MG, flags) as s:
        phi = BoxData(v, 1, 1)
        rep = s.vcycle(phi, rhs, bc, True, 1e-10, maxiters)
    return rep, phi.interior().copy()


def _lockstep(M, probs, flags, maxiters=60):
    phis = [BoxData(p[0], 1, 1) for p in probs]
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, flags | M.FLAG_LOCKSTEP, nstreams=2) as b:
        reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, maxiters)
    return reps, [p.interior().copy() for p in phis]


@pytest.mark.parametrize("mixed,bottom", [(False, "reference"), (True, "reference"), (True, "large")])
def test_lockstep_same_bits_as_each_problem_alone(M, probs, mixed, bottom):
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | (M.FLAG_MIXED if mixed else 0)
    if bottom == "large":   # the exact bottom on the coarse-cycle level, a batched matrix-vector product
        flags |= M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE
    reps, sols = _lockstep(M, probs, flags)
    its = set()
    for k, prob in enumerate(probs):
        ra, sa = _alone(M, prob, flags)
        assert reps[k].iterations == ra.iterations, (PROBS[k], reps[k].iterations, ra.iterations)
        assert reps[k].final_relres <= 1e-10 and not reps[k].diverged
        np.testing.assert_allclose(reps[k].relres, ra.relres, rtol=1e-12, atol=0)
        assert np.array_equal(sols[k].view(np.uint64), sa.view(np.uint64)), PROBS[k]
        its.add(ra.iterations)
    assert len(its) > 1   # the problems leave the batch at different V-cycles


def test_lockstep_same_alone_and_in_the_mix(M, probs):
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_MIXED
    _, mix = _lockstep(M, probs, flags)
    for k in (0, 3, 7):
        _, one = _lockstep(M, [probs[k]], flags)
        assert np.array_equal(one[0].view(np.uint64), mix[k].view(np.uint64))


@pytest.mark.parametrize("mixed,large", [(False, False), (True, False), (True, True)])
def test_lockstep_against_oracle(M, probs, mixed, large):
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | (M.FLAG_MIXED if mixed else 0)
    flags |= M.FLAG_DIRECT_LARGE if large else 0
    reps, sols = _lockstep(M, probs, flags)
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(1)
    try:
        for k, (v, geo, rhs, bc) in enumerate(probs):
            assert reps[k].final_relres <= 1e-10
            for order in (1, 0):
                po = BoxData(v, 1, 1)
                ro = O.vcycle(po, rhs, geo, bc, True, 1e-10, 200, gs_order=order)
                ref = po.interior()
                rel_l2 = np.linalg.norm(sols[k] - ref) / np.linalg.norm(ref)
                rel_max = np.abs(sols[k] - ref).max() / np.abs(ref).max()
                assert rel_l2 <= 1e-8 and rel_max <= 1e-7, (PROBS[k], order, rel_l2, rel_max)
    finally:
        O.lib().or_set_dirichlet_coupled_diagonal(0)


def test_lockstep_falls_back_for_krylov_and_odd_counts(M, probs):
    """Flags or counts the lockstep path does not serve run the concurrent
    per-problem path: same answers as solving alone."""
    sub = probs[:3]
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV
    reps, sols = _lockstep(M, sub, flags)
    for k, prob in enumerate(sub):
        ra, sa = _alone(M, prob, flags)
        assert np.array_equal(sols[k], sa)
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG
    phis = [BoxData(p[0], 1, 1) for p in sub]
    with M.Batch([(p[0], p[1], p[3]) for p in sub], M.KIND_MG, flags | M.FLAG_LOCKSTEP) as b:
        reps = b.vcycle(phis, [p[2] for p in sub], [p[3] for p in sub], True, 1e-10, 60, 1, 7, 7, 7)
    for k, prob in enumerate(sub):
        v, geo, rhs, bc = prob
        with M.Solver(v, geo, bc, M.KIND_MG, flags) as s:
            phi = BoxData(v, 1, 1)
            s.vcycle(phi, rhs, bc, True, 1e-10, 60, 1, 7, 7, 7)
        assert np.array_equal(phis[k].interior(), phi.interior())


def _solve_with(M, probs, flags, groups, pairs):
    phis = [BoxData(p[0], 1, 1) for p in probs]
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, flags | M.FLAG_LOCKSTEP, nstreams=4) as b:
        b.set_tuning(groups, pairs)
        assert b.tuning() == {"groups": groups, "pairs": pairs}
        reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, 60)
    return [r.iterations for r in reps], [p.interior().copy() for p in phis]


def test_lockstep_tuning_changes_no_bits(M, probs):
    """Concurrent groups and two sweeps per launch change speed only: the
    same V-cycle counts and the same bits for every setting."""
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_MIXED | M.FLAG_DIRECT_COARSE
    its0, sols0 = _solve_with(M, probs, flags, 1, 0)
    for groups, pairs in ((2, 0), (4, 1), (1, 1), (3, 1)):
        its, sols = _solve_with(M, probs, flags, groups, pairs)
        assert its == its0
        for a, b in zip(sols, sols0):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_lockstep_autotune_keeps_fastest_and_caches(M, probs, tmp_path):
    import json
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_MIXED
    cache = str(tmp_path / "tune.json")
    sub = probs[:6]
    phis = [BoxData(p[0], 1, 1) for p in sub]
    args = ([p[2] for p in sub], [p[3] for p in sub], True, 1e-10, 60)
    with M.Batch([(p[0], p[1], p[3]) for p in sub], M.KIND_MG, flags | M.FLAG_LOCKSTEP, nstreams=4) as b:
        got = b.autotune(phis, *args, cache_path=cache, key="six")
        assert not got["cached"] and len(got["seconds"]) == 6
        best = min(got["seconds"], key=got["seconds"].get)
        assert best == f"{got['groups']},{got['pairs']}" and b.tuning() == {"groups": got["groups"], "pairs": got["pairs"]}
    assert json.load(open(cache))["six"]["groups"] == got["groups"]
    with M.Batch([(p[0], p[1], p[3]) for p in sub], M.KIND_MG, flags | M.FLAG_LOCKSTEP, nstreams=4) as b:
        again = b.autotune(phis, *args, cache_path=cache, key="six")
        assert again["cached"] and b.tuning() == {"groups": got["groups"], "pairs": got["pairs"]}


def test_cluster_coarse_cycle_same_bits_as_lockstep(M):
    """A coarse level of 2 K - 8 K cells that one CTA cannot stage (sides
    8 x 61 and 8 x 45 stop the schedule at 61 x 45) runs on a thread-block
    cluster when the problem is solved alone and on one CTA in a lockstep
    batch; the cluster keeps the one-CTA reduction order, so the bits agree."""
    probs = [W.skew_stretched(360, nx=488), W.skew_stretched(488, nx=360)]
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_MIXED
    alone = []
    for v, geo, rhs, bc, _ in probs:
        with M.Solver(v, geo, bc, M.KIND_MG, flags) as s:
            phi = BoxData(v, 1, 1)
            rep = s.vcycle(phi, rhs, bc, False, 1e-10, 60)
        assert rep.final_relres <= 1e-10
        alone.append((rep.iterations, phi.interior().copy()))
    phis = [BoxData(p[0], 1, 1) for p in probs]
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, flags | M.FLAG_LOCKSTEP) as b:
        reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], False, 1e-10, 60)
    for k in range(2):
        assert reps[k].iterations == alone[k][0]
        assert np.array_equal(phis[k].interior().view(np.uint64), alone[k][1].view(np.uint64))
