"""Failure detection without a GPU fault.

The reference stops the process on an allocation failure (MGPoisson2D.f90:441-443)
and undoes a correction whose residual grew (MG:630-639); it has no device
waits.  Here every failure comes back as a status code and the device context
stays usable:

* non-finite data -> MGP_EDIVERGED, through the Fortran-signature driver, the
  resident solver with its Krylov/mixed forms, the solve server, and both
  bottom-solver entry points (the allocating one and the no-allocation one
  report the same status);
* a request larger than the server's memory budget -> MGP_ENOMEM, for two such
  requests at once with nothing else running (no admission deadlock), and
  requests that fit one at a time are served in turn;
* a grid-barrier wait made to run out (one CTA of a cooperative grid exits
  before the barrier, a short limit) -> MGP_ETIMEOUT in bounded time, after
  which a normal solve still runs.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

from mgpoisson2d_b200 import workloads as W
from mgpoisson2d_b200.types import BoxData

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MGP_OK, MGP_ENOMEM, MGP_EDIVERGED, MGP_EMAXITER, MGP_ETIMEOUT = 0, 2, 3, 4, 5


@pytest.fixture(scope="module")
def M():
    assert torch.cuda.is_available(), "needs a CUDA device"
    import mgpoisson2d_b200.api as api
    return api


def _nan_problem(n=32):
    v, geo, rhs, bc, _ = W.identity_dirichlet(n)
    rhs.interior()[5, 7] = np.nan
    return v, geo, rhs, bc


def test_nan_rhs_fortran_driver(M):
    v, geo, rhs, bc = _nan_problem()
    with pytest.raises(M.MGPError) as ei:
        M.vcycle(BoxData(v, 1, 1), rhs, geo, bc, True, 1e-10, 10)
    assert ei.value.status == MGP_EDIVERGED


@pytest.mark.parametrize("flags", [0, 4 | 8, 32 | 8 | 16])   # plain; BiCGStab + mixed; GMRES + mixed + exact bottom
def test_nan_rhs_resident_solver(M, flags):
    v, geo, rhs, bc = _nan_problem(64)
    with M.Solver(v, geo, bc, M.KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | flags) as s:
        with pytest.raises(M.MGPError) as ei:
            s.vcycle(BoxData(v, 1, 1), rhs, bc, True, 1e-10, 10)
        assert ei.value.status == MGP_EDIVERGED
        # the same solver then solves a finite problem
        v2, geo2, rhs2, bc2, _ = W.identity_dirichlet(64)
        rep = s.vcycle(BoxData(v, 1, 1), rhs2, bc, True, 1e-10, 60)
        assert rep.final_relres <= 1e-10


def test_nan_rhs_server(M):
    v, geo, rhs, bc = _nan_problem()
    with M.Server(2, 0, M.FLAG_DIRICHLET_COUPLED_DIAG) as srv:
        t = srv.submit(v, geo, bc, BoxData(v, 1, 1), rhs, True, 1e-10, 10, key=7)
        with pytest.raises(M.MGPError) as ei:
            srv.wait(t)
        assert ei.value.status == MGP_EDIVERGED


def test_nan_rhs_bicgstab2_both_entry_points(M):
    """mgp_solve_bicgstab2 and mgp_solve_bicgstab2_noalloc return the same
    status on a non-finite right-hand side."""
    v, geo, rhs, bc = _nan_problem(24)
    inv = BoxData(v)
    M.compute_invdiags(inv, geo, bc, True)
    with pytest.raises(M.MGPError) as ea:
        M.solve_bicgstab2(BoxData(v, 1, 1), rhs, geo, bc, True, inv, 1e-10, 40, 3, True)
    with pytest.raises(M.MGPError) as eb:
        M.solve_bicgstab2_noalloc(BoxData(v, 1, 1).to_device(), rhs.to_device(), geo.to_device(), bc, True,
                                  inv.to_device(), 1e-10, 40, 3, True)
    assert ea.value.status == eb.value.status == MGP_EDIVERGED


def _run_with_deadline(fn, seconds):
    """Run fn in a thread; fail (instead of hanging the suite) if it does not return."""
    out = {}

    def body():
        try:
            out["value"] = fn()
        except BaseException as e:   # noqa: BLE001
            out["error"] = e
    th = threading.Thread(target=body, daemon=True)
    th.start()
    th.join(seconds)
    assert not th.is_alive(), f"did not return within {seconds} s"
    if "error" in out:
        raise out["error"]
    return out.get("value")


def test_server_refuses_requests_larger_than_the_budget(M):
    """Two requests that can never fit a 1 MB budget, submitted together to two
    workers with nothing else running: both come back MGP_ENOMEM, and the
    server shuts down."""
    v, geo, rhs, bc, _ = W.identity_dirichlet(64)

    def run():
        srv = M.Server(2, 1 << 20, M.FLAG_DIRICHLET_COUPLED_DIAG)
        try:
            tickets = [srv.submit(v, geo, bc, BoxData(v, 1, 1), rhs, True, 1e-10, 20) for _ in range(2)]
            codes = []
            for t in tickets:
                try:
                    srv.wait(t)
                    codes.append(MGP_OK)
                except M.MGPError as e:
                    codes.append(e.status)
            return codes
        finally:
            srv.close()
    assert _run_with_deadline(run, 120) == [MGP_ENOMEM, MGP_ENOMEM]


def test_server_serialises_requests_that_fit_one_at_a_time(M):
    """A budget that holds one 64^2 hierarchy but not two: four requests on two
    workers are admitted one after another, and each is solved."""
    v, geo, rhs, bc, _ = W.identity_dirichlet(64)
    budget = 14 << 20   # the server's estimate for 64^2 is ~8.7 MB

    def run():
        srv = M.Server(2, budget, M.FLAG_DIRICHLET_COUPLED_DIAG)
        try:
            phis = [BoxData(v, 1, 1) for _ in range(4)]
            tickets = [srv.submit(v, geo, bc, p, rhs, True, 1e-10, 40) for p in phis]
            reps = [srv.wait(t)[0] for t in tickets]
            return reps, phis
        finally:
            srv.close()
    reps, phis = _run_with_deadline(run, 120)
    for r, p in zip(reps, phis):
        assert r.final_relres <= 1e-10
        assert np.array_equal(p.interior(), phis[0].interior())


def test_grid_barrier_wait_runs_out_and_returns(M):
    """One CTA of a cooperative grid never arrives at the barrier: the others'
    waits end after the 50 ms limit with MGP_ETIMEOUT, every later barrier is
    skipped (64 barriers do not cost 64 limits), and the context stays usable."""
    st, sec = M.selftest_grid_barrier(8, 3, 64, 0.05)
    assert st == MGP_ETIMEOUT, st
    assert 0.04 <= sec < 1.0, sec
    st, sec = M.selftest_grid_barrier(8, -1, 64, 0.05)
    assert st == MGP_OK and sec < 0.05, (st, sec)
    v, geo, rhs, bc, _ = W.identity_dirichlet(32)
    old = M.set_flags(M.FLAG_DIRICHLET_COUPLED_DIAG)
    try:
        rep = M.vcycle(BoxData(v, 1, 1), rhs, geo, bc, True, 1e-10, 30)
    finally:
        M.set_flags(old)
    assert rep.final_relres <= 1e-10


def test_grid_barrier_selftest_rejects_bad_arguments(M):
    assert M.selftest_grid_barrier(1, -1, 4, 0.05)[0] == 1          # MGP_EINVAL: one CTA
    assert M.selftest_grid_barrier(4, 4, 4, 0.05)[0] == 1           # skip index out of range
    assert M.selftest_grid_barrier(4, -1, 4, 0.0)[0] == 1           # no limit
    assert M.selftest_grid_barrier(100000, -1, 4, 0.05)[0] == 1     # more CTAs than stay resident


@pytest.mark.parametrize("flags", [0, 4 | 8, 32 | 8 | 16 | 64])   # plain; BiCGStab + mixed; GMRES + exact bottom
def test_maxiter_status_only_with_the_flag(M, flags):
    """A solve capped by maxiters returns OK as the Fortran drivers do, and
    MGP_EMAXITER with MGP_FLAG_REPORT_MAXITER; the iterate is the same either way,
    and a solve that reaches tol under the flag still returns OK."""
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    base = M.FLAG_DIRICHLET_COUPLED_DIAG | flags
    with M.Solver(v, geo, bc, M.KIND_MG, base) as s:
        phi0 = BoxData(v, 1, 1)
        rep0 = s.vcycle(phi0, rhs, bc, True, 1e-10, 2)
    assert rep0.iterations == 2 and rep0.final_relres > 1e-10
    with M.Solver(v, geo, bc, M.KIND_MG, base | M.FLAG_REPORT_MAXITER) as s:
        phi1 = BoxData(v, 1, 1)
        with pytest.raises(M.MGPError) as ei:
            s.vcycle(phi1, rhs, bc, True, 1e-10, 2)
        assert ei.value.status == MGP_EMAXITER
        assert np.array_equal(phi1.interior(), phi0.interior())
        rep = s.vcycle(BoxData(v, 1, 1), rhs, bc, True, 1e-10, 400)
        assert rep.final_relres <= 1e-10


def test_maxiter_status_in_a_lockstep_batch(M):
    """Under lockstep each report carries its own status: the problems that
    reach tol within maxiters report OK, the rest MGP_EMAXITER, and the call
    returns MGP_EMAXITER."""
    probs = [W.batch_problem(i) for i in (0, 1, 2, 5, 6, 7, 8, 13, 14, 20)]
    phis = [BoxData(p[0], 1, 1) for p in probs]
    fl = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_LOCKSTEP
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, fl) as b:
        reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, 60)
    its = sorted(r.iterations for r in reps)
    cap = its[len(its) // 2]
    assert its[0] <= cap < its[-1]
    phis = [BoxData(p[0], 1, 1) for p in probs]
    with M.Batch([(p[0], p[1], p[3]) for p in probs], M.KIND_MG, fl | M.FLAG_REPORT_MAXITER) as b:
        with pytest.raises(M.MGPError) as ei:
            b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, cap)
        assert ei.value.status == MGP_EMAXITER
        st = b.last_statuses()
    for r, s in zip(reps, st):
        assert s == (MGP_OK if r.iterations <= cap else MGP_EMAXITER)
