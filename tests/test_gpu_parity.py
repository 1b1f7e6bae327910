"""CUDA library vs the CPU oracle on the same seeded inputs.

Operator-level results must be bit-identical: both sides evaluate each cell
with the same FP64 operations in the same order (no FMA contraction on either
side).  Solves are compared against the oracle run in the device's colour
order (tight tolerance: only reduction order differs) and against the oracle
run in the reference's lexicographic order (converged-solution tolerance).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import BC_CASES, hierarchy_geo, rand_bc, rand_field, rand_geo, same
from mgpoisson2d_b200.types import (BCMODE_LAH, BCMODE_UNIFORM, BCTYPE_DIRI, BCTYPE_EXTRAP0, BCTYPE_EXTRAP1,
                                    BCTYPE_EXTRAP2, BCTYPE_NEUM, BCTYPE_NONE, BD_CELL, BD_NODE, KIND_DD, KIND_MG,
                                    BdryData, Box, BoxData)
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def M():
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import mgpoisson2d_b200.api as api
    return api


SIZES = [(16, 12), (9, 7), (24, 24)]


def _problem(case, nx, ny, seed):
    rng = np.random.default_rng(seed)
    v = Box.of_size(nx, ny)
    types, modes = BC_CASES[case]
    if case in ("NNNN-NU",) and ny > nx:
        pytest.skip("north Neumann data is read at index jhi, which needs ny <= nx")
    return v, rand_geo(v, rng), rand_field(v, rng), rand_bc(v, types, modes, rng), rng


@pytest.mark.parametrize("case", list(BC_CASES))
@pytest.mark.parametrize("nx,ny", SIZES)
@pytest.mark.parametrize("homog", [False, True])
def test_laplacian_bitexact(M, case, nx, ny, homog):
    v, geo, phi, bc, rng = _problem(case, nx, ny, 11)
    lap_o, lap_d = BoxData(v), BoxData(v)
    phi_o, phi_d = phi.copy(), phi.copy()
    O.compute_laplacian(lap_o, phi_o, geo, bc, homog)
    M.compute_laplacian(lap_d, phi_d, geo, bc, homog)
    assert same(lap_o.data, lap_d.data)
    assert same(phi_o.data, phi_d.data)   # ghost state after the call


@pytest.mark.parametrize("case", ["DDDD-U", "NNNN-NU", "DNND-mixed"])
@pytest.mark.parametrize("jscale", [False, True])
def test_residual_bitexact(M, case, jscale):
    v, geo, phi, bc, rng = _problem(case, 16, 12, 12)
    rhs = rand_field(v, rng, 0)
    r_o, r_d = BoxData(v), BoxData(v)
    O.compute_residual(r_o, rhs, phi.copy(), geo, bc, False, jscale)
    M.compute_residual(r_d, rhs, phi.copy(), geo, bc, False, jscale)
    assert same(r_o.data, r_d.data)


@pytest.mark.parametrize("case", list(BC_CASES))
@pytest.mark.parametrize("coupled", [0, 1])
def test_invdiags_bitexact(M, case, coupled):
    import ctypes
    v, geo, phi, bc, rng = _problem(case, 16, 12, 13)
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(coupled)
    old = M.set_flags(coupled)
    try:
        d_o, d_d = BoxData(v), BoxData(v)
        O.compute_invdiags(d_o, geo, bc, True)
        M.compute_invdiags(d_d, geo, bc, True)
        assert same(d_o.data, d_d.data)
    finally:
        M.set_flags(old)
        O.lib().or_set_dirichlet_coupled_diagonal(0)


FILL_TYPES = [
    ([BCTYPE_DIRI] * 4, [BCMODE_UNIFORM] * 4),
    ([BCTYPE_NEUM] * 4, [BCMODE_UNIFORM] * 4),
    ([BCTYPE_NEUM] * 4, [1] * 4),
    ([BCTYPE_NEUM, BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_DIRI], [1, 0, 0, 1]),
    ([BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_DIRI, BCTYPE_NEUM], [BCMODE_LAH] * 4),
    ([BCTYPE_EXTRAP0, BCTYPE_EXTRAP1, BCTYPE_EXTRAP2, BCTYPE_NONE], [0] * 4),
    ([2, 2, BCTYPE_DIRI, BCTYPE_NEUM], [0, 0, 1, 0]),
    ([BCTYPE_NEUM, BCTYPE_DIRI, 2, 2], [0, 1, 0, 0]),
]


@pytest.mark.parametrize("k", range(len(FILL_TYPES)))
@pytest.mark.parametrize("homog", [False, True])
@pytest.mark.parametrize("do_neum", [False, True])
def test_fill_ghosts_bitexact(M, k, homog, do_neum):
    types, modes = FILL_TYPES[k]
    rng = np.random.default_rng(100 + k)
    v = Box.of_size(12, 10)
    geo = rand_geo(v, rng)
    phi = rand_field(v, rng)
    bc = rand_bc(v, types, modes, rng)
    a, b = phi.copy(), phi.copy()
    O.fill_ghosts(a, bc, geo, homog, do_neum)
    M.fill_ghosts(b, bc, geo, homog, do_neum)
    assert same(a.data, b.data)


@pytest.mark.parametrize("order", range(4))
def test_extrapolate_ghosts_bitexact(M, order):
    rng = np.random.default_rng(5)
    v = Box.of_size(10, 9)
    phi = rand_field(v, rng)
    a, b = phi.copy(), phi.copy()
    O.extrapolate_ghosts(a, order)
    M.extrapolate_ghosts(b, order)
    assert same(a.data, b.data)


@pytest.mark.parametrize("case", ["DDDD-U", "NNNN-NU", "DNND-mixed", "PPDD"])
@pytest.mark.parametrize("omega", [1.0, 2.0 / 3.0])
def test_relax_gs_colour_bitexact(M, case, omega):
    v, geo, phi, bc, rng = _problem(case, 16, 12, 14)
    rhs = rand_field(v, rng, 0)
    inv = BoxData(v)
    O.compute_invdiags(inv, geo, bc, True)
    a, b = phi.copy(), phi.copy()
    O.relax_gs(a, rhs, geo, bc, True, inv, omega, -1.0, 3, False, 0, gs_order=1)
    M.relax_gs(b, rhs, geo, bc, True, inv, omega, -1.0, 3, False, 0)
    assert same(a.data, b.data)


@pytest.mark.parametrize("case", ["DDDD-U", "NNNN-NU", "DNND-mixed", "PPDD", "DDPP", "PPPP", "DDNN-U"])
@pytest.mark.parametrize("nx,ny", [(200, 150), (300, 262), (64, 96), (257, 33)])
def test_relax_gs_multitile_bitexact(M, case, nx, ny):
    """Grids of many tiles (sizes not multiples of the tile): the halo
    recomputation of the one-launch sweep must reproduce the sub-pass order."""
    if case == "NNNN-NU" and ny > nx:
        pytest.skip("north Neumann data is read at index jhi, which needs ny <= nx")
    v, geo, phi, bc, rng = _problem(case, nx, ny, 15)
    rhs = rand_field(v, rng, 0)
    inv = BoxData(v)
    O.compute_invdiags(inv, geo, bc, True)
    a, b = phi.copy(), phi.copy()
    O.relax_gs(a, rhs, geo, bc, True, inv, 1.0, -1.0, 3, False, 0, gs_order=1)
    M.relax_gs(b, rhs, geo, bc, True, inv, 1.0, -1.0, 3, False, 0)
    assert same(a.data, b.data)


@pytest.mark.parametrize("offi,offj", [(1, 1), (0, 1), (1, 0), (0, 0)])
@pytest.mark.parametrize("ref", [(2, 2), (2, 1), (1, 2)])
def test_restrict_bitexact(M, offi, offj, ref):
    rng = np.random.default_rng(7)
    v = Box.of_size(16, 12)
    c = v.coarsened(*ref)
    f = rand_field(v, rng, 0, offi, offj)
    a, b = BoxData(c, 0, 0, offi, offj), BoxData(c, 0, 0, offi, offj)
    O.restrict(f, a)
    M.restrict(f, b)
    assert same(a.data, b.data)


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("ref", [(2, 2), (2, 1), (1, 2)])
@pytest.mark.parametrize("types", [[BCTYPE_DIRI] * 4, [BCTYPE_DIRI, BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_NEUM]])
def test_prolong_bitexact(M, order, ref, types):
    rng = np.random.default_rng(8)
    v = Box.of_size(16, 12)
    geo = rand_geo(v, rng)
    c = v.coarsened(*ref)
    cgeo = rand_geo(c, rng)
    fine = rand_field(v, rng)
    crse = rand_field(c, rng)
    cbc = BdryData.uniform(c, types)
    fa, fb, ca, cb = fine.copy(), fine.copy(), crse.copy(), crse.copy()
    O.prolong(fa, ca, geo, cgeo, cbc, order)
    M.prolong(fb, cb, geo, cgeo, cbc, order)
    assert same(fa.data, fb.data)
    assert same(ca.data, cb.data)


def test_prolong_remove_mean(M):
    """All-Neumann coarse BCs remove the J-weighted mean (MG:371-383); the
    mean is a reduction, so equality is to rounding."""
    rng = np.random.default_rng(9)
    v = Box.of_size(16, 16)
    geo = rand_geo(v, rng)
    c, cgeo = hierarchy_geo(v, geo, O.restrict)
    fine, crse = rand_field(v, rng), rand_field(c, rng)
    cbc = BdryData.uniform(c, [BCTYPE_NEUM] * 4)
    fa, fb = fine.copy(), fine.copy()
    O.prolong(fa, crse.copy(), geo, cgeo, cbc, 1)
    M.prolong(fb, crse.copy(), geo, cgeo, cbc, 1)
    np.testing.assert_allclose(fb.interior(), fa.interior(), rtol=0, atol=1e-13)


def test_norms(M):
    rng = np.random.default_rng(10)
    v = Box.of_size(33, 17)
    a, b = rand_field(v, rng, 0), rand_field(v, rng, 0)
    for p in (0, 1, 2):
        np.testing.assert_allclose(M.pnorm(a, p), O.pnorm(a, p), rtol=1e-13)
    np.testing.assert_allclose(M.inner_prod(a, b), O.inner_prod(a, b), rtol=1e-12)


def test_bicgstab(M):
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(8)
    inv = BoxData(v)
    O.compute_invdiags(inv, geo, bc, True)
    a, b = BoxData(v, 1, 1), BoxData(v, 1, 1)
    O.solve_bicgstab2(a, rhs, geo, bc, True, inv, 1e-10, 80, 5, False, 0, gs_order=1)
    M.solve_bicgstab2(b, rhs, geo, bc, True, inv, 1e-10, 80, 5, False, 0)
    np.testing.assert_allclose(b.interior(), a.interior(), rtol=1e-9, atol=1e-12)


# ---------------------------------------------------------------------------
# Solves
# ---------------------------------------------------------------------------
def _set_coupled(M, on):
    import ctypes
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(int(on))
    return M.set_flags(int(on))


@pytest.mark.parametrize("n", [32, 64, 128, 256])
def test_vcycle_matches_oracle(M, n):
    from mgpoisson2d_b200 import workloads as W
    old = _set_coupled(M, True)
    try:
        v, geo, rhs, bc, u = W.identity_dirichlet(n)
        pa, pb, pc = BoxData(v, 1, 1), BoxData(v, 1, 1), BoxData(v, 1, 1)
        ra = O.vcycle(pa, rhs, geo, bc, True, 1e-10, 30, gs_order=1)
        rb = M.vcycle(pb, rhs, geo, bc, True, 1e-10, 30)
        rc = O.vcycle(pc, rhs, geo, bc, True, 1e-10, 30, gs_order=0)
    finally:
        _set_coupled(M, old)
    assert rb.iterations == ra.iterations
    np.testing.assert_allclose(rb.relres, ra.relres, rtol=1e-7, atol=1e-14)
    np.testing.assert_allclose(pb.interior(), pa.interior(), rtol=0, atol=1e-11 * np.abs(pa.interior()).max())
    # against the reference's lexicographic order: same converged solution
    assert rb.relres[-1] <= 1e-10 and rc.relres[-1] <= 1e-10
    err = pb.interior() - pc.interior()
    assert np.linalg.norm(err) / np.linalg.norm(pc.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(pc.interior()).max() < 1e-7


def test_vcycle_reference_diverges_like_oracle(M):
    """With the reference's own diagonal the V-cycle diverges on a Dirichlet
    problem and stops after undoing the correction (MG:630-639); both sides
    must take that same path."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(32)
    pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
    ra = O.vcycle(pa, rhs, geo, bc, True, 1e-10, 20, gs_order=1)
    rb = M.vcycle(pb, rhs, geo, bc, True, 1e-10, 20)
    assert ra.diverged and rb.diverged and ra.iterations == rb.iterations == 1
    np.testing.assert_allclose(rb.relres, ra.relres, rtol=1e-9)


def test_fmg_terrain_neumann(M):
    """The reference's solver test: FMG on the terrain map with all-Neumann data."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, soln = W.terrain_neumann(64, O.boundary_fluxes, O.compute_laplacian)
    pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
    ra = O.fmg(pa, rhs, geo, bc, False, 1e-30, 3, gs_order=1)
    rb = M.fmg(pb, rhs, geo, bc, False, 1e-30, 3)
    np.testing.assert_allclose(rb.relres, ra.relres, rtol=1e-6)
    np.testing.assert_allclose(pb.interior(), pa.interior(), rtol=0, atol=1e-10 * np.abs(pa.interior()).max())


def test_dc_vcycle(M):
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(64)
    f = rhs.copy()
    f.interior()[:] /= geo.J.interior()
    fa, fb = f.copy(), f.copy()
    pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
    ra = O.dc_vcycle(pa, fa, geo, bc, True, 1e-10, 60, smooth_down=8, smooth_up=8, smooth_bottom=8, gs_order=1)
    rb = M.dc_vcycle(pb, fb, geo, bc, True, 1e-10, 60, smooth_down=8, smooth_up=8, smooth_bottom=8)
    assert rb.iterations == ra.iterations
    np.testing.assert_allclose(rb.relres, ra.relres, rtol=1e-6, atol=1e-14)
    np.testing.assert_allclose(pb.interior(), pa.interior(), rtol=0, atol=1e-10 * np.abs(pa.interior()).max())
    assert same(fa.data, fb.data)   # rhs*J/J written back exactly like the reference


@pytest.mark.parametrize("kind", ["mg", "dd"])
def test_grid_coarse_cycle_matches_oracle(M, kind):
    """Depth capped at 1 on 256^2 leaves a 128 x 128 bottom (16384 cells, as an
    odd side leaves on many grids): the coarse cycle -- the bottom's 8 sweeps
    and BiCGStab -- then runs as a cooperative grid of CTAs.  Its reductions
    combine in another order than the oracle's, and BiCGStab's iterates
    amplify that rounding: the bottom solve (to 1e-6) differs at that level,
    so the histories agree to 1e-3 relative, not to rounding.  Same V-cycle
    count, and the converged solutions agree to 1e-9 of the maximum."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(256)
    pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
    if kind == "mg":
        old = _set_coupled(M, True)
        try:
            ra = O.vcycle(pa, rhs, geo, bc, True, 1e-10, 30, maxdepth_user=1, gs_order=1)
            rb = M.vcycle(pb, rhs, geo, bc, True, 1e-10, 30, maxdepth_user=1)
        finally:
            _set_coupled(M, old)
    else:
        f = rhs.copy()
        f.interior()[:] /= geo.J.interior()
        fa, fb = f.copy(), f.copy()
        ra = O.dc_vcycle(pa, fa, geo, bc, True, 1e-10, 60, maxdepth_user=1, smooth_down=8, smooth_up=8,
                         smooth_bottom=8, gs_order=1)
        rb = M.dc_vcycle(pb, fb, geo, bc, True, 1e-10, 60, maxdepth_user=1, smooth_down=8, smooth_up=8,
                         smooth_bottom=8)
    assert rb.status == 0 and rb.maxdepth == 1
    assert rb.iterations == ra.iterations
    np.testing.assert_allclose(rb.relres, ra.relres, rtol=1e-3, atol=1e-14)
    np.testing.assert_allclose(pb.interior(), pa.interior(), rtol=0, atol=1e-9 * np.abs(pa.interior()).max())


def test_grid_coarse_cycle_in_resident_solver(M):
    """The resident solver with the grid coarse cycle inside its replayed
    V-cycle graphs (BiCGStab-accelerated): converges, and a second solve on
    the same hierarchy gives the same bits."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(256)
    fl = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV
    outs = []
    with M.Solver(v, geo, bc, KIND_MG, fl, maxdepth_user=1) as s:
        for _ in range(2):
            p = BoxData(v, 1, 1)
            r = s.vcycle(p, rhs, bc, True, 1e-10, 100)
            assert r.status == 0 and r.final_relres <= 1e-10
            outs.append(p)
    assert same(outs[0].data, outs[1].data)


def test_resident_solver_equals_oneshot_and_device_arrays(M):
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.wavy_stretched(64)
    old = M.set_flags(M.FLAG_DIRICHLET_COUPLED_DIAG)
    try:
        pa = BoxData(v, 1, 1)
        ra = M.vcycle(pa, rhs, geo, bc, True, 1e-10, 15)
    finally:
        M.set_flags(old)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG) as s:
        for _ in range(2):   # a second solve on the same hierarchy gives the same bits
            pb = BoxData(v, 1, 1)
            rb = s.vcycle(pb, rhs, bc, True, 1e-10, 15)
            assert same(pa.data, pb.data) and np.array_equal(ra.relres, rb.relres)
        pd, rd_ = BoxData(v, 1, 1).to_device(), rhs.to_device()
        rd = s.vcycle(pd, rd_, bc, True, 1e-10, 15)
        assert same(pa.data, pd.to_host().data) and np.array_equal(ra.relres, rd.relres)


# ---------------------------------------------------------------------------
# BiCGStab-accelerated V-cycle (MGP_FLAG_KRYLOV; no reference counterpart)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n", [64, 128])
def test_krylov_vcycle_matches_oracle(M, n):
    """Same V-cycles as the oracle (bit-exact in the device order); the inner
    products are summed in a different order, so the histories agree to
    rounding.  The converged solution must match the plain V-cycle's."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(n)
    old = _set_coupled(M, True)
    try:
        pa, pc = BoxData(v, 1, 1), BoxData(v, 1, 1)
        ra = O.krylov_vcycle(pa, rhs, geo, bc, True, 1e-10, 400)
        O.vcycle(pc, rhs, geo, bc, True, 1e-10, 2000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV) as s:
        pb = BoxData(v, 1, 1)
        rb = s.vcycle(pb, rhs, bc, True, 1e-10, 400)
        pd = BoxData(v, 1, 1)
        rd = s.vcycle(pd, rhs, bc, True, 1e-10, 400)
    assert rb.status == 0 and rb.final_relres <= 1e-10 and rb.relres[-1] == rb.final_relres
    assert abs(rb.iterations - (len(ra) - 1)) <= 2
    k = min(12, len(ra), len(rb.relres))
    np.testing.assert_allclose(rb.relres[:k], ra[:k], rtol=1e-6)
    assert same(pb.data, pd.data) and np.array_equal(rb.relres, rd.relres)   # deterministic
    for ref in (pa, pc):
        err = pb.interior() - ref.interior()
        assert np.linalg.norm(err) / np.linalg.norm(ref.interior()) < 1e-8
    np.testing.assert_allclose(pb.data, pa.data, rtol=0, atol=1e-9 * np.abs(pa.data).max())   # ghosts too


def test_krylov_oneshot_device_arrays_and_maxiters(M):
    """The flag through mgp_set_flags and the one-shot driver, device arrays,
    and the V-cycle budget: an odd maxiters stops after the first half step
    with the true residual as the last entry."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, u = W.identity_dirichlet(64)
    old = M.set_flags(M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV)
    try:
        pa = BoxData(v, 1, 1)
        ra = M.vcycle(pa, rhs, geo, bc, True, 1e-11, 50)
        pd, rd_ = BoxData(v, 1, 1).to_device(), rhs.to_device()
        rd = M.vcycle(pd, rd_, geo, bc, True, 1e-11, 50)
        pe = BoxData(v, 1, 1)
        re = M.vcycle(pe, rhs, geo, bc, True, 1e-30, 3)
    finally:
        M.set_flags(old)
    assert ra.final_relres <= 1e-11 and ra.iterations < 20
    assert same(pa.data, pd.to_host().data) and np.array_equal(ra.relres, rd.relres)
    assert re.iterations == 3 and len(re.relres) == 4 and re.final_relres == re.relres[-1] > 0
    oa = BoxData(v, 1, 1)
    O.lib().or_set_dirichlet_coupled_diagonal(1)
    try:
        ro = O.krylov_vcycle(oa, rhs, geo, bc, True, 1e-30, 3)
    finally:
        O.lib().or_set_dirichlet_coupled_diagonal(0)
    np.testing.assert_allclose(re.relres, ro, rtol=1e-7)
    np.testing.assert_allclose(pe.data, oa.data, rtol=0, atol=1e-10 * np.abs(oa.data).max())


# ---------------------------------------------------------------------------
# Mixed precision (MGP_FLAG_MIXED; no reference counterpart): FP32 grid levels
# inside the FP64 outer iteration
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("krylov", [False, True])
def test_mixed_vcycle_converges_to_fp64_solution(M, krylov):
    """The outer iteration and its residual stay FP64, so the mixed solve must
    reach the same 1e-10 relative residual and the same solution as the FP64
    oracle, in about as many V-cycles as the FP64 device solve."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    base = M.FLAG_DIRICHLET_COUPLED_DIAG | (M.FLAG_KRYLOV if krylov else 0)
    old = _set_coupled(M, True)
    try:
        po = BoxData(v, 1, 1)
        O.vcycle(po, rhs, geo, bc, True, 1e-11, 3000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, base) as s:
        p64 = BoxData(v, 1, 1)
        r64 = s.vcycle(p64, rhs, bc, True, 1e-10, 3000)
    with M.Solver(v, geo, bc, KIND_MG, base | M.FLAG_MIXED) as s:
        p32 = BoxData(v, 1, 1)
        r32 = s.vcycle(p32, rhs, bc, True, 1e-10, 3000)
        p32b = BoxData(v, 1, 1)
        r32b = s.vcycle(p32b, rhs, bc, True, 1e-10, 3000)
    assert r32.status == 0 and not r32.diverged and r32.final_relres <= 1e-10
    # the plain iteration contracts at the same rate in FP32; BiCGStab's count
    # moves with the preconditioner's rounding, within a fifth either way
    assert abs(r32.iterations - r64.iterations) <= max(3, r64.iterations // (5 if krylov else 10))
    assert same(p32.data, p32b.data) and np.array_equal(r32.relres, r32b.relres)   # deterministic
    err = p32.interior() - po.interior()
    assert np.linalg.norm(err) / np.linalg.norm(po.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(po.interior()).max() < 1e-7


@pytest.mark.parametrize("which", ["skew", "identity"])
def test_mixed_dc_vcycle_converges_to_fp64_solution(M, which):
    """The deferred-correction solve (DD kind) with FP32 grid levels: the
    outer residual is the FP64 9-point one, so it reaches the FP64 DC solve's
    tolerance and solution, in about as many iterations.  (On the wavy 64:1
    grid the reference DC iteration itself diverges, FP64 or not.)"""
    from mgpoisson2d_b200 import workloads as W
    if which == "skew":
        v, geo, rhs, bc, _ = W.skew_stretched(128)
        homog = False
    else:
        v, geo, rhs, bc, _ = W.identity_dirichlet(128)
        homog = True
    f = rhs.copy()
    f.interior()[:] /= geo.J.interior()
    sols, reps = [], []
    for fl in (0, M.FLAG_MIXED, M.FLAG_MIXED):
        with M.Solver(v, geo, bc, KIND_DD, fl) as s:
            p = BoxData(v, 1, 1)
            r = s.dc_vcycle(p, f.copy(), bc, homog, 1e-10, 400, 1, 8, 8, 8)
        assert r.status == 0 and not r.diverged and r.final_relres <= 1e-10, (fl, r.iterations, r.final_relres)
        sols.append(p)
        reps.append(r)
    assert abs(reps[1].iterations - reps[0].iterations) <= max(3, reps[0].iterations // 10)
    assert same(sols[1].data, sols[2].data)   # deterministic
    err = sols[1].interior() - sols[0].interior()
    assert np.linalg.norm(err) / np.linalg.norm(sols[0].interior()) < 1e-8
    assert np.abs(err).max() / np.abs(sols[0].interior()).max() < 1e-7


@pytest.mark.parametrize("kind", ["krylov", "dc"])
def test_bf16_coarse_values_converge_to_fp64_solution(M, kind):
    """MGP_FLAG_BF16_COARSE (a numerics study of BF16 storage below the
    finest level): the FP64 outer iteration still reaches 1e-10 and the FP64
    solution; the flag changes the iterates (the coarse levels hold other
    values) and stays deterministic."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.skew_stretched(128)
    f = rhs.copy()
    f.interior()[:] /= geo.J.interior()

    def run(fl):
        if kind == "dc":
            with M.Solver(v, geo, bc, KIND_DD, fl) as s:
                p = BoxData(v, 1, 1)
                r = s.dc_vcycle(p, f.copy(), bc, False, 1e-10, 400, 1, 8, 8, 8)
        else:
            with M.Solver(v, geo, bc, KIND_MG, fl | M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV) as s:
                p = BoxData(v, 1, 1)
                r = s.vcycle(p, rhs, bc, False, 1e-10, 400)
        assert r.status == 0 and not r.diverged and r.final_relres <= 1e-10, (fl, r.iterations, r.final_relres)
        return p, r
    p64, r64 = run(0)
    p32, r32 = run(M.FLAG_MIXED)
    pb, rb = run(M.FLAG_MIXED | M.FLAG_BF16_COARSE)
    pb2, _ = run(M.FLAG_MIXED | M.FLAG_BF16_COARSE)
    assert same(pb.data, pb2.data)
    assert not same(pb.data, p32.data)
    assert rb.iterations <= 2 * r64.iterations + 2
    err = pb.interior() - p64.interior()
    assert np.linalg.norm(err) / np.linalg.norm(p64.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(p64.interior()).max() < 1e-7


# ---------------------------------------------------------------------------
# GMRES-accelerated V-cycle (MGP_FLAG_GMRES; no reference counterpart)
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("mixed", [False, True])
def test_gmres_vcycle_converges_to_oracle_solution(M, mixed):
    """Right-preconditioned GMRES(m) with one V-cycle per application reaches
    1e-10 and the oracle's FP64 solution, in no more V-cycles than BiCGStab
    with the same preconditioner, and repeats bit for bit."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    base = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | (M.FLAG_MIXED if mixed else 0)
    old = _set_coupled(M, True)
    try:
        po = BoxData(v, 1, 1)
        O.vcycle(po, rhs, geo, bc, True, 1e-11, 3000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, base | M.FLAG_KRYLOV) as s:
        pk = BoxData(v, 1, 1)
        rk = s.vcycle(pk, rhs, bc, True, 1e-10, 3000)
    with M.Solver(v, geo, bc, KIND_MG, base | M.FLAG_GMRES) as s:
        pg = BoxData(v, 1, 1)
        rg = s.vcycle(pg, rhs, bc, True, 1e-10, 3000)
        pg2 = BoxData(v, 1, 1)
        rg2 = s.vcycle(pg2, rhs, bc, True, 1e-10, 3000)
    assert rg.status == 0 and not rg.diverged and rg.final_relres <= 1e-10, (rg.iterations, rg.final_relres)
    assert rg.iterations <= rk.iterations, (rg.iterations, rk.iterations)
    assert same(pg.data, pg2.data) and np.array_equal(rg.relres, rg2.relres)
    err = pg.interior() - po.interior()
    assert np.linalg.norm(err) / np.linalg.norm(po.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(po.interior()).max() < 1e-7


@pytest.mark.parametrize("n", [64, 128])
def test_gmres_vcycle_matches_oracle(M, n):
    """Same V-cycles as the oracle's GMRES restatement (bit-exact in the device
    order, the reference bottom); inner products are summed in a different
    order, so the histories agree to rounding.  The converged solution
    matches the oracle's GMRES and plain V-cycle solutions."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(n)
    old = _set_coupled(M, True)
    try:
        pa, pc = BoxData(v, 1, 1), BoxData(v, 1, 1)
        ra = O.gmres_vcycle(pa, rhs, geo, bc, True, 1e-10, 400)
        O.vcycle(pc, rhs, geo, bc, True, 1e-10, 2000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_GMRES) as s:
        pb = BoxData(v, 1, 1)
        rb = s.vcycle(pb, rhs, bc, True, 1e-10, 400)
    assert rb.status == 0 and rb.final_relres <= 1e-10 and rb.relres[-1] == rb.final_relres
    assert abs(rb.iterations - (len(ra) - 1)) <= 2, (rb.iterations, len(ra) - 1)
    k = min(12, len(ra), len(rb.relres))
    np.testing.assert_allclose(rb.relres[:k], ra[:k], rtol=1e-6)
    for ref in (pa, pc):
        err = pb.interior() - ref.interior()
        assert np.linalg.norm(err) / np.linalg.norm(ref.interior()) < 1e-8
    np.testing.assert_allclose(pb.data, pa.data, rtol=0, atol=1e-9 * np.abs(pa.data).max())   # ghosts too


def test_gmres_restarts(M):
    """One sweep down and up per V-cycle on 256^2: the solve needs more V-cycles
    than the restart length (64), so it restarts from the true residual and
    still reaches the oracle's solution."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(256)
    old = _set_coupled(M, True)
    try:
        po = BoxData(v, 1, 1)
        O.vcycle(po, rhs, geo, bc, True, 1e-11, 5000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_GMRES) as s:
        pg = BoxData(v, 1, 1)
        rg = s.vcycle(pg, rhs, bc, True, 1e-10, 2000, 1, 1, 1, 8)
    assert rg.status == 0 and rg.final_relres <= 1e-10, (rg.iterations, rg.final_relres)
    assert rg.iterations > 64, rg.iterations
    err = pg.interior() - po.interior()
    assert np.linalg.norm(err) / np.linalg.norm(po.interior()) < 1e-8


def test_mixed_all_neumann_and_identity(M):
    """Mixed precision with the mean removal of an all-Neumann hierarchy (the
    terrain solver test) and on the identity map with Dirichlet sides."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, soln = W.terrain_neumann(64, O.boundary_fluxes, O.compute_laplacian)
    pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
    with M.Solver(v, geo, bc, KIND_MG, 0) as s:
        ra = s.vcycle(pa, rhs, bc, False, 1e-9, 200)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_MIXED) as s:
        rb = s.vcycle(pb, rhs, bc, False, 1e-9, 200)
    assert ra.final_relres <= 1e-9 and rb.final_relres <= 1e-9
    d = (pb.interior() - pb.interior().mean()) - (pa.interior() - pa.interior().mean())
    assert np.abs(d).max() < 1e-7 * np.abs(pa.interior()).max()
    v, geo, rhs, bc, u = W.identity_dirichlet(96)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_MIXED | M.FLAG_KRYLOV) as s:
        pc = BoxData(v, 1, 1)
        rc = s.vcycle(pc, rhs, bc, True, 1e-11, 100)
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG) as s:
        pd = BoxData(v, 1, 1)
        s.vcycle(pd, rhs, bc, True, 1e-11, 100)
    assert rc.final_relres <= 1e-11
    assert np.abs(pc.interior() - pd.interior()).max() < 1e-8 * np.abs(pd.interior()).max()


# ---------------------------------------------------------------------------
# Exact coarse solve (MGP_FLAG_DIRECT_COARSE; no reference counterpart): the
# V-cycle's bottom is the first level of at most 64 cells, solved with the
# inverse of its operator
# ---------------------------------------------------------------------------
def _oracle_operator(v, geo, bc):
    """Dense matrix of the oracle's operator with homogeneous BCs: column k is
    compute_laplacian of the k-th unit vector (cells numbered i fastest)."""
    n = v.nx * v.ny
    A = np.zeros((n, n))
    for k in range(n):
        e = BoxData(v, 1, 1)
        e.interior()[k % v.nx, k // v.nx] = 1.0
        lap = BoxData(v)
        O.compute_laplacian(lap, e, geo, bc, True)
        A[:, k] = lap.interior().reshape(-1, order="F")
    return A


@pytest.mark.parametrize("case", ["DDDD-U", "DNND-mixed", "PPDD", "DDNN-U"])
@pytest.mark.parametrize("nx,ny", [(8, 8), (16, 4)])
def test_direct_coarse_solves_a_bottom_sized_grid_in_one_cycle(M, case, nx, ny):
    """A grid of 64 cells is its own bottom level: one V-cycle is the exact
    solve, phi = A^-1 (rhs - L[0]), against numpy's dense solve of the
    oracle's operator."""
    v, geo, rhs, bc, _ = _problem(case, nx, ny, 5)
    res = BoxData(v)
    O.compute_residual(res, rhs, BoxData(v, 1, 1), geo, bc, False)
    A = _oracle_operator(v, geo, bc)
    want = np.linalg.solve(A, res.interior().reshape(-1, order="F")).reshape((nx, ny), order="F")
    with M.Solver(v, geo, bc, KIND_MG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE) as s:
        phi = BoxData(v, 1, 1)
        r = s.vcycle(phi, rhs, bc, False, 1e-12, 5)
    assert r.status == 0 and r.iterations == 1 and r.final_relres <= 1e-12, (r.iterations, r.final_relres)
    assert np.abs(phi.interior() - want).max() <= 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("mixed", [False, True])
def test_direct_coarse_vcycle_converges_to_oracle_solution(M, mixed):
    """On the stretched grid (bottom 8 x 8 instead of 4 x 4 with BiCGStab) the
    BiCGStab(V-cycle) solve reaches 1e-10 in no more V-cycles than with the
    reference bottom, and the oracle's FP64 solution."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    base = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV | (M.FLAG_MIXED if mixed else 0)
    old = _set_coupled(M, True)
    try:
        po = BoxData(v, 1, 1)
        O.vcycle(po, rhs, geo, bc, True, 1e-11, 3000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, base) as s:
        pr = BoxData(v, 1, 1)
        rr = s.vcycle(pr, rhs, bc, True, 1e-10, 3000)
    with M.Solver(v, geo, bc, KIND_MG, base | M.FLAG_DIRECT_COARSE) as s:
        pd = BoxData(v, 1, 1)
        rd = s.vcycle(pd, rhs, bc, True, 1e-10, 3000)
        pd2 = BoxData(v, 1, 1)
        rd2 = s.vcycle(pd2, rhs, bc, True, 1e-10, 3000)
    assert rd.status == 0 and not rd.diverged and rd.final_relres <= 1e-10
    assert rd.iterations <= rr.iterations + 2, (rd.iterations, rr.iterations)
    assert same(pd.data, pd2.data)   # deterministic
    err = pd.interior() - po.interior()
    assert np.linalg.norm(err) / np.linalg.norm(po.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(po.interior()).max() < 1e-7


def test_direct_coarse_keeps_the_reference_bottom_when_singular(M):
    """All-Neumann: the bottom operator is singular, the flag changes nothing
    (same bits as without it)."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.terrain_neumann(64, O.boundary_fluxes, O.compute_laplacian)
    out = []
    for fl in (0, M.FLAG_DIRECT_COARSE):
        with M.Solver(v, geo, bc, KIND_MG, fl) as s:
            p = BoxData(v, 1, 1)
            r = s.vcycle(p, rhs, bc, False, 1e-9, 200)
        out.append((p, r))
    assert same(out[0][0].data, out[1][0].data) and np.array_equal(out[0][1].relres, out[1][1].relres)


def test_direct_coarse_with_fmg(M):
    """fmg's cycles that start below the direct level keep the reference
    bottom; the solve still reaches the same solution."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    sols = []
    for fl in (M.FLAG_DIRICHLET_COUPLED_DIAG, M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE):
        with M.Solver(v, geo, bc, KIND_MG, fl) as s:
            p = BoxData(v, 1, 1)
            r = s.fmg(p, rhs, bc, True, 1e-10, 2000)
        assert r.status == 0 and r.final_relres <= 1e-10
        sols.append(p.interior())
    assert np.abs(sols[1] - sols[0]).max() <= 1e-7 * np.abs(sols[0]).max()


# MGP_FLAG_DIRECT_LARGE: the bottom is the first level of at most 1024 cells,
# inverted on the device by Gauss-Jordan elimination
@pytest.mark.parametrize("case", ["DDDD-U", "DNND-mixed", "PPDD", "DDNN-U"])
@pytest.mark.parametrize("nx,ny", [(32, 32), (64, 16), (12, 20)])
def test_direct_large_solves_a_coarse_sized_grid_in_one_cycle(M, case, nx, ny):
    """A grid of 240..1024 cells is its own bottom level: one V-cycle is the
    exact solve, against numpy's dense solve of the oracle's operator."""
    v, geo, rhs, bc, _ = _problem(case, nx, ny, 5)
    res = BoxData(v)
    O.compute_residual(res, rhs, BoxData(v, 1, 1), geo, bc, False)
    A = _oracle_operator(v, geo, bc)
    want = np.linalg.solve(A, res.interior().reshape(-1, order="F")).reshape((nx, ny), order="F")
    fl = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE
    with M.Solver(v, geo, bc, KIND_MG, fl) as s:
        phi = BoxData(v, 1, 1)
        r = s.vcycle(phi, rhs, bc, False, 1e-11, 5)
    assert r.status == 0 and r.iterations == 1 and r.final_relres <= 1e-11, (r.iterations, r.final_relres)
    assert np.abs(phi.interior() - want).max() <= 1e-10 * np.abs(want).max()


@pytest.mark.parametrize("solver", ["krylov", "gmres"])
@pytest.mark.parametrize("mixed", [False, True])
def test_direct_large_vcycle_converges_to_oracle_solution(M, solver, mixed):
    """On the stretched grid the bottom is 32 x 32 instead of 8 x 8: the
    Krylov(V-cycle) solve reaches 1e-10, deterministically, and the oracle's
    FP64 solution.  The coarse operators are restrictions of the geometry,
    not Galerkin products, so the exact 32 x 32 solve is not always the
    better preconditioner: BiCGStab took 64 V-cycles against 57 with the 8 x 8
    bottom (71 against 55 in mixed precision); GMRES no more."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    base = (M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | (M.FLAG_MIXED if mixed else 0) |
            (M.FLAG_KRYLOV if solver == "krylov" else M.FLAG_GMRES))
    old = _set_coupled(M, True)
    try:
        po = BoxData(v, 1, 1)
        O.vcycle(po, rhs, geo, bc, True, 1e-11, 3000, gs_order=1)
    finally:
        _set_coupled(M, old)
    with M.Solver(v, geo, bc, KIND_MG, base) as s:
        ps = BoxData(v, 1, 1)
        rs = s.vcycle(ps, rhs, bc, True, 1e-10, 3000)
    with M.Solver(v, geo, bc, KIND_MG, base | M.FLAG_DIRECT_LARGE) as s:
        pd = BoxData(v, 1, 1)
        rd = s.vcycle(pd, rhs, bc, True, 1e-10, 3000)
        pd2 = BoxData(v, 1, 1)
        rd2 = s.vcycle(pd2, rhs, bc, True, 1e-10, 3000)
    assert rd.status == 0 and not rd.diverged and rd.final_relres <= 1e-10
    assert rd.iterations <= (rs.iterations if solver == "gmres" else 1.5 * rs.iterations), (rd.iterations,
                                                                                         rs.iterations)
    assert same(pd.data, pd2.data) and np.array_equal(rd.relres, rd2.relres)   # deterministic
    err = pd.interior() - po.interior()
    assert np.linalg.norm(err) / np.linalg.norm(po.interior()) < 1e-8
    assert np.abs(err).max() / np.abs(po.interior()).max() < 1e-7


def test_direct_large_keeps_the_reference_bottom_when_singular(M):
    """All-Neumann: the bottom operator is singular, the flags change nothing."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.terrain_neumann(64, O.boundary_fluxes, O.compute_laplacian)
    out = []
    for fl in (0, M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE):
        with M.Solver(v, geo, bc, KIND_MG, fl) as s:
            p = BoxData(v, 1, 1)
            r = s.vcycle(p, rhs, bc, False, 1e-9, 200)
        out.append((p, r))
    assert same(out[0][0].data, out[1][0].data) and np.array_equal(out[0][1].relres, out[1][1].relres)


def test_direct_large_with_fmg(M):
    """fmg's cycles that start below the 32 x 32 level keep the reference
    bottom; the solve reaches the same solution as without the flags."""
    from mgpoisson2d_b200 import workloads as W
    v, geo, rhs, bc, _ = W.wavy_stretched(128)
    sols = []
    for fl in (M.FLAG_DIRICHLET_COUPLED_DIAG,
               M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_DIRECT_COARSE | M.FLAG_DIRECT_LARGE):
        with M.Solver(v, geo, bc, KIND_MG, fl) as s:
            p = BoxData(v, 1, 1)
            r = s.fmg(p, rhs, bc, True, 1e-10, 2000)
        assert r.status == 0 and r.final_relres <= 1e-10
        sols.append(p.interior())
    assert np.abs(sols[1] - sols[0]).max() <= 1e-7 * np.abs(sols[0]).max()


# ---------------------------------------------------------------------------
# Batches and the solve server: every result identical to solving alone
# ---------------------------------------------------------------------------
def _alone(M, prob, flags, tol=1e-10, maxiters=400):
    v, geo, rhs, bc = prob
    with M.Solver(v, geo, bc, KIND_MG, flags) as s:
        p = BoxData(v, 1, 1)
        r = s.vcycle(p, rhs, bc, True, tol, maxiters)
    return p, r


def test_batch_matches_individual_solves(M):
    from mgpoisson2d_b200 import workloads as W
    probs = [W.batch_problem(i, nmax=192) for i in range(5)]
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV | M.FLAG_MIXED
    with M.Batch([(v, g, bc) for v, g, _, bc in probs], KIND_MG, flags, nstreams=3) as b:
        phis = [BoxData(p[0], 1, 1) for p in probs]
        reps = b.vcycle(phis, [p[2] for p in probs], [p[3] for p in probs], True, 1e-10, 400)
    for k, prob in enumerate(probs):
        pa, ra = _alone(M, prob, flags)
        assert reps[k].status == 0 and reps[k].final_relres <= 1e-10
        assert same(phis[k].data, pa.data) and np.array_equal(reps[k].relres, ra.relres)


@pytest.mark.parametrize("solver", ["krylov", "gmres_mixed"])
def test_server_results_same_alone_and_in_the_mix(M, solver):
    """Requests overlap on the device (3 slots, 7 requests, two keys reused);
    each result must equal the same solve run alone (BiCGStab, and the
    served leg's GMRES mixed with the exact bottom)."""
    from mgpoisson2d_b200 import workloads as W
    probs = [W.batch_problem(i, nmax=160) for i in range(4)]
    flags = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV
    if solver == "gmres_mixed":
        flags = (M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_GMRES | M.FLAG_MIXED | M.FLAG_DIRECT_COARSE |
                 M.FLAG_DIRECT_LARGE)
    order = [0, 1, 2, 3, 0, 1, 0]
    with M.Server(nworkers=3, flags=flags) as srv:
        outs, tickets = [], []
        for n, k in enumerate(order):
            v, geo, rhs, bc = probs[k]
            p = BoxData(v, 1, 1)
            outs.append(p)
            tickets.append(srv.submit(v, geo, bc, p, rhs, True, 1e-10, 400, key=(k + 1 if k < 2 else 0)))
        results = [srv.wait(t) for t in tickets]
    for n, k in enumerate(order):
        pa, ra = _alone(M, probs[k], flags)
        rep, lat, qt = results[n]
        assert rep.status == 0 and lat >= qt >= 0.0
        assert same(outs[n].data, pa.data) and np.array_equal(rep.relres, ra.relres)


# ---------------------------------------------------------------------------
# Gradient and divergence (compute_pd, compute_grad, compute_div,
# fill_boundary_fluxes): bit-exact
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dir,nodedir", [(1, 1), (2, 1), (1, 2), (2, 2)])
@pytest.mark.parametrize("nx,ny", [(16, 12), (9, 7), (40, 33)])
def test_compute_pd_bitexact(M, dir, nodedir, nx, ny):
    rng = np.random.default_rng(nx * 100 + ny + 7 * dir + nodedir)
    v = Box.of_size(nx, ny)
    phi = rand_field(v, rng)
    offs = (BD_NODE, BD_CELL) if nodedir == 1 else (BD_CELL, BD_NODE)
    a, b = BoxData(v, 0, 0, *offs), BoxData(v, 0, 0, *offs)
    O.compute_pd(a, phi, dir, nodedir)
    M.compute_pd(b, phi, dir, nodedir)
    assert same(a.data, b.data)


@pytest.mark.parametrize("case", list(BC_CASES))
@pytest.mark.parametrize("homog", [False, True])
def test_compute_grad_div_bitexact(M, case, homog):
    v, geo, phi, bc, rng = _problem(case, 20, 14, 77)
    xa, ya = BoxData(v, 0, 0, BD_NODE, BD_CELL), BoxData(v, 0, 0, BD_CELL, BD_NODE)
    xb, yb = BoxData(v, 0, 0, BD_NODE, BD_CELL), BoxData(v, 0, 0, BD_CELL, BD_NODE)
    pa, pb = phi.copy(), phi.copy()
    O.compute_grad(xa, ya, pa, geo, bc, homog)
    M.compute_grad(xb, yb, pb, geo, bc, homog)
    assert same(xa.data, xb.data) and same(ya.data, yb.data)
    assert same(pa.data, pb.data)   # the ghosts compute_grad fills
    da, db = BoxData(v), BoxData(v)
    O.compute_div(da, xa, ya)
    M.compute_div(db, xa, ya)
    assert same(da.data, db.data)


@pytest.mark.parametrize("case", ["NNNN-U", "NNNN-NU", "DNND-mixed"])
@pytest.mark.parametrize("homog", [False, True])
def test_fill_boundary_fluxes_bitexact(M, case, homog):
    v, geo, phi, bc, rng = _problem(case, 12, 10, 5)
    xa, ya = rand_field(v, rng, 0, BD_NODE, BD_CELL), rand_field(v, rng, 0, BD_CELL, BD_NODE)
    xb, yb = xa.copy(), ya.copy()
    O.fill_boundary_fluxes(xa, ya, bc, homog)
    M.fill_boundary_fluxes(xb, yb, bc, homog)
    assert same(xa.data, xb.data) and same(ya.data, yb.data)


@pytest.mark.parametrize("case", ["DDDD-U", "NNNN-NU", "DNND-mixed", "PPDD"])
@pytest.mark.parametrize("omega", [1.0, 0.8])
def test_relax_jacobi_bitexact(M, case, omega):
    v, geo, phi, bc, rng = _problem(case, 18, 14, 31)
    rhs, d = rand_field(v, rng, 0), BoxData(v)
    d.data[:] = rng.uniform(-0.5, -0.1, d.data.shape)
    pa, pb = phi.copy(), phi.copy()
    O.relax_jacobi(pa, rhs, geo, bc, False, d, omega, -1.0, 5, False)
    M.relax_jacobi(pb, rhs, geo, bc, False, d, omega, -1.0, 5)
    assert same(pa.data, pb.data)


# ---------------------------------------------------------------------------
# Metric terms and rhs generated on the device from analytic maps
# ---------------------------------------------------------------------------
def _close(a, b, rel):
    a, b = a.host(), b.host()
    assert np.abs(a - b).max() <= rel * np.abs(b).max(), np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("which", ["identity", "wavy", "skew"])
def test_map_geometry_matches_host_generator(M, which):
    """Same formulas as the host generator; only the rounding of the map's
    transcendentals differs, amplified by the one-cell differences."""
    import math
    from mgpoisson2d_b200 import geometry as G
    v = Box.of_size(96, 80)
    if which == "identity":
        kind, params, fmap = M.MAP_IDENTITY, (), G.map_identity()
    elif which == "wavy":
        beta = G.exp_stretch_beta(64.0)
        kind, params, fmap = M.MAP_WAVY_EXP, (0.1, beta), G.map_wavy_exp(0.1, 64.0)
    else:
        kind, params = M.MAP_SKEW_LAYER, (math.tan(math.radians(20.0)), 1.05, 24.0, 80.0)
        fmap = G.map_skew_stretch(20.0, 1.05, 24.0 / 80.0, 80)
    gd = M.map_geometry(v, kind, params)
    gh = G.mapped_geometry(v, fmap)
    for a, b in zip((gd.J, gd.Jgup_xx, gd.Jgup_xy, gd.Jgup_yx, gd.Jgup_yy),
                    (gh.J, gh.Jgup_xx, gh.Jgup_xy, gh.Jgup_yx, gh.Jgup_yy)):
        if np.abs(b.host()).max() == 0:
            assert np.abs(a.host()).max() < 1e-12
        else:
            _close(a, b, 1e-9)
    gc = M.map_geometry(v, kind, params, device=False)   # host arrays: the same bits
    for a, b in zip((gd.J, gd.Jgup_xx, gd.Jgup_yy), (gc.J, gc.Jgup_xx, gc.Jgup_yy)):
        assert same(a.host(), b.host())


def test_batch_problem_device_matches_host(M):
    from mgpoisson2d_b200 import workloads as W
    for i in (0, 3):
        vh, gh, rh, bh = W.batch_problem(i, nmax=256)
        vd, gd, rd, bd = W.batch_problem_device(i, nmax=256)
        assert (vh.nx, vh.ny) == (vd.nx, vd.ny)
        _close(gd.J, gh.J, 1e-9)
        _close(gd.Jgup_xy, gh.Jgup_xy, 1e-8)
        _close(rd, rh, 1e-9)


def test_skew_stretched_device_matches_host(M):
    """The device-assembled manufactured problem equals the host one: metric
    from the same map, u and rhs from the same formulas, Dirichlet data at the
    same face centres."""
    from mgpoisson2d_b200 import workloads as W
    vh, gh, rh, bh, uh = W.skew_stretched(128)
    vd, gd, rd, bd, ud = W.skew_stretched_device(128)
    assert (vh.nx, vh.ny) == (vd.nx, vd.ny)
    _close(gd.J, gh.J, 1e-9)
    _close(gd.Jgup_xx, gh.Jgup_xx, 1e-8)
    _close(gd.Jgup_xy, gh.Jgup_xy, 1e-8)
    _close(rd, rh, 1e-9)
    u = ud.cpu().numpy().T     # (ny, nx) row-major view -> (nx, ny)
    assert np.abs(u - uh).max() <= 1e-12 * np.abs(uh).max()
    for s in range(4):
        assert np.abs(bd.data[s] - bh.data[s]).max() <= 1e-12 * np.abs(bh.data[s]).max()


def test_manufactured_solution_second_order_mixed_and_fp64(M):
    """Solving the skewed, stretched manufactured problem to 1e-10 with the
    BiCGStab(V-cycle) solver: the error against the exact solution falls at
    second order, and the mixed-precision solution sits far below the
    discretisation error from the FP64 one (relative L2 < 1e-8)."""
    from mgpoisson2d_b200 import workloads as W
    kry = M.FLAG_DIRICHLET_COUPLED_DIAG | M.FLAG_KRYLOV
    err = {}
    for n in (256, 512):
        v, geo, rhs, bc, u = W.skew_stretched_device(n)
        sols = {}
        for name, fl in (("mixed", kry | M.FLAG_MIXED), ("fp64", kry)):
            with M.Solver(v, geo, bc, KIND_MG, fl) as s:
                phi = BoxData.device_zeros(v, 1, 1)
                r = s.vcycle(phi, rhs, bc, False, 1e-10, 400)
            assert r.final_relres <= 1e-10 and not r.diverged
            p = phi.data[1:-1, 1:-1]
            sols[name] = p
            err[name, n] = float(torch.linalg.norm(p - u) / torch.linalg.norm(u))
        d = float(torch.linalg.norm(sols["mixed"] - sols["fp64"]) / torch.linalg.norm(sols["fp64"]))
        assert d < 1e-8, d
        assert d < 1e-3 * err["fp64", n]
    for name in ("mixed", "fp64"):
        order = math.log2(err[name, 256] / err[name, 512])
        assert 1.8 < order < 2.2, (name, order, err)
