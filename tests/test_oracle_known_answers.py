"""The CPU oracle against the reference's own known-answer tests
(src/tests/test.f90): manufactured solutions on the reference's terrain map and
the convergence rates they must show.  The reference ships no golden numbers
and cannot be built here (no Fortran compiler), so these rates are what pins
the restatement.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import pytest

from helpers import hierarchy_geo
from mgpoisson2d_b200 import geometry as G
from mgpoisson2d_b200 import workloads as W
from mgpoisson2d_b200.types import (BCMODE_NONUNIFORM, BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_PERIODIC, BD_CELL, BD_NODE,
                                    BdryData, Box, BoxData)
from oracle import oracle as O

LEVELS = [32, 64, 128, 256]


def rates(errs):
    return [math.log2(errs[k] / errs[k + 1]) for k in range(len(errs) - 1)]


def smooth_phi(X, Y, modes=(2,)):
    return sum(np.cos(i * math.pi * X) * np.cos(i * math.pi * Y) / i for i in modes)


def smooth_lap(X, Y, modes=(2,)):
    return sum(-i * 2 * math.pi ** 2 * np.cos(i * math.pi * X) * np.cos(i * math.pi * Y) for i in modes)


def laplacian_error(n, bctype, modes=(2,)):
    """test_laplacian (test.f90:1898-2058) with the smooth solution of its
    commented variant; Neumann data from the operator's own boundary fluxes."""
    v = Box.of_size(n, n)
    geo = G.terrain_geometry(v)
    X, Y = G.terrain_positions(v, BD_CELL, BD_CELL, 1)
    phi = BoxData(v, 1, 1)
    phi.data[:] = smooth_phi(X, Y, modes)
    exact = smooth_lap(X[1:-1, 1:-1], Y[1:-1, 1:-1], modes) * geo.J.interior()
    if bctype == BCTYPE_NEUM:
        bc = BdryData(v, [BCTYPE_NEUM] * 4, [BCMODE_NONUNIFORM] * 4, O.boundary_fluxes(phi, geo))
    else:
        Xf, Yf = G.terrain_positions(v, BD_NODE, BD_CELL, 0)
        Xg, Yg = G.terrain_positions(v, BD_CELL, BD_NODE, 0)
        f = lambda x, y: smooth_phi(x, y, modes)
        bc = BdryData(v, [BCTYPE_DIRI] * 4, [BCMODE_NONUNIFORM] * 4,
                      [f(Xf[0], Yf[0]), f(Xf[-1], Yf[-1]), f(Xg[:, 0], Yg[:, 0]), f(Xg[:, -1], Yg[:, -1])])
    lap = BoxData(v)
    O.compute_laplacian(lap, phi, geo, bc, False)
    return np.abs(exact - lap.interior()).max()


@pytest.mark.parametrize("bctype", [BCTYPE_NEUM, BCTYPE_DIRI])
def test_laplacian_second_order(bctype):
    r = rates([laplacian_error(n, bctype) for n in LEVELS])
    assert all(x > 1.85 for x in r), r


def test_laplacian_reference_modes_converge():
    """The reference's own 117-mode solution (test.f90:1945-1958) is under-
    resolved on these grids; its error still falls with refinement."""
    e = [laplacian_error(n, BCTYPE_NEUM, tuple(range(8, 241, 2))) for n in (64, 128, 256)]
    assert e[0] > e[1] > e[2]


def ghost_error(n, bctype):
    """test_nonuniform_diri_bcs / _neum_bcs (test.f90:1099-1368): fill ghosts
    from exact boundary data, compare with the exact solution there."""
    v = Box.of_size(n, n)
    geo = G.terrain_geometry(v)
    X, Y = G.terrain_positions(v, BD_CELL, BD_CELL, 1)
    if bctype == BCTYPE_DIRI:
        u = lambda x, y: np.sin((0.5 + 4 * y) * math.pi * x)
        Xf, Yf = G.terrain_positions(v, BD_NODE, BD_CELL, 0)
        Xg, Yg = G.terrain_positions(v, BD_CELL, BD_NODE, 0)
        data = [u(Xf[0], Yf[0]), u(Xf[-1], Yf[-1]), u(Xg[:, 0], Yg[:, 0]), u(Xg[:, -1], Yg[:, -1])]
    else:
        # x^3 y^3 (test.f90:1294).  The boundary data is the flux the operator
        # uses, J g^{n xi} d_xi u + J g^{n eta} d_eta u, in computational
        # derivatives (the reference test multiplies physical derivatives by
        # Jgup, which is not that flux on mapped y faces).
        u = lambda x, y: x ** 3 * y ** 3

        def dxi_deta(xi, eta):
            x = xi
            el = 0.25 * np.sin(math.pi * x) ** 2
            y = el + (1 - el) * eta
            y_xi = 0.25 * math.pi * np.sin(2 * math.pi * x) * (1 - eta)
            y_eta = 1 - el
            ux, uy = 3 * x ** 2 * y ** 3, 3 * x ** 3 * y ** 2
            return ux + uy * y_xi, uy * y_eta

        xi_f, eta_f = G._coords(v, BD_NODE, BD_CELL, 0)
        xi_g, eta_g = G._coords(v, BD_CELL, BD_NODE, 0)
        jxx, jxy = geo.Jgup_xx.interior(), geo.Jgup_xy.interior()
        jyx, jyy = geo.Jgup_yx.interior(), geo.Jgup_yy.interior()
        a, b = dxi_deta(xi_f, eta_f)
        c, d = dxi_deta(xi_g, eta_g)
        fxf, fyf = jxx * a + jxy * b, jyx * c + jyy * d
        data = [fxf[0], fxf[-1], fyf[:, 0], fyf[:, -1]]
    bc = BdryData(v, [bctype] * 4, [BCMODE_NONUNIFORM] * 4, data)
    soln = u(X, Y)
    state = BoxData(v, 1, 1)
    state.data[:] = soln   # ghosts start exact, so the centred Neumann stencil reads sane values
    state.data[1:-1, 1:-1] = soln[1:-1, 1:-1]
    ghosts_before = state.data.copy()
    O.fill_ghosts(state, bc, geo, False)
    assert np.array_equal(state.interior(), ghosts_before[1:-1, 1:-1])   # valid cells untouched (test.f90:1202-1213)
    err = state.data - soln
    g = np.concatenate([err[0, 1:-1], err[-1, 1:-1], err[1:-1, 0], err[1:-1, -1]])
    return np.abs(g).max()


def test_dirichlet_ghosts_third_order():
    r = rates([ghost_error(n, BCTYPE_DIRI) for n in LEVELS])
    assert all(x > 2.8 for x in r), r


def test_neumann_ghosts_zero_flux_third_order():
    """Homogeneous Neumann ghosts (the fill prolong uses, MG:318) for a field
    with zero normal derivative on an orthogonal grid: third order."""
    errs = []
    for n in LEVELS:
        v = Box.of_size(n, n)
        geo = G.mapped_geometry(v, G.map_identity())
        X, Y = G.positions(v, G.map_identity(), ng=1)
        f = lambda t: t ** 2 - 2.0 * t ** 3 / 3.0   # f'(0) = f'(1) = 0, not symmetric
        soln = f(X) * f(Y) + f(X)
        st = BoxData(v, 1, 1)
        st.data[:] = soln
        O.fill_ghosts(st, BdryData.uniform(v, [BCTYPE_NEUM] * 4), geo, True)
        err = st.data - soln
        errs.append(max(np.abs(err[0, 1:-1]).max(), np.abs(err[-1, 1:-1]).max(),
                        np.abs(err[1:-1, 0]).max(), np.abs(err[1:-1, -1]).max()))
    assert all(x > 2.8 for x in rates(errs)), rates(errs)


def test_neumann_ghost_formula_as_written():
    """fill_ghosts_neum_dir_side (AU:926-960) sets the ghost to
    cell - (g - cross) * dx / Jgup_xx with dx negated on the low side, reading
    Jgup at the cell's own low face on both sides (AU:943, AU:1008)."""
    v = Box.of_size(8, 8)
    geo = G.mapped_geometry(v, G.map_identity())
    rng = np.random.default_rng(3)
    st = BoxData(v, 1, 1)
    st.data[:] = rng.standard_normal(st.data.shape)
    g = rng.standard_normal(8)
    bc = BdryData(v, [BCTYPE_NEUM] * 4, [BCMODE_NONUNIFORM] * 4, [g, g, g, g])
    O.fill_ghosts(st, bc, geo, False)
    p = st.interior()
    jxx = geo.Jgup_xx.interior()
    # identity map: the cross terms vanish
    np.testing.assert_allclose(st.data[0, 1:-1], p[0, :] + g * v.dx / jxx[0, :], rtol=1e-13)
    np.testing.assert_allclose(st.data[-1, 1:-1], p[-1, :] - g * v.dx / jxx[-2, :], rtol=1e-13)


def test_restrict_face_second_order():
    """test_restrict (test.f90:2063-2177): refine-by-4 restriction of x^3 y^3
    face data converges at second order."""
    errs = []
    for n in LEVELS:
        v = Box.of_size(n, n)
        c = v.coarsened(4, 4)
        out = []
        for offi, offj in ((BD_NODE, BD_CELL), (BD_CELL, BD_NODE)):
            X, Y = G.terrain_positions(v, offi, offj, 0)
            f = BoxData(v, 0, 0, offi, offj, data=np.asfortranarray(X ** 3 * Y ** 3))
            cr = BoxData(c, 0, 0, offi, offj)
            O.restrict(f, cr)
            Xc, Yc = G.terrain_positions(c, offi, offj, 0)
            out.append(np.abs(cr.data - Xc ** 3 * Yc ** 3).max())
        errs.append(max(out))
    assert all(x > 1.8 for x in rates(errs)), rates(errs)


def test_prolong_order2_periodic():
    """test_prolong (test.f90:2182-2331): order-2 prolongation of a periodic
    field, error of (fine - P crse)."""
    errs = []
    for n in LEVELS:
        v = Box.of_size(n, n)
        geo = G.terrain_geometry(v)
        c, cgeo = hierarchy_geo(v, geo, O.restrict)
        X, Y = G.positions(v, G.map_identity())
        Xc, Yc = G.positions(c, G.map_identity(), ng=1)
        k = 8 * math.pi
        fine = BoxData(v, 0, 0)
        fine.interior()[:] = np.cos(k * X) * np.cos(k * Y)
        crse = BoxData(c, 1, 1)
        crse.data[:] = -np.cos(k * Xc) * np.cos(k * Yc)
        bc = BdryData.uniform(c, [BCTYPE_PERIODIC] * 4)
        O.prolong(fine, crse, geo, cgeo, bc, 2)
        errs.append(np.abs(fine.interior()).max())
    assert all(x > 1.8 for x in rates(errs)), rates(errs)


def test_schedule():
    """create_mgschedule (MG:67-129): 128^2 gives depth 5, 1024^2 depth 8,
    and unequal spacings semicoarsen."""
    assert O.create_mgschedule(O.estimate_maxdepth(1000, Box.of_size(128, 128)), Box.of_size(128, 128))[2] == 5
    assert O.create_mgschedule(O.estimate_maxdepth(1000, Box.of_size(1024, 1024)), Box.of_size(1024, 1024))[2] == 8
    b = Box.of_size(64, 256)
    rx, ry, md = O.create_mgschedule(O.estimate_maxdepth(1000, b), b)
    assert (rx[0], ry[0]) == (1, 2) and (rx[1], ry[1]) == (1, 2) and (rx[2], ry[2]) == (2, 2)
    # odd sizes stop at depth 0 (MG:90-91)
    b = Box.of_size(63, 64)
    assert O.create_mgschedule(O.estimate_maxdepth(1000, b), b)[2] == 0


def _solver_error(n, use_fmg):
    v, geo, rhs, bc, soln = W.terrain_neumann(n, O.boundary_fluxes, O.compute_laplacian)
    phi = BoxData(v, 1, 1)
    if use_fmg:
        rep = O.fmg(phi, rhs, geo, bc, False, 1e-30, 1)
    else:
        rep = O.vcycle(phi, rhs, geo, bc, False, 1e-9, 40)
    e = phi.interior() - soln.interior()
    e -= e.mean()   # all-Neumann: defined up to a constant
    return np.abs(e).max(), rep


def test_fmg_solver_test():
    """test_solver (test.f90:2336-2583): one FMG cycle, nu = 8/8/8, on the
    discrete problem whose exact solution is the sampled 117-mode field."""
    e64, r64 = _solver_error(64, True)
    e128, r128 = _solver_error(128, True)
    assert r64.relres[-1] < 0.1 and r128.relres[-1] < 0.1
    assert e128 < e64


def test_vcycle_converges_on_all_neumann():
    e, rep = _solver_error(64, False)
    assert rep.relres[-1] <= 1e-9 and not rep.diverged


def _coupled(on):
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(int(on))


def test_reference_diagonal_diverges_on_dirichlet():
    """With compute_invdiags as written (P2:29-33) the Dirichlet ghost's
    dependence on the cell is left out and the sweep amplifies errors at
    Dirichlet corners: the reference V-cycle stops after one diverging cycle."""
    v, geo, rhs, bc, u = W.identity_dirichlet(64)
    phi = BoxData(v, 1, 1)
    rep = O.vcycle(phi, rhs, geo, bc, True, 1e-10, 20)
    assert rep.diverged and rep.iterations == 1


@pytest.mark.parametrize("gs_order", [0, 1])
def test_coupled_diagonal_converges_second_order(gs_order):
    """128^2 identity-map Dirichlet problem, coupled diagonal: converges to 1e-10 and the
    discretisation error vs u falls at second order."""
    _coupled(True)
    try:
        errs = []
        for n in (32, 64, 128):
            v, geo, rhs, bc, u = W.identity_dirichlet(n, seed=None)
            rhs.interior()[:] = -13 * math.pi ** 2 * u   # noise-free for the rate
            phi = BoxData(v, 1, 1)
            rep = O.vcycle(phi, rhs, geo, bc, True, 1e-10, 40, gs_order=gs_order)
            assert rep.relres[-1] <= 1e-10 and not rep.diverged
            errs.append(np.abs(phi.interior() - u).max())
        assert all(x > 1.9 for x in rates(errs)), rates(errs)
    finally:
        _coupled(False)


def test_colour_and_lexicographic_agree():
    _coupled(True)
    try:
        v, geo, rhs, bc, u = W.identity_dirichlet(64)
        a, b = BoxData(v, 1, 1), BoxData(v, 1, 1)
        O.vcycle(a, rhs, geo, bc, True, 1e-11, 40, gs_order=0)
        O.vcycle(b, rhs, geo, bc, True, 1e-11, 40, gs_order=1)
        assert np.linalg.norm(a.interior() - b.interior()) / np.linalg.norm(a.interior()) < 1e-9
    finally:
        _coupled(False)


def test_dc_vcycle_dirichlet_converges():
    """The deferred-correction driver (DD:589-862) converges on a Dirichlet
    problem as written: its LAH ghosts are stable."""
    v, geo, rhs, bc, u = W.identity_dirichlet(64)
    f = rhs.copy()
    f.interior()[:] /= geo.J.interior()
    phi = BoxData(v, 1, 1)
    rep = O.dc_vcycle(phi, f, geo, bc, True, 1e-10, 60, smooth_down=8, smooth_up=8, smooth_bottom=8)
    assert rep.relres[-1] <= 1e-10
    assert np.abs(phi.interior() - u).max() < 2e-3


def test_krylov_oracle_same_solution_fewer_vcycles():
    """The BiCGStab restatement behind MGP_FLAG_KRYLOV reaches the plain
    V-cycle's converged solution on the stretched wavy grid with several
    times fewer V-cycles."""
    v, geo, rhs, bc, _ = W.wavy_stretched(64)
    _coupled(True)
    try:
        pa, pb = BoxData(v, 1, 1), BoxData(v, 1, 1)
        ra = O.vcycle(pa, rhs, geo, bc, True, 1e-10, 2000, gs_order=1)
        rk = O.krylov_vcycle(pb, rhs, geo, bc, True, 1e-10, 2000)
    finally:
        _coupled(False)
    assert ra.relres[-1] <= 1e-10 and rk[-1] <= 1e-10
    assert 3 * (len(rk) - 1) < ra.iterations
    err = pb.interior() - pa.interior()
    assert np.linalg.norm(err) / np.linalg.norm(pa.interior()) < 1e-8


def test_gmres_oracle_same_solution_fewer_vcycles():
    """The GMRES restatement behind MGP_FLAG_GMRES reaches the plain
    V-cycle's converged solution on the stretched wavy grid in fewer V-cycles
    than the BiCGStab one; with a restart every 5 V-cycles it restarts from
    the true residual and still converges."""
    v, geo, rhs, bc, _ = W.wavy_stretched(64)
    _coupled(True)
    try:
        pa, pb, pc, pd = (BoxData(v, 1, 1) for _ in range(4))
        ra = O.vcycle(pa, rhs, geo, bc, True, 1e-10, 2000, gs_order=1)
        rk = O.krylov_vcycle(pb, rhs, geo, bc, True, 1e-10, 2000)
        rg = O.gmres_vcycle(pc, rhs, geo, bc, True, 1e-10, 2000)
        rr = O.gmres_vcycle(pd, rhs, geo, bc, True, 1e-10, 2000, restart=5)
    finally:
        _coupled(False)
    assert rg[-1] <= 1e-10 and rr[-1] <= 1e-10
    assert len(rg) < len(rk) and 4 * (len(rg) - 1) < ra.iterations
    assert len(rr) - 1 > 5 and len(rr) > len(rg)
    assert all(b <= a * (1 + 1e-12) for a, b in zip(rg, rg[1:]))   # minimal residual: no increase
    for p in (pc, pd):
        err = p.interior() - pa.interior()
        assert np.linalg.norm(err) / np.linalg.norm(pa.interior()) < 1e-8


def test_batch_problem_generator():
    """The batched workload: seeded, sides multiples of 16 within [64, 1024],
    Dirichlet all round, the rhs with zero J-weighted mean."""
    a, b = W.batch_problem(7), W.batch_problem(7)
    assert a[0].nx == b[0].nx and a[0].ny == b[0].ny
    assert np.array_equal(a[2].interior(), b[2].interior())
    for i in range(12):
        v, geo, rhs, bc = W.batch_problem(i, nmax=256)
        assert v.nx % 16 == 0 and v.ny % 16 == 0 and 64 <= v.nx <= 256 and 64 <= v.ny <= 256
        assert bc.types == [BCTYPE_DIRI] * 4
        assert np.all(geo.J.interior() > 0)
        assert abs(rhs.interior().sum()) < 1e-9 * np.abs(rhs.interior()).sum()


@pytest.mark.parametrize("case", ["DDDD-U", "NNNN-NU", "DDNN-U", "NNDD-NU"])
def test_div_grad_is_the_laplacian(case):
    """compute_pd uses compute_laplacian's stencils (P2:396-398), so
    compute_div(compute_grad(phi)) is compute_laplacian(phi) up to rounding,
    Neumann faces replaced by the BC data in both."""
    from helpers import BC_CASES, rand_bc, rand_field, rand_geo
    rng = np.random.default_rng(11)
    v = Box.of_size(24, 18)
    types, modes = BC_CASES[case]
    geo, phi, bc = rand_geo(v, rng), rand_field(v, rng), rand_bc(v, types, modes, rng)
    xf, yf = BoxData(v, 0, 0, BD_NODE, BD_CELL), BoxData(v, 0, 0, BD_CELL, BD_NODE)
    O.compute_grad(xf, yf, phi, geo, bc, False)
    div, lap = BoxData(v), BoxData(v)
    O.compute_div(div, xf, yf)
    O.compute_laplacian(lap, phi, geo, bc, False)
    scale = np.abs(lap.interior()).max()
    d, l = div.interior(), lap.interior()
    if types[3] == BCTYPE_NEUM and modes[3] == BCMODE_NONUNIFORM:
        # compute_laplacian reads the north Neumann data at index jhi for every
        # column (P2:1220, P2:1256, P2:1303); fill_boundary_fluxes uses the
        # column's own value
        d, l = d[:, :-1], l[:, :-1]
    np.testing.assert_allclose(d, l, rtol=0, atol=1e-12 * scale)


def test_compute_pd_exact_for_quadratics():
    """Every compute_pd stencil -- the centred and one-sided differences and
    the quadratic extrapolation of the region values -- is exact for a
    quadratic in (xi, eta): the derivatives on both face families must match
    the analytic ones to rounding."""
    v = Box.of_size(20, 14)
    c = (0.3, 1.7, -0.8, 0.9, -1.3, 0.6)

    def q(xi, eta):
        return c[0] + c[1] * xi + c[2] * eta + c[3] * xi * xi + c[4] * xi * eta + c[5] * eta * eta

    i = np.arange(-1, v.nx + 1)[:, None]
    j = np.arange(-1, v.ny + 1)[None, :]
    phi = BoxData(v, 1, 1)
    phi.data[:] = q((i + 0.5) * v.dx, (j + 0.5) * v.dy)
    for nodedir, offs in ((1, (BD_NODE, BD_CELL)), (2, (BD_CELL, BD_NODE))):
        fi = np.arange(v.nx + (nodedir == 1))[:, None] + (0.0 if nodedir == 1 else 0.5)
        fj = np.arange(v.ny + (nodedir == 2))[None, :] + (0.0 if nodedir == 2 else 0.5)
        XI, ETA = fi * v.dx, fj * v.dy
        exact = {1: c[1] + 2 * c[3] * XI + c[4] * ETA, 2: c[2] + c[4] * XI + 2 * c[5] * ETA}
        for d in (1, 2):
            pd = BoxData(v, 0, 0, *offs)
            O.compute_pd(pd, phi, d, nodedir)
            np.testing.assert_allclose(pd.interior(), exact[d], rtol=0, atol=1e-10)


def test_relax_jacobi_converges_and_matches_a_manual_sweep():
    """relax_jacobi (P2:1358-1451): one iteration is phi += omega r invdiag
    with the residual of the sweep-start phi; repeated weighted-Jacobi
    iterations reduce the residual of a Dirichlet problem."""
    from helpers import rand_field
    rng = np.random.default_rng(3)
    v = Box.of_size(16, 16)
    geo = G.mapped_geometry(v, G.map_identity())
    bc = BdryData.uniform(v, [BCTYPE_DIRI] * 4)
    rhs, phi = rand_field(v, rng, 0), rand_field(v, rng)
    d = BoxData(v)
    _coupled(True)
    try:
        O.compute_invdiags(d, geo, bc, True)
    finally:
        _coupled(False)
    r = BoxData(v)
    p1 = phi.copy()
    O.compute_residual(r, rhs, p1, geo, bc, True)
    manual = p1.interior() + 0.8 * (r.interior() * d.interior())
    p2 = phi.copy()
    O.relax_jacobi(p2, rhs, geo, bc, True, d, 0.8, -1.0, 1, False)
    np.testing.assert_allclose(p2.interior(), manual, rtol=1e-15, atol=1e-15)
    r0 = np.linalg.norm(r.interior())
    O.relax_jacobi(p2, rhs, geo, bc, True, d, 0.8, -1.0, 200, False)
    O.compute_residual(r, rhs, p2, geo, bc, True)
    assert np.linalg.norm(r.interior()) < 0.5 * r0
