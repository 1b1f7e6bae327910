"""Python face of the CPU oracle (oracle/mgp_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() to
check the device result, and by bench.py's CPU-baseline and reference legs.  The product
package never imports it.

Function names and argument lists follow the Fortran routines they restate
(see mgp_oracle.h for the citations), with containers from
mgpoisson2d_b200.types.  ``gs_order`` = 0 visits cells lexicographically like
the reference; 1 visits them in the device's colour order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mgpoisson2d_b200.types import (BdryData, Box, BoxData, GeoData, MgpArray, MgpBdry,
                                    MgpBox, MgpGeo, MgpReport, make_report, read_report)

_HERE = os.path.dirname(os.path.abspath(__file__))
# MGP_ORACLE_NATIVE=1 selects the copy built with -march=native for this host
# (the timed CPU baseline; same arithmetic, same bits)
_NATIVE = os.environ.get("MGP_ORACLE_NATIVE", "0") == "1"
_SO = os.path.join(_HERE, "_build", "libmgp_oracle_native.so" if _NATIVE else "libmgp_oracle.so")


def build(force: bool = False) -> str:
    src = [os.path.join(_HERE, f) for f in ("mgp_oracle.c", "mgp_oracle.h")]
    stale = not os.path.exists(_SO) or any(os.path.getmtime(s) > os.path.getmtime(_SO) for s in src)
    if force or stale:
        subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []) + (["native"] if _NATIVE else []),
                       check=True)
    return _SO


def _load():
    if not os.path.exists(_SO):
        build()
    lib = C.CDLL(_SO)
    P = C.POINTER
    B, A, BC, G, R = P(MgpBox), P(MgpArray), P(MgpBdry), P(MgpGeo), P(MgpReport)
    i, d = C.c_int, C.c_double
    sig = {
        "or_estimate_maxdepth": [P(C.c_int), B],
        "or_create_mgschedule": [P(C.c_int), P(C.c_int), P(C.c_int), B],
        "or_fill_ghosts": [B, A, BC, G, i, i],
        "or_extrapolate_ghosts": [B, A, i],
        "or_compute_invdiags": [B, A, G, BC, i],
        "or_compute_laplacian": [B, A, A, G, BC, i, i],
        "or_compute_residual": [B, A, A, A, G, BC, i, i],
        "or_relax_gs": [B, A, A, G, BC, i, A, d, d, i, i, i, i],
        "or_relax_jacobi": [B, A, A, G, BC, i, A, d, d, i, i, i],
        "or_compute_pd": [B, A, A, i, i],
        "or_fill_boundary_fluxes": [B, A, A, BC, i],
        "or_compute_grad": [B, A, A, A, G, BC, i],
        "or_compute_div": [B, A, A, A],
        "or_solve_bicgstab2": [B, A, A, G, BC, i, A, d, i, i, i, i, i],
        "or_restrict": [B, A, B, A, i, i],
        "or_prolong": [B, A, B, A, G, G, BC, i],
        "or_boundary_fluxes": [B, A, G, P(d), P(d), P(d), P(d)],
        "or_dd_compute_invdiags": [B, A, G],
        "or_dd_compute_laplacian": [B, A, A, G, BC, i],
        "or_dd_compute_residual": [B, A, A, A, G, BC, i],
        "or_dd_relax_gs": [B, A, A, G, BC, i, A, d, d, i, i, i, i],
        "or_vcycle": [B, A, A, G, BC, i, d, i, i, i, i, i, i, i, i, i, R],
        "or_fmg": [B, A, A, G, BC, i, d, i, i, i, i, i, i, i, i, i, R],
        "or_dc_vcycle": [B, A, A, G, BC, i, d, i, i, i, i, i, i, i, i, i, R],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    for name in ("or_pnorm", "or_inner_prod", "or_integrate2d"):
        getattr(lib, name).restype = C.c_double
    lib.or_pnorm.argtypes = [B, A, i]
    lib.or_inner_prod.argtypes = [B, A, A]
    lib.or_integrate2d.argtypes = [B, A, G, i]
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


class OracleError(RuntimeError):
    pass


def _ck(rc: int, what: str):
    if rc != 0:
        raise OracleError(f"{what} returned status {rc}")


def _r(x):
    return C.byref(x)


def _host(bd: BoxData):
    assert not bd.is_device, "the oracle works on host arrays"
    return bd.c()


# ---- schedule ------------------------------------------------------------- #
def estimate_maxdepth(maxdepth: int, valid: Box) -> int:
    m = C.c_int(maxdepth)
    _ck(lib().or_estimate_maxdepth(_r(m), _r(valid.c())), "estimate_maxdepth")
    return m.value


def create_mgschedule(maxdepth: int, valid: Box):
    m = C.c_int(maxdepth)
    rx = (C.c_int * max(maxdepth, 1))()
    ry = (C.c_int * max(maxdepth, 1))()
    _ck(lib().or_create_mgschedule(rx, ry, _r(m), _r(valid.c())), "create_mgschedule")
    return list(rx)[:m.value], list(ry)[:m.value], m.value


# ---- operators ------------------------------------------------------------ #
def fill_ghosts(phi: BoxData, bc: BdryData, geo: GeoData, homog: bool, do_neum: bool = True):
    a, b, g = _host(phi), bc.c(), geo.c()
    _ck(lib().or_fill_ghosts(_r(phi.valid.c()), _r(a), _r(b), _r(g), int(homog), int(do_neum)), "fill_ghosts")


def extrapolate_ghosts(phi: BoxData, order: int):
    a = _host(phi)
    _ck(lib().or_extrapolate_ghosts(_r(phi.valid.c()), _r(a), order), "extrapolate_ghosts")


def compute_invdiags(invdiags: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    a, b, g = _host(invdiags), bc.c(), geo.c()
    _ck(lib().or_compute_invdiags(_r(invdiags.valid.c()), _r(a), _r(g), _r(b), int(homog)), "compute_invdiags")


def compute_laplacian(lap: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool, jscale=False):
    l, p, b, g = _host(lap), _host(phi), bc.c(), geo.c()
    _ck(lib().or_compute_laplacian(_r(lap.valid.c()), _r(l), _r(p), _r(g), _r(b), int(homog), int(jscale)),
        "compute_laplacian")


def compute_residual(res: BoxData, rhs: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool,
                     jscale=False):
    r, f, p, b, g = _host(res), _host(rhs), _host(phi), bc.c(), geo.c()
    _ck(lib().or_compute_residual(_r(res.valid.c()), _r(r), _r(f), _r(p), _r(g), _r(b), int(homog),
                                  int(jscale)), "compute_residual")


def relax_gs(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
             omega: float, tol: float, maxiters: int, zerophi: bool, verbosity: int = 0, gs_order: int = 0):
    p, f, b, g, d = _host(phi), _host(rhs), bc.c(), geo.c(), _host(invdiags)
    _ck(lib().or_relax_gs(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), omega, tol,
                          maxiters, int(zerophi), verbosity, gs_order), "relax_gs")


def relax_jacobi(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
                 omega: float, tol: float, maxiters: int, zerophi: bool, verbosity: int = 0):
    """relax_jacobi (P2:1358-1451)."""
    p, f, b, g, d = _host(phi), _host(rhs), bc.c(), geo.c(), _host(invdiags)
    _ck(lib().or_relax_jacobi(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), omega, tol,
                              maxiters, int(zerophi), verbosity), "relax_jacobi")


def solve_bicgstab2(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
                    tol: float, max_iters: int, max_restarts: int, zerophi: bool, verbosity: int = 0,
                    gs_order: int = 0):
    p, f, b, g, d = _host(phi), _host(rhs), bc.c(), geo.c(), _host(invdiags)
    _ck(lib().or_solve_bicgstab2(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), tol,
                                 max_iters, max_restarts, int(zerophi), verbosity, gs_order), "solve_bicgstab2")


def restrict(fine: BoxData, crse: BoxData):
    f, c = _host(fine), _host(crse)
    _ck(lib().or_restrict(_r(fine.valid.c()), _r(f), _r(crse.valid.c()), _r(c), fine.offi, fine.offj),
        "restrict")


def prolong(fine: BoxData, crse: BoxData, fine_geo: GeoData, crse_geo: GeoData, crse_bc: BdryData, order: int):
    f, c, fg, cg, b = _host(fine), _host(crse), fine_geo.c(), crse_geo.c(), crse_bc.c()
    _ck(lib().or_prolong(_r(fine.valid.c()), _r(f), _r(crse.valid.c()), _r(c), _r(fg), _r(cg), _r(b), order),
        "prolong")


def pnorm(bd: BoxData, p: int) -> float:
    a = _host(bd)
    return lib().or_pnorm(_r(bd.valid.c()), _r(a), p)


def inner_prod(a: BoxData, b: BoxData) -> float:
    x, y = _host(a), _host(b)
    return lib().or_inner_prod(_r(a.valid.c()), _r(x), _r(y))


def integrate2d(bd: BoxData, geo: GeoData, jscale: bool = True) -> float:
    a, g = _host(bd), geo.c()
    return lib().or_integrate2d(_r(bd.valid.c()), _r(a), _r(g), int(jscale))


def boundary_fluxes(phi: BoxData, geo: GeoData):
    """The operator's face fluxes on the boundary faces (compute_grad there)."""
    v = phi.valid
    out = [np.zeros(v.ny), np.zeros(v.ny), np.zeros(v.nx), np.zeros(v.nx)]
    a, g = _host(phi), geo.c()
    ptr = [o.ctypes.data_as(C.POINTER(C.c_double)) for o in out]
    _ck(lib().or_boundary_fluxes(_r(v.c()), _r(a), _r(g), *ptr), "boundary_fluxes")
    return out


def compute_pd(pd: BoxData, phi: BoxData, dir: int, nodedir: int):
    """compute_pd (P2:404-795); pd nodal in x (nodedir 1) or y (2)."""
    a, p = _host(pd), _host(phi)
    _ck(lib().or_compute_pd(_r(phi.valid.c()), _r(a), _r(p), dir, nodedir), "compute_pd")


def fill_boundary_fluxes(xflux: BoxData, yflux: BoxData, bc: BdryData, homog: bool):
    x, y, b = _host(xflux), _host(yflux), bc.c()
    _ck(lib().or_fill_boundary_fluxes(_r(xflux.valid.c()), _r(x), _r(y), _r(b), int(homog)), "fill_boundary_fluxes")


def compute_grad(xflux: BoxData, yflux: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    """compute_grad (P2:809-850): J Grad[phi] on x- and y-faces."""
    x, y, p, g, b = _host(xflux), _host(yflux), _host(phi), geo.c(), bc.c()
    _ck(lib().or_compute_grad(_r(phi.valid.c()), _r(x), _r(y), _r(p), _r(g), _r(b), int(homog)), "compute_grad")


def compute_div(div: BoxData, xflux: BoxData, yflux: BoxData):
    """compute_div (P2:860-879)."""
    d, x, y = _host(div), _host(xflux), _host(yflux)
    _ck(lib().or_compute_div(_r(div.valid.c()), _r(d), _r(x), _r(y)), "compute_div")


# ---- deferred correction -------------------------------------------------- #
def dd_compute_invdiags(invdiags: BoxData, geo: GeoData):
    a, g = _host(invdiags), geo.c()
    _ck(lib().or_dd_compute_invdiags(_r(invdiags.valid.c()), _r(a), _r(g)), "dd_compute_invdiags")


def dd_compute_laplacian(lap: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    l, p, b, g = _host(lap), _host(phi), bc.c(), geo.c()
    _ck(lib().or_dd_compute_laplacian(_r(lap.valid.c()), _r(l), _r(p), _r(g), _r(b), int(homog)),
        "dd_compute_laplacian")


def dd_compute_residual(res: BoxData, rhs: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    r, f, p, b, g = _host(res), _host(rhs), _host(phi), bc.c(), geo.c()
    _ck(lib().or_dd_compute_residual(_r(res.valid.c()), _r(r), _r(f), _r(p), _r(g), _r(b), int(homog)),
        "dd_compute_residual")


def dd_relax_gs(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
                omega: float, tol: float, maxiters: int, zerophi: bool, verbosity: int = 0, gs_order: int = 0):
    p, f, b, g, d = _host(phi), _host(rhs), bc.c(), geo.c(), _host(invdiags)
    _ck(lib().or_dd_relax_gs(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), omega, tol,
                             maxiters, int(zerophi), verbosity, gs_order), "dd_relax_gs")


# ---- drivers -------------------------------------------------------------- #
def _driver(fn, name, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles, smooth_down,
            smooth_up, smooth_bottom, zerophi, verbosity, gs_order):
    rep, buf = make_report(maxiters)
    p, f, b, g = _host(phi), _host(rhs), bc.c(), geo.c()
    rc = fn(_r(rhs.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), tol, maxiters, maxdepth_user, numcycles,
            smooth_down, smooth_up, smooth_bottom, int(zerophi), verbosity, gs_order, _r(rep))
    _ck(rc, name)
    return read_report(rep, buf)


def vcycle(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=8, smooth_up=8,
           smooth_bottom=8, zerophi=False, verbosity=0, gs_order=0):
    return _driver(lib().or_vcycle, "vcycle", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                   smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order)


def fmg(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=8, smooth_up=8,
        smooth_bottom=8, zerophi=False, verbosity=0, gs_order=0):
    return _driver(lib().or_fmg, "fmg", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                   smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order)


def dc_vcycle(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=1, smooth_up=1,
              smooth_bottom=1, zerophi=False, verbosity=0, gs_order=0):
    return _driver(lib().or_dc_vcycle, "dc_vcycle", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user,
                   numcycles, smooth_down, smooth_up, smooth_bottom, zerophi, verbosity, gs_order)


def krylov_vcycle(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, tol: float,
                  maxiters: int, numcycles: int = 1, smooth_down: int = 8, smooth_up: int = 8,
                  smooth_bottom: int = 8, gs_order: int = 1):
    """Oracle for the solver's MGP_FLAG_KRYLOV mode (no Fortran counterpart).

    Right-preconditioned BiCGStab (van der Vorst 1992) on L_h e = r0, where
    L_h is compute_laplacian with homogeneous BCs and the preconditioner is one
    V-cycle of ``vcycle`` (MG:400-670) started from phi = 0 with the input as
    its rhs -- exactly the set_guess + vcycle_noinit step of MG:600-606.
    Returns the relative-residual history (one entry per V-cycle, the last one
    recomputed as rhs - L[phi]).  Norms and inner products are numpy sums, so
    the history agrees with the device's to rounding, not bitwise.
    """
    v = rhs.valid
    vol = v.dx * v.dy

    def nrm(a):
        return float(np.sqrt(vol * np.sum(a * a)))

    def dot(a, b):
        return float(vol * np.sum(a * b))

    def true_residual():
        rb = BoxData(v)
        compute_residual(rb, rhs, phi, geo, bc, homog)
        return rb.interior().copy()

    def precond(x):
        e, f = BoxData(v, 1, 1), BoxData(v)
        f.interior()[:] = x
        rep = vcycle(e, f, geo, bc, True, 0.0, 1, numcycles=numcycles, smooth_down=smooth_down,
                     smooth_up=smooth_up, smooth_bottom=smooth_bottom, zerophi=True, gs_order=gs_order)
        if rep.diverged:
            raise RuntimeError("preconditioning V-cycle raised the residual")
        lap = BoxData(v)
        compute_laplacian(lap, e, geo, bc, True)
        return e.interior().copy(), lap.interior().copy()

    r = true_residual()
    rscale = nrm(r)
    relres = [1.0]
    if rscale == 0.0:
        relres, rscale = [0.0], 1.0
    if relres[0] <= tol:
        return relres
    x = phi.interior()
    k = 0
    while True:
        rh, p = r.copy(), r.copy()
        rho = dot(rh, r)
        passed = False
        while k < maxiters:
            y, vv = precond(p)
            k += 1
            alpha = rho / dot(rh, vv)
            if not np.isfinite(alpha):
                relres.append(relres[-1])
                break
            x[:] = x + alpha * y
            r = r - alpha * vv
            relres.append(nrm(r) / rscale)
            if relres[-1] <= tol:
                passed = True
                break
            if k >= maxiters:
                break
            z, t = precond(r)
            k += 1
            omega = dot(t, r) / dot(t, t)
            if not np.isfinite(omega) or omega == 0.0:
                relres.append(relres[-1])
                break
            x[:] = x + omega * z
            r = r - omega * t
            relres.append(nrm(r) / rscale)
            if relres[-1] <= tol:
                passed = True
                break
            rho_new = dot(rh, r)
            beta = (rho_new / rho) * (alpha / omega)
            if not np.isfinite(beta) or rho_new == 0.0:
                break
            rho = rho_new
            p = p - omega * vv
            p = beta * p + r
        r = true_residual()
        relres[k] = nrm(r) / rscale
        del relres[k + 1:]
        if (passed and relres[k] <= tol) or k >= maxiters:
            fill_ghosts(phi, bc, geo, homog, False)
            return relres


def gmres_vcycle(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, tol: float,
                 maxiters: int, restart: int = 64, numcycles: int = 1, smooth_down: int = 8, smooth_up: int = 8,
                 smooth_bottom: int = 8, gs_order: int = 1):
    """Oracle for the solver's MGP_FLAG_GMRES mode (no Fortran counterpart).

    Restarted, right-preconditioned GMRES(restart) (Saad and Schultz, SIAM J.
    Sci. Stat. Comput. 7, 1986) on L_h e = r0, L_h and the V-cycle
    preconditioner as in ``krylov_vcycle``, the preconditioned vectors kept
    (flexible form).  Each step: one V-cycle, w = L_h z_j, one pass of
    classical Gram-Schmidt (every coefficient from the same w), Givens
    rotations.  At convergence of the rotated residual, a breakdown or
    ``restart`` steps: phi += Z y, the true residual rhs - L[phi] replaces the
    last history entry, and the solve restarts from it if it has not passed.
    Inner products are unweighted; the history is weighted like the
    reference's norms (sqrt(dx dy)).  Returns the relative-residual history,
    one entry per V-cycle; it agrees with the device's to rounding.
    """
    v = rhs.valid
    vol = v.dx * v.dy
    sv = float(np.sqrt(vol))

    def true_residual():
        rb = BoxData(v)
        compute_residual(rb, rhs, phi, geo, bc, homog)
        return rb.interior().copy()

    def precond(x):
        e, f = BoxData(v, 1, 1), BoxData(v)
        f.interior()[:] = x
        rep = vcycle(e, f, geo, bc, True, 0.0, 1, numcycles=numcycles, smooth_down=smooth_down,
                     smooth_up=smooth_up, smooth_bottom=smooth_bottom, zerophi=True, gs_order=gs_order)
        if rep.diverged:
            raise RuntimeError("preconditioning V-cycle raised the residual")
        lap = BoxData(v)
        compute_laplacian(lap, e, geo, bc, True)
        return e.interior().copy(), lap.interior().copy()

    m = restart
    r = true_residual()
    rscale = sv * float(np.sqrt(np.sum(r * r)))
    relres = [1.0]
    if rscale == 0.0:
        relres, rscale = [0.0], 1.0
    if relres[0] <= tol:
        return relres
    x = phi.interior()
    k = 0
    while True:
        beta = float(np.sqrt(np.sum(r * r)))
        if not (beta > 0.0) or not np.isfinite(beta):
            return relres
        V, Z = [r / beta], []
        H = np.zeros((m + 1, m))
        cs, sn, g = np.zeros(m), np.zeros(m), np.zeros(m + 1)
        g[0] = beta
        jend = 0
        for j in range(m):
            if k >= maxiters:
                break
            z, w = precond(V[j])
            k += 1
            Z.append(z)
            h = np.array([float(np.sum(w * V[i])) for i in range(j + 1)])
            for i in range(j + 1):
                w = w - h[i] * V[i]
            hn = float(np.sqrt(np.sum(w * w)))
            col = np.zeros(m + 1)
            col[:j + 1] = h
            col[j + 1] = hn
            for i in range(j):   # earlier rotations
                t = cs[i] * col[i] + sn[i] * col[i + 1]
                col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1]
                col[i] = t
            den = float(np.hypot(col[j], col[j + 1]))
            cs[j] = col[j] / den if den > 0.0 else 1.0
            sn[j] = col[j + 1] / den if den > 0.0 else 0.0
            col[j], col[j + 1] = den, 0.0
            H[:, j] = col
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            jend = j + 1
            relres.append(float(abs(g[j + 1]) * sv / rscale))
            if relres[-1] <= tol or not (hn > 0.0) or not (den > 0.0):
                break
            V.append(w * (1.0 / hn))
        if jend == 0:
            return relres
        y = np.zeros(jend)
        for i in range(jend - 1, -1, -1):   # H y = g, upper triangular
            y[i] = (g[i] - float(np.dot(H[i, i + 1:jend], y[i + 1:jend]))) / H[i, i]
        for i in range(jend):
            x[:] = x + y[i] * Z[i]
        r = true_residual()
        relres[k] = sv * float(np.sqrt(np.sum(r * r))) / rscale
        if relres[k] <= tol or k >= maxiters:
            fill_ghosts(phi, bc, geo, homog, False)
            return relres
