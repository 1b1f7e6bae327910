"""Python binding of the C ABI (include/mgp2d.h) with the call shapes of the
Fortran module procedures it replaces.

    from mgpoisson2d_b200 import vcycle, fmg, dc_vcycle, Solver
    report = vcycle(phi, rhs, geo, bc, homog, tol=1e-10, maxiters=100)

Arrays are ``BoxData`` (host NumPy or device torch); the library stages host
arrays through device memory itself.  Every call raises ``MGPError`` on a
non-zero status.  The library file must have been built
(``python -m mgpoisson2d_b200.build``); importing this module raises
ImportError otherwise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .types import (BD_CELL, BD_NODE, KIND_DD, KIND_MG, STATUS_NAMES, BdryData, Box, BoxData, GeoData, MgpArray,
                    MgpBdry, MgpBox, MgpGeo, MgpReport, Report, make_report, read_report)

FLAG_DIRICHLET_COUPLED_DIAG = 1
FLAG_TIME_SMOOTHER = 2
FLAG_KRYLOV = 4
FLAG_MIXED = 8
FLAG_DIRECT_COARSE = 16
FLAG_GMRES = 32
FLAG_DIRECT_LARGE = 64
FLAG_LOCKSTEP = 128
FLAG_REPORT_MAXITER = 256
FLAG_BF16_COARSE = 512

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmgp2d.so")

if not os.path.exists(_LIB_PATH):
    raise ImportError(f"mgpoisson2d_b200: CUDA library {_LIB_PATH} is missing; "
                      "build it with `python -m mgpoisson2d_b200.build`")

_lib = C.CDLL(_LIB_PATH)

_P = C.POINTER
_B, _A, _BC, _G, _R = _P(MgpBox), _P(MgpArray), _P(MgpBdry), _P(MgpGeo), _P(MgpReport)
_i, _d, _vp = C.c_int, C.c_double, C.c_void_p

_SIGS = {
    "mgp_set_flags": [_i],
    "mgp_estimate_maxdepth": [_P(_i), _B],
    "mgp_create_mgschedule": [_P(_i), _P(_i), _P(_i), _B],
    "mgp_fill_ghosts": [_B, _A, _BC, _G, _i, _i],
    "mgp_extrapolate_ghosts": [_B, _A, _i],
    "mgp_compute_invdiags": [_B, _A, _G, _BC, _i],
    "mgp_compute_laplacian": [_B, _A, _A, _G, _BC, _i, _i],
    "mgp_compute_residual": [_B, _A, _A, _A, _G, _BC, _i, _i],
    "mgp_relax_gs": [_B, _A, _A, _G, _BC, _i, _A, _d, _d, _i, _i, _i],
    "mgp_relax_jacobi": [_B, _A, _A, _G, _BC, _i, _A, _d, _d, _i, _i, _i],
    "mgp_solve_bicgstab2": [_B, _A, _A, _G, _BC, _i, _A, _d, _i, _i, _i, _i],
    "mgp_solve_bicgstab2_noalloc": [_B, _A, _A, _G, _BC, _i, _A, _d, _i, _i, _i, _i],
    "mgp_restrict": [_B, _A, _B, _A, _i, _i],
    "mgp_compute_pd": [_B, _A, _A, _i, _i],
    "mgp_compute_grad": [_B, _A, _A, _A, _G, _BC, _i],
    "mgp_fill_boundary_fluxes": [_B, _A, _A, _BC, _i],
    "mgp_compute_div": [_B, _A, _A, _A],
    "mgp_prolong": [_B, _A, _B, _A, _G, _G, _BC, _i],
    "mgp_pnorm": [_B, _A, _i, _P(_d)],
    "mgp_inner_prod": [_B, _A, _A, _P(_d)],
    "mgp_vcycle": [_B, _A, _A, _G, _BC, _i, _i, _i, _d, _i, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_fmg": [_B, _A, _A, _G, _BC, _i, _i, _i, _d, _i, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_dc_vcycle": [_B, _A, _A, _G, _BC, _i, _i, _i, _d, _i, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_solver_create": [_B, _G, _BC, _i, _i, _i, _P(_vp)],
    "mgp_solver_destroy": [_vp],
    "mgp_solver_set_stream": [_vp, _vp],
    "mgp_solver_maxdepth": [_vp, _P(_i)],
    "mgp_solver_vcycle": [_vp, _A, _A, _BC, _i, _d, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_solver_fmg": [_vp, _A, _A, _BC, _i, _d, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_solver_dc_vcycle": [_vp, _A, _A, _BC, _i, _d, _i, _i, _i, _i, _i, _i, _i, _R],
    "mgp_map_geometry": [_B, _i, _P(_d), _G],
    "mgp_map_fourier_rhs": [_B, _i, _P(_d), _i, _P(_d), _P(_i), _P(_i), _A, _A],
    "mgp_batch_create": [_i, _B, _G, _BC, _i, _i, _i, _i, _P(_vp)],
    "mgp_batch_destroy": [_vp],
    "mgp_batch_size": [_vp, _P(_i)],
    "mgp_batch_vcycle": [_vp, _A, _A, _BC, _i, _d, _i, _i, _i, _i, _i, _i, _R],
    "mgp_batch_set_tuning": [_vp, _i, _i],
    "mgp_batch_get_tuning": [_vp, _P(_i), _P(_i)],
    "mgp_server_create": [_i, C.c_size_t, _i, _P(_vp)],
    "mgp_server_submit": [_vp, C.c_ulonglong, _B, _G, _BC, _A, _A, _i, _d, _i, _i, _i, _i, _i, _i,
                          _P(C.c_longlong)],
    "mgp_server_wait": [_vp, C.c_longlong, _R, _P(_d), _P(_d)],
    "mgp_server_destroy": [_vp],
    "mgp_selftest_grid_barrier": [_i, _i, _i, _d, _P(_d)],
}
for _name, _args in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.argtypes = _args
    _f.restype = _i
_lib.mgp_version.restype = C.c_char_p
_lib.mgp_last_error.restype = C.c_char_p
_lib.mgp_kernel_launch_count.restype = C.c_longlong

#: every symbol include/mgp2d.h declares
EXPORTS = sorted(list(_SIGS) + ["mgp_version", "mgp_last_error", "mgp_kernel_launch_count"])


class MGPError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = _lib.mgp_last_error().decode(errors="replace")
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def _ck(rc: int, where: str):
    if rc != 0:
        raise MGPError(rc, where)


def _r(x):
    return C.byref(x)


def library_path() -> str:
    return _LIB_PATH


def kernel_launch_count() -> int:
    return int(_lib.mgp_kernel_launch_count())


def selftest_grid_barrier(nctas: int, skip_cta: int = -1, nbarriers: int = 64, wait_s: float = 0.05):
    """Run the coarse cycle's bounded grid barrier (mgp_selftest_grid_barrier).
    Returns (status, device seconds); the status is not raised."""
    sec = C.c_double(0.0)
    rc = _lib.mgp_selftest_grid_barrier(nctas, skip_cta, nbarriers, wait_s, _r(sec))
    return int(rc), sec.value


def set_flags(flags: int) -> int:
    """Process-wide flags for the calls without a flags argument (mgp_set_flags)."""
    return int(_lib.mgp_set_flags(flags))


# ---- schedule (MG:38-129) -------------------------------------------------- #
def estimate_maxdepth(maxdepth: int, valid: Box) -> int:
    m = C.c_int(maxdepth)
    _ck(_lib.mgp_estimate_maxdepth(_r(m), _r(valid.c())), "estimate_maxdepth")
    return m.value


def create_mgschedule(maxdepth: int, valid: Box):
    m = C.c_int(maxdepth)
    rx = (C.c_int * max(maxdepth, 1))()
    ry = (C.c_int * max(maxdepth, 1))()
    _ck(_lib.mgp_create_mgschedule(rx, ry, _r(m), _r(valid.c())), "create_mgschedule")
    return list(rx)[:m.value], list(ry)[:m.value], m.value


# ---- operator-level calls --------------------------------------------------- #
def fill_ghosts(phi: BoxData, bc: BdryData, geo: GeoData, homog: bool, do_neum: bool = True):
    """fill_ghosts, arrayutils.f90:1277-1492."""
    a, b, g = phi.c(), bc.c(), geo.c()
    _ck(_lib.mgp_fill_ghosts(_r(phi.valid.c()), _r(a), _r(b), _r(g), int(homog), int(do_neum)), "fill_ghosts")


def extrapolate_ghosts(phi: BoxData, order: int):
    """extrapolate_ghosts, arrayutils.f90:1497-1566."""
    a = phi.c()
    _ck(_lib.mgp_extrapolate_ghosts(_r(phi.valid.c()), _r(a), order), "extrapolate_ghosts")


def compute_invdiags(invdiags: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    """compute_invdiags, poisson2d.f90:16-388."""
    a, b, g = invdiags.c(), bc.c(), geo.c()
    _ck(_lib.mgp_compute_invdiags(_r(invdiags.valid.c()), _r(a), _r(g), _r(b), int(homog)), "compute_invdiags")


def compute_laplacian(lap: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool, jscale: bool = False):
    """compute_laplacian, poisson2d.f90:886-1319."""
    l, p, b, g = lap.c(), phi.c(), bc.c(), geo.c()
    _ck(_lib.mgp_compute_laplacian(_r(lap.valid.c()), _r(l), _r(p), _r(g), _r(b), int(homog), int(jscale)),
        "compute_laplacian")


def compute_pd(pd: BoxData, phi: BoxData, dir: int, nodedir: int):
    """compute_pd, poisson2d.f90:404-795 (pd nodal in x for nodedir 1, y for 2)."""
    d, p = pd.c(), phi.c()
    _ck(_lib.mgp_compute_pd(_r(phi.valid.c()), _r(d), _r(p), dir, nodedir), "compute_pd")


def compute_grad(xflux: BoxData, yflux: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool):
    """compute_grad, poisson2d.f90:809-850: J Grad[phi] on x- and y-faces."""
    x, y, p, g, b = xflux.c(), yflux.c(), phi.c(), geo.c(), bc.c()
    _ck(_lib.mgp_compute_grad(_r(phi.valid.c()), _r(x), _r(y), _r(p), _r(g), _r(b), int(homog)), "compute_grad")


def fill_boundary_fluxes(xflux: BoxData, yflux: BoxData, bc: BdryData, homog: bool):
    """fill_boundary_fluxes, arrayutils.f90:1574-1622."""
    x, y, b = xflux.c(), yflux.c(), bc.c()
    _ck(_lib.mgp_fill_boundary_fluxes(_r(xflux.valid.c()), _r(x), _r(y), _r(b), int(homog)),
        "fill_boundary_fluxes")


def compute_div(div: BoxData, xflux: BoxData, yflux: BoxData):
    """compute_div, poisson2d.f90:860-879."""
    d, x, y = div.c(), xflux.c(), yflux.c()
    _ck(_lib.mgp_compute_div(_r(div.valid.c()), _r(d), _r(x), _r(y)), "compute_div")


def compute_residual(res: BoxData, rhs: BoxData, phi: BoxData, geo: GeoData, bc: BdryData, homog: bool,
                     jscale: bool = False):
    """compute_residual, poisson2d.f90:1327-1353."""
    r, f, p, b, g = res.c(), rhs.c(), phi.c(), bc.c(), geo.c()
    _ck(_lib.mgp_compute_residual(_r(res.valid.c()), _r(r), _r(f), _r(p), _r(g), _r(b), int(homog), int(jscale)),
        "compute_residual")


def relax_jacobi(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
                 omega: float, tol: float, maxiters: int, zerophi: bool = False, verbosity: int = 0):
    """relax_jacobi, poisson2d.f90:1358-1451."""
    p, f, b, g, d = phi.c(), rhs.c(), bc.c(), geo.c(), invdiags.c()
    _ck(_lib.mgp_relax_jacobi(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), omega, tol,
                              maxiters, int(zerophi), verbosity), "relax_jacobi")


def relax_gs(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData, omega: float,
             tol: float, maxiters: int, zerophi: bool, verbosity: int = 0):
    """relax_gs, poisson2d.f90:1460-1988 (4-colour order on the device)."""
    p, f, b, g, d = phi.c(), rhs.c(), bc.c(), geo.c(), invdiags.c()
    _ck(_lib.mgp_relax_gs(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), omega, tol, maxiters,
                          int(zerophi), verbosity), "relax_gs")


def solve_bicgstab2(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool, invdiags: BoxData,
                    tol: float, max_iters: int, max_restarts: int, zerophi: bool, verbosity: int = 0):
    """solve_bicgstab2, poisson2d.f90:2253-2477."""
    p, f, b, g, d = phi.c(), rhs.c(), bc.c(), geo.c(), invdiags.c()
    _ck(_lib.mgp_solve_bicgstab2(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), tol, max_iters,
                                 max_restarts, int(zerophi), verbosity), "solve_bicgstab2")


NOALLOC_MAX_SIDE = 128


def solve_bicgstab2_noalloc(phi: BoxData, rhs: BoxData, geo: GeoData, bc: BdryData, homog: bool,
                            invdiags: BoxData, tol: float, max_iters: int, max_restarts: int, zerophi: bool,
                            verbosity: int = 0):
    """mgp_solve_bicgstab2_noalloc: the bottom solver on device arrays without
    allocating device memory (for callers that cannot allocate; grids of at
    most NOALLOC_MAX_SIDE cells per side; concurrent calls share one scratch
    array and must not overlap on the device)."""
    p, f, b, g, d = phi.c(), rhs.c(), bc.c(), geo.c(), invdiags.c()
    _ck(_lib.mgp_solve_bicgstab2_noalloc(_r(phi.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), _r(d), tol,
                                         max_iters, max_restarts, int(zerophi), verbosity), "solve_bicgstab2_noalloc")


def restrict(fine: BoxData, crse: BoxData):
    """restrict, MGPoisson2D.f90:135-257."""
    f, c = fine.c(), crse.c()
    _ck(_lib.mgp_restrict(_r(fine.valid.c()), _r(f), _r(crse.valid.c()), _r(c), fine.offi, fine.offj), "restrict")


def prolong(fine: BoxData, crse: BoxData, fine_geo: GeoData, crse_geo: GeoData, crse_bc: BdryData, order: int):
    """prolong, MGPoisson2D.f90:262-394."""
    f, c, fg, cg, b = fine.c(), crse.c(), fine_geo.c(), crse_geo.c(), crse_bc.c()
    _ck(_lib.mgp_prolong(_r(fine.valid.c()), _r(f), _r(crse.valid.c()), _r(c), _r(fg), _r(cg), _r(b), order),
        "prolong")


def pnorm(bd: BoxData, p: int) -> float:
    """pnorm, arrayutils.f90:753-796 (p = 0, 1, 2)."""
    out = C.c_double()
    a = bd.c()
    _ck(_lib.mgp_pnorm(_r(bd.valid.c()), _r(a), p, _r(out)), "pnorm")
    return out.value


def inner_prod(a: BoxData, b: BoxData) -> float:
    """inner_prod, arrayutils.f90:637-661."""
    out = C.c_double()
    x, y = a.c(), b.c()
    _ck(_lib.mgp_inner_prod(_r(a.valid.c()), _r(x), _r(y), _r(out)), "inner_prod")
    return out.value


# ---- drivers with the Fortran argument lists ------------------------------- #
def _driver(fn, name, phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles, smooth_down, smooth_up,
            smooth_bottom, zerophi, verbosity) -> Report:
    rep, buf = make_report(maxiters)
    p, f, b, g = phi.c(), rhs.c(), bc.c(), geo.c()
    rc = fn(_r(rhs.valid.c()), _r(p), _r(f), _r(g), _r(b), int(homog), 0, 0, tol, maxiters, maxdepth_user, numcycles,
            smooth_down, smooth_up, smooth_bottom, int(zerophi), verbosity, _r(rep))
    _ck(rc, name)
    return read_report(rep, buf)


def vcycle(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=8, smooth_up=8,
           smooth_bottom=8, zerophi=False, verbosity=0) -> Report:
    """MGPoisson2D::vcycle, MGPoisson2D.f90:400-670."""
    return _driver(_lib.mgp_vcycle, "vcycle", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                   smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)


def fmg(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=8, smooth_up=8,
        smooth_bottom=8, zerophi=False, verbosity=0) -> Report:
    """MGPoisson2D::fmg, MGPoisson2D.f90:860-1122."""
    return _driver(_lib.mgp_fmg, "fmg", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user, numcycles,
                   smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)


def dc_vcycle(phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user=-1, numcycles=1, smooth_down=1, smooth_up=1,
              smooth_bottom=1, zerophi=False, verbosity=0) -> Report:
    """DeferredMGPoisson2D::vcycle, MGPoisson2D_DD.f90:589-862."""
    return _driver(_lib.mgp_dc_vcycle, "dc_vcycle", phi, rhs, geo, bc, homog, tol, maxiters, maxdepth_user,
                   numcycles, smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)


class Solver:
    """A hierarchy built once and kept in HBM (mgp_solver_create).

    ``kind`` is KIND_MG (vcycle / fmg) or KIND_DD (deferred-correction vcycle);
    ``flags`` e.g. FLAG_DIRICHLET_COUPLED_DIAG | FLAG_KRYLOV.
    """

    def __init__(self, valid: Box, geo: GeoData, bc: BdryData, kind: int = KIND_MG, flags: int = 0,
                 maxdepth_user: int = -1):
        self._h = C.c_void_p()
        b, g = bc.c(), geo.c()
        _ck(_lib.mgp_solver_create(_r(valid.c()), _r(g), _r(b), kind, flags, maxdepth_user, _r(self._h)),
            "solver_create")
        self.valid, self.kind, self.flags = valid, kind, flags
        md = C.c_int()
        _lib.mgp_solver_maxdepth(self._h, _r(md))
        self.maxdepth = md.value

    def close(self):
        if self._h:
            _lib.mgp_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_stream(self, stream_handle: int):
        _ck(_lib.mgp_solver_set_stream(self._h, C.c_void_p(stream_handle)), "solver_set_stream")

    def _solve(self, fn, name, phi, rhs, bc, homog, tol, maxiters, numcycles, nd, nu, nb, zerophi, verbosity):
        rep, buf = make_report(maxiters)
        p, f, b = phi.c(), rhs.c(), bc.c()
        _ck(fn(self._h, _r(p), _r(f), _r(b), int(homog), tol, maxiters, numcycles, nd, nu, nb, int(zerophi),
               verbosity, _r(rep)), name)
        return read_report(rep, buf)

    def vcycle(self, phi, rhs, bc, homog, tol, maxiters, numcycles=1, smooth_down=8, smooth_up=8, smooth_bottom=8,
               zerophi=False, verbosity=0) -> Report:
        return self._solve(_lib.mgp_solver_vcycle, "solver_vcycle", phi, rhs, bc, homog, tol, maxiters, numcycles,
                           smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)

    def fmg(self, phi, rhs, bc, homog, tol, maxiters, numcycles=1, smooth_down=8, smooth_up=8, smooth_bottom=8,
            zerophi=False, verbosity=0) -> Report:
        return self._solve(_lib.mgp_solver_fmg, "solver_fmg", phi, rhs, bc, homog, tol, maxiters, numcycles,
                           smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)

    def dc_vcycle(self, phi, rhs, bc, homog, tol, maxiters, numcycles=1, smooth_down=1, smooth_up=1, smooth_bottom=1,
                  zerophi=False, verbosity=0) -> Report:
        return self._solve(_lib.mgp_solver_dc_vcycle, "solver_dc_vcycle", phi, rhs, bc, homog, tol, maxiters,
                           numcycles, smooth_down, smooth_up, smooth_bottom, zerophi, verbosity)


MAP_IDENTITY, MAP_WAVY_EXP, MAP_SKEW_LAYER = 0, 1, 2


def _params(params):
    arr = (C.c_double * max(1, len(params)))(*params)
    return arr


def map_geometry(valid: Box, kind: int, params=(), device: bool = True, ng: int = 1) -> GeoData:
    """Metric terms of an analytic map, generated on the device
    (mgp_map_geometry); the arrays stay on the device unless device=False."""
    mk = (lambda oi, oj: BoxData.device_zeros(valid, ng, ng, oi, oj)) if device else \
        (lambda oi, oj: BoxData(valid, ng, ng, oi, oj))
    geo = GeoData(mk(BD_CELL, BD_CELL), mk(BD_NODE, BD_CELL), mk(BD_NODE, BD_CELL), mk(BD_CELL, BD_NODE),
                  mk(BD_CELL, BD_NODE), valid.dx, valid.dy)
    g = geo.c()
    _ck(_lib.mgp_map_geometry(_r(valid.c()), kind, _params(params), _r(g)), "map_geometry")
    return geo


def map_fourier_rhs(valid: Box, kind: int, params, amp, mx, my, J: BoxData, device: bool = True) -> BoxData:
    """rhs = J (f - <f>_J), f = sum amp cos(pi mx x) cos(pi my y) at the mapped
    cell centres (mgp_map_fourier_rhs)."""
    rhs = BoxData.device_zeros(valid) if device else BoxData(valid)
    n = len(amp)
    a = (C.c_double * max(1, n))(*amp)
    m1 = (C.c_int * max(1, n))(*[int(v) for v in mx])
    m2 = (C.c_int * max(1, n))(*[int(v) for v in my])
    j, r = J.c(), rhs.c()
    _ck(_lib.mgp_map_fourier_rhs(_r(valid.c()), kind, _params(params), n, a, m1, m2, _r(j), _r(r)),
        "map_fourier_rhs")
    return rhs


class Batch:
    """Independent problems solved concurrently (mgp_batch_*): one resident
    hierarchy per problem, ``nstreams`` host workers with their own streams.
    ``problems`` is a list of (valid, geo, bc)."""

    def __init__(self, problems, kind: int = KIND_MG, flags: int = 0, maxdepth_user: int = -1, nstreams: int = 8):
        n = len(problems)
        self._boxes = (MgpBox * n)(*[p[0].c() for p in problems])
        self._geos = (MgpGeo * n)(*[p[1].c() for p in problems])
        self._bcs = (MgpBdry * n)(*[p[2].c() for p in problems])
        self._keep = problems   # the geometry arrays must outlive the batch's set-up
        self._h = C.c_void_p()
        _ck(_lib.mgp_batch_create(n, self._boxes, self._geos, self._bcs, kind, flags, maxdepth_user, nstreams,
                                  _r(self._h)), "batch_create")
        self.n = n
        self._statuses = []
        self._nstreams = max(1, min(nstreams, n))

    def close(self):
        if self._h:
            _lib.mgp_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_tuning(self, groups: int = 0, pairs: int = 0):
        """Lockstep knobs (mgp_batch_set_tuning): concurrent groups, two sweeps per launch."""
        _ck(_lib.mgp_batch_set_tuning(self._h, groups, pairs), "batch_set_tuning")

    def tuning(self):
        g, p = C.c_int(), C.c_int()
        _ck(_lib.mgp_batch_get_tuning(self._h, _r(g), _r(p)), "batch_get_tuning")
        return {"groups": g.value, "pairs": p.value}

    def autotune(self, phis, rhss, bcs, homog, tol, maxiters, cache_path=None, key=None, groups=(1, 2, 4),
                 pairs=(0, 1), numcycles=1, smooth_down=8, smooth_up=8, smooth_bottom=8):
        """Time the lockstep knobs (every combination of `groups` and `pairs`,
        one solve each, device-timed) and keep the fastest.  Every combination
        gives the same bits, so the search changes nothing but speed.  With
        `cache_path` the choice is stored under `key` in that JSON file and read
        back instead of searching.  Returns the chosen knobs with the timings."""
        import json
        import os
        import time
        if cache_path and key and os.path.exists(cache_path):
            try:
                hit = json.load(open(cache_path)).get(key)
            except (OSError, ValueError):
                hit = None
            if hit:
                self.set_tuning(hit["groups"], hit["pairs"])
                return dict(hit, cached=True)
        sync = None
        try:
            import torch
            if torch.cuda.is_available():
                sync = torch.cuda.synchronize
        except ImportError:
            pass
        times = {}
        for g in groups:
            for p in pairs:
                if g > self._nstreams:
                    continue
                self.set_tuning(g, p)
                for x in phis:
                    x.data[...] = 0.0
                if sync:
                    sync()
                t0 = time.perf_counter()
                self.vcycle(phis, rhss, bcs, homog, tol, maxiters, numcycles, smooth_down, smooth_up, smooth_bottom)
                if sync:
                    sync()
                times[f"{g},{p}"] = time.perf_counter() - t0
        best = min(times, key=times.get)
        g, p = (int(x) for x in best.split(","))
        self.set_tuning(g, p)
        out = {"groups": g, "pairs": p, "seconds": times}
        if cache_path and key:
            try:
                cache = json.load(open(cache_path)) if os.path.exists(cache_path) else {}
            except (OSError, ValueError):
                cache = {}
            cache[key] = out
            with open(cache_path, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
        return dict(out, cached=False)

    def vcycle(self, phis, rhss, bcs, homog, tol, maxiters, numcycles=1, smooth_down=8, smooth_up=8,
               smooth_bottom=8, zerophi=False):
        n = self.n
        reps, bufs = zip(*[make_report(maxiters) for _ in range(n)])
        rarr = (MgpReport * n)(*reps)
        parr = (MgpArray * n)(*[p.c() for p in phis])
        farr = (MgpArray * n)(*[f.c() for f in rhss])
        barr = (MgpBdry * n)(*[b.c() for b in bcs])
        rc = _lib.mgp_batch_vcycle(self._h, parr, farr, barr, int(homog), tol, maxiters, numcycles, smooth_down,
                                   smooth_up, smooth_bottom, int(zerophi), rarr)
        self._statuses = [int(rarr[k].status) for k in range(n)]
        _ck(rc, "batch_vcycle")
        return [read_report(rarr[k], bufs[k]) for k in range(n)]

    def last_statuses(self):
        """Each problem's status from the last vcycle call (also after it raised)."""
        return list(self._statuses)


class Server:
    """A solve server (mgp_server_*): ``nworkers`` slots, admission by device
    memory (``mem_budget`` bytes, 0 = 90 % of the free memory), resident
    hierarchies reused per nonzero ``key``.  ``submit`` returns a ticket;
    ``wait`` returns (Report, latency_s, queue_s)."""

    def __init__(self, nworkers: int = 8, mem_budget: int = 0, flags: int = 0):
        self._h = C.c_void_p()
        _ck(_lib.mgp_server_create(nworkers, mem_budget, flags, _r(self._h)), "server_create")
        self._live = {}

    def submit(self, valid: Box, geo: GeoData, bc: BdryData, phi: BoxData, rhs: BoxData, homog, tol, maxiters,
               key: int = 0, numcycles=1, smooth_down=8, smooth_up=8, smooth_bottom=8, zerophi=False) -> int:
        t = C.c_longlong()
        b, g, c, p, f = valid.c(), geo.c(), bc.c(), phi.c(), rhs.c()
        _ck(_lib.mgp_server_submit(self._h, key, _r(b), _r(g), _r(c), _r(p), _r(f), int(homog), tol, maxiters,
                                   numcycles, smooth_down, smooth_up, smooth_bottom, int(zerophi), _r(t)),
            "server_submit")
        # the arrays (and the structs describing them) must outlive the request
        self._live[t.value] = (b, g, c, p, f, valid, geo, bc, phi, rhs, maxiters)
        return t.value

    def wait(self, ticket: int):
        maxiters = self._live[ticket][-1]
        rep, buf = make_report(maxiters)
        lat, qt = C.c_double(), C.c_double()
        rc = _lib.mgp_server_wait(self._h, ticket, _r(rep), _r(lat), _r(qt))
        self._live.pop(ticket, None)
        _ck(rc, "server_wait")
        return read_report(rep, buf), lat.value, qt.value

    def close(self):
        if self._h:
            _lib.mgp_server_destroy(self._h)
            self._h = C.c_void_p()
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


__all__ = ["vcycle", "fmg", "dc_vcycle", "Solver", "fill_ghosts", "extrapolate_ghosts", "compute_invdiags",
           "compute_laplacian", "compute_residual", "compute_pd", "compute_grad", "fill_boundary_fluxes", "compute_div", "relax_gs", "relax_jacobi", "solve_bicgstab2", "solve_bicgstab2_noalloc", "NOALLOC_MAX_SIDE", "restrict", "prolong", "pnorm",
           "inner_prod", "estimate_maxdepth", "create_mgschedule", "MGPError", "library_path", "kernel_launch_count",
           "set_flags", "FLAG_DIRICHLET_COUPLED_DIAG", "FLAG_TIME_SMOOTHER", "FLAG_KRYLOV", "FLAG_MIXED", "FLAG_DIRECT_COARSE", "FLAG_GMRES", "FLAG_DIRECT_LARGE", "FLAG_LOCKSTEP", "FLAG_REPORT_MAXITER", "FLAG_BF16_COARSE", "Batch", "Server", "map_geometry", "map_fourier_rhs",
           "MAP_IDENTITY", "MAP_WAVY_EXP", "MAP_SKEW_LAYER", "EXPORTS", "KIND_MG", "KIND_DD"]
