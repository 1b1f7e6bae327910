"""Metric generation: computational grid -> (J, J g^ij) on the staggered layout
the solver takes as input.

The reference builds its geometry in its test program (src/tests/test.f90:320-716):
positions are evaluated at cell centres, faces and nodes, and the metric
derivatives are one-cell differences of those positions (fill_dxdXi,
test.f90:566-646).  ``terrain_geometry`` reproduces that generator for the
reference's own map (x = xi, y = el(x) + (H - el) * eta / H, el = sin^2(pi x/L)/4,
test.f90:396-440, 528) with the reference's closed forms for x = xi maps
(test.f90:685-716).  ``mapped_geometry`` takes any smooth map x(xi, eta),
y(xi, eta) and uses the general forms

    J = x_xi y_eta - x_eta y_xi,
    J g^{xi xi}   = (x_eta^2 + y_eta^2) / J,
    J g^{xi eta}  = J g^{eta xi} = -(x_xi x_eta + y_xi y_eta) / J,
    J g^{eta eta} = (x_xi^2 + y_xi^2) / J,

which reduce to the reference's formulas when x = xi.  Both return arrays with
``ng`` ghost layers, as the reference's define_geometry does (ng = 1).
"""
from __future__ import annotations

import math
from typing import Callable, Tuple

import numpy as np

from .types import BD_CELL, BD_NODE, Box, BoxData, GeoData

MapFn = Callable[[np.ndarray, np.ndarray], Tuple[np.ndarray, np.ndarray]]


def _coords(valid: Box, offi: int, offj: int, ng: int, shift_i: float = 0.0, shift_j: float = 0.0):
    """Computational coordinates of the points of a centred array with ghosts.

    Point (i, j) of centring (offi, offj) sits at xi = (i + offx) * dx with
    offx = 1/2 for cell centring, 0 for nodes (define_box_data, AU:389-451;
    fill_x, test.f90:370-390).  ``shift_*`` moves by half a cell.
    """
    nvx = valid.nx + (1 if offi == BD_NODE else 0)
    nvy = valid.ny + (1 if offj == BD_NODE else 0)
    offx = 0.5 if offi == BD_CELL else 0.0
    offy = 0.5 if offj == BD_CELL else 0.0
    i = np.arange(valid.ilo - ng, valid.ilo + nvx + ng, dtype=np.float64)
    j = np.arange(valid.jlo - ng, valid.jlo + nvy + ng, dtype=np.float64)
    xi = (i + offx + shift_i) * valid.dx
    eta = (j + offy + shift_j) * valid.dy
    XI, ETA = np.meshgrid(xi, eta, indexing="ij")
    return XI, ETA


def _bd(valid, ng, offi, offj, arr):
    return BoxData(valid, ng, ng, offi, offj, data=np.asfortranarray(arr))


# --------------------------------------------------------------------------- #
# The reference's own terrain-following map (test.f90:320-716)
# --------------------------------------------------------------------------- #
def terrain_y(xi: np.ndarray, eta: np.ndarray, L: float = 1.0, H: float = 1.0) -> np.ndarray:
    """fill_y + fill_elevation (test.f90:396-440, 528): sinusoidal bottom."""
    el = 0.25 * np.sin(math.pi * xi / L) ** 2
    return el + (H - el) * (eta / H)


def terrain_geometry(valid: Box, L: float = 1.0, H: float = 1.0, ng: int = 1) -> GeoData:
    """define_geometry, test.f90:320-346, for the x = xi terrain map."""
    sx, sy = 1.0 / valid.dx, 1.0 / valid.dy
    h = 0.5

    def Y(XI, ETA):
        return terrain_y(XI, ETA, L, H)

    # J = y_eta at cell centres (fill_J -> fill_dxdXi(dest, 2, 2))
    XI, ETA = _coords(valid, BD_CELL, BD_CELL, ng)
    J = (Y(XI, ETA + h * valid.dy) - Y(XI, ETA - h * valid.dy)) * sy
    # x-faces: Jgup_xx = y_eta (nodes above/below), Jgup_xy = -y_xi (cells left/right)
    XI, ETA = _coords(valid, BD_NODE, BD_CELL, ng)
    y_eta = (Y(XI, ETA + h * valid.dy) - Y(XI, ETA - h * valid.dy)) * sy
    y_xi = (Y(XI + h * valid.dx, ETA) - Y(XI - h * valid.dx, ETA)) * sx
    Jxx, Jxy = y_eta, -y_xi
    # y-faces: Jgup_yx = -y_xi (nodes left/right), Jgup_yy = (1 + y_xi^2) / y_eta (cells below/above)
    XI, ETA = _coords(valid, BD_CELL, BD_NODE, ng)
    y_xi = (Y(XI + h * valid.dx, ETA) - Y(XI - h * valid.dx, ETA)) * sx
    y_eta = (Y(XI, ETA + h * valid.dy) - Y(XI, ETA - h * valid.dy)) * sy
    Jyx, Jyy = -y_xi, (1.0 + y_xi ** 2) / y_eta
    return GeoData(_bd(valid, ng, BD_CELL, BD_CELL, J), _bd(valid, ng, BD_NODE, BD_CELL, Jxx),
                   _bd(valid, ng, BD_NODE, BD_CELL, Jxy), _bd(valid, ng, BD_CELL, BD_NODE, Jyx),
                   _bd(valid, ng, BD_CELL, BD_NODE, Jyy), valid.dx, valid.dy)


def terrain_positions(valid: Box, offi: int, offj: int, ng: int, L: float = 1.0, H: float = 1.0):
    """Cartesian (x, y) of the points of a centred array (fill_x / fill_y)."""
    XI, ETA = _coords(valid, offi, offj, ng)
    return XI.copy(), terrain_y(XI, ETA, L, H)


# --------------------------------------------------------------------------- #
# General maps
# --------------------------------------------------------------------------- #
def mapped_geometry(valid: Box, fmap: MapFn, ng: int = 1) -> GeoData:
    """Metrics of a general map by one-cell differences of staggered positions."""
    sx, sy = 1.0 / valid.dx, 1.0 / valid.dy
    hx, hy = 0.5 * valid.dx, 0.5 * valid.dy

    def derivs(XI, ETA):
        xe, ye = fmap(XI + hx, ETA)
        xw, yw = fmap(XI - hx, ETA)
        xn, yn = fmap(XI, ETA + hy)
        xs, ys = fmap(XI, ETA - hy)
        return (xe - xw) * sx, (xn - xs) * sy, (ye - yw) * sx, (yn - ys) * sy

    XI, ETA = _coords(valid, BD_CELL, BD_CELL, ng)
    x_xi, x_eta, y_xi, y_eta = derivs(XI, ETA)
    J = x_xi * y_eta - x_eta * y_xi

    XI, ETA = _coords(valid, BD_NODE, BD_CELL, ng)
    x_xi, x_eta, y_xi, y_eta = derivs(XI, ETA)
    Jf = x_xi * y_eta - x_eta * y_xi
    Jxx = (x_eta ** 2 + y_eta ** 2) / Jf
    Jxy = -(x_xi * x_eta + y_xi * y_eta) / Jf

    XI, ETA = _coords(valid, BD_CELL, BD_NODE, ng)
    x_xi, x_eta, y_xi, y_eta = derivs(XI, ETA)
    Jf = x_xi * y_eta - x_eta * y_xi
    Jyx = -(x_xi * x_eta + y_xi * y_eta) / Jf
    Jyy = (x_xi ** 2 + y_xi ** 2) / Jf
    return GeoData(_bd(valid, ng, BD_CELL, BD_CELL, J), _bd(valid, ng, BD_NODE, BD_CELL, Jxx),
                   _bd(valid, ng, BD_NODE, BD_CELL, Jxy), _bd(valid, ng, BD_CELL, BD_NODE, Jyx),
                   _bd(valid, ng, BD_CELL, BD_NODE, Jyy), valid.dx, valid.dy)


def positions(valid: Box, fmap: MapFn, offi: int = BD_CELL, offj: int = BD_CELL, ng: int = 0):
    XI, ETA = _coords(valid, offi, offj, ng)
    return fmap(XI, ETA)


# --------------------------------------------------------------------------- #
# Maps of the synthetic workloads
# --------------------------------------------------------------------------- #
def map_identity() -> MapFn:
    return lambda XI, ETA: (XI.copy(), ETA.copy())


def exp_stretch_beta(aspect: float) -> float:
    """beta with (e^beta - 1) / beta = aspect, so that y = (e^{beta eta} - 1)/(e^beta - 1)
    has first-cell height 1/aspect of the uniform one."""
    lo, hi = 1e-9, 60.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.expm1(mid) / mid < aspect:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def map_wavy_exp(amplitude: float = 0.1, aspect: float = 64.0) -> MapFn:
    """x = xi + a sin(2 pi xi) sin(2 pi eta), y = (e^{beta eta} - 1)/(e^beta - 1)."""
    beta = exp_stretch_beta(aspect)
    den = math.expm1(beta)

    def f(XI, ETA):
        x = XI + amplitude * np.sin(2 * math.pi * XI) * np.sin(2 * math.pi * ETA)
        y = np.expm1(beta * ETA) / den
        return x, y
    return f


def layer_stretch(ratio: float, layer: float, n_ref: int):
    """y(eta) whose cell height grows by ``ratio`` per cell (at n_ref cells) inside
    a wall layer of thickness ``layer`` (fraction of eta), uniform beyond it,
    normalised to [0, 1].  Returned as a smooth function of eta."""
    if abs(ratio - 1.0) < 1e-14:
        return lambda ETA: ETA.copy()
    lr = math.log(ratio)
    tstar = layer * n_ref

    def prim(t):
        t = np.asarray(t, dtype=np.float64)
        inner = np.expm1(lr * np.minimum(t, tstar)) / lr
        outer = np.exp(lr * tstar) * np.maximum(t - tstar, 0.0)
        # extend below 0 linearly so ghost points stay well defined
        below = np.minimum(t, 0.0)
        return np.where(t < 0, below, inner + outer)
    total = float(prim(np.array(float(n_ref))))
    return lambda ETA: prim(ETA * n_ref) / total


def map_skew_stretch(angle_deg: float, ratio: float, layer: float, n_ref: int) -> MapFn:
    """y stretched near y = 0 (layer_stretch), then sheared: x = xi + tan(angle) y."""
    ys = layer_stretch(ratio, layer, n_ref)
    t = math.tan(math.radians(angle_deg))

    def f(XI, ETA):
        y = ys(ETA)
        return XI + t * y, y
    return f
