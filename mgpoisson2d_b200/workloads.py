"""Seeded synthetic inputs of the benchmark workloads and of the reference's
own known-answer tests.  All functions return host containers
(``Box``, ``GeoData``, ``BoxData`` rhs, ``BdryData``) plus whatever exact
solution the workload has.

* ``identity_dirichlet``  -- unit square, identity map, homogeneous Dirichlet,
  rhs = Laplacian of sin(2 pi x) sin(3 pi y) plus seeded noise of amplitude 1e-3.
* ``wavy_stretched``      -- x = xi + 0.1 sin(2 pi xi) sin(2 pi eta),
  y = (e^{beta eta} - 1)/(e^beta - 1) with a 64:1 first-cell aspect ratio,
  Dirichlet x sides, Neumann y sides, rhs = J f with f a seeded sum of 16
  Fourier modes (J-weighted mean removed).
* ``skew_stretched``      -- shear x = xi + tan(angle) y over a wall-layer
  stretched y, nonuniform Dirichlet data from u = e^x cos(4 pi y).
* ``terrain_neumann``     -- the reference's own solver test problem
  (src/tests/test.f90:2336-2583): terrain map, 117-mode cosine solution, all
  Neumann BCs from the operator's boundary fluxes.
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as G
from .types import (BCMODE_NONUNIFORM, BCMODE_UNIFORM, BCTYPE_DIRI, BCTYPE_NEUM, BD_CELL, BD_NODE, BdryData, Box,
                    BoxData)


def identity_dirichlet(n: int = 128, seed: int = 1):
    v = Box.of_size(n, n)
    fmap = G.map_identity()
    geo = G.mapped_geometry(v, fmap)
    X, Y = G.positions(v, fmap)
    rng = np.random.default_rng(seed)
    u = np.sin(2 * math.pi * X) * np.sin(3 * math.pi * Y)
    f = -13.0 * math.pi ** 2 * u + rng.uniform(-1e-3, 1e-3, size=u.shape)
    rhs = BoxData(v)
    rhs.interior()[:] = f * geo.J.interior()
    bc = BdryData.uniform(v, [BCTYPE_DIRI] * 4)
    return v, geo, rhs, bc, u


def fourier_modes(seed, modes=16, kmax=8):
    """Amplitudes U(-1,1) and wave numbers U{1..kmax} of the seeded rhs."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(-1, 1, modes)
    m = rng.integers(1, kmax + 1, modes)
    nn = rng.integers(1, kmax + 1, modes)
    return a, m, nn


def fourier_rhs(v, geo, fmap, seed, modes=16, kmax=8):
    X, Y = G.positions(v, fmap)
    a, m, nn = fourier_modes(seed, modes, kmax)
    f = np.zeros_like(X)
    for k in range(modes):
        f += a[k] * np.cos(math.pi * m[k] * X) * np.cos(math.pi * nn[k] * Y)
    J = geo.J.interior()
    f -= (f * J).sum() / J.sum()
    rhs = BoxData(v)
    rhs.interior()[:] = J * f
    return rhs


def wavy_stretched(n: int = 1024, seed: int = 2, aspect: float = 64.0):
    v = Box.of_size(n, n)
    fmap = G.map_wavy_exp(0.1, aspect)
    geo = G.mapped_geometry(v, fmap)
    rhs = fourier_rhs(v, geo, fmap, seed)
    bc = BdryData.uniform(v, [BCTYPE_DIRI, BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_NEUM])
    return v, geo, rhs, bc, None


def skew_stretched(n: int = 256, angle: float = 30.0, ratio: float = 1.05, layer: float = 96 / 4096,
                   n_ref: int = 4096, nx: int = None):
    nx = nx or n
    v = Box.of_size(nx, n)
    fmap = G.map_skew_stretch(angle, ratio, layer, n_ref)
    geo = G.mapped_geometry(v, fmap)
    X, Y = G.positions(v, fmap)
    u = np.exp(X) * np.cos(4 * math.pi * Y)
    rhs = BoxData(v)
    rhs.interior()[:] = geo.J.interior() * (1.0 - 16 * math.pi ** 2) * u
    # Dirichlet data at the boundary face centres
    Xf, Yf = G.positions(v, fmap, BD_NODE, BD_CELL)
    Xg, Yg = G.positions(v, fmap, BD_CELL, BD_NODE)
    ue = lambda x, y: np.exp(x) * np.cos(4 * math.pi * y)
    data = [ue(Xf[0], Yf[0]), ue(Xf[-1], Yf[-1]), ue(Xg[:, 0], Yg[:, 0]), ue(Xg[:, -1], Yg[:, -1])]
    bc = BdryData(v, [BCTYPE_DIRI] * 4, [BCMODE_NONUNIFORM] * 4, data)
    return v, geo, rhs, bc, u


def terrain_solution(X, Y, L=1.0, H=1.0):
    s = np.zeros_like(X)
    for i in range(8, 241, 2):
        s += np.cos(i * math.pi * X / L) * np.cos(i * math.pi * Y / H) / i
    return s


def terrain_neumann(n: int, boundary_fluxes, compute_laplacian):
    """The problem of test_solver (test.f90:2336-2470).  ``boundary_fluxes`` and
    ``compute_laplacian`` are the operator routines used to build the Neumann
    data and the rhs (the reference uses its own compute_grad and
    compute_laplacian there)."""
    v = Box.of_size(n, n)
    geo = G.terrain_geometry(v)
    X, Y = G.terrain_positions(v, BD_CELL, BD_CELL, 1)
    soln = BoxData(v, 1, 1)
    soln.data[:] = terrain_solution(X, Y)
    fl = boundary_fluxes(soln, geo)
    bc = BdryData(v, [BCTYPE_NEUM] * 4, [BCMODE_NONUNIFORM] * 4, fl)
    rhs = BoxData(v)
    compute_laplacian(rhs, soln.copy(), geo, bc, False)
    return v, geo, rhs, bc, soln


def batch_problem(i: int, seed: int = 4, nmin: int = 64, nmax: int = 1024, round_to: int = 16):
    """Problem i of the batched workload (seed*10^6 + i): each side
    log-uniform in [nmin, nmax], rounded to a multiple of round_to (the reference
    schedule stops at depth 0 on odd sizes); y stretched by a ratio U[1, 1.08]
    per cell in a wall layer of min(64, ny/4) cells, then sheared by U[0, 25]
    degrees; the 16-mode Fourier rhs of wavy_stretched; homogeneous Dirichlet
    on all sides."""
    nx, ny, angle, ratio, layer_cells = batch_problem_params(i, seed, nmin, nmax, round_to)
    v = Box.of_size(nx, ny)
    fmap = G.map_skew_stretch(angle, ratio, layer_cells / ny, ny)
    geo = G.mapped_geometry(v, fmap)
    rhs = fourier_rhs(v, geo, fmap, seed * 1_000_000 + i)
    bc = BdryData.uniform(v, [BCTYPE_DIRI] * 4)
    return v, geo, rhs, bc


def batch_problem_params(i: int, seed: int = 4, nmin: int = 64, nmax: int = 1024, round_to: int = 16):
    """The parameters batch_problem(i) draws: (nx, ny, angle, ratio, layer cells)."""
    rng = np.random.default_rng(seed * 1_000_000 + i)

    def side():
        n = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        return int(max(nmin, min(nmax, round_to * round(n / round_to))))

    nx, ny = side(), side()
    ratio = float(rng.uniform(1.0, 1.08))
    angle = float(rng.uniform(0.0, 25.0))
    return nx, ny, angle, ratio, min(64, ny // 4)


def batch_problem_device(i: int, seed: int = 4, nmin: int = 64, nmax: int = 1024, round_to: int = 16):
    """batch_problem(i) with the geometry and the rhs generated on the device
    (mgp_map_geometry, mgp_map_fourier_rhs): equal to the host version to the
    rounding of the map's transcendentals."""
    from . import api as M
    nx, ny, angle, ratio, layer_cells = batch_problem_params(i, seed, nmin, nmax, round_to)
    v = Box.of_size(nx, ny)
    params = (math.tan(math.radians(angle)), ratio, float(layer_cells), float(ny))
    geo = M.map_geometry(v, M.MAP_SKEW_LAYER, params)
    a, m, nn = fourier_modes(seed * 1_000_000 + i)
    rhs = M.map_fourier_rhs(v, M.MAP_SKEW_LAYER, params, a, m, nn, geo.J)
    bc = BdryData.uniform(v, [BCTYPE_DIRI] * 4)
    return v, geo, rhs, bc


def skew_stretched_device(n: int, angle: float = 30.0, ratio: float = 1.05, layer_cells: float = 96.0,
                          n_ref: int = 4096):
    """skew_stretched(n) with the metric terms generated on the device
    (mgp_map_geometry) and the manufactured rhs and exact solution assembled
    on the device from 1-D factors: x = xi + tan(angle) y(eta), so
    u = e^x cos(4 pi y) = e^xi * (e^{tan(angle) y} cos(4 pi y)).  Returns
    (valid, geo, rhs, bc, u_exact) with rhs and u_exact on the device."""
    import torch
    from . import api as M
    v = Box.of_size(n, n)
    t = math.tan(math.radians(angle))
    params = (t, ratio, float(layer_cells), float(n_ref))
    geo = M.map_geometry(v, M.MAP_SKEW_LAYER, params)
    ys = G.layer_stretch(ratio, layer_cells / n_ref, n_ref)
    xi = (np.arange(n) + 0.5) * v.dx
    yc = ys((np.arange(n) + 0.5) * v.dy)
    fx = np.exp(xi)
    fy = np.exp(t * yc) * np.cos(4 * math.pi * yc)
    dev = geo.J.data.device
    # device arrays are (ny, nx) row-major views of the column-major fields
    u = torch.outer(torch.from_numpy(fy).to(dev), torch.from_numpy(fx).to(dev))
    rhs = BoxData.device_zeros(v)
    rhs.data[:] = geo.J.data[1:-1, 1:-1] * ((1.0 - 16 * math.pi ** 2) * u)
    ue = lambda x, y: np.exp(x) * np.cos(4 * math.pi * y)
    y_side = yc
    data = [ue(t * y_side, y_side), ue(1.0 + t * y_side, y_side), ue(xi, np.zeros(n)), ue(xi + t * 1.0, np.ones(n))]
    bc = BdryData(v, [BCTYPE_DIRI] * 4, [BCMODE_NONUNIFORM] * 4, data)
    return v, geo, rhs, bc, u
