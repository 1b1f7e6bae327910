"""Shared builders for the tests: seeded random geometry / fields / BCs."""
from __future__ import annotations

import numpy as np

from mgpoisson2d_b200.types import (BCMODE_LAH, BCMODE_NONUNIFORM, BCMODE_UNIFORM, BCTYPE_DIRI, BCTYPE_EXTRAP0,
                                    BCTYPE_EXTRAP1, BCTYPE_EXTRAP2, BCTYPE_NEUM, BCTYPE_NONE, BCTYPE_PERIODIC,
                                    BD_CELL, BD_NODE, BdryData, Box, BoxData, GeoData)

D, N, P = BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_PERIODIC
U, NU = BCMODE_UNIFORM, BCMODE_NONUNIFORM

# (types, modes) combinations exercised by the operator tests
BC_CASES = {
    "DDDD-U": ([D, D, D, D], [U] * 4),
    "DDDD-NU": ([D, D, D, D], [NU] * 4),
    "NNNN-U": ([N, N, N, N], [U] * 4),
    "NNNN-NU": ([N, N, N, N], [NU] * 4),
    "DDNN-U": ([D, D, N, N], [U] * 4),
    "NNDD-NU": ([N, N, D, D], [NU] * 4),
    "DNND-mixed": ([D, N, N, D], [U, NU, U, NU]),
    "PPDD": ([P, P, D, D], [U, U, NU, U]),
    "DDPP": ([D, D, P, P], [NU, U, U, U]),
    "PPPP": ([P, P, P, P], [U] * 4),
}


def rand_geo(v: Box, rng, cross: float = 0.3) -> GeoData:
    def arr(offi, offj, lo, hi):
        b = BoxData(v, 1, 1, offi, offj)
        b.data[:] = rng.uniform(lo, hi, b.data.shape)
        return b
    return GeoData(arr(BD_CELL, BD_CELL, 0.5, 2.0), arr(BD_NODE, BD_CELL, 0.5, 2.0),
                   arr(BD_NODE, BD_CELL, -cross, cross), arr(BD_CELL, BD_NODE, -cross, cross),
                   arr(BD_CELL, BD_NODE, 0.5, 2.0), v.dx, v.dy)


def rand_field(v: Box, rng, ng=1, offi=BD_CELL, offj=BD_CELL) -> BoxData:
    b = BoxData(v, ng, ng, offi, offj)
    b.data[:] = rng.standard_normal(b.data.shape)
    return b


def rand_bc(v: Box, types, modes, rng) -> BdryData:
    data = []
    for s in range(4):
        n = 1 if modes[s] != BCMODE_NONUNIFORM else (v.ny if s < 2 else v.nx)
        data.append(rng.standard_normal(n))
    return BdryData(v, types, modes, data)


def same(a: np.ndarray, b: np.ndarray) -> bool:
    """Bitwise equality (NaN-aware)."""
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def hierarchy_geo(v: Box, fine: GeoData, restrict):
    """Coarsen a geometry by (2,2) with the given restrict routine."""
    c = v.coarsened(2, 2)
    g = GeoData(BoxData(c), BoxData(c, 0, 0, BD_NODE, BD_CELL), BoxData(c, 0, 0, BD_NODE, BD_CELL),
                BoxData(c, 0, 0, BD_CELL, BD_NODE), BoxData(c, 0, 0, BD_CELL, BD_NODE), c.dx, c.dy)
    for a, b in ((fine.J, g.J), (fine.Jgup_xx, g.Jgup_xx), (fine.Jgup_xy, g.Jgup_xy), (fine.Jgup_yx, g.Jgup_yx),
                 (fine.Jgup_yy, g.Jgup_yy)):
        restrict(a, b)
    return c, g
