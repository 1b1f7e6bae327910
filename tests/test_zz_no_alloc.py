"""mgp_solve_bicgstab2_noalloc: the BiCGStab bottom solver for callers that
cannot allocate device memory (a service that reserves its device-memory
budget at start-up and forbids later allocation, or code running while another
component owns the allocator).  It keeps its work arrays in one file-scope
device array, so it must give the same result as the allocating
mgp_solve_bicgstab2 -- here on two calls in a row, since every call reuses the
array the previous call left behind.  This file sorts last so that a run that
stops at the first failure has already run every other test.
"""
from __future__ import annotations

import numpy as np
import pytest

from mgpoisson2d_b200 import geometry as G
from mgpoisson2d_b200.types import BCMODE_NONUNIFORM, BCTYPE_DIRI, BCTYPE_NEUM, BdryData, Box, BoxData

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _problem(nx=40, ny=32, seed=21):
    rng = np.random.default_rng(seed)
    v = Box.of_size(nx, ny)
    geo = G.mapped_geometry(v, G.map_wavy_exp(0.1, 8.0))
    rhs = BoxData(v)
    rhs.interior()[:] = rng.standard_normal((nx, ny))
    types = [BCTYPE_DIRI, BCTYPE_NEUM, BCTYPE_DIRI, BCTYPE_NEUM]
    data = [rng.standard_normal(ny), rng.standard_normal(ny), rng.standard_normal(nx), rng.standard_normal(nx)]
    bc = BdryData(v, types, [BCMODE_NONUNIFORM] * 4, data)
    return v, geo, rhs, bc


def _allocating(v, geo, rhs, bc, M):
    inv = BoxData(v)
    M.compute_invdiags(inv, geo, bc, True)
    ref = BoxData(v, 1, 1)
    M.solve_bicgstab2(ref, rhs, geo, bc, False, inv, 1e-10, 80, 5, False)
    return inv, ref


def _noalloc(v, geo, rhs, bc, inv, M):
    phi_d = BoxData(v, 1, 1).to_device()
    M.solve_bicgstab2_noalloc(phi_d, rhs.to_device(), geo.to_device(), bc, False, inv.to_device(), 1e-10, 80, 5,
                              False)
    return phi_d.to_host().interior().copy()


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    """Problem A, then a different problem B (another size and data), then A
    again: each no-allocation result matches the allocating entry point's, so
    no call reads what the previous one left in the shared scratch array."""
    assert torch.cuda.is_available(), "needs a CUDA device"
    import mgpoisson2d_b200.api as M
    pa = _problem()
    pb = _problem(36, 28, seed=5)
    inv_a, ref_a = _allocating(*pa, M)
    inv_b, ref_b = _allocating(*pb, M)
    outs = []
    for (v, geo, rhs, bc), inv, ref in ((pa, inv_a, ref_a), (pb, inv_b, ref_b), (pa, inv_a, ref_a)):
        got = _noalloc(v, geo, rhs, bc, inv, M)
        np.testing.assert_allclose(got, ref.interior(), rtol=1e-9, atol=1e-12)
        outs.append(got)
    np.testing.assert_array_equal(outs[0], outs[2])


def test_noalloc_rejects_oversized_grid_and_host_arrays():
    import mgpoisson2d_b200.api as M
    n = M.NOALLOC_MAX_SIDE + 2
    v, geo, rhs, bc = _problem(n, 8)
    inv = BoxData(v)
    inv.interior()[:] = -1.0
    with pytest.raises(M.MGPError, match="MGP_EINVAL"):
        M.solve_bicgstab2_noalloc(BoxData(v, 1, 1).to_device(), rhs.to_device(), geo.to_device(), bc, False,
                                  inv.to_device(), 1e-10, 80, 5, False)
    v, geo, rhs, bc = _problem(16, 16)
    inv = BoxData(v)
    inv.interior()[:] = -1.0
    with pytest.raises(M.MGPError, match="device memory"):
        M.solve_bicgstab2_noalloc(BoxData(v, 1, 1), rhs, geo, bc, False, inv, 1e-10, 80, 5, False)
