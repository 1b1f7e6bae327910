"""The committed golden fixtures (tests/golden/make_fixtures.py) against the
oracle and the workload generators, on the CPU.

* the 128^2 identity-map fixture is reproduced bit for bit by a fresh oracle solve (the
  oracle is deterministic), and its solution has the manufactured solution's
  discretisation error;
* the 1024^2 stretched wavy-map fixtures were made from the same inputs the generators give now
  (checksums), and records a converged, non-diverged lexicographic solve whose
  residual history falls monotonically (the stationary V-cycle, MG:630-639).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import pytest

from mgpoisson2d_b200 import workloads as W
from mgpoisson2d_b200.types import BoxData
from oracle import oracle as O

from golden.make_fixtures import input_sums

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _coupled(on):
    O.lib().or_set_dirichlet_coupled_diagonal.argtypes = [ctypes.c_int]
    O.lib().or_set_dirichlet_coupled_diagonal(int(on))


def test_identity128_fixture_reproduced_by_the_oracle():
    fx = np.load(os.path.join(GOLDEN, "identity128.npz"))
    v, geo, rhs, bc, u = W.identity_dirichlet(128)
    np.testing.assert_allclose(input_sums(geo, rhs), fx["inputs"], rtol=1e-12, atol=1e-12)
    _coupled(True)
    try:
        phi = BoxData(v, 1, 1)
        rep = O.vcycle(phi, rhs, geo, bc, True, 1e-10, 100, smooth_down=8, smooth_up=8, smooth_bottom=8)
    finally:
        _coupled(False)
    assert rep.iterations == int(fx["iterations"])
    assert np.array_equal(rep.relres, fx["relres"])
    assert np.array_equal(phi.interior(), fx["solution"])
    # second-order scheme at h = 1/128 with 1e-3 noise in the rhs
    assert np.abs(fx["solution"] - u).max() < 2e-3


@pytest.mark.parametrize("name", ["wavy1024.npz", "wavy1024_colour.npz"])
def test_wavy1024_fixture_inputs_and_history(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"{name} not generated")
    fx = np.load(path)
    v, geo, rhs, bc, _ = W.wavy_stretched(1024)
    np.testing.assert_allclose(input_sums(geo, rhs), fx["inputs"], rtol=1e-12, atol=1e-12)
    h = fx["relres"]
    assert not bool(fx["diverged"])
    assert h[0] == 1.0 and h[-1] <= 1e-10 and len(h) == int(fx["iterations"]) + 1
    assert np.all(np.diff(h) < 0)
    assert fx["strided"].shape == (128, 128) and fx["sample"].shape == (16384,)
    assert np.isclose(np.abs(fx["strided"]).max(), float(fx["maxabs"]), rtol=0.05)
