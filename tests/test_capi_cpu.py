"""The C-ABI library on a host without a GPU: it loads, exports every symbol
include/mgp2d.h declares, and its host-side logic (schedule, argument checks)
behaves like the reference routines.  No call here reaches a kernel."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from mgpoisson2d_b200.types import (BCTYPE_CF, BCTYPE_DIRI, MgpArray, MgpBdry, MgpBox, MgpGeo, MgpReport, Box)
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "mgp2d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]*?\b(mgp_\w+)\s*\(", src, flags=re.M)))


def test_library_exports_every_declared_symbol():
    import mgpoisson2d_b200.api as api
    lib = C.CDLL(api.library_path())
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(api.EXPORTS)


def test_header_constants_match_the_python_binding():
    """Every MGP_FLAG_*, MGP_KIND_*, MGP_BCTYPE_*, MGP_MAP_* and the no-alloc
    side limit of include/mgp2d.h has the same value in the Python binding,
    and the flags are distinct powers of two."""
    import mgpoisson2d_b200 as pkg
    import mgpoisson2d_b200.api as api
    import mgpoisson2d_b200.types as T
    src = open(os.path.join(ROOT, "include", "mgp2d.h")).read()
    defs = dict(re.findall(r"^#define MGP_(\w+)\s+\(?(-?\d+)\)?", src, flags=re.M))
    flags = {k: int(v) for k, v in defs.items() if k.startswith("FLAG_")}
    assert len(flags) >= 7
    for k, v in flags.items():
        assert getattr(api, k) == v and getattr(pkg, k) == v, k
        assert v > 0 and v & (v - 1) == 0, k
    assert len(set(flags.values())) == len(flags)
    for k, v in defs.items():
        if k.startswith(("KIND_", "MAP_")) or k == "NOALLOC_MAX_SIDE":
            assert getattr(api, k) == int(v), k
        elif k.startswith("BCTYPE_"):
            assert getattr(T, k) == int(v), k


def test_version_and_error_strings():
    import mgpoisson2d_b200.api as api
    assert b"sm_100a" in api._lib.mgp_version()
    assert isinstance(api._lib.mgp_last_error(), bytes)


@pytest.mark.parametrize("nx,ny", [(128, 128), (1024, 1024), (64, 256), (96, 40), (63, 64), (80, 1024)])
def test_schedule_matches_oracle(nx, ny):
    import mgpoisson2d_b200.api as api
    b = Box.of_size(nx, ny)
    m1 = api.estimate_maxdepth(1000, b)
    assert m1 == O.estimate_maxdepth(1000, b)
    assert api.create_mgschedule(m1, b) == O.create_mgschedule(m1, b)


def test_invalid_arguments_return_einval():
    """Checks that run before any device work: odd ilo, bad BC type,
    CF type (the reference reads uninitialised coefficients there)."""
    import mgpoisson2d_b200.api as api
    lib = api._lib
    box = MgpBox(1, 16, 0, 15, 16, 16, 1 / 16, 1 / 16)   # odd ilo
    arr = MgpArray(None, 0, 1, 1)
    geo = MgpGeo()
    bc = MgpBdry()
    rep = MgpReport()
    rc = lib.mgp_vcycle(C.byref(box), C.byref(arr), C.byref(arr), C.byref(geo), C.byref(bc), 1, 0, 0, 1e-10, 10,
                        -1, 1, 8, 8, 8, 0, 0, C.byref(rep))
    assert rc == 1   # MGP_EINVAL
    box = MgpBox(0, 15, 0, 15, 16, 16, 1 / 16, 1 / 16)
    for t in range(4):
        bc.type[t] = BCTYPE_DIRI
    bc.type[2] = BCTYPE_CF
    h = C.c_void_p()
    rc = lib.mgp_solver_create(C.byref(box), C.byref(geo), C.byref(bc), 0, 0, -1, C.byref(h))
    assert rc in (1, 7)
    bc.type[2] = 42
    rc = lib.mgp_solver_create(C.byref(box), C.byref(geo), C.byref(bc), 0, 0, -1, C.byref(h))
    assert rc == 1
    bad = MgpBox(0, 15, 0, 15, 17, 16, 1 / 16, 1 / 16)   # inconsistent nx
    rc = lib.mgp_compute_laplacian(C.byref(bad), C.byref(arr), C.byref(arr), C.byref(geo), C.byref(bc), 1, 0)
    assert rc == 1
    assert b"inconsistent" in lib.mgp_last_error()
