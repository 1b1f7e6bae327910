"""ctypes mirrors of the C structs in include/mgp2d.h, and the Python-side
containers that mirror the Fortran derived types of arrayutils.f90.

Nothing here loads a shared library; it is safe to import on a host without a
GPU.  The containers follow the reference's types:

* ``Box``       -- type(box), arrayutils.f90:10-15
* ``BoxData``   -- type(box_data), arrayutils.f90:83-96 (column-major data with
                   ghosts; ``offi``/``offj`` = BD_NODE/BD_CELL centring)
* ``BdryData``  -- type(bdry_data), arrayutils.f90:55-70
* ``GeoData``   -- type(geo_data), arrayutils.f90:109-116

``BoxData.data`` is either a NumPy array in Fortran order with shape
(allocated nx, allocated ny), or a torch CUDA tensor of shape (allocated ny,
allocated nx) -- the same memory layout, i fastest.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

# BC types / modes, arrayutils.f90:27-49
BCTYPE_UNDEFINED = -2
BCTYPE_NONE = -1
BCTYPE_NEUM = 0
BCTYPE_DIRI = 1
BCTYPE_PERIODIC = 2
BCTYPE_CF = 3
BCTYPE_EXTRAP0 = 4
BCTYPE_EXTRAP1 = 5
BCTYPE_EXTRAP2 = 6

BCMODE_UNIFORM = 0
BCMODE_NONUNIFORM = 1
BCMODE_LAH = 2

BD_NODE = 0
BD_CELL = 1

XLO, XHI, YLO, YHI = 0, 1, 2, 3
BOGUS_VAL = 1.2345e300

KIND_MG = 0
KIND_DD = 1

STATUS_NAMES = {0: "MGP_OK", 1: "MGP_EINVAL", 2: "MGP_ENOMEM", 3: "MGP_EDIVERGED",
                4: "MGP_EMAXITER", 5: "MGP_ETIMEOUT", 6: "MGP_ECUDA", 7: "MGP_ENOTSUP"}


class MgpBox(C.Structure):
    _fields_ = [("ilo", C.c_int), ("ihi", C.c_int), ("jlo", C.c_int), ("jhi", C.c_int),
                ("nx", C.c_int), ("ny", C.c_int), ("dx", C.c_double), ("dy", C.c_double)]


class MgpArray(C.Structure):
    _fields_ = [("data", C.c_void_p), ("ld", C.c_int), ("ngx", C.c_int), ("ngy", C.c_int)]


class MgpBdry(C.Structure):
    _fields_ = [("type", C.c_int * 4), ("mode", C.c_int * 4), ("data", C.c_void_p * 4)]


class MgpGeo(C.Structure):
    _fields_ = [("J", MgpArray), ("Jgup_xx", MgpArray), ("Jgup_xy", MgpArray),
                ("Jgup_yx", MgpArray), ("Jgup_yy", MgpArray), ("dx", C.c_double), ("dy", C.c_double)]


class MgpReport(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("maxdepth", C.c_int),
                ("diverged", C.c_int), ("rscale", C.c_double), ("final_relres", C.c_double),
                ("relres", C.c_void_p), ("seconds", C.c_double), ("smooth0_seconds", C.c_double),
                ("smooth0_sweeps", C.c_longlong)]


@dataclass
class Box:
    """type(box): lower/upper cell indices and spacings (arrayutils.f90:10-15)."""
    ilo: int
    ihi: int
    jlo: int
    jhi: int
    dx: float
    dy: float

    @property
    def nx(self) -> int:
        return self.ihi - self.ilo + 1

    @property
    def ny(self) -> int:
        return self.jhi - self.jlo + 1

    @staticmethod
    def of_size(nx: int, ny: int, L: float = 1.0, H: float = 1.0, ilo: int = 0, jlo: int = 0) -> "Box":
        return Box(ilo, ilo + nx - 1, jlo, jlo + ny - 1, L / nx, H / ny)

    def coarsened(self, refx: int, refy: int) -> "Box":
        """coarsen_box, arrayutils.f90:154-170."""
        ilo, ihi = int(self.ilo / refx), int(self.ihi / refx)
        jlo, jhi = int(self.jlo / refy), int(self.jhi / refy)
        return Box(ilo, ihi, jlo, jhi, self.dx * refx, self.dy * refy)

    def c(self) -> MgpBox:
        return MgpBox(self.ilo, self.ihi, self.jlo, self.jhi, self.nx, self.ny, self.dx, self.dy)


class BoxData:
    """type(box_data): centred data with ghosts, stored column-major.

    ``valid`` is the cell-centred box the data is defined over (as passed to
    define_box_data, arrayutils.f90:389-451); node centring adds one point in
    that direction.
    """

    def __init__(self, valid: Box, ngx: int = 0, ngy: int = 0, offi: int = BD_CELL,
                 offj: int = BD_CELL, data=None, fill: float = 0.0):
        self.valid = valid
        self.ngx, self.ngy = ngx, ngy
        self.offi, self.offj = offi, offj
        self.nvx = valid.nx + (1 if offi == BD_NODE else 0)
        self.nvy = valid.ny + (1 if offj == BD_NODE else 0)
        shape = (self.nvx + 2 * ngx, self.nvy + 2 * ngy)
        if data is None:
            data = np.full(shape, fill, dtype=np.float64, order="F")
        self.data = data
        if self.is_device:
            assert tuple(data.shape) == (shape[1], shape[0]) and data.is_contiguous()
        else:
            assert data.shape == shape and data.flags.f_contiguous and data.dtype == np.float64

    # -- views -------------------------------------------------------------
    @property
    def is_device(self) -> bool:
        return not isinstance(self.data, np.ndarray)

    @property
    def ld(self) -> int:
        return self.nvx + 2 * self.ngx

    def interior(self) -> np.ndarray:
        """Valid region as a (nvx, nvy) NumPy view (host data only)."""
        a = self.host()
        return a[self.ngx:self.ngx + self.nvx, self.ngy:self.ngy + self.nvy]

    def host(self) -> np.ndarray:
        if self.is_device:
            return self.data.detach().cpu().numpy().T
        return self.data

    def copy(self) -> "BoxData":
        d = self.data.clone() if self.is_device else self.data.copy(order="F")
        return BoxData(self.valid, self.ngx, self.ngy, self.offi, self.offj, data=d)

    def like(self, fill: float = 0.0) -> "BoxData":
        """define_box_data_dup (arrayutils.f90:458-475): same shape, new storage."""
        if self.is_device:
            import torch
            d = torch.full_like(self.data, fill)
        else:
            d = np.full(self.data.shape, fill, dtype=np.float64, order="F")
        return BoxData(self.valid, self.ngx, self.ngy, self.offi, self.offj, data=d)

    @staticmethod
    def device_zeros(valid: Box, ngx: int = 0, ngy: int = 0, offi: int = BD_CELL, offj: int = BD_CELL,
                     device="cuda") -> "BoxData":
        """Zero-filled storage allocated on the device (no host copy)."""
        import torch
        nvx = valid.nx + (1 if offi == BD_NODE else 0)
        nvy = valid.ny + (1 if offj == BD_NODE else 0)
        t = torch.zeros((nvy + 2 * ngy, nvx + 2 * ngx), dtype=torch.float64, device=device)
        return BoxData(valid, ngx, ngy, offi, offj, data=t)

    def to_device(self, device="cuda") -> "BoxData":
        import torch
        t = torch.from_numpy(np.ascontiguousarray(self.host().T)).to(device)
        return BoxData(self.valid, self.ngx, self.ngy, self.offi, self.offj, data=t)

    def to_host(self) -> "BoxData":
        return BoxData(self.valid, self.ngx, self.ngy, self.offi, self.offj,
                       data=np.asfortranarray(self.host().copy()))

    def c(self) -> MgpArray:
        ptr = self.data.data_ptr() if self.is_device else self.data.ctypes.data
        return MgpArray(ptr, self.ld, self.ngx, self.ngy)


class BdryData:
    """type(bdry_data): per-side BC type, mode and values (arrayutils.f90:55-70).

    ``data`` holds, per side, one value (UNIFORM/LAH) or the side's values
    (NONUNIFORM: ny for x sides, nx for y sides).
    """

    def __init__(self, valid: Box, types: Sequence[int], modes: Sequence[int],
                 data: Optional[Sequence[Optional[np.ndarray]]] = None):
        self.valid = valid
        self.types = list(types)
        self.modes = list(modes)
        self.data = []
        for s in range(4):
            n = 1 if self.modes[s] != BCMODE_NONUNIFORM else (valid.ny if s < 2 else valid.nx)
            v = None if data is None else data[s]
            if v is None:
                v = np.zeros(n)
            self.data.append(np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(-1)))

    @staticmethod
    def uniform(valid: Box, types: Sequence[int], values=(0.0, 0.0, 0.0, 0.0)) -> "BdryData":
        return BdryData(valid, types, [BCMODE_UNIFORM] * 4, [np.array([v]) for v in values])

    def c(self) -> MgpBdry:
        b = MgpBdry()
        for s in range(4):
            b.type[s] = self.types[s]
            b.mode[s] = self.modes[s]
            b.data[s] = self.data[s].ctypes.data
        return b


@dataclass
class GeoData:
    """type(geo_data) (arrayutils.f90:109-116)."""
    J: BoxData
    Jgup_xx: BoxData
    Jgup_xy: BoxData
    Jgup_yx: BoxData
    Jgup_yy: BoxData
    dx: float
    dy: float

    def c(self) -> MgpGeo:
        return MgpGeo(self.J.c(), self.Jgup_xx.c(), self.Jgup_xy.c(), self.Jgup_yx.c(),
                      self.Jgup_yy.c(), self.dx, self.dy)

    def to_device(self, device="cuda") -> "GeoData":
        return GeoData(self.J.to_device(device), self.Jgup_xx.to_device(device),
                       self.Jgup_xy.to_device(device), self.Jgup_yx.to_device(device),
                       self.Jgup_yy.to_device(device), self.dx, self.dy)


@dataclass
class Report:
    status: int = 0
    iterations: int = 0
    maxdepth: int = 0
    diverged: bool = False
    rscale: float = 0.0
    final_relres: float = 0.0
    relres: np.ndarray = field(default_factory=lambda: np.zeros(0))
    seconds: float = 0.0
    smooth0_seconds: float = 0.0
    smooth0_sweeps: int = 0


def make_report(maxiters: int):
    buf = np.zeros(max(maxiters, 0) + 1)
    rep = MgpReport()
    rep.relres = buf.ctypes.data
    return rep, buf


def read_report(rep: MgpReport, buf: np.ndarray) -> Report:
    n = rep.iterations
    return Report(rep.status, rep.iterations, rep.maxdepth, bool(rep.diverged), rep.rscale,
                  rep.final_relres, buf[:n + 1].copy(), rep.seconds, rep.smooth0_seconds, rep.smooth0_sweeps)
