"""The reference's case files through the C-ABI (include/cosa_io.h):
input.dat (input(), src/input.f90:2271-4392), mesh.dat (readgrid,
src/input.f90:4482-4570) and the restart file (readrest,
src/input.f90:4620-4716; writerest, src/output.f90:3484-3566).

The readers and writers are host code in libcosa_gpu.so (csrc/io.cpp); they
need no GPU.  Arrays are the library's flat layouts: node arrays P2 per
block at the setoffs offsets, displacement scales P1, states P3 with npde
variables and S = 2 nharms + 1 snapshots.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np

from . import gpu
from .params import CosaParams
from .tables import LevelTables

SYMBOLS = [
    "cosa_io_default_params", "cosa_io_read_input", "cosa_io_input_level", "cosa_io_free_input",
    "cosa_io_write_input", "cosa_io_read_mesh", "cosa_io_write_mesh", "cosa_io_read_restart",
    "cosa_io_write_restart",
]


class RunOpts(C.Structure):
    """cosa_run_opts: the input.dat controls that are not cosa_params fields."""
    _fields_ = [(n, C.c_int32) for n in (
        "debug", "exter", "irest", "srest", "lmax", "nl_fmg", "dgn_cell", "wri_res", "wri_tec", "calfor",
        "nsurface", "ntime", "nsave")] + [
        ("wrifl", C.c_int32 * 3),
        ("toler", C.c_double), ("tref", C.c_double), ("dt", C.c_double),
        ("xmom", C.c_double * 3), ("lngth", C.c_double * 3),
        ("flow_kind", C.c_char * 16), ("out_format", C.c_char * 16),
        ("n_surblo", C.c_int32 * 8), ("i_surbl", (C.c_int32 * 64) * 8),
    ]


class CaseFileError(RuntimeError):
    def __init__(self, what: str, code: int):
        super().__init__(f"{what} failed with status 0x{code:x}")
        self.code = code


def _lib():
    L = gpu.load()
    for n in SYMBOLS:
        getattr(L, n).restype = C.c_int
    return L


def _check(code: int, what: str):
    if code != 0:
        raise CaseFileError(what, code)


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dims(t: LevelTables) -> np.ndarray:
    return np.ascontiguousarray(t.dims.ravel(), dtype=np.int32)


def default_params() -> CosaParams:
    p = CosaParams()
    _check(_lib().cosa_io_default_params(C.byref(p)), "cosa_io_default_params")
    return p


def read_input(path: str) -> Tuple[CosaParams, RunOpts, LevelTables]:
    """(params, run controls, fine-level tables) of an input.dat."""
    L = _lib()
    p, r, h = CosaParams(), RunOpts(), C.c_void_p()
    _check(L.cosa_io_read_input(str(path).encode(), C.byref(p), C.byref(r), C.byref(h)), "cosa_io_read_input")
    try:
        d = gpu.LevelDesc()
        _check(L.cosa_io_input_level(h, C.byref(d)), "cosa_io_input_level")
        nb = d.nblocks
        dims = np.ctypeslib.as_array(d.dims, (3 * nb,)).reshape(nb, 3).copy()
        nbcs = np.ctypeslib.as_array(d.nbcs, (nb,)).copy()
        nbc = int(nbcs.sum())
        bct = (np.ctypeslib.as_array(d.bctopo, (10 * nbc,)).reshape(nbc, 10).copy() if nbc
               else np.zeros((0, 10), np.int32))
        cut = (np.ctypeslib.as_array(d.cutopo, (21 * d.ncuts,)).reshape(d.ncuts, 21).copy() if d.ncuts
               else np.zeros((0, 21), np.int32))
    finally:
        L.cosa_io_free_input(h)
    return p, r, LevelTables(dims.astype(np.int32), nbcs.astype(np.int32), bct.astype(np.int32),
                             cut.astype(np.int32))


def write_input(path: str, params: CosaParams, run: RunOpts, tables: LevelTables) -> None:
    arrs = [_dims(tables), np.ascontiguousarray(tables.nbcs, dtype=np.int32),
            np.ascontiguousarray(tables.bctopo.ravel(), dtype=np.int32),
            np.ascontiguousarray(tables.cutopo.ravel(), dtype=np.int32)]
    ip = C.POINTER(C.c_int32)
    d = gpu.LevelDesc(tables.nblocks, arrs[0].ctypes.data_as(ip), arrs[1].ctypes.data_as(ip),
                      arrs[2].ctypes.data_as(ip), tables.ncuts, arrs[3].ctypes.data_as(ip))
    _check(_lib().cosa_io_write_input(str(path).encode(), C.byref(params), C.byref(run), C.byref(d)),
           "cosa_io_write_input")


def read_mesh(path: str, tables: LevelTables, with_disp: bool = False):
    """x, y, z as P2 node arrays (and dx, dy, dz as P1 arrays with_disp);
    nodes outside 1..imax stay zero."""
    _, tot = tables.offsets()
    xyz = [np.zeros(tot["p2"]) for _ in range(3)]
    dxyz = [np.zeros(tot["p1"]) for _ in range(3)] if with_disp else [None] * 3
    args = [_p(a) for a in xyz] + [(_p(a) if a is not None else None) for a in dxyz]
    _check(_lib().cosa_io_read_mesh(str(path).encode(), C.c_int32(tables.nblocks), _p(_dims(tables)),
                                    C.c_int32(int(with_disp)), *args), "cosa_io_read_mesh")
    return (*xyz, *dxyz) if with_disp else tuple(xyz)


def write_mesh(path: str, tables: LevelTables, x, y, z, dx=None, dy=None, dz=None) -> None:
    with_disp = dx is not None
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z)]
    b = [np.ascontiguousarray(v, dtype=np.float64) for v in (dx, dy, dz)] if with_disp else [None] * 3
    args = [_p(v) for v in a] + [(_p(v) if v is not None else None) for v in b]
    _check(_lib().cosa_io_write_mesh(str(path).encode(), C.c_int32(tables.nblocks), _p(_dims(tables)),
                                     C.c_int32(int(with_disp)), *args), "cosa_io_write_mesh")


def read_restart(path: str, tables: LevelTables, npde: int, nharms: int = 0, with_q1: bool = False,
                 with_mut: bool = False):
    """(q, q1 or None, mut or None) in the P3 layouts."""
    _, tot = tables.offsets()
    S = 2 * nharms + 1
    q = np.zeros(tot["p3"] * npde * S)
    q1 = np.zeros(tot["p3"] * npde) if with_q1 else None
    mut = np.zeros(tot["p3"] * S) if with_mut else None
    _check(_lib().cosa_io_read_restart(str(path).encode(), C.c_int32(tables.nblocks), _p(_dims(tables)),
                                       C.c_int32(npde), C.c_int32(nharms), C.c_int32(int(with_q1)),
                                       C.c_int32(int(with_mut)), _p(q), _p(q1) if with_q1 else None,
                                       _p(mut) if with_mut else None), "cosa_io_read_restart")
    return q, q1, mut


def write_restart(path: str, tables: LevelTables, npde: int, q, nharms: int = 0, q1: Optional[np.ndarray] = None,
                  mut: Optional[np.ndarray] = None) -> None:
    qa = np.ascontiguousarray(q, dtype=np.float64)
    q1a = np.ascontiguousarray(q1, dtype=np.float64) if q1 is not None else None
    ma = np.ascontiguousarray(mut, dtype=np.float64) if mut is not None else None
    _, tot = tables.offsets()
    S = 2 * nharms + 1
    if qa.size != tot["p3"] * npde * S or (q1a is not None and q1a.size != tot["p3"] * npde) or \
            (ma is not None and ma.size != tot["p3"] * S):
        raise CaseFileError("write_restart: array sizes", 0x10)
    _check(_lib().cosa_io_write_restart(str(path).encode(), C.c_int32(tables.nblocks), _p(_dims(tables)),
                                        C.c_int32(npde), C.c_int32(nharms), C.c_int32(int(q1a is not None)),
                                        C.c_int32(int(ma is not None)), _p(qa),
                                        _p(q1a) if q1a is not None else None,
                                        _p(ma) if ma is not None else None), "cosa_io_write_restart")
