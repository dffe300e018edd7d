"""The reference's case files through the C-ABI (include/cosa_io.h):
input.dat (input(), src/input.f90:2271-4392), mesh.dat (readgrid,
src/input.f90:4482-4570), the restart file (readrest,
src/input.f90:4620-4716; writerest, src/output.f90:3484-3566) and the
history and force files of output() and force() (src/output.f90:4100-4386,
4941-4965).

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
    "cosa_io_write_restart", "cosa_io_hist_record", "cosa_io_force_header", "cosa_io_force_record",
]

# column order of the force files per surface, as indices into the (S, 12)
# rows of gpu.Context.force (cl_p, cd_p, cz_p, cmx_p, cmy_p, cm_p, then the
# viscous six): cl_p, cl_v, cd_p, cd_v, cz_p, cz_v, cmx_p, cmx_v, cmy_p,
# cmy_v, cm_p, cm_v
FORCE_FILE_COLUMNS = [0, 6, 1, 7, 2, 8, 3, 9, 4, 10, 5, 11]


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


_BUF = 1 << 16


def hist_record(itime: int, it: int, res) -> str:
    """A line of hist.dat / histur.dat / histg.dat, format
    (i7,2x,i7,5(1x,e13.5)) (src/output.f90:4941-4965)."""
    r = np.ascontiguousarray(res, dtype=np.float64)
    buf = C.create_string_buffer(_BUF)
    _check(_lib().cosa_io_hist_record(C.c_int32(itime), C.c_int32(it), _p(r), C.c_int32(r.size), buf,
                                      C.c_int64(_BUF)), "cosa_io_hist_record")
    return buf.value.decode()


def force_header(params: CosaParams, nsurface: int = 1, n: int = 0) -> str:
    buf = C.create_string_buffer(_BUF)
    _check(_lib().cosa_io_force_header(C.byref(params), C.c_int32(nsurface), C.c_int32(n), buf, C.c_int64(_BUF)),
           "cosa_io_force_header")
    return buf.value.decode()


def force_record(params: CosaParams, it: int, coef_rows, itime: int = 0, time: float = 0.0, zeit: float = 0.0,
                 alpha_deg: float = 0.0) -> str:
    """coef_rows: one (12,) row of gpu.Context.force per surface (its column
    order); written in the force file's order."""
    rows = np.atleast_2d(np.asarray(coef_rows, dtype=np.float64))
    c = np.ascontiguousarray(rows[:, FORCE_FILE_COLUMNS].ravel())
    buf = C.create_string_buffer(_BUF)
    _check(_lib().cosa_io_force_record(C.byref(params), C.c_int32(rows.shape[0]), C.c_int32(itime), C.c_int32(it),
                                       C.c_double(time), C.c_double(zeit), _p(c), C.c_double(alpha_deg), buf,
                                       C.c_int64(_BUF)), "cosa_io_force_record")
    return buf.value.decode()


class OutputFiles:
    """The history and force files of a steady or harmonic-balance run in a
    directory, written as output() and force() write them
    (src/output.f90:4889-5010): hist.dat (and histur.dat for k-omega) on
    cycle 1, every iprint-th cycle and the last one; histg.dat on the last
    one; forces_tec.dat (steady) or forces_hb_<nnn>.dat per snapshot
    (harmonic balance), created with their header on cycle 1 and appended
    after that.  hist(it, resrms_row) takes a row of the library's residual
    history (npde + 1 values; the last is the total); forces(it, coef) the
    (S, 12) array of gpu.Context.force of surface 1."""

    def __init__(self, directory: str, params: CosaParams, iprint: int = 10, itime: int = 0):
        import os
        self.dir, self.p, self.iprint, self.itime = directory, params, max(1, iprint), itime
        self.kom = bool(params.kom or params.kom_bsl or params.kom_sst)
        os.makedirs(directory, exist_ok=True)
        for name in ("hist.dat", "histg.dat") + (("histur.dat",) if self.kom else ()):
            open(os.path.join(directory, name), "w").close()

    def _due(self, it: int, last: bool) -> bool:
        return it != 0 and (it == 1 or it % self.iprint == 0 or last)

    def hist(self, it: int, row, last: bool = False) -> None:
        import os
        if not self._due(it, last):
            return
        r = np.asarray(row, dtype=np.float64)
        with open(os.path.join(self.dir, "hist.dat"), "a") as f:
            f.write(hist_record(self.itime, it, r[:5]))
        if self.kom:
            with open(os.path.join(self.dir, "histur.dat"), "a") as f:
                f.write(hist_record(self.itime, it, r[5:self.p.npde]))
        if last:
            with open(os.path.join(self.dir, "histg.dat"), "a") as f:
                f.write(hist_record(self.itime, it, r[:5]))

    def forces(self, it: int, coef, last: bool = False, alpha_deg=None) -> None:
        import os
        if not self._due(it, last):
            return
        p = self.p
        coef = np.atleast_2d(coef)
        S = 2 * p.nharms + 1
        for n in range(S if p.harbal else 1):
            name = f"forces_hb_{n:03d}.dat" if p.harbal else "forces_tec.dat"
            path = os.path.join(self.dir, name)
            mode = "w" if it == 1 else "a"
            with open(path, mode) as f:
                if it == 1:
                    f.write(force_header(p, 1, n))
                zeit = 0.0
                if p.harbal and p.omegas != 0:
                    zeit = n * 2 * np.pi / abs(p.omegas) / S
                a = 0.0 if alpha_deg is None else float(np.atleast_1d(alpha_deg)[min(n, np.size(alpha_deg) - 1)])
                f.write(force_record(p, it, coef[n:n + 1], self.itime, 0.0, zeit, a))
