"""ctypes binding of libcosa_gpu.so (include/cosa_gpu.h) and a small host driver.

This is the Python mirror of the Fortran side of the boundary: the same
entry points a Fortran ``interface ... bind(C)`` block would declare, called
with device pointers to arrays in COSA's layout.  There is no CPU fallback:
if the CUDA library or a GPU is missing, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from . import build as _build
from .params import CosaParams
from .tables import LevelTables

_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)

ERR = {0x001: "NEG_P", 0x002: "NEG_RHO", 0x004: "INFLOW", 0x008: "NAN", 0x010: "ARG", 0x020: "CUDA",
       0x040: "TIMEOUT", 0x080: "UNSUPPORTED"}


class CosaError(RuntimeError):
    def __init__(self, code: int, what: str):
        names = [v for k, v in ERR.items() if code & k]
        super().__init__(f"{what}: status 0x{code:x} ({'|'.join(names) or '?'})")
        self.code = code


class LevelDesc(C.Structure):
    _fields_ = [("nblocks", C.c_int32), ("dims", _ip), ("nbcs", _ip), ("bctopo", _ip),
                ("ncuts", C.c_int32), ("cutopo", _ip)]


class LevelPtrs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "q", "qold", "res", "rhs", "dtvol", "dtvolt", "si", "sj", "sk", "vol",
        "qp", "qm", "dq", "dqp", "dqm", "flux", "betaxi", "betaeta", "betazeta",
        "mut", "dist", "xdot", "ydot", "zdot", "fvi", "fvj", "fvk")]


# public symbols of include/cosa_gpu.h
SYMBOLS = [
    "cosa_gpu_params_size", "cosa_gpu_init", "cosa_gpu_finalize", "cosa_gpu_set_params",
    "cosa_gpu_level_sizes", "cosa_gpu_malloc", "cosa_gpu_memcpy_h2d", "cosa_gpu_memcpy_d2h",
    "cosa_gpu_synchronize", "cosa_gpu_bind_level", "cosa_gpu_cons2prim", "cosa_gpu_prim2cons",
    "cosa_gpu_bc", "cosa_gpu_cutman_q", "cosa_gpu_prtest", "cosa_gpu_lambda", "cosa_gpu_deltat",
    "cosa_gpu_muscl", "cosa_gpu_roflux", "cosa_gpu_resid", "cosa_gpu_update", "cosa_gpu_resg_rms",
    "cosa_gpu_zero", "cosa_gpu_smooth", "cosa_gpu_smooth_host", "cosa_gpu_launch_count",
    "cosa_gpu_status", "cosa_gpu_imetrix", "cosa_gpu_vols", "cosa_gpu_profile", "cosa_gpu_stream",
    "cosa_gpu_resg_rms_noalloc", "cosa_gpu_scalef", "cosa_gpu_scaleb", "cosa_gpu_cirs", "cosa_gpu_ccirs",
    "cosa_gpu_src_hb", "cosa_gpu_q_edges", "cosa_gpu_q_corns", "cosa_gpu_fixq", "cosa_gpu_tur_vis",
    "cosa_gpu_rest1", "cosa_gpu_rest2", "cosa_gpu_prol_bln", "cosa_gpu_prol_lin", "cosa_gpu_restrict",
    "cosa_gpu_prolong", "cosa_gpu_smooth_level", "cosa_gpu_mg", "cosa_gpu_nr_selftest",
    "cosa_serve_create", "cosa_serve_destroy", "cosa_serve_submit", "cosa_serve_step", "cosa_serve_result",
    "cosa_serve_free_slots", "cosa_gpu_coordex", "cosa_gpu_cutman_x", "cosa_gpu_volex", "cosa_gpu_cutman_v",
    "cosa_gpu_vmetrix", "cosa_gpu_viscous_setup", "cosa_gpu_q_face", "cosa_gpu_q_der", "cosa_gpu_vflux",
    "cosa_gpu_lambda_ns", "cosa_gpu_deltat_ns", "cosa_gpu_q_face_mut", "cosa_gpu_rtst", "cosa_gpu_vflux_kom",
    "cosa_gpu_q_der_c", "cosa_gpu_turprod", "cosa_gpu_srckw", "cosa_gpu_update_kom", "cosa_gpu_cutman_mut",
    "cosa_gpu_autotune", "cosa_gpu_set_schedule", "cosa_gpu_force", "cosa_gpu_rest2_ho", "cosa_gpu_bc_res",
    "cosa_gpu_movegrid", "cosa_gpu_face_vel", "cosa_gpu_vert2cell", "cosa_gpu_facedist", "cosa_gpu_update_ttrm",
    "cosa_gpu_srckw_sst", "cosa_gpu_tur_vis_sst", "cosa_gpu_src_uns", "cosa_gpu_rhs_uns", "cosa_gpu_rkuns",
    "cosa_gpu_copy_interior", "cosa_gpu_lm_cutoff_pg", "cosa_gpu_lm_viscoff", "cosa_gpu_rest3", "cosa_gpu_proflux",
    "cosa_gpu_lambda_p", "cosa_gpu_lsp", "cosa_gpu_precres", "cosa_gpu_lsp_cutoffs",
]


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libcosa_gpu.so (building it in-tree first if needed)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if not build_if_missing:
            raise OSError(f"{path} missing: run cosa_b200.build.build()")
        _build.build()
    L = C.CDLL(path)
    L.cosa_gpu_params_size.restype = C.c_int64
    L.cosa_gpu_launch_count.restype = C.c_int64
    L.cosa_gpu_stream.restype = C.c_void_p
    L.cosa_serve_free_slots.restype = C.c_int64
    L.cosa_gpu_init.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]
    for name in SYMBOLS:
        if name not in ("cosa_gpu_params_size", "cosa_gpu_launch_count", "cosa_gpu_stream", "cosa_serve_free_slots"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _ptr(x) -> C.c_void_p:
    return C.c_void_p(int(x)) if x is not None else C.c_void_p(0)


class DevArray:
    """A device float64 array owned by a Context."""

    def __init__(self, ctx: "Context", n: int):
        self.ctx = ctx
        self.n = int(n)
        p = C.c_void_p()
        ctx._check(load().cosa_gpu_malloc(ctx.h, C.c_int64(self.n), C.byref(p)), "cosa_gpu_malloc")
        self.ptr = p.value

    def upload(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.size == self.n, (a.size, self.n)
        self.ctx._check(load().cosa_gpu_memcpy_h2d(self.ctx.h, _ptr(self.ptr), a.ctypes.data_as(C.c_void_p),
                                                   C.c_int64(self.n)), "h2d")
        self.ctx.sync()
        return self

    def download(self) -> np.ndarray:
        out = np.empty(self.n)
        self.ctx._check(load().cosa_gpu_memcpy_d2h(self.ctx.h, out.ctypes.data_as(C.c_void_p), _ptr(self.ptr),
                                                   C.c_int64(self.n)), "d2h")
        return out


class Context:
    """cosa_ctx: module state of one solve on one GPU."""

    def __init__(self, levels: Sequence[LevelTables], params: CosaParams, device: int = 0):
        L = load()
        if L.cosa_gpu_params_size() != C.sizeof(CosaParams):
            raise RuntimeError("cosa_params ABI mismatch between Python and libcosa_gpu.so")
        self.params = params
        self.levels = list(levels)
        self._keep = []
        descs = (LevelDesc * len(self.levels))()
        for i, t in enumerate(self.levels):
            arrs = [np.ascontiguousarray(t.dims.ravel(), dtype=np.int32),
                    np.ascontiguousarray(t.nbcs, dtype=np.int32),
                    np.ascontiguousarray(t.bctopo.ravel(), dtype=np.int32),
                    np.ascontiguousarray(t.cutopo.ravel(), dtype=np.int32)]
            self._keep.append(arrs)
            ip = lambda a: a.ctypes.data_as(_ip)
            descs[i] = LevelDesc(t.nblocks, ip(arrs[0]), ip(arrs[1]), ip(arrs[2]), t.ncuts, ip(arrs[3]))
        h = C.c_void_p()
        self.h = None
        self._check(L.cosa_gpu_init(C.byref(params), len(self.levels), descs, device, C.byref(h)), "cosa_gpu_init")
        self.h = h
        self.S = 2 * params.nharms + 1

    def _check(self, st: int, what: str):
        if st != 0:
            raise CosaError(st, what)

    def close(self):
        if self.h is not None:
            load().cosa_gpu_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        self._check(load().cosa_gpu_synchronize(self.h), "sync")

    def sizes(self, nl: int = 1):
        s = (C.c_int64 * 5)()
        self._check(load().cosa_gpu_level_sizes(self.h, nl, s), "level_sizes")
        return list(s)

    def set_params(self, p: CosaParams):
        self._check(load().cosa_gpu_set_params(self.h, C.byref(p)), "set_params")
        self.params = p

    def alloc_p3(self, nl=1, nvar=None):
        n3 = self.sizes(nl)[0]
        return DevArray(self, n3 * (nvar or self.params.npde) * self.S)

    def alloc_p2(self, nl=1, ncomp=4):
        return DevArray(self, self.sizes(nl)[1] * ncomp)

    def alloc_p1(self, nl=1, nsnap=1):
        return DevArray(self, self.sizes(nl)[2] * nsnap)

    def alloc_f0(self, nl=1):
        return DevArray(self, self.sizes(nl)[3] * self.params.npde * self.S)

    def alloc_f0s(self, nl=1):
        """One F0 scalar (imax, jmax, kmax) per block, no snapshots (face wall distance)."""
        return DevArray(self, self.sizes(nl)[3])

    def status(self, reset: bool = False) -> int:
        return load().cosa_gpu_status(self.h, 1 if reset else 0)

    def launch_count(self, reset: bool = False) -> int:
        return int(load().cosa_gpu_launch_count(self.h, 1 if reset else 0))

    # ---- level drivers -------------------------------------------------------
    def cons2prim(self, nl, q, xtnd=0):
        self._check(load().cosa_gpu_cons2prim(self.h, nl, xtnd, _ptr(q.ptr)), "cons2prim")

    def prim2cons(self, nl, q):
        self._check(load().cosa_gpu_prim2cons(self.h, nl, _ptr(q.ptr)), "prim2cons")

    def bc(self, nl, q, si, sj, sk):
        self._check(load().cosa_gpu_bc(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                       _ptr(None)), "bc")

    def cutman_q(self, nl, q):
        self._check(load().cosa_gpu_cutman_q(self.h, nl, _ptr(q.ptr)), "cutman_q")

    def prtest(self, nl, q) -> int:
        return load().cosa_gpu_prtest(self.h, nl, _ptr(q.ptr))

    def lambda_(self, nl, q, si, sj, sk, vol, lam):
        self._check(load().cosa_gpu_lambda(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                           _ptr(vol.ptr if vol else None), _ptr(lam.ptr)), "lambda")

    def deltat(self, nl, dtvol, lam, bx=None, by=None, bz=None):
        self._check(load().cosa_gpu_deltat(self.h, nl, _ptr(dtvol.ptr), _ptr(lam.ptr),
                                           _ptr(bx.ptr if bx else None), _ptr(by.ptr if by else None),
                                           _ptr(bz.ptr if bz else None)), "deltat")

    def muscl(self, idir, nl, q, qp, qm, dq, dqp, dqm):
        self._check(load().cosa_gpu_muscl(self.h, idir, nl, _ptr(q.ptr), _ptr(qp.ptr), _ptr(qm.ptr), _ptr(dq.ptr),
                                          _ptr(dqp.ptr), _ptr(dqm.ptr)), "muscl")

    def roflux(self, idir, nl, qr, ql, flux, sijk):
        self._check(load().cosa_gpu_roflux(self.h, idir, nl, _ptr(qr.ptr), _ptr(ql.ptr), _ptr(flux.ptr),
                                           _ptr(sijk.ptr)), "roflux")

    def resid(self, idir, nl, flux, res):
        self._check(load().cosa_gpu_resid(self.h, idir, nl, _ptr(flux.ptr), _ptr(res.ptr)), "resid")

    def update(self, nl, res, q, qold, dtvol, ar):
        self._check(load().cosa_gpu_update(self.h, nl, _ptr(res.ptr), _ptr(q.ptr), _ptr(qold.ptr), _ptr(dtvol.ptr),
                                           C.c_double(ar)), "update")

    def zero(self, nl, a):
        self._check(load().cosa_gpu_zero(self.h, nl, _ptr(a.ptr)), "zero")

    def resg_rms(self, nl, res, rhs=None):
        out = np.zeros(self.params.npde + 1)
        self._check(load().cosa_gpu_resg_rms(self.h, nl, _ptr(res.ptr), _ptr(rhs.ptr if rhs else None),
                                             out.ctypes.data_as(_dp)), "resg_rms")
        return out

    def src_hb(self, nl, q, vol, res):
        self._check(load().cosa_gpu_src_hb(self.h, nl, _ptr(q.ptr), _ptr(vol.ptr), _ptr(res.ptr)), "src_hb")

    def scalef(self, nl, res, dtvol, dtvolt=None):
        self._check(load().cosa_gpu_scalef(self.h, nl, _ptr(res.ptr), _ptr(dtvol.ptr),
                                           _ptr(dtvolt.ptr if dtvolt else None)), "scalef")

    def scaleb(self, nl, res, dtvol, dtvolt=None):
        self._check(load().cosa_gpu_scaleb(self.h, nl, _ptr(res.ptr), _ptr(dtvol.ptr),
                                           _ptr(dtvolt.ptr if dtvolt else None)), "scaleb")

    def cirs(self, nl, res, dtvol, bx=None, by=None, bz=None):
        self._check(load().cosa_gpu_cirs(self.h, nl, _ptr(res.ptr), _ptr(dtvol.ptr), _ptr(bx.ptr if bx else None),
                                         _ptr(by.ptr if by else None), _ptr(bz.ptr if bz else None)), "cirs")

    def ccirs(self, nl, res, ores, bx=None, by=None, bz=None):
        self._check(load().cosa_gpu_ccirs(self.h, nl, _ptr(res.ptr), _ptr(ores.ptr), _ptr(bx.ptr if bx else None),
                                          _ptr(by.ptr if by else None), _ptr(bz.ptr if bz else None)), "ccirs")

    def imetrix(self, nl, x, y, z, si, sj, sk):
        self._check(load().cosa_gpu_imetrix(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr), _ptr(si.ptr),
                                            _ptr(sj.ptr), _ptr(sk.ptr)), "imetrix")

    def vols(self, nl, x, y, z, vol):
        self._check(load().cosa_gpu_vols(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr), _ptr(vol.ptr)), "vols")

    # ---- moving grids (harmonic balance of a pitching body) -----------------------------
    def movegrid(self, nl, x0, y0, z0, dx, dy, dz, x, y, z, xdot, ydot, zdot):
        self._check(load().cosa_gpu_movegrid(self.h, nl, *(_ptr(a.ptr) for a in (x0, y0, z0, dx, dy, dz, x, y, z,
                                                                                 xdot, ydot, zdot))), "movegrid")

    def face_vel(self, nl, xdot, ydot, zdot, fvi, fvj, fvk):
        self._check(load().cosa_gpu_face_vel(self.h, nl, *(_ptr(a.ptr) for a in (xdot, ydot, zdot, fvi, fvj, fvk))),
                    "face_vel")

    def vert2cell(self, nl, w):
        self._check(load().cosa_gpu_vert2cell(self.h, nl, _ptr(w.ptr)), "vert2cell")

    def pitching_setup(self, nl, case):
        """The moving grid of a pitching harmonic-balance case in the
        reference's set-up order: movegrid, vols, imetrix (per snapshot),
        face velocities, vert2cell of the grid velocities.  Returns a dict of
        device arrays (x, y, z, xdot, ydot, zdot, si, sj, sk, vol, fvi, fvj,
        fvk); the displacement scales are 1 (rigid motion)."""
        S = self.S
        n1 = self.sizes(nl)[2]
        x0, y0, z0 = (self.alloc_p2(nl, ncomp=1).upload(a) for a in (case.x, case.y, case.z))
        dxyz = [self.alloc_p1(nl).upload(np.ones(n1)) for _ in range(3)]
        m = {k: self.alloc_p2(nl, ncomp=S) for k in ("x", "y", "z", "xdot", "ydot", "zdot")}
        self.movegrid(nl, x0, y0, z0, *dxyz, m["x"], m["y"], m["z"], m["xdot"], m["ydot"], m["zdot"])
        m["vol"] = self.alloc_p1(nl)
        self.vols(nl, m["x"], m["y"], m["z"], m["vol"])
        for k in ("si", "sj", "sk"):
            m[k] = self.alloc_p2(nl, ncomp=4 * S)
        self.imetrix(nl, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"])
        for k in ("fvi", "fvj", "fvk"):
            m[k] = self.alloc_p2(nl, ncomp=3 * S)
        self.face_vel(nl, m["xdot"], m["ydot"], m["zdot"], m["fvi"], m["fvj"], m["fvk"])
        for k in ("xdot", "ydot", "zdot"):
            self.vert2cell(nl, m[k])
        return m

    def profile(self, nl, niter):
        ms = (C.c_double * 4)()
        cnt = (C.c_int64 * 4)()
        self._check(load().cosa_gpu_profile(self.h, nl, niter, ms, cnt), "profile")
        return list(ms), list(cnt)

    def autotune(self, nl=1, niter=5):
        """Time the fused-tile and face-split stage schedules on level nl and
        keep the faster; returns (ms_tile, ms_split, choice)."""
        ms = (C.c_double * 2)()
        ch = C.c_int32()
        self._check(load().cosa_gpu_autotune(self.h, nl, niter, ms, C.byref(ch)), "autotune")
        return ms[0], ms[1], ch.value

    def set_schedule(self, nl, schedule):
        self._check(load().cosa_gpu_set_schedule(self.h, nl, schedule), "set_schedule")

    def stream(self) -> int:
        return int(load().cosa_gpu_stream(self.h) or 0)

    def bind_level(self, nl, **arrays):
        p = LevelPtrs()
        for k, v in arrays.items():
            setattr(p, k, v.ptr if v is not None else None)
        self._check(load().cosa_gpu_bind_level(self.h, nl, C.byref(p)), "bind_level")

    def smooth(self, nl, niter, mgit0=1, rms_every=1, want_hist=True):
        hist = np.full((max(niter, 1), self.params.npde + 1), np.nan) if want_hist else None
        st = load().cosa_gpu_smooth(self.h, nl, niter, mgit0, rms_every,
                                    hist.ctypes.data_as(_dp) if want_hist else _dp())
        return (hist[:niter] if want_hist else None), st

    # ---- laminar viscous terms -------------------------------------------------------
    def alloc_vm(self, nl=1):
        """The nine face inverse-metric arrays of level nl (27 * n0 doubles);
        on a moving grid one set per node snapshot."""
        nsnap = self.S if self.params.moving and self.params.hbmove else 1
        return DevArray(self, self.sizes(nl)[3] * 27 * nsnap)

    def coordex(self, nl, x, y, z):
        self._check(load().cosa_gpu_coordex(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr)), "coordex")

    def cutman_x(self, nl, x, y, z):
        self._check(load().cosa_gpu_cutman_x(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr)), "cutman_x")

    def volex(self, nl, vol):
        self._check(load().cosa_gpu_volex(self.h, nl, _ptr(vol.ptr)), "volex")

    def cutman_v(self, nl, vol):
        self._check(load().cosa_gpu_cutman_v(self.h, nl, _ptr(vol.ptr)), "cutman_v")

    def vmetrix(self, nl, x, y, z, vol, vm):
        self._check(load().cosa_gpu_vmetrix(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr), _ptr(vol.ptr),
                                            _ptr(vm.ptr)), "vmetrix")

    def viscous_setup(self, nl, x, y, z, vol, vm):
        self._check(load().cosa_gpu_viscous_setup(self.h, nl, _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr), _ptr(vol.ptr),
                                                  _ptr(vm.ptr)), "viscous_setup")

    def q_face(self, idir, nl, q, qf):
        self._check(load().cosa_gpu_q_face(self.h, idir, nl, _ptr(q.ptr), _ptr(qf.ptr)), "q_face")

    def q_der(self, idir, nl, q, dqxi, dqeta, dqzeta):
        self._check(load().cosa_gpu_q_der(self.h, idir, nl, _ptr(q.ptr), _ptr(dqxi.ptr), _ptr(dqeta.ptr),
                                          _ptr(dqzeta.ptr)), "q_der")

    def vflux(self, idir, nl, qf, dqxi, dqeta, dqzeta, vm, sijk, flux):
        self._check(load().cosa_gpu_vflux(self.h, idir, nl, _ptr(qf.ptr), _ptr(dqxi.ptr), _ptr(dqeta.ptr),
                                          _ptr(dqzeta.ptr), _ptr(vm.ptr), _ptr(sijk.ptr), _ptr(flux.ptr)), "vflux")

    def lambda_ns(self, nl, q, si, sj, sk, vol, lam, lamv, mut=None):
        self._check(load().cosa_gpu_lambda_ns(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                              _ptr(vol.ptr), _ptr(mut.ptr if mut else None), _ptr(lam.ptr),
                                              _ptr(lamv.ptr)), "lambda_ns")

    def deltat_ns(self, nl, dtvol, lam, lamv, bx=None, by=None, bz=None, dtvolt=None, tbx=None, tby=None, tbz=None):
        o = lambda a: _ptr(a.ptr if a else None)
        self._check(load().cosa_gpu_deltat_ns(self.h, nl, _ptr(dtvol.ptr), _ptr(lam.ptr), _ptr(lamv.ptr), o(bx), o(by),
                                              o(bz), o(dtvolt), o(tbx), o(tby), o(tbz)), "deltat_ns")

    # ---- Wilcox k-omega ---------------------------------------------------------------
    def alloc_p3s(self, nl=1):
        """A scalar P3 array (mut, prd, divvel, delpls) with S snapshots."""
        return DevArray(self, self.sizes(nl)[0] * self.S)

    def bc_dist(self, nl, q, si, sj, sk, dist):
        self._check(load().cosa_gpu_bc(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                       _ptr(dist.ptr)), "bc")

    def q_face_mut(self, idir, nl, mut, flux):
        self._check(load().cosa_gpu_q_face_mut(self.h, idir, nl, _ptr(mut.ptr), _ptr(flux.ptr)), "q_face_mut")

    def rtst(self, idir, nl, qf, dqxi, dqeta, dqzeta, vm, flux, tau1):
        self._check(load().cosa_gpu_rtst(self.h, idir, nl, _ptr(qf.ptr), _ptr(dqxi.ptr), _ptr(dqeta.ptr),
                                         _ptr(dqzeta.ptr), _ptr(vm.ptr), _ptr(flux.ptr), _ptr(tau1.ptr)), "rtst")

    def vflux_kom(self, idir, nl, qf, dqxi, dqeta, dqzeta, tau1, vm, sijk, flux, fdist=None):
        """fdist: the face wall distances of family idir (BSL/SST)."""
        self._check(load().cosa_gpu_vflux_kom(self.h, idir, nl, _ptr(qf.ptr), _ptr(dqxi.ptr), _ptr(dqeta.ptr),
                                              _ptr(dqzeta.ptr), _ptr(tau1.ptr), _ptr(vm.ptr), _ptr(sijk.ptr),
                                              _ptr(flux.ptr), _ptr(fdist.ptr if fdist is not None else None)),
                    "vflux_kom")

    def q_der_c(self, idir, nl, qf, dqc):
        self._check(load().cosa_gpu_q_der_c(self.h, idir, nl, _ptr(qf.ptr), _ptr(dqc.ptr)), "q_der_c")

    def turprod(self, nl, dqxi, dqeta, dqzeta, vm, prd, divvel, delpls):
        self._check(load().cosa_gpu_turprod(self.h, nl, _ptr(dqxi.ptr), _ptr(dqeta.ptr), _ptr(dqzeta.ptr),
                                            _ptr(vm.ptr), _ptr(prd.ptr), _ptr(divvel.ptr), _ptr(delpls.ptr)),
                    "turprod")

    def srckw(self, nl, q, mut, prd, divvel, res, vol):
        self._check(load().cosa_gpu_srckw(self.h, nl, _ptr(q.ptr), _ptr(mut.ptr), _ptr(prd.ptr), _ptr(divvel.ptr),
                                          _ptr(res.ptr), _ptr(vol.ptr)), "srckw")

    def update_kom(self, nl, res, q, qold, vol, dtvolt, delpls, prd, ar, ttrm=None):
        self._check(load().cosa_gpu_update_kom(self.h, nl, _ptr(res.ptr), _ptr(q.ptr), _ptr(qold.ptr), _ptr(vol.ptr),
                                               _ptr(dtvolt.ptr), _ptr(delpls.ptr), _ptr(prd.ptr), C.c_double(ar),
                                               _ptr(ttrm.ptr if ttrm is not None else None)), "update_kom")

    # ---- low-speed preconditioning -------------------------------------------------
    def alloc_m1(self, nl=1, nvar=1):
        """An interior-cell array x S (x nvar): the cut-off layout; nvar =
        npde^2 for a preconditioner array."""
        return DevArray(self, self.sizes(nl)[4] * self.S * nvar)

    def lm_cutoff_pg(self, nl, q, cut):
        self._check(load().cosa_gpu_lm_cutoff_pg(self.h, nl, _ptr(q.ptr), _ptr(cut.ptr)), "lm_cutoff_pg")

    def lm_viscoff(self, nl, q, si, sj, sk, cut):
        self._check(load().cosa_gpu_lm_viscoff(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                               _ptr(cut.ptr)), "lm_viscoff")

    def rest3(self, nl, c1, c2, vol1, vol2):
        self._check(load().cosa_gpu_rest3(self.h, nl, _ptr(c1.ptr), _ptr(c2.ptr), _ptr(vol1.ptr), _ptr(vol2.ptr)),
                    "rest3")

    def proflux(self, idir, nl, qr, ql, flux, sijk, cpg, cvs):
        self._check(load().cosa_gpu_proflux(self.h, idir, nl, _ptr(qr.ptr), _ptr(ql.ptr), _ptr(flux.ptr),
                                            _ptr(sijk.ptr), _ptr(cpg.ptr), _ptr(cvs.ptr)), "proflux")

    def lambda_p(self, nl, q, si, sj, sk, lam, cpg, cvs, vol=None, lamv=None):
        self._check(load().cosa_gpu_lambda_p(self.h, nl, _ptr(q.ptr), _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                             _ptr(vol.ptr if vol is not None else None), _ptr(lam.ptr),
                                             _ptr(lamv.ptr if lamv is not None else None), _ptr(cpg.ptr),
                                             _ptr(cvs.ptr)), "lambda_p")

    def lsp(self, nl, q, cpg, cvs, prec):
        self._check(load().cosa_gpu_lsp(self.h, nl, _ptr(q.ptr), _ptr(cpg.ptr), _ptr(cvs.ptr), _ptr(prec.ptr)), "lsp")

    def precres(self, nl, res, prec):
        self._check(load().cosa_gpu_precres(self.h, nl, _ptr(res.ptr), _ptr(prec.ptr)), "precres")

    def lsp_cutoffs(self, nl=1):
        """The level's own pressure-gradient and viscous cut-offs (host arrays)."""
        pgr, vis = self.alloc_m1(nl), self.alloc_m1(nl)
        self._check(load().cosa_gpu_lsp_cutoffs(self.h, nl, _ptr(pgr.ptr), _ptr(vis.ptr)), "lsp_cutoffs")
        return pgr.download(), vis.download()

    # ---- time-accurate runs -------------------------------------------------------
    def src_uns(self, nl, q, vol, res):
        self._check(load().cosa_gpu_src_uns(self.h, nl, _ptr(q.ptr), _ptr(vol.ptr), _ptr(res.ptr)), "src_uns")

    def rhs_uns(self, nl, rhs, q1, q2, vol):
        self._check(load().cosa_gpu_rhs_uns(self.h, nl, _ptr(rhs.ptr), _ptr(q1.ptr), _ptr(q2.ptr), _ptr(vol.ptr)),
                    "rhs_uns")

    def copy_interior(self, nl, dst, src):
        self._check(load().cosa_gpu_copy_interior(self.h, nl, _ptr(dst.ptr), _ptr(src.ptr)), "copy_interior")

    def rkuns(self, ntime, iprint=1):
        """rkuns on level 1: (hist (ntime, npde+1), status)."""
        hist = np.full((max(ntime, 1), self.params.npde + 1), np.nan)
        st = load().cosa_gpu_rkuns(self.h, ntime, iprint, hist.ctypes.data_as(C.c_void_p))
        return hist[:ntime], st

    def facedist(self, nl, dist, fidist, fjdist, fkdist):
        self._check(load().cosa_gpu_facedist(self.h, nl, _ptr(dist.ptr), _ptr(fidist.ptr), _ptr(fjdist.ptr),
                                             _ptr(fkdist.ptr)), "facedist")

    def update_ttrm(self, nl, q, dqxi, dqeta, dqzeta, vm, ttrm, dist):
        self._check(load().cosa_gpu_update_ttrm(self.h, nl, _ptr(q.ptr), _ptr(dqxi.ptr), _ptr(dqeta.ptr),
                                                _ptr(dqzeta.ptr), _ptr(vm.ptr), _ptr(ttrm.ptr), _ptr(dist.ptr)),
                    "update_ttrm")

    def srckw_sst(self, nl, q, prd, divvel, res, mut, ttrm, vol):
        self._check(load().cosa_gpu_srckw_sst(self.h, nl, _ptr(q.ptr), _ptr(prd.ptr), _ptr(divvel.ptr), _ptr(res.ptr),
                                              _ptr(mut.ptr), _ptr(ttrm.ptr), _ptr(vol.ptr)), "srckw_sst")

    def tur_vis_sst(self, nl, q, mut, dqxi, dqeta, dqzeta, vm, dist):
        self._check(load().cosa_gpu_tur_vis_sst(self.h, nl, _ptr(q.ptr), _ptr(mut.ptr), _ptr(dqxi.ptr),
                                                _ptr(dqeta.ptr), _ptr(dqzeta.ptr), _ptr(vm.ptr), _ptr(dist.ptr)),
                    "tur_vis_sst")

    def cutman_mut(self, nl, mut):
        self._check(load().cosa_gpu_cutman_mut(self.h, nl, _ptr(mut.ptr)), "cutman_mut")

    # ---- wall forces -------------------------------------------------------------
    def force(self, nl, q, x, y, z, si, sj, sk, vm=None, isurf=1, xmom=(0.25, 0.0, 0.0), lngth=(1.0, 1.0, 1.0)):
        """(S, 12) force and moment coefficients of surface isurf, columns
        cl_p, cd_p, cz_p, cmx_p, cmy_p, cm_p, then the viscous six."""
        S = self.S
        out = (C.c_double * (12 * S))()
        xm = (C.c_double * 3)(*xmom)
        ln = (C.c_double * 3)(*lngth)
        self._check(load().cosa_gpu_force(self.h, nl, _ptr(q.ptr), _ptr(x.ptr), _ptr(y.ptr), _ptr(z.ptr),
                                          _ptr(si.ptr), _ptr(sj.ptr), _ptr(sk.ptr),
                                          _ptr(vm.ptr if vm is not None else None), C.c_int32(isurf), xm, ln, out),
                    "force")
        return np.array(out[:], dtype=np.float64).reshape(S, 12)

    # ---- multigrid ---------------------------------------------------------------
    def q_edges(self, nl, q, mut=None):
        self._check(load().cosa_gpu_q_edges(self.h, nl, _ptr(q.ptr), _ptr(mut.ptr if mut else None)), "q_edges")

    def q_corns(self, nl, q, mut=None):
        self._check(load().cosa_gpu_q_corns(self.h, nl, _ptr(q.ptr), _ptr(mut.ptr if mut else None)), "q_corns")

    def fixq(self, nl, q):
        self._check(load().cosa_gpu_fixq(self.h, nl, _ptr(q.ptr)), "fixq")

    def tur_vis(self, nl, q, mut):
        self._check(load().cosa_gpu_tur_vis(self.h, nl, _ptr(q.ptr), _ptr(mut.ptr)), "tur_vis")

    def rest1(self, nl, q1, q2, vol1, vol2):
        self._check(load().cosa_gpu_rest1(self.h, nl, _ptr(q1.ptr), _ptr(q2.ptr), _ptr(vol1.ptr), _ptr(vol2.ptr)),
                    "rest1")

    def rest2(self, nl, rhs2, res1):
        self._check(load().cosa_gpu_rest2(self.h, nl, _ptr(rhs2.ptr), _ptr(res1.ptr)), "rest2")

    def rest2_ho(self, nl, rhs2, res1):
        self._check(load().cosa_gpu_rest2_ho(self.h, nl, _ptr(rhs2.ptr), _ptr(res1.ptr)), "rest2_ho")

    def bc_res(self, nl, res):
        self._check(load().cosa_gpu_bc_res(self.h, nl, _ptr(res.ptr)), "bc_res")

    def prol_bln(self, nl, q1, q2):
        self._check(load().cosa_gpu_prol_bln(self.h, nl, _ptr(q1.ptr), _ptr(q2.ptr)), "prol_bln")

    def prol_lin(self, nl, q1, q2, vol1):
        self._check(load().cosa_gpu_prol_lin(self.h, nl, _ptr(q1.ptr), _ptr(q2.ptr), _ptr(vol1.ptr)), "prol_lin")

    def restrict(self, nl):
        self._check(load().cosa_gpu_restrict(self.h, nl), "restrict")

    def prolong(self, nl) -> int:
        return load().cosa_gpu_prolong(self.h, nl)

    def smooth_level(self, nl, niter, from_fine, to_coarse, mgit=1, ncycle=1, rms_every=1, want_rms=True):
        out = np.full(self.params.npde + 1, np.nan)
        st = load().cosa_gpu_smooth_level(self.h, nl, niter, int(from_fine), int(to_coarse), mgit, ncycle, rms_every,
                                          out.ctypes.data_as(_dp) if want_rms else _dp())
        return out, st

    def mg(self, mgit0, ncycles, ncycle, rms_every=1, want_hist=True):
        hist = np.full((max(ncycles, 1), self.params.npde + 1), np.nan) if want_hist else None
        st = load().cosa_gpu_mg(self.h, mgit0, ncycles, ncycle, rms_every,
                                hist.ctypes.data_as(_dp) if want_hist else _dp())
        return (hist[:ncycles] if want_hist else None), st

    def smooth_host(self, nl, q_host: np.ndarray, niter, mgit0=1, rms_every=1, want_hist=True):
        hist = np.full((max(niter, 1), self.params.npde + 1), np.nan) if want_hist else None
        st = load().cosa_gpu_smooth_host(self.h, nl, q_host.ctypes.data_as(_dp), niter, mgit0, rms_every,
                                         hist.ctypes.data_as(_dp) if want_hist else _dp())
        return (hist[:niter] if want_hist else None), st


SOLVE_STATES = {0: "queued", 1: "active", 2: "converged", 3: "stopped", 4: "failed"}


class Server:
    """cosa_serve: steady solves of different grids and flow conditions
    resident on one GPU and advanced together (continuous batching)."""

    def __init__(self, scheme: CosaParams, budget_bytes: int, device: int = 0, check_every: int = 10):
        L = load()
        h = C.c_void_p()
        st = L.cosa_serve_create(C.byref(scheme), C.c_int64(int(budget_bytes)), device, check_every, C.byref(h))
        if st:
            raise CosaError(st, "cosa_serve_create")
        self.h = h
        self.npde = scheme.npde
        self._sizes = {}

    def close(self):
        if self.h is not None:
            load().cosa_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, tables: LevelTables, x, y, z, q0, flow: CosaParams, tol: float, max_iter: int) -> int:
        arrs = [np.ascontiguousarray(tables.dims.ravel(), dtype=np.int32),
                np.ascontiguousarray(tables.nbcs, dtype=np.int32),
                np.ascontiguousarray(tables.bctopo.ravel(), dtype=np.int32),
                np.ascontiguousarray(tables.cutopo.ravel(), dtype=np.int32)]
        ip = lambda a: a.ctypes.data_as(_ip)
        d = LevelDesc(tables.nblocks, ip(arrs[0]), ip(arrs[1]), ip(arrs[2]), tables.ncuts, ip(arrs[3]))
        dp = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)
        xs = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z, q0)]
        rid = C.c_int64()
        st = load().cosa_serve_submit(self.h, C.byref(d), *(a.ctypes.data_as(_dp) for a in xs), C.byref(flow),
                                      C.c_double(tol), C.c_int32(max_iter), C.byref(rid))
        if st:
            raise CosaError(st, "cosa_serve_submit")
        self._sizes[rid.value] = xs[3].size
        return rid.value

    def step(self, niter: int):
        na, nq = C.c_int32(), C.c_int32()
        st = load().cosa_serve_step(self.h, niter, C.byref(na), C.byref(nq))
        if st:
            raise CosaError(st, "cosa_serve_step")
        return na.value, nq.value

    def result(self, rid: int, want_state: bool = False):
        s, it, drop = C.c_int32(), C.c_int32(), C.c_double()
        t = (C.c_double * 3)()
        q = np.zeros(self._sizes[rid]) if want_state else None
        st = load().cosa_serve_result(self.h, C.c_int64(rid), C.byref(s), C.byref(it), C.byref(drop), t,
                                      q.ctypes.data_as(_dp) if want_state else _dp())
        if st:
            raise CosaError(st, "cosa_serve_result")
        return {"state": SOLVE_STATES[s.value], "iters": it.value, "rms_drop": drop.value,
                "t_submit": t[0], "t_admit": t[1], "t_done": t[2], "q": q}

    def free_slots(self) -> int:
        return int(load().cosa_serve_free_slots(self.h))


def nr_selftest(x: np.ndarray):
    """Largest relative differences of the fused kernel's Newton-Raphson 1/x
    and 1/sqrt(x) from IEEE division and square root, on the GPU."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    err = (C.c_double * 2)()
    st = load().cosa_gpu_nr_selftest(C.c_int64(x.size), x.ctypes.data_as(_dp), err)
    if st:
        raise CosaError(st, "cosa_gpu_nr_selftest")
    return float(err[0]), float(err[1])


class Solver:
    """Single-level explicit RK solve on one GPU (mg() with nlevel = 1):
    device-resident state, metrics uploaded once, smooth() iterations fused."""

    def __init__(self, tables: LevelTables, params: CosaParams, si: np.ndarray, sj: np.ndarray, sk: np.ndarray,
                 vol: Optional[np.ndarray], q0: np.ndarray, device: int = 0):
        self.ctx = Context([tables], params, device)
        c = self.ctx
        self.q = c.alloc_p3().upload(q0)
        self.qold = c.alloc_p3()
        self.dtvol = c.alloc_p1(nsnap=c.S)
        self.si = c.alloc_p2().upload(si)
        self.sj = c.alloc_p2().upload(sj)
        self.sk = c.alloc_p2().upload(sk)
        self.vol = c.alloc_p1().upload(vol) if vol is not None else None
        c.bind_level(1, q=self.q, qold=self.qold, dtvol=self.dtvol, si=self.si, sj=self.sj, sk=self.sk,
                     vol=self.vol)
        self.mgit = 1

    def run(self, ncycles: int, rms_every: int = 1):
        hist, st = self.ctx.smooth(1, ncycles, self.mgit, rms_every)
        if st:
            raise CosaError(st, "cosa_gpu_smooth")
        self.mgit += ncycles
        return hist

    def state(self) -> np.ndarray:
        return self.q.download()

    def close(self):
        self.ctx.close()
