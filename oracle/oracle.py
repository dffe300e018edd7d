"""ORACLE -- test infrastructure only (ctypes wrapper of liboracle_cosa.so).

Used by tests/, by __graft_entry__.smoke() as the checker, and by bench.py's
cpu_baseline / --impl reference legs.  The product (cosa_b200) never imports
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle_cosa.so")
_lib = None

_dp = C.POINTER(C.c_double)


class _LevelDesc(C.Structure):
    _fields_ = [("nblocks", C.c_int32), ("dims", C.POINTER(C.c_int32)),
                ("nbcs", C.POINTER(C.c_int32)), ("bctopo", C.POINTER(C.c_int32)),
                ("ncuts", C.c_int32), ("cutopo", C.POINTER(C.c_int32))]


class _LevelPtrs(C.Structure):
    # cosa_level_ptrs of include/cosa_gpu.h
    _fields_ = [(n, _dp) for n in (
        "q", "qold", "res", "rhs", "dtvol", "dtvolt", "si", "sj", "sk", "vol",
        "qp", "qm", "dq", "dqp", "dqm", "flux", "betaxi", "betaeta", "betazeta",
        "mut", "dist", "xdot", "ydot", "zdot", "fvi", "fvj", "fvk")]


def build(force: bool = False) -> str:
    srcs = [os.path.join(_HERE, f) for f in ("cosa_oracle.cpp", "lsp_oracle.inc", "Makefile")]
    srcs.append(os.path.join(_HERE, "..", "include", "cosa_gpu.h"))
    if force or not os.path.exists(_LIB) or any(os.path.getmtime(_LIB) < os.path.getmtime(f) for f in srcs):
        subprocess.run(["make", "-C", _HERE], check=True, stdout=subprocess.DEVNULL)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
        _lib.orc_level_new.restype = C.c_void_p
        _lib.orc_level_new.argtypes = [C.POINTER(_LevelDesc), C.c_int, C.c_int]
        _lib.orc_level_free.argtypes = [C.c_void_p]
        _lib.orc_level_sizes.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _par(p):
    return C.byref(p)


class OracleLevel:
    """One level of the oracle with its own copy of the block tables."""

    def __init__(self, tables, params):
        self.t = tables
        self.p = params
        self._keep = [np.ascontiguousarray(tables.dims.ravel(), dtype=np.int32),
                      np.ascontiguousarray(tables.nbcs, dtype=np.int32),
                      np.ascontiguousarray(tables.bctopo.ravel(), dtype=np.int32),
                      np.ascontiguousarray(tables.cutopo.ravel(), dtype=np.int32)]
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        d = _LevelDesc(tables.nblocks, ip(self._keep[0]), ip(self._keep[1]), ip(self._keep[2]),
                       tables.ncuts, ip(self._keep[3]))
        self.h = C.c_void_p(lib().orc_level_new(C.byref(d), params.npde, params.nharms))
        s = (C.c_int64 * 5)()
        lib().orc_level_sizes(self.h, s)
        self.n3, self.n2, self.n1, self.n0, self.nm1 = list(s)
        self.S = 2 * params.nharms + 1

    def __del__(self):
        try:
            lib().orc_level_free(self.h)
        except Exception:
            pass

    # allocation helpers (zeroed, like cosa_all)
    def p3(self):
        return np.zeros(self.n3 * self.p.npde * self.S)

    def p2(self, ncomp=4):
        return np.zeros(self.n2 * ncomp)

    def p1(self, nsnap=1):
        return np.zeros(self.n1 * nsnap)

    def f0(self):
        return np.zeros(self.n0 * self.p.npde * self.S)

    def metrics(self, x, y, z):
        si, sj, sk = self.p2(), self.p2(), self.p2()
        vol = self.p1()
        lib().orc_imetrix(self.h, _p(x), _p(y), _p(z), _p(si), _p(sj), _p(sk))
        lib().orc_vols(self.h, _p(x), _p(y), _p(z), _p(vol))
        return si, sj, sk, vol

    def cons2prim(self, q, xtnd=0):
        lib().orc_cons2prim(self.h, _par(self.p), C.c_int(xtnd), _p(q))

    def prim2cons(self, q):
        lib().orc_prim2cons(self.h, _par(self.p), _p(q))

    def bc(self, q, si, sj, sk):
        return lib().orc_bc(self.h, _par(self.p), _p(q), _p(si), _p(sj), _p(sk))

    def cutman_q(self, q):
        lib().orc_cutman_q(self.h, _p(q))

    def prtest(self, q):
        return lib().orc_prtest(self.h, _par(self.p), _p(q))

    def lambda_(self, q, si, sj, sk, lam):
        lib().orc_lambda(self.h, _par(self.p), _p(q), _p(si), _p(sj), _p(sk), _p(lam))

    def deltat(self, dtvol, lam, bx=None, by=None, bz=None):
        nul = C.cast(None, _dp)
        lib().orc_deltat(self.h, _par(self.p), _p(dtvol), _p(lam),
                         _p(bx) if bx is not None else nul, _p(by) if by is not None else nul,
                         _p(bz) if bz is not None else nul)

    def muscl(self, idir, nl, q, qp, qm, dq, dqp, dqm):
        lib().orc_muscl(self.h, _par(self.p), C.c_int(idir), C.c_int(nl), _p(q), _p(qp), _p(qm),
                        _p(dq), _p(dqp), _p(dqm))

    def roflux(self, idir, qr, ql, flux, sijk):
        lib().orc_roflux(self.h, _par(self.p), C.c_int(idir), _p(qr), _p(ql), _p(flux), _p(sijk))

    def resid(self, idir, flux, res):
        lib().orc_resid(self.h, C.c_int(idir), _p(flux), _p(res))

    def update(self, res, q, qold, dtvol, ar):
        lib().orc_update(self.h, _p(res), _p(q), _p(qold), _p(dtvol), C.c_double(ar))

    def resg_rms(self, res, rhs):
        out = np.zeros(self.p.npde + 1)
        lib().orc_resg_rms(self.h, _p(res), _p(rhs), _p(out))
        return out

    def zero_res(self, res):
        lib().orc_zero_res(self.h, _p(res))

    def copy_interior(self, dst, src):
        lib().orc_copy_interior(self.h, _p(dst), _p(src))

    def residual(self, q, si, sj, sk, nl=1, want_dt=True, work=None):
        """Stage-1 residual as smooth() computes it; returns (res, dtvol, status).
        q is modified in place exactly as smooth() modifies it."""
        w = work or {k: self.p3() for k in ("res", "qp", "qm", "dq", "dqp", "dqm")}
        flux = self.f0()
        dtvol = self.p1(self.S)
        st = lib().orc_residual(self.h, _par(self.p), C.c_int(nl), _p(q), _p(si), _p(sj), _p(sk),
                                _p(w["res"]), _p(w["qp"]), _p(w["qm"]), _p(w["dq"]), _p(w["dqp"]),
                                _p(w["dqm"]), _p(flux), _p(dtvol), C.c_int(1 if want_dt else 0))
        return w["res"], dtvol, st

    def smooth(self, q, si, sj, sk, ncycles, mgit0=1, rms_every=1):
        """ncycles single-level cycles of smooth(); q updated in place.
        Returns (hist[ncycles, npde+1], status)."""
        qold = self.p3()
        res, rhs = self.p3(), self.p3()
        qp, qm, dq, dqp, dqm = (self.p3() for _ in range(5))
        flux = self.f0()
        dtvol = self.p1(self.S)
        hist = np.full((ncycles, self.p.npde + 1), np.nan)
        st = lib().orc_smooth(self.h, _par(self.p), C.c_int(ncycles), C.c_int(mgit0), C.c_int(rms_every),
                              _p(q), _p(qold), _p(si), _p(sj), _p(sk), _p(res), _p(rhs), _p(qp), _p(qm),
                              _p(dq), _p(dqp), _p(dqm), _p(flux), _p(dtvol), _p(hist))
        return hist, st


def hb_motion(p, S):
    """Snapshot times and pitch angles of harmonic balance."""
    zeit, dth = np.zeros(S), np.zeros(S)
    lib().orc_hb_motion(_par(p), C.c_int(S), _p(zeit), _p(dth))
    return zeit, dth


def moving_setup(O, x0, y0, z0, dx, dy, dz):
    """The moving grid of a pitching harmonic-balance case as the reference's
    set-up builds it (movegrid, imetrix with the face velocities, vols,
    vert2cell_g of the grid velocities), bound to O: returns a dict with the
    per-snapshot node arrays x, y, z, the cell grid velocities cx, cy, cz, the
    face velocities fvi, fvj, fvk, the metrics si, sj, sk and vol."""
    S = O.S
    m = {k: np.zeros(O.n2 * S) for k in ("x", "y", "z", "cx", "cy", "cz")}
    for k in ("fvi", "fvj", "fvk"):
        m[k] = np.zeros(O.n2 * 3 * S)
    lib().orc_set_moving(O.h, C.c_int(1), None, None, None, None, None, None)
    lib().orc_pitch(O.h, _par(O.p), _p(x0), _p(y0), _p(z0), _p(dx), _p(dy), _p(dz), _p(m["x"]), _p(m["y"]),
                    _p(m["z"]), _p(m["cx"]), _p(m["cy"]), _p(m["cz"]))
    lib().orc_face_vel(O.h, _p(m["cx"]), _p(m["cy"]), _p(m["cz"]), _p(m["fvi"]), _p(m["fvj"]), _p(m["fvk"]))
    for k in ("cx", "cy", "cz"):
        lib().orc_vert2cell(O.h, _p(m[k]))
    m["si"], m["sj"], m["sk"] = (np.zeros(O.n2 * 4 * S) for _ in range(3))
    m["vol"] = O.p1()
    lib().orc_imetrix(O.h, _p(m["x"]), _p(m["y"]), _p(m["z"]), _p(m["si"]), _p(m["sj"]), _p(m["sk"]))
    lib().orc_vols(O.h, _p(m["x"]), _p(m["y"]), _p(m["z"]), _p(m["vol"]))
    lib().orc_set_moving(O.h, C.c_int(1), _p(m["fvi"]), _p(m["fvj"]), _p(m["fvk"]), _p(m["cx"]), _p(m["cy"]),
                         _p(m["cz"]))
    O._moving = m  # keeps the arrays the oracle points to alive
    return m


def smooth_irs(O, q, si, sj, sk, ncycles, mgit0=1, rms_every=1):
    """Single-level cycles with implicit residual smoothing (irsop > 0)."""
    qold = O.p3()
    res, rhs = O.p3(), O.p3()
    qp, qm, dq, dqp, dqm = (O.p3() for _ in range(5))
    flux = O.f0()
    dtvol = O.p1(O.S)
    bx, by, bz = (O.p1(O.S) for _ in range(3))
    hist = np.full((ncycles, O.p.npde + 1), np.nan)
    st = lib().orc_smooth_irs(O.h, _par(O.p), C.c_int(ncycles), C.c_int(mgit0), C.c_int(rms_every),
                              _p(q), _p(qold), _p(si), _p(sj), _p(sk), _p(res), _p(rhs), _p(qp), _p(qm),
                              _p(dq), _p(dqp), _p(dqm), _p(flux), _p(dtvol), _p(bx), _p(by), _p(bz), _p(hist))
    return hist, st, dtvol, (bx, by, bz)


def smooth_hb(O, q, si, sj, sk, vol, ncycles, mgit0=1, rms_every=1):
    """Harmonic-balance cycles: explicit (src_hb in the residual, resg_rms_hb)
    or, with params.rkimp, the time-spectral term solved per cell in
    update_bhb and added to the residual norm."""
    qold = O.p3()
    res = O.p3()
    qp, qm, dq, dqp, dqm = (O.p3() for _ in range(5))
    flux = O.f0()
    dtvol = O.p1(O.S)
    hist = np.full((ncycles, O.p.npde + 1), np.nan)
    st = lib().orc_smooth_hb(O.h, _par(O.p), C.c_int(ncycles), C.c_int(mgit0), C.c_int(rms_every),
                             _p(q), _p(qold), _p(si), _p(sj), _p(sk), _p(vol), _p(res), _p(qp), _p(qm),
                             _p(dq), _p(dqp), _p(dqm), _p(flux), _p(dtvol), _p(hist))
    return hist, st


def src_uns(O, q, vol, res):
    lib().orc_src_uns(O.h, _par(O.p), _p(q), _p(vol), _p(res))


def rhs_uns(O, rhs, q1, q2, vol):
    lib().orc_rhs_uns(O.h, _par(O.p), _p(rhs), _p(q1), _p(q2), _p(vol))


def rkuns(O, A, ntime, iprint=1, vm=None):
    """rkuns on one level (LevelArrays with vol; vm for laminar): (hist, status)."""
    hist = np.full((max(ntime, 1), O.p.npde + 1), np.nan)
    pt = A.ptrs()
    st = lib().orc_rkuns(O.h, _par(O.p), C.byref(pt), _opt(vm), C.c_int(ntime), C.c_int(iprint), _p(hist))
    return hist[:ntime], st


def copy_interior(O, dst, src):
    lib().orc_copy_interior(O.h, _p(dst), _p(src))


def src_hb(O, q, vol, res):
    lib().orc_src_hb(O.h, _par(O.p), _p(q), _p(vol), _p(res))


def irs(O, res, dtvol, bx, by, bz):
    lib().orc_irs(O.h, _par(O.p), _p(res), _p(dtvol), _p(bx), _p(by), _p(bz))


def tridi(a, b, c, x):
    x = np.ascontiguousarray(x, dtype=np.float64).copy()
    lib().orc_tridi(_p(np.ascontiguousarray(a, dtype=np.float64)), _p(np.ascontiguousarray(b, dtype=np.float64)),
                    _p(np.ascontiguousarray(c, dtype=np.float64)), _p(x), C.c_int(len(x)))
    return x


def roe_face(params, nrm, qr, ql):
    """roflux_b's face flux; nrm = (kx, ky, kz, ds) or (kx, ky, kz, ds, ubn)
    with the face's normal grid speed ubn."""
    f = np.zeros(5)
    n = np.ascontiguousarray(nrm, dtype=np.float64)
    a = np.ascontiguousarray(qr, dtype=np.float64)
    b = np.ascontiguousarray(ql, dtype=np.float64)
    lib().orc_roe_face(C.byref(params), _p(n), _p(a), _p(b), _p(f), C.c_int(1 if n.size > 4 else 0))
    return f


def num_threads() -> int:
    return int(lib().orc_num_threads())


# ---- multigrid ---------------------------------------------------------------------
def _opt(a):
    return _p(a) if a is not None else C.cast(None, _dp)


def q_edges(O, q, mut=None):
    lib().orc_q_edges(O.h, _p(q), _opt(mut))


def q_corns(O, q, mut=None):
    lib().orc_q_corns(O.h, _p(q), _opt(mut))


def fixq(O, q):
    lib().orc_fixq(O.h, _par(O.p), _p(q))


def tur_vis(O, q, mut):
    lib().orc_tur_vis(O.h, _par(O.p), _p(q), _p(mut))


def add_array(O, v1, v2, fact, off_l):
    lib().orc_add_array(O.h, _p(v1), _p(v2), C.c_double(fact), C.c_int(off_l))


def rest1(Of, Oc, q1, q2, vol1, vol2):
    lib().orc_rest1(Of.h, Oc.h, _p(q1), _p(q2), _p(vol1), _p(vol2))


def rest2(Of, Oc, rhs2, res1):
    lib().orc_rest2(Of.h, Oc.h, _p(rhs2), _p(res1))


def rest2_ho(Of, Oc, rhs2, res1):
    lib().orc_rest2_ho(Of.h, Oc.h, _p(rhs2), _p(res1))


def bc_res(O, res):
    lib().orc_bc_res(O.h, _p(res))


def prol_bln(Of, Oc, q1, q2, lim_corr=0):
    lib().orc_prol_bln(Of.h, Oc.h, _p(q1), _p(q2), C.c_int(lim_corr))


def prol_lin(Of, Oc, q1, q2, vol1):
    lib().orc_prol_lin(Of.h, Oc.h, _p(q1), _p(q2), _p(vol1))


class LevelArrays:
    """The arrays smooth()/restrict()/prolong() touch on one level, zeroed like
    cosa_all; q, si, sj, sk, vol are set by the caller."""

    P3 = ("q", "qold", "res", "rhs", "qp", "qm", "dq", "dqp", "dqm")

    def __init__(self, O):
        self.O = O
        for n in self.P3:
            setattr(self, n, O.p3())
        self.flux = O.f0()
        self.dtvol = O.p1(O.S)
        self.betaxi, self.betaeta, self.betazeta = (O.p1(O.S) for _ in range(3))
        self.si = self.sj = self.sk = self.vol = None

    def ptrs(self):
        p = _LevelPtrs()
        for n in self.P3 + ("flux", "dtvol", "betaxi", "betaeta", "betazeta", "si", "sj", "sk", "vol"):
            a = getattr(self, n)
            if a is not None:
                setattr(p, n, _p(a))
        return p


def restrict(Of, Oc, A1, A2):
    p1, p2 = A1.ptrs(), A2.ptrs()
    return lib().orc_restrict(Of.h, Oc.h, _par(Of.p), C.byref(p1), C.byref(p2))


def prolong(Of, Oc, A1, A2):
    p1, p2 = A1.ptrs(), A2.ptrs()
    return lib().orc_prolong(Of.h, Oc.h, _par(Of.p), C.byref(p1), C.byref(p2))


def smooth_level(O, nl, A, niter, from_fine, to_coarse, mgit=1, ncycle=1, rms_every=1):
    row = np.full(O.p.npde + 1, np.nan)
    pt = A.ptrs()
    st = lib().orc_smooth_level(O.h, _par(O.p), C.c_int(nl), C.byref(pt), C.c_int(niter), C.c_int(int(from_fine)),
                                C.c_int(int(to_coarse)), C.c_int(mgit), C.c_int(ncycle), C.c_int(rms_every),
                                _p(row))
    return row, st


def mg(levels, arrays, mgit0, ncycles, ncycle, rms_every=1):
    """mg() cycles on oracle levels (levels[0] finest) with LevelArrays each."""
    n = len(levels)
    hs = (C.c_void_p * n)(*[O.h.value for O in levels])
    ps = (_LevelPtrs * n)(*[A.ptrs() for A in arrays])
    p = levels[0].p
    hist = np.full((max(ncycles, 1), p.npde + 1), np.nan)
    st = lib().orc_mg(hs, C.c_int(n), _par(p), ps, C.c_int(mgit0), C.c_int(ncycles), C.c_int(ncycle),
                      C.c_int(rms_every), _p(hist))
    return hist[:ncycles], st


# ---- viscous path ------------------------------------------------------------------
def vm_alloc(O):
    """The 9 face inverse-metric arrays (3 x imax x jmax x kmax each) of a level
    in one buffer: array (d, m) at offset ((d-1)*3 + m) * 3 * n0; on a moving
    grid (moving_setup) one such set per snapshot, snapshot nh at nh * 27 n0."""
    return np.zeros(27 * O.n0 * (O.S if getattr(O, "_moving", None) is not None else 1))


def coordex(O, x, y, z):
    lib().orc_coordex(O.h, _p(x), _p(y), _p(z))


def cutman_x(O, x, y, z):
    lib().orc_cutman_x(O.h, _p(x), _p(y), _p(z))


def volex(O, vol):
    lib().orc_volex(O.h, _p(vol))


def cutman_v(O, vol):
    lib().orc_cutman_v(O.h, _p(vol))


def vmetrix(O, x, y, z, vol, vm):
    lib().orc_vmetrix(O.h, _p(x), _p(y), _p(z), _p(vol), _p(vm))


def viscous_setup(O, x, y, z, vol):
    """volex + cutman_v + coordex + cutman_x (x, y, z, vol updated in place)
    and vmetrix; returns vm."""
    vm = vm_alloc(O)
    lib().orc_viscous_setup(O.h, _p(x), _p(y), _p(z), _p(vol), _p(vm))
    return vm


def q_face(O, idir, q, qf):
    lib().orc_q_face(O.h, C.c_int(idir), _p(q), _p(qf))


def q_der(O, idir, q, dqxi, dqeta, dqzeta):
    lib().orc_q_der(O.h, C.c_int(idir), _p(q), _p(dqxi), _p(dqeta), _p(dqzeta))


def vflux(O, idir, qf, dqxi, dqeta, dqzeta, vm, sijk, flux):
    lib().orc_vflux(O.h, _par(O.p), C.c_int(idir), _p(qf), _p(dqxi), _p(dqeta), _p(dqzeta), _p(vm), _p(sijk),
                    _p(flux))


def lambda_ns(O, q, si, sj, sk, vol, lam, lamv, mut=None):
    lib().orc_lambda_ns(O.h, _par(O.p), _p(q), _p(si), _p(sj), _p(sk), _p(vol), _opt(mut), _p(lam), _p(lamv))


def deltat_ns(O, dtvol, lam, lamv, bx=None, by=None, bz=None):
    lib().orc_deltat_ns(O.h, _par(O.p), _p(dtvol), _p(lam), _p(lamv), _opt(bx), _opt(by), _opt(bz))


def residual_ns(O, q, si, sj, sk, vol, vm, nl=1, want_dt=True):
    """Stage-1 viscous residual; returns (res, dtvol, status), q modified in
    place as smooth() modifies it."""
    w = {k: O.p3() for k in ("res", "qp", "qm", "dq", "dqp", "dqm")}
    flux = O.f0()
    dtvol = O.p1(O.S)
    bx, by, bz = (O.p1(O.S) for _ in range(3))
    st = lib().orc_residual_ns(O.h, _par(O.p), C.c_int(nl), _p(q), _p(si), _p(sj), _p(sk), _p(vol), _p(vm),
                               _p(w["res"]), _p(w["qp"]), _p(w["qm"]), _p(w["dq"]), _p(w["dqp"]), _p(w["dqm"]),
                               _p(flux), _p(dtvol), C.c_int(1 if want_dt else 0), _p(bx), _p(by), _p(bz))
    return w["res"], dtvol, st


def smooth_ns(O, q, si, sj, sk, vol, vm, ncycles, mgit0=1, rms_every=1):
    """Single-level viscous cycles; q updated in place.  Returns (hist, status)."""
    qold, res, rhs = O.p3(), O.p3(), O.p3()
    qp, qm, dq, dqp, dqm = (O.p3() for _ in range(5))
    flux = O.f0()
    dtvol = O.p1(O.S)
    bx, by, bz = (O.p1(O.S) for _ in range(3))
    hist = np.full((ncycles, O.p.npde + 1), np.nan)
    st = lib().orc_smooth_ns(O.h, _par(O.p), C.c_int(ncycles), C.c_int(mgit0), C.c_int(rms_every), _p(q),
                             _p(qold), _p(si), _p(sj), _p(sk), _p(vol), _p(vm), _p(res), _p(rhs), _p(qp), _p(qm),
                             _p(dq), _p(dqp), _p(dqm), _p(flux), _p(dtvol), _p(bx), _p(by), _p(bz), _p(hist))
    return hist, st


# ---- k-omega (Wilcox) ------------------------------------------------------------
class RansArrays(LevelArrays):
    """LevelArrays plus what the viscous / k-omega residual reads: mut (P3
    scalar), dist (P1), dtvolt, the turbulence IRS coefficients, production,
    div u, delta+ and the face inverse metrics vm (set by the caller)."""

    def __init__(self, O):
        super().__init__(O)
        n3s = O.n3 * O.S
        self.mut = np.zeros(n3s)
        self.dist = O.p1()
        self.dtvolt = O.p1(O.S)
        self.prd, self.divvel, self.delpls = (np.zeros(n3s) for _ in range(3))
        self.tbx, self.tby, self.tbz = (O.p1(O.S) for _ in range(3))
        self.vm = None
        # BSL/SST: blended coefficients per cell and the face wall distances
        self.ttrm = np.zeros(O.n3 * 3 * O.S)
        self.fdist = np.zeros(3 * O.n0)
        self._O = O

    def ptrs(self):
        p = super().ptrs()
        for n in ("mut", "dist", "dtvolt"):
            setattr(p, n, _p(getattr(self, n)))
        return p

    def extras(self):
        if self._O.p.kom_bsl or self._O.p.kom_sst:
            facedist(self._O, self.dist, self.fdist)
        return (_p(self.vm), _p(self.prd), _p(self.divvel), _p(self.delpls), _p(self.tbx), _p(self.tby), _p(self.tbz),
                _p(self.ttrm), _p(self.fdist))


def smooth_rans(O, A, ncycles, mgit0=1, rms_every=1):
    hist = np.full((ncycles, O.p.npde + 1), np.nan)
    pt = A.ptrs()
    st = lib().orc_smooth_rans(O.h, _par(O.p), C.c_int(ncycles), C.c_int(mgit0), C.c_int(rms_every), C.byref(pt),
                               *A.extras(), _p(hist))
    return hist, st


def residual_rans(O, A, nl=1, want_dt=True):
    pt = A.ptrs()
    return lib().orc_residual_rans(O.h, _par(O.p), C.c_int(nl), C.byref(pt), *A.extras(), C.c_int(int(want_dt)))


def cutman_mut(O, mut):
    lib().orc_cutman_mut(O.h, _p(mut))


def bc_dist(O, q, si, sj, sk, dist):
    return lib().orc_bc_dist(O.h, _par(O.p), _p(q), _p(si), _p(sj), _p(sk), _p(dist))


def q_face_mut(O, idir, mut, flux):
    lib().orc_q_face_mut(O.h, C.c_int(idir), _p(mut), _p(flux))


def rtst(O, idir, qf, dqxi, dqeta, dqzeta, vm, tau1, flux):
    lib().orc_rtst(O.h, _par(O.p), C.c_int(idir), _p(qf), _p(dqxi), _p(dqeta), _p(dqzeta), _p(vm), _p(tau1),
                   _p(flux))


def vflux_kom(O, idir, qf, dqxi, dqeta, dqzeta, tau1, vm, sijk, flux, fdist=None):
    """fdist: the face wall distances of family idir (BSL/SST)."""
    lib().orc_vflux_kom(O.h, _par(O.p), C.c_int(idir), _p(qf), _p(dqxi), _p(dqeta), _p(dqzeta), _p(tau1), _p(vm),
                        _p(sijk), _p(flux), _opt(fdist))


def q_der_c(O, idir, qf, dqc):
    lib().orc_q_der_c(O.h, _par(O.p), C.c_int(idir), _p(qf), _p(dqc))


def facedist(O, dist, fdist):
    """facedist_b: the three face-distance arrays (F0 each) into fdist (3 n0)."""
    lib().orc_facedist(O.h, _p(dist), _p(fdist))


def update_ttrm(O, q, dqxi, dqeta, dqzeta, vm, ttrm, dist):
    lib().orc_update_ttrm(O.h, _par(O.p), _p(q), _p(dqxi), _p(dqeta), _p(dqzeta), _p(vm), _p(ttrm), _p(dist))


def srckw_sst(O, nl, q, mut, prd, divvel, res, ttrm, vol):
    lib().orc_srckw_sst(O.h, _par(O.p), C.c_int(nl), _p(q), _p(mut), _p(prd), _p(divvel), _p(res), _p(ttrm), _p(vol))


def tur_vis_sst(O, q, mut, dqxi, dqeta, dqzeta, vm, dist):
    lib().orc_tur_vis_sst(O.h, _par(O.p), _p(q), _p(mut), _p(dqxi), _p(dqeta), _p(dqzeta), _p(vm), _p(dist))


def turprod(O, q, dqxi, dqeta, dqzeta, vm, prd, divvel, delpls):
    lib().orc_turprod(O.h, _par(O.p), _p(q), _p(dqxi), _p(dqeta), _p(dqzeta), _p(vm), _p(prd), _p(divvel),
                      _p(delpls))


def srckw(O, nl, q, mut, prd, divvel, res, vol):
    lib().orc_srckw(O.h, _par(O.p), C.c_int(nl), _p(q), _p(mut), _p(prd), _p(divvel), _p(res), _p(vol))


def update_kom(O, res, q, qold, vol, dtvolt, delpls, prd, ar, ttrm=None):
    lib().orc_update_kom(O.h, _par(O.p), _p(res), _p(q), _p(qold), _p(vol), _p(dtvolt), _p(delpls), _p(prd),
                         C.c_double(ar), _opt(ttrm))


def deltat_ns_full(O, dtvol, lam, lamv, bx, by, bz, dtvolt, tbx, tby, tbz):
    lib().orc_deltat_ns_full(O.h, _par(O.p), _p(dtvol), _p(lam), _p(lamv), _opt(bx), _opt(by), _opt(bz),
                             _opt(dtvolt), _opt(tbx), _opt(tby), _opt(tbz))


FORCE_NAMES = ("cl_p", "cd_p", "cz_p", "cmx_p", "cmy_p", "cm_p",
               "cl_v", "cd_v", "cz_v", "cmx_v", "cmy_v", "cm_v")


def force(O, q, x, y, z, si, sj, sk, vm, isurf=1, xmom=(0.25, 0.0, 0.0), lngth=(1.0, 1.0, 1.0)):
    """force_b summed over blocks (src/output.f90:4283-4900): (S, 12) force
    and moment coefficients of wall surface isurf, columns FORCE_NAMES."""
    out = np.zeros(O.S * 12)
    xm = np.ascontiguousarray(xmom, dtype=np.float64)
    ln = np.ascontiguousarray(lngth, dtype=np.float64)
    lib().orc_force(O.h, _par(O.p), _p(q), _p(x), _p(y), _p(z), _p(si), _p(sj), _p(sk), _opt(vm),
                    C.c_int(isurf), _p(xm), _p(ln), _p(out))
    return out.reshape(O.S, 12)


# ---- k-omega multigrid ---------------------------------------------------------------
class _VExtra(C.Structure):
    _fields_ = [(n, _dp) for n in ("vm", "prd", "divvel", "delpls", "tbx", "tby", "tbz", "ttrm", "fdist")]


def _vextra(A):
    return _VExtra(*A.extras())


def rest4(Of, Oc, f1, f2, vol1, vol2):
    lib().orc_rest4(Of.h, Oc.h, _p(f1), _p(f2), _p(vol1), _p(vol2))


def lim_prod_mg(O, q, prd, mut):
    lib().orc_lim_prod_mg(O.h, _par(O.p), _p(q), _p(prd), _p(mut))


def lim_res_ome(O, res, q, vol, dtvolt, delpls, prd, ar):
    lib().orc_lim_res_ome(O.h, _par(O.p), _p(res), _p(q), _p(vol), _p(dtvolt), _p(delpls), _p(prd), C.c_double(ar))


def smooth_level_rans(O, nl, nlevel, A, niter, from_fine, to_coarse, mgit=1, ncycle=1, rms_every=1):
    row = np.full(O.p.npde + 1, np.nan)
    pt, ex = A.ptrs(), _vextra(A)
    st = lib().orc_smooth_level_rans(O.h, _par(O.p), C.c_int(nl), C.c_int(nlevel), C.byref(pt), C.byref(ex),
                                     C.c_int(niter), C.c_int(int(from_fine)), C.c_int(int(to_coarse)), C.c_int(mgit),
                                     C.c_int(ncycle), C.c_int(rms_every), _p(row))
    return row, st


def restrict_rans(Of, Oc, A1, A2):
    p1, p2, e1, e2 = A1.ptrs(), A2.ptrs(), _vextra(A1), _vextra(A2)
    return lib().orc_restrict_rans(Of.h, Oc.h, _par(Of.p), C.byref(p1), C.byref(p2), C.byref(e1), C.byref(e2))


def mg_rans(levels, arrays, mgit0, ncycles, ncycle, rms_every=1):
    """mg() cycles of the k-omega path on oracle levels (levels[0] finest)
    with RansArrays each."""
    n = len(levels)
    hs = (C.c_void_p * n)(*[O.h.value for O in levels])
    ps = (_LevelPtrs * n)(*[A.ptrs() for A in arrays])
    es = (_VExtra * n)(*[_vextra(A) for A in arrays])
    p = levels[0].p
    hist = np.full((max(ncycles, 1), p.npde + 1), np.nan)
    st = lib().orc_mg_rans(hs, C.c_int(n), _par(p), ps, es, C.c_int(mgit0), C.c_int(ncycles), C.c_int(ncycle),
                           C.c_int(rms_every), _p(hist))
    return hist[:ncycles], st


def lu_solve(a, b):
    """x with a x = b (partial-pivot LU in DGETF2/DGETRS order); a (n, n),
    b (n,) or (n, nrhs)."""
    n = a.shape[0]
    af = np.asfortranarray(a, dtype=np.float64).ravel(order="F").copy()
    bb = np.asarray(b, dtype=np.float64)
    nrhs = 1 if bb.ndim == 1 else bb.shape[1]
    bf = bb.reshape(n, nrhs).ravel(order="F").copy()
    lib().orc_lu_solve(C.c_int(n), _p(af), _p(bf), C.c_int(nrhs))
    x = bf.reshape((n, nrhs), order="F")
    return x[:, 0] if bb.ndim == 1 else x


# ---- low-speed preconditioning (src/losp.f90, src/flux.f90:390-830) ----------
def m1(O):
    """An interior-cell array x S (cutoff_pgr / cutoff_vis layout)."""
    return np.zeros(O.nm1 * O.S)


def lm_cutoff_pg(O, q, cut):
    lib().orc_lm_cutoff_pg(O.h, _par(O.p), _p(q), _p(cut))


def lm_viscoff(O, q, si, sj, sk, cut):
    lib().orc_lm_viscoff(O.h, _par(O.p), _p(q), _p(si), _p(sj), _p(sk), _p(cut))


def proflux(O, idir, nl, qr, ql, flux, sijk, cpg, cvs):
    lib().orc_proflux(O.h, _par(O.p), C.c_int(idir), C.c_int(nl), _p(qr), _p(ql), _p(flux), _p(sijk), _p(cpg),
                      _p(cvs))


def lambda_p(O, nl, q, si, sj, sk, lam, cpg, cvs, vol=None, lamv=None):
    lib().orc_lambda_p(O.h, _par(O.p), C.c_int(nl), _p(q), _p(si), _p(sj), _p(sk), _opt(vol), _p(lam), _opt(lamv),
                       _p(cpg), _p(cvs))


def lsp_prec(O, nl, q, cpg, cvs):
    """blsp's preconditioner of every interior cell of the conservative q,
    (imax-1, jmax-1, kmax-1, npde, npde, S) per block."""
    prec = np.zeros(O.nm1 * O.p.npde * O.p.npde * O.S)
    lib().orc_lsp_prec(O.h, _par(O.p), C.c_int(nl), _p(q), _p(cpg), _p(cvs), _p(prec))
    return prec


def precres(O, res, prec):
    lib().orc_precres(O.h, _p(res), _p(prec))


def rest3(Of, Oc, c1, c2, vol1, vol2):
    lib().orc_rest3(Of.h, Oc.h, _p(c1), _p(c2), _p(vol1), _p(vol2))


def get_cutoffs(O):
    """The level's own pressure-gradient and viscous cut-offs."""
    pgr, vis = m1(O), m1(O)
    lib().orc_get_cutoffs(O.h, _p(pgr), _p(vis))
    return pgr, vis


def set_cutoffs(O, pgr, vis):
    lib().orc_set_cutoffs(O.h, _p(pgr), _p(vis))
