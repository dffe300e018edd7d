"""cosa_params: the module globals of COSA's hot path as a ctypes struct.

Mirrors ``struct cosa_params`` in ``include/cosa_gpu.h`` field for field.
Defaults follow ``input()`` (src/input.f90:2400-2540): RK coefficients
``ar4 = (0.25, 0.333333, 0.5, 1.0)`` (the literal 0.333333, read as FP64
because every build uses -fdefault-real-8), k-omega constants, qmin, and the
boundary values the reference hard-wires in bc_insub / bc_outsub
(src/bc.f90:996-1000, 1310-1312).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

MAX_SNAP = 15
MAX_LEVELS = 3

PREC_FP64 = 0
PREC_MIXED = 1


class CosaParams(C.Structure):
    _fields_ = [
        ("gamma", C.c_double), ("machfs", C.c_double), ("alpha", C.c_double),
        ("beta", C.c_double), ("reyno", C.c_double), ("pranl", C.c_double),
        ("prant", C.c_double), ("stemp", C.c_double),
        ("pinf", C.c_double), ("rhoinf", C.c_double), ("ainf", C.c_double),
        ("tinf", C.c_double),
        ("rkap", C.c_double), ("epslimf", C.c_double), ("epslimt", C.c_double),
        ("ilimf", C.c_int32), ("ilimt", C.c_int32),
        ("nl_crs", C.c_int32), ("foturb", C.c_int32),
        ("efx_setup_f", C.c_int32), ("efx_all_f", C.c_int32),
        ("eig_limit_f", C.c_int32), ("eig_lim_all_f", C.c_int32),
        ("efx_setup_t", C.c_int32), ("efx_all_t", C.c_int32),
        ("eig_limit_t", C.c_int32), ("eig_lim_all_t", C.c_int32),
        ("entfx_f_w", C.c_int32 * 3), ("entfx_t_w", C.c_int32 * 3),
        ("cntrpy_f", C.c_double), ("entfxctf_f", C.c_double), ("eig_cutoff_f", C.c_double),
        ("cntrpy_t", C.c_double), ("entfxctf_t", C.c_double), ("eig_cutoff_t", C.c_double),
        ("cfl", C.c_double), ("cflt", C.c_double), ("cdff", C.c_double),
        ("rat", C.c_double), ("ratt", C.c_double), ("psirs", C.c_double),
        ("irsop", C.c_int32), ("cutcirs", C.c_int32), ("iupdt", C.c_int32),
        ("nstage", C.c_int32),
        ("alphas", C.c_double * 5),
        ("npde", C.c_int32), ("nharms", C.c_int32), ("hbmove", C.c_int32),
        ("lmet", C.c_int32),
        ("viscous", C.c_int32), ("kom", C.c_int32), ("kom_bsl", C.c_int32),
        ("kom_sst", C.c_int32), ("harbal", C.c_int32), ("rkimp", C.c_int32),
        ("moving", C.c_int32),
        ("aircraft", C.c_int32), ("rgkuns", C.c_int32), ("dualt", C.c_int32),
        ("nlevel", C.c_int32),
        ("qmin", C.c_double * 7),
        ("tkefar", C.c_double), ("omefar", C.c_double), ("mutfar", C.c_double),
        ("cmu", C.c_double), ("bstrkw", C.c_double), ("gkw", C.c_double),
        ("bkw", C.c_double), ("sigk", C.c_double), ("sigw", C.c_double),
        ("epst", C.c_double), ("kappa", C.c_double),
        ("inlet_t0", C.c_double), ("inlet_p0", C.c_double), ("inlet_dir", C.c_double * 3),
        ("outlet_p", C.c_double * 3),
        ("omega", C.c_double),
        ("dhb", C.c_double * (MAX_SNAP * MAX_SNAP)),
        ("precision", C.c_int32),
        ("nstart", C.c_int32), ("npre", C.c_int32), ("npost", C.c_int32), ("ncrs", C.c_int32),
        ("bln_prol", C.c_int32), ("lim_corr", C.c_int32),
        ("lim_prodtke", C.c_int32), ("lim_prodomega", C.c_int32), ("prd_all_lvls", C.c_int32),
        ("ifixq", C.c_int32), ("wallwilc", C.c_int32), ("ho_rest", C.c_int32),
        ("turcmp", C.c_double), ("prdlim", C.c_double), ("roughk", C.c_double),
        ("dtheta0", C.c_double), ("omegas", C.c_double), ("xh", C.c_double), ("yh", C.c_double),
        ("dt", C.c_double), ("bdf1", C.c_int32), ("reserved_t", C.c_int32),
        ("lomach", C.c_int32), ("cutoff_type", C.c_int32), ("visprec", C.c_int32), ("mixpi", C.c_int32),
        ("uprv", C.c_double), ("epsp", C.c_double * MAX_LEVELS),
    ]


def default_params() -> CosaParams:
    """A CosaParams holding input()'s defaults (src/input.f90:2400-2540)."""
    p = CosaParams()
    p.gamma = 1.4
    p.pranl = 0.72
    p.prant = 0.9
    p.stemp = 110.4 / 288.15
    p.rhoinf = 1.0
    p.ainf = 1.0
    p.tinf = 1.0
    p.pinf = 1.0 / p.gamma
    p.rkap = 1.0 / 3.0
    p.epslimf = 1.0e-6
    p.epslimt = 1.0e-6
    p.ilimf = 1
    p.ilimt = 1
    p.nl_crs = 99
    p.cfl = 2.0
    p.cflt = 2.0
    p.cdff = 1.0
    p.rat = 1.0
    p.ratt = 1.0
    p.iupdt = 1
    p.nstage = 4
    for i, a in enumerate((0.25, 0.333333, 0.5, 1.0, 0.0)):
        p.alphas[i] = a
    p.npde = 5
    p.lmet = 4
    p.aircraft = 1
    p.nlevel = 1
    for i, v in enumerate((1.0e-8, 1.0, 1.0, 1.0, 1.0e-8, 1.0e-12, 1.0e-8)):
        p.qmin[i] = v
    # k-omega (src/input.f90:2513-2521)
    p.epst = 1.0e-12
    p.kappa = 0.41
    p.cmu = 1.0
    p.sigk = 0.5
    p.sigw = 0.5
    p.bkw = 3.0 / 40.0
    p.bstrkw = 0.09
    p.gkw = p.bkw / p.bstrkw - p.sigw * p.kappa ** 2 / math.sqrt(p.bstrkw)
    # reference hard-wired inlet / outlet values (src/bc.f90:996-1000, 1310-1312)
    p.inlet_t0 = 1.008
    p.inlet_p0 = 0.734486515085076
    p.inlet_dir[0] = 1.0
    p.inlet_dir[1] = 0.0
    p.inlet_dir[2] = 0.0
    for i in range(3):
        p.outlet_p[i] = 0.714285714285714
    p.precision = PREC_FP64
    # multigrid: one smoothing iteration per visit, bilinear prolongation
    p.nstart = p.npre = p.npost = p.ncrs = 1
    p.bln_prol = 1
    p.lim_corr = 0
    # time-accurate runs start with a first-order step (src/src.f90:420-432)
    p.bdf1 = 1
    # low-speed preconditioning off; cut-off type 1 (none) when switched on
    p.cutoff_type = 1
    return p


def set_low_speed(p: CosaParams, cutoff_type: int = 2, visprec: bool = False, epsp=(1.0e-5, 1.0e-5, 1.0e-5),
                  mixpi: int = 0, uprv: float = 0.0) -> CosaParams:
    """Switch on low-speed preconditioning (the input file's `lomach`
    line and its constant cut-offs per level, src/input.f90:3585-3700)."""
    p.lomach = 1
    p.cutoff_type = cutoff_type
    p.visprec = 1 if visprec else 0
    p.mixpi = mixpi
    p.uprv = uprv
    for i in range(MAX_LEVELS):
        p.epsp[i] = epsp[min(i, len(epsp) - 1)]
    return p


def subsonic_inlet_total_state(gamma: float, mach: float):
    """T0 and p0 of the subsonic inlet for a free stream at `mach` with the
    non-dimensionalisation rho=1, p=1/gamma, a=1 (T = gamma p / rho = a^2)."""
    t0 = 1.0 + 0.5 * (gamma - 1.0) * mach * mach
    p0 = (1.0 / gamma) * t0 ** (gamma / (gamma - 1.0))
    return t0, p0


def hb_matrix(nharms: int, omega: float) -> np.ndarray:
    """Time-spectral operator D = E^-1 A E of mathb (src/input.f90:5206-5284)
    on the 2*nharms+1 equispaced instants zeit(n) = n * 2 pi / omega / S
    (src/input.f90:3180-3193); D @ u(t_n) is d/dt u at the instants for
    every Fourier mode up to nharms."""
    S = 2 * nharms + 1
    dt = 2 * math.pi / omega / S
    zeit = [n * dt for n in range(S)]
    ahb = np.zeros((S, S)); eihb = np.zeros((S, S)); ehb = np.zeros((S, S))
    for i in range(1, nharms + 1):
        ahb[2 * (i - 1) + 1, 2 * (i - 1) + 2] = i
        ahb[2 * (i - 1) + 2, 2 * (i - 1) + 1] = -i
    for i in range(S):
        eihb[i, 0] = 1.0
    for j in range(1, nharms + 1):
        for i in range(S):
            eihb[i, 2 * (j - 1) + 1] = math.cos(j * omega * zeit[i])
            eihb[i, 2 * (j - 1) + 2] = math.sin(j * omega * zeit[i])
    fact = 2.0 / S
    for j in range(S):
        ehb[0, j] = fact / 2
    for i in range(1, nharms + 1):
        for j in range(S):
            ehb[2 * (i - 1) + 1, j] = fact * math.cos(i * omega * zeit[j])
            ehb[2 * (i - 1) + 2, j] = fact * math.sin(i * omega * zeit[j])
    # the reference accumulates the two products with explicit k loops
    t = np.zeros((S, S))
    for i in range(S):
        for j in range(S):
            acc = 0.0
            for k in range(S):
                acc = acc + ahb[i, k] * ehb[k, j]
            t[i, j] = acc
    d = np.zeros((S, S))
    for i in range(S):
        for j in range(S):
            acc = 0.0
            for k in range(S):
                acc = acc + eihb[i, k] * t[k, j]
            d[i, j] = acc
    return d


def set_harmonic_balance(p: CosaParams, nharms: int, omega: float) -> CosaParams:
    """Switch p to harmonic balance with nharms harmonics at frequency omega
    (rad per unit time): S = 2 nharms + 1 snapshots and D in p.dhb."""
    p.harbal = 1
    p.nharms = nharms
    p.omega = omega
    d = hb_matrix(nharms, omega)
    S = 2 * nharms + 1
    for i in range(S):
        for j in range(S):
            p.dhb[i * S + j] = d[i, j]
    return p


def hb_harmonics(values, nharms: int, omega: float) -> np.ndarray:
    """Fourier coefficients of a periodic quantity from its S = 2 nharms + 1
    snapshot values through the matrix E of mathb (src/input.f90:5240-5251):
    [a0, a1, b1, a2, b2, ...] with v(t) = a0 + sum a_i cos(i omega t) +
    b_i sin(i omega t)."""
    S = 2 * nharms + 1
    dt = 2 * math.pi / omega / S
    zeit = [n * dt for n in range(S)]
    fact = 2.0 / S
    e = np.zeros((S, S))
    e[0, :] = fact / 2
    for i in range(1, nharms + 1):
        for j in range(S):
            e[2 * (i - 1) + 1, j] = fact * math.cos(i * omega * zeit[j])
            e[2 * (i - 1) + 2, j] = fact * math.sin(i * omega * zeit[j])
    return e @ np.asarray(values, dtype=np.float64)


def set_pitching(p: CosaParams, nharms: int, amp_deg: float, kred: float, xh: float = 0.25,
                 yh: float = 0.0) -> CosaParams:
    """Harmonic balance of a rigid pitching motion theta(t) = amp sin(omega t)
    about (xh, yh): reduced frequency kred = omega c / (2 U) with chord 1 and
    U = machfs (a_inf = 1), so omega = 2 kred machfs; every snapshot has its
    own grid and metrics (moving = hbmove = 1)."""
    omega = 2.0 * kred * p.machfs
    set_harmonic_balance(p, nharms, omega)
    p.moving = 1
    p.hbmove = 1
    p.omegas = omega
    p.dtheta0 = math.radians(amp_deg)
    p.xh = xh
    p.yh = yh
    return p


def params_bytes(p: CosaParams) -> bytes:
    return bytes(memoryview(p))


def cfl_ramp(mgit: int, mode: int, ncycr, vcfli, vcflit, current=None):
    """(cfl, cflt) of cycle mgit under the k-omega CFL ramps of bdeltat
    (src/cosa.f90:4763-4815).  mode 1: cubic then linear growth, re-evaluated
    on cycle 1 and every 100th cycle (in between the previous value, passed
    as `current`, holds); mode 2: constant, linear, constant, linear, every
    cycle.  ncycr = (n0, n1, n2, n3), vcfli/vcflit = the three CFL levels of
    the mean-flow and turbulence equations."""
    n0, n1, n2, n3 = ncycr
    if mode == 1:
        if not (mgit == 1 or mgit % 100 == 0):
            return current
        s3 = 3.0 ** 0.5
        d1, d2 = (vcfli[1] - vcfli[0]) * s3 ** 3, vcfli[2] - vcfli[1]
        t1, t2 = (vcflit[1] - vcflit[0]) * s3 ** 3, vcflit[2] - vcflit[1]
        if mgit <= n1:
            return vcfli[0], vcflit[0]
        if mgit <= n2:
            f = (float(mgit - n1) / (n2 - n1) / s3) ** 3
            return vcfli[0] + d1 * f, vcflit[0] + t1 * f
        if mgit <= n3:
            f = float(mgit - n2) / (n3 - n2)
            return vcfli[1] + d2 * f, vcflit[1] + t2 * f
        return vcfli[2], vcflit[2]
    d1, d2 = vcfli[1] - vcfli[0], vcfli[2] - vcfli[1]
    t1, t2 = vcflit[1] - vcflit[0], vcflit[2] - vcflit[1]
    if mgit <= n0:
        return vcfli[0], vcflit[0]
    if mgit <= n1:
        f = float(mgit - n0) / (n1 - n0)
        return vcfli[0] + d1 * f, vcflit[0] + t1 * f
    if mgit <= n2:
        return vcfli[1], vcflit[1]
    if mgit <= n3:
        f = float(mgit - n2) / (n3 - n2)
        return vcfli[1] + d2 * f, vcflit[1] + t2 * f
    return vcfli[2], vcflit[2]
