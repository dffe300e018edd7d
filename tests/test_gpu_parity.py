"""Parity of the sm_100a path (through the C-ABI) with the CPU oracle.

Tolerance (FP64 path): the GPU build contracts multiply-adds (FMA) where the
oracle keeps the Fortran operation order, so results differ by rounding only.
Per-cell errors are measured relative to the magnitude of the terms being
combined: for fluxes and residuals, relative to the largest face flux of the
same equation (a residual is a sum of face fluxes); for states, relative to
the largest value of the same variable.  The bar is 1e-12.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p3_views
from cosa_b200.params import PREC_MIXED

import casekit

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _setup(case, oracle_mod, seed=3, perturb=True):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = cases.perturbed_state(case, seed=seed) if perturb else case.q0.copy()
    ctx = gpu.Context([case.tables], case.params)
    return O, ctx, (si, sj, sk, vol), q


def _rel(a, b, case, nvar=5, scale=None):
    """max |a-b| over interior cells, relative to the largest value of each
    variable; the three momentum components share the momentum scale (the
    largest of the three), so a component that is small everywhere (rho w
    of a quasi-2D flow) is not measured against its own tiny values."""
    A = casekit.interior_cells(case, a, nvar)
    B = casekit.interior_cells(case, b, nvar)
    if scale is None:
        scale = np.abs(B).reshape(-1, nvar).max(axis=0) + 1e-300
        scale[1:4] = scale[1:4].max()
    return float((np.abs(A - B) / scale[None, :, None]).max())


def _flux_scale(flux, case):
    nvar = 5
    F = flux.reshape(nvar, -1)  # one block of F0 is (i,j,k,v): use per-variable max over all
    return np.array([np.abs(f).max() for f in F]) + 1e-300


@pytest.mark.parametrize("which", ["channel", "partitioned", "naca_far1"])
def test_routines_match_oracle(oracle_mod, which):
    """Each level driver against the oracle routine it replaces, chained as
    smooth() chains them for one stage (src/cosa.f90:1721-2000)."""
    case = {"channel": casekit.small_channel, "partitioned": casekit.small_partitioned,
            "naca_far1": lambda: _naca_euler(31)}[which]()
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod)
    d = {k: ctx.alloc_p2().upload(v) for k, v in (("si", si), ("sj", sj), ("sk", sk))}
    dq_ = ctx.alloc_p3().upload(q)
    qh = q.copy()
    # cons2prim
    O.cons2prim(qh)
    ctx.cons2prim(1, dq_)
    assert _rel(dq_.download(), qh, case) <= TOL
    # bc + cutman_q (+ prtest): full arrays, halos included
    O.bc(qh, si, sj, sk)
    O.cutman_q(qh)
    ctx.bc(1, dq_, d["si"], d["sj"], d["sk"])
    ctx.cutman_q(1, dq_)
    assert ctx.prtest(1, dq_) == 0 and O.prtest(qh) == 0
    g = dq_.download()
    for vg, vo in zip(p3_views(case.tables, g, 5, 1), p3_views(case.tables, qh, 5, 1)):
        sc = np.abs(vo).reshape(-1, 5).max(axis=0)
        assert (np.abs(vg - vo) / sc[None, None, None, :, None]).max() <= TOL
    # lambda + deltat
    lam_o, lam_g = O.p3(), ctx.alloc_p3()
    O.lambda_(qh, si, sj, sk, lam_o)
    ctx.lambda_(1, dq_, d["si"], d["sj"], d["sk"], None, lam_g)
    dt_o, dt_g = O.p1(), ctx.alloc_p1()
    O.deltat(dt_o, lam_o)
    ctx.deltat(1, dt_g, lam_g)
    np.testing.assert_allclose(dt_g.download(), dt_o, rtol=TOL, atol=0)
    # muscl + roflux + resid in the three directions
    res_o, res_g = O.p3(), ctx.alloc_p3()
    O.zero_res(res_o)
    ctx.zero(1, res_g)
    fscale = np.zeros(5)
    for idir, s_o, s_g in ((1, si, d["si"]), (2, sj, d["sj"]), (3, sk, d["sk"])):
        bufs_o = [O.p3() for _ in range(5)]
        bufs_g = [ctx.alloc_p3() for _ in range(5)]
        O.muscl(idir, 1, qh, *bufs_o)
        ctx.muscl(idir, 1, dq_, *bufs_g)
        for k in (0, 1):  # qp, qm on the faces
            a, b = bufs_g[k].download(), bufs_o[k]
            sc = np.abs(b).max()
            # compare the face entries the reference writes (interior of the face range)
            for vg, vo in zip(p3_views(case.tables, a, 5, 1), p3_views(case.tables, b, 5, 1)):
                sl = [slice(2, -2)] * 3
                sl[idir - 1] = slice(2, -1)
                assert (np.abs(vg[tuple(sl)] - vo[tuple(sl)])).max() <= TOL * sc
        fo, fg = O.f0(), ctx.alloc_f0()
        O.roflux(idir, bufs_o[0], bufs_o[1], fo, s_o)
        ctx.roflux(idir, 1, bufs_g[0], bufs_g[1], fg, s_g)
        fgh = fg.download()
        sc = np.abs(fo).max()
        assert np.abs(fgh - fo).max() <= TOL * sc
        fscale = np.maximum(fscale, sc)
        O.resid(idir, fo, res_o)
        ctx.resid(idir, 1, fg, res_g)
    assert _rel(res_g.download(), res_o, case, scale=fscale) <= TOL
    rms_o = O.resg_rms(res_o, O.p3())
    rms_g = ctx.resg_rms(1, res_g)
    np.testing.assert_allclose(rms_g, rms_o, rtol=1e-9)
    # prim2cons + update
    O.prim2cons(qh)
    ctx.prim2cons(1, dq_)
    qold_o = q.copy()
    qold_g = ctx.alloc_p3().upload(q)
    O.update(res_o, qh, qold_o, dt_o, 0.25)
    ctx.update(1, res_g, dq_, qold_g, dt_g, 0.25)
    assert _rel(dq_.download(), qh, case) <= TOL
    ctx.close()


def _naca_euler(far):
    p = cases.naca_params("euler", mach=0.5, alpha_deg=3.0, eps_irs=0.0)
    p.cfl = 2.0
    return cases.naca0012_ogrid(blocks=(12, 20, 20, 12), nj=12, nk=2, rfar=10.0, h1=5e-3, params=p, wall=14, far=far)


FUSED_CASES = {
    "channel": lambda: casekit.small_channel(),
    # extrapolated z faces and 5 k-planes: planes k0-2 and k0+2 differ, which
    # a missing barrier between the first k-face and the ring refill exposes
    "channel_extrap_nk5": lambda: cases.bump_channel(40, 20, 5, kface_bc=4),
    "jsplit_10_14": lambda: cases.partitioned_channel(48, 24, 2, isplit=(), jsplit=(10,), permute_last=False),
    "partitioned": lambda: casekit.small_partitioned(),
    "duct": lambda: casekit.small_duct(),
    # Euler NACA O-grid: seam cut, slip wall, far field 30 (bc_far0) or 31 (bc_far1)
    "naca_far0": lambda: _naca_euler(30),
    "naca_far1": lambda: _naca_euler(31),
}


@pytest.mark.parametrize("which", list(FUSED_CASES))
def test_fused_smooth_matches_oracle(oracle_mod, which):
    """cosa_gpu_smooth (fused halo + tile kernels in a CUDA graph) against the
    oracle's smooth() for several RK cycles: state, q^n copy, time step and
    the residual history."""
    case = FUSED_CASES[which]()
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=11)
    ncyc = 6
    qo = q.copy()
    hist_o, st_o = O.smooth(qo, si, sj, sk, ncyc, rms_every=2)
    assert st_o == 0
    dq_ = ctx.alloc_p3().upload(q)
    qold = ctx.alloc_p3()
    dtv = ctx.alloc_p1(nsnap=1)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    ctx.bind_level(1, q=dq_, qold=qold, dtvol=dtv, si=m[0], sj=m[1], sk=m[2])
    hist_g, st = ctx.smooth(1, ncyc, 1, 2)
    assert st == 0
    err = _rel(dq_.download(), qo, case)
    assert err <= TOL, err
    rows = ~np.isnan(hist_o[:, 0])
    assert np.array_equal(rows, ~np.isnan(hist_g[:, 0]))
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)
    ctx.close()


def test_smooth_host_buffers_equal_device_path(oracle_mod):
    """cosa_gpu_smooth_host (state copied in and out each call) gives the
    device-resident result."""
    case = casekit.small_partitioned()
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=2)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    dq_ = ctx.alloc_p3().upload(q)
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    ctx.smooth(1, 3, 1, 1)
    a = dq_.download()
    qh = q.copy()
    _, st = ctx.smooth_host(1, qh, 3, 1, 1)
    assert st == 0
    assert np.array_equal(casekit.interior_cells(case, a, 5), casekit.interior_cells(case, qh, 5))
    ctx.close()


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("ilimf", [1, 2, 3, 4])
def test_mixed_precision_close_to_fp64(oracle_mod, schedule, ilimf):
    """Mixed precision (FP32 limiter and Roe flux on FP64 differences; in the
    face-split schedule also the FP32 change of the central flux from the
    left cell's FP64 flux): after 20 cycles the state stays within 1e-6
    (relative) of the FP64 path, for both schedules; the other limiters,
    less dissipative on this perturbed state, over 4 cycles."""
    case = casekit.small_partitioned()
    case.params.ilimf = ilimf
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=4)
    p = case.params
    p.precision = PREC_MIXED
    ctx2 = gpu.Context([case.tables], p)
    out = []
    for c in (ctx, ctx2):
        m = [c.alloc_p2().upload(a) for a in (si, sj, sk)]
        dq_ = c.alloc_p3().upload(q)
        c.bind_level(1, q=dq_, qold=c.alloc_p3(), dtvol=c.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
        c.set_schedule(1, schedule)
        ncyc = 20 if ilimf == 1 else 4
        _, st = c.smooth(1, ncyc, 1, ncyc)
        assert st == 0
        out.append(dq_.download())
    err = _rel(out[1], out[0], case)
    assert 0 < err < 1e-6, err
    ctx.close(); ctx2.close()


@pytest.mark.parametrize("schedule", [0, 1])
def test_negative_pressure_sets_status_not_fault(oracle_mod, schedule):
    """A state with a non-physical pressure is reported through the status
    word (src/cosa.f90:1000-1040 stops there); the context stays usable.
    Both stage schedules test positivity where they convert the state."""
    case = casekit.small_channel(16, 8, 2)
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, perturb=False)
    v = p3_views(case.tables, q, 5, 1)[0]
    v[6, 4, 2, 4, 0] = -5.0  # rho*E far below the kinetic energy -> p < 0
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    dq_ = ctx.alloc_p3().upload(q)
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    ctx.set_schedule(1, schedule)
    _, st = ctx.smooth(1, 1, 1, 1)
    assert st & 0x1
    ctx.status(reset=True)
    dq_.upload(case.q0)
    _, st = ctx.smooth(1, 1, 1, 1)
    assert st == 0
    ctx.close()


@pytest.mark.parametrize("which", ["channel", "duct"])
def test_device_metrics_match_oracle(oracle_mod, which):
    """imetrix / vols on the device against the oracle's restatement of
    src/grid.f90 (the host precompute the GPU path replaces)."""
    case = casekit.small_channel() if which == "channel" else casekit.small_duct()
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    ctx = gpu.Context([case.tables], case.params)
    X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
    gs = [ctx.alloc_p2() for _ in range(3)]
    gv = ctx.alloc_p1()
    ctx.imetrix(1, X, Y, Z, *gs)
    ctx.vols(1, X, Y, Z, gv)
    for g, o in zip(gs, (si, sj, sk)):
        np.testing.assert_allclose(g.download(), o, rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(gv.download(), vol, rtol=1e-12, atol=1e-18)
    ctx.close()


def _irs_case(irsop, cutcirs, long_lines=False):
    # long_lines: 800-cell i-lines, above the cyclic-reduction limit (768),
    # so the i sweeps take the Thomas kernel
    case = cases.bump_channel(800, 6, 2) if long_lines else casekit.small_partitioned()
    p = case.params
    p.irsop = irsop
    p.cutcirs = cutcirs
    p.psirs = 0.125
    p.rat = float(np.sqrt(1 + 4 * 0.6))
    p.cfl = 2.0 * p.rat
    return case


@pytest.mark.parametrize("irsop,cutcirs,long_lines", [(1, 0, False), (1, 1, False), (3, 0, False), (3, 1, False),
                                                      (2, 1, False), (3, 0, True)])
def test_irs_routines_match_oracle(oracle_mod, irsop, cutcirs, long_lines):
    """cirs (cutcirs 0) and scalef + 2 x (cutman_q + ccirs) + scaleb (cutcirs 1)
    on a residual field, against the oracle's restatement of
    src/cosa.f90:1977-1998, 2035-2443, 5206-5773 (cyclic reduction on the
    device up to 768-cell lines, Thomas sweeps beyond)."""
    case = _irs_case(irsop, cutcirs, long_lines)
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=9)
    qh = q.copy()
    res_o, dt_o, st = O.residual(qh, si, sj, sk)
    lam = O.p3()
    qp_ = q.copy()
    O.cons2prim(qp_)
    O.lambda_(qp_, si, sj, sk, lam)
    bx, by, bz = (O.p1() for _ in range(3))
    O.deltat(dt_o, lam, bx, by, bz)
    rg = ctx.alloc_p3().upload(res_o)
    dtg = ctx.alloc_p1().upload(dt_o)
    bg = [ctx.alloc_p1().upload(a) for a in (bx, by, bz)]
    oracle_mod.irs(O, res_o, dt_o, bx, by, bz)
    if cutcirs == 0:
        ctx.cirs(1, rg, dtg, *bg)
    else:
        ctx.scalef(1, rg, dtg)
        ores = ctx.alloc_p3().upload(rg.download())
        for _ in range(2):
            ctx.cutman_q(1, rg)
            ctx.ccirs(1, rg, ores, *bg)
        ctx.scaleb(1, rg, dtg)
    scale = np.abs(casekit.interior_cells(case, res_o, 5)).reshape(-1, 5).max(axis=0)
    assert _rel(rg.download(), res_o, case, scale=scale) <= TOL
    ctx.close()


@pytest.mark.parametrize("irsop,cutcirs", [(1, 0), (3, 1)])
def test_fused_smooth_irs_matches_oracle(oracle_mod, irsop, cutcirs):
    """The fused smooth with implicit residual smoothing (tile kernel writes R
    and beta, Thomas sweeps, stage update) against the oracle for 5 cycles."""
    case = _irs_case(irsop, cutcirs)
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=13)
    qo = q.copy()
    hist_o, st_o, dto, _ = oracle_mod.smooth_irs(O, qo, si, sj, sk, 5, rms_every=2)
    assert st_o == 0
    dq_ = ctx.alloc_p3().upload(q)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    hist_g, st = ctx.smooth(1, 5, 1, 2)
    assert st == 0
    err = _rel(dq_.download(), qo, case)
    assert err <= TOL, err
    rows = ~np.isnan(hist_o[:, 0])
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)
    ctx.close()


def _hb_case(nharms):
    from cosa_b200.params import set_harmonic_balance
    case = casekit.small_partitioned()
    p = set_harmonic_balance(case.params, nharms, 0.16)
    case.q0 = cases._freestream_state(case.tables, p)
    return case


def _hb_state(case, seed):
    """Snapshot-dependent perturbation of the free stream."""
    p = case.params
    S = 2 * p.nharms + 1
    q = cases.perturbed_state(case, seed=seed)
    base = case.q0
    for v, v0 in zip(p3_views(case.tables, q, 5, S), p3_views(case.tables, base, 5, S)):
        for n in range(S):
            v[..., n] = v0[..., n] + (v[..., n] - v0[..., n]) * (1.0 + 0.5 * np.sin(2 * np.pi * n / S + 0.3))
    return q


def test_src_hb_matches_oracle(oracle_mod):
    case = _hb_case(2)
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = _hb_state(case, 5)
    res = np.random.default_rng(1).standard_normal(q.size) * 1e-3
    ro = res.copy()
    oracle_mod.src_hb(O, q, vol, ro)
    ctx = gpu.Context([case.tables], case.params)
    rg = ctx.alloc_p3().upload(res)
    ctx.src_hb(1, ctx.alloc_p3().upload(q), ctx.alloc_p1().upload(vol), rg)
    S = 5
    a = casekit.interior_cells(case, rg.download(), 5, S)
    b = casekit.interior_cells(case, ro, 5, S)
    scale = np.abs(b).max()
    assert np.abs(a - b).max() <= TOL * scale
    ctx.close()


@pytest.mark.parametrize("nharms,rkimp,irsop,cutcirs", [(1, 0, 0, 0), (3, 0, 0, 0), (1, 1, 0, 0), (3, 1, 0, 0),
                                                       (1, 1, 1, 0), (2, 1, 2, 1), (2, 0, 2, 1)])
def test_fused_smooth_hb_matches_oracle(oracle_mod, nharms, rkimp, irsop, cutcirs):
    """Harmonic balance with all snapshots batched in the tile launch:
    per-snapshot time steps, the coupling source and the snapshot-averaged
    residual norm (resg_rms_hb) against the oracle for 4 cycles; with rkimp
    the time-spectral term leaves the residual and each cell's snapshots are
    coupled by the LU solve of update_bhb (its norm adds the term back).
    With IRS (rkimp or not) the term is in the smoothed residual and
    update_bhb takes the unsmoothed term out again."""
    case = _hb_case(nharms)
    p = case.params
    p.rkimp = rkimp
    if irsop:
        p.irsop, p.cutcirs, p.rat = irsop, cutcirs, float(np.sqrt(1 + 4 * 0.6))
    S = 2 * nharms + 1
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = _hb_state(case, 21)
    qo = q.copy()
    hist_o, st_o = oracle_mod.smooth_hb(O, qo, si, sj, sk, vol, 4, rms_every=2)
    assert st_o == 0
    ctx = gpu.Context([case.tables], case.params)
    dq_ = ctx.alloc_p3().upload(q)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    extra = {k: ctx.alloc_p1(nsnap=S) for k in ("betaxi", "betaeta", "betazeta")} if irsop >= 2 else {}
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(nsnap=S), si=m[0], sj=m[1], sk=m[2],
                   vol=ctx.alloc_p1().upload(vol), **extra)
    hist_g, st = ctx.smooth(1, 4, 1, 2)
    assert st == 0
    a = casekit.interior_cells(case, dq_.download(), 5, S)
    b = casekit.interior_cells(case, qo, 5, S)
    scale = np.abs(b).reshape(-1, 5, S).max(axis=(0, 2))
    assert (np.abs(a - b) / scale[None, :, None]).max() <= TOL
    rows = ~np.isnan(hist_o[:, 0])
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)
    ctx.close()


def test_newton_raphson_reciprocals_within_ulps():
    """The tile kernel's 1/x and 1/sqrt(x) (Newton-Raphson on the PTX
    approximations) stay within a few ulp of IEEE division and square root
    over the range of densities, sound speeds and limiter denominators."""
    rng = np.random.default_rng(0)
    x = np.exp(rng.uniform(np.log(1e-8), np.log(1e8), 200_000))
    x = np.concatenate([x, [1.0, 2.0, 0.5, 1.4, 1e-6, 3.0e5]])
    e_rcp, e_rsq = gpu.nr_selftest(x)
    eps = np.finfo(np.float64).eps
    assert e_rcp <= 4 * eps, e_rcp / eps
    assert e_rsq <= 4 * eps, e_rsq / eps


@pytest.mark.parametrize("which", ["channel", "partitioned", "duct"])
def test_split_schedule_matches_oracle(oracle_mod, which):
    """The face-split stage schedule (face fluxes through HBM, then the cell
    pass) against the oracle, like the fused tile kernel."""
    case = FUSED_CASES[which]()
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=11)
    ncyc = 6
    qo = q.copy()
    hist_o, st_o = O.smooth(qo, si, sj, sk, ncyc, rms_every=2)
    assert st_o == 0
    dq_ = ctx.alloc_p3().upload(q)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    ctx.set_schedule(1, 1)
    hist_g, st = ctx.smooth(1, ncyc, 1, 2)
    assert st == 0
    assert _rel(dq_.download(), qo, case) <= TOL
    rows = ~np.isnan(hist_o[:, 0])
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)
    ctx.close()


def _schedule_run(case, q, schedule, ncyc, nsnap=1, vol=None, si=None, sj=None, sk=None):
    ctx = gpu.Context([case.tables], case.params)
    dq_ = ctx.alloc_p3().upload(q)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    extra = {} if vol is None else dict(vol=ctx.alloc_p1().upload(vol))
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(nsnap=nsnap), si=m[0], sj=m[1], sk=m[2],
                   **extra)
    ctx.set_schedule(1, schedule)
    hist, st = ctx.smooth(1, ncyc, 1, 1)
    out = dq_.download()
    ctx.close()
    return out, hist, st


@pytest.mark.parametrize("which", ["channel_extrap_nk5", "partitioned", "duct", "naca_far1", "hb1"])
@pytest.mark.parametrize("ilimf", [1, 2, 3, 4])
def test_split_schedule_bits_equal_tile(oracle_mod, which, ilimf):
    """In FP64 the face-split schedule computes the tile kernel's arithmetic
    with the same device functions in the same order: the states of both
    schedules are bit for bit the same, for every limiter, strong
    boundaries, cuts and harmonic-balance snapshots; the residual norms,
    summed in a different order, agree to rounding.  (The mixed path is not
    bit-equal across schedules; it is held to its own tolerance against
    FP64 elsewhere.)"""
    if which == "hb1":
        case = _hb_case(1)
        q = _hb_state(case, 21)
        nsnap = 3
    else:
        case = FUSED_CASES[which]()
        q = cases.perturbed_state(case, seed=13)
        nsnap = 1
    case.params.ilimf = ilimf
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    kw = dict(nsnap=nsnap, vol=vol if which == "hb1" else None, si=si, sj=sj, sk=sk)
    q0, h0, st0 = _schedule_run(case, q, 0, 3, **kw)
    q1, h1, st1 = _schedule_run(case, q, 1, 3, **kw)
    assert st0 == 0 and st1 == 0
    assert np.array_equal(q0, q1)
    # the norms' partial sums are reduced in a different order per schedule
    np.testing.assert_allclose(h1, h0, rtol=1e-12, atol=0)


def test_autotune_restores_state_and_picks_a_schedule(oracle_mod):
    case = casekit.small_duct()
    O, ctx, (si, sj, sk, vol), q = _setup(case, oracle_mod, seed=3)
    dq_ = ctx.alloc_p3().upload(q)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    t0, t1, choice = ctx.autotune(1, 3)
    assert t0 > 0 and t1 > 0 and choice in (0, 1)
    assert choice == (1 if t1 < t0 else 0)
    assert np.array_equal(dq_.download(), q)
    _, st = ctx.smooth(1, 2, 1, 1)
    assert st == 0
    ctx.close()
