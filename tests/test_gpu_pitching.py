"""Harmonic balance of a rigidly pitching NACA 0012 on the device against the
oracle, through the C-ABI: the moving-grid set-up (movegrid, per-snapshot
metrics, face velocities, vert2cell), the per-routine face flux and
spectral radii with the grid speeds, the inviscid and 1500 walls moving with
the body, the fused harmonic-balance cycles on the face-split schedule
(S = 3, 5, 7) and the per-snapshot forces with the moment centre carried
with the body.

Tolerances as elsewhere: states 1e-12 relative to the largest value of each
variable, residual norms 1e-9, forces 1e-10 of the largest coefficient."""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p3_views
from cosa_b200.params import PREC_MIXED, hb_harmonics

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _case(nharms, **kw):
    kw.setdefault("blocks", (16, 16, 16, 16))
    kw.setdefault("nj", 16)
    kw.setdefault("rfar", 12.0)
    kw.setdefault("h1", 5e-3)
    return cases.naca_pitching(nharms=nharms, **kw)


def _state(case, seed):
    """A snapshot-dependent perturbation of the free stream."""
    S = 2 * case.params.nharms + 1
    q = cases.perturbed_state(case, amp=0.01, seed=seed)
    for v, v0 in zip(p3_views(case.tables, q, 5, S), p3_views(case.tables, case.q0, 5, S)):
        for n in range(S):
            v[..., n] = v0[..., n] + (v[..., n] - v0[..., n]) * (1.0 + 0.5 * np.sin(2 * np.pi * n / S + 0.3))
    return q


def _rel(a, b, tables, S):
    worst = 0.0
    for va, vb in zip(p3_views(tables, a, 5, S), p3_views(tables, b, 5, S)):
        ia, ib = cases.interior(va), cases.interior(vb)
        sc = np.abs(ib).reshape(-1, 5, S).max(axis=(0, 2))
        sc[1:4] = max(sc[1:4].max(), 1e-300)  # momentum components share one scale
        worst = max(worst, float((np.abs(ia - ib) / sc[None, None, None, :, None]).max()))
    return worst


def _device(case, precision=None):
    p = case.params
    if precision is not None:
        p.precision = precision
    ctx = gpu.Context([case.tables], p)
    m = ctx.pitching_setup(1, case)
    return ctx, m


def _bind(ctx, m, q):
    dq = ctx.alloc_p3().upload(q)
    ctx.bind_level(1, q=dq, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(nsnap=ctx.S), si=m["si"], sj=m["sj"],
                   sk=m["sk"], vol=m["vol"], xdot=m["xdot"], ydot=m["ydot"], zdot=m["zdot"], fvi=m["fvi"],
                   fvj=m["fvj"], fvk=m["fvk"])
    return dq


@pytest.mark.parametrize("nharms", [1, 3])
def test_moving_grid_setup_matches_oracle(nharms):
    case = _case(nharms)
    O = oracle.OracleLevel(case.tables, case.params)
    ones = np.ones(O.n1)
    mo = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    ctx, m = _device(case)
    for k, ko in (("x", "x"), ("y", "y"), ("z", "z"), ("xdot", "cx"), ("ydot", "cy"), ("zdot", "cz"),
                  ("si", "si"), ("sj", "sj"), ("sk", "sk"), ("vol", "vol"), ("fvi", "fvi"), ("fvj", "fvj"),
                  ("fvk", "fvk")):
        a, b = m[k].download(), mo[ko]
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-13 * scale, (k, np.abs(a - b).max(), scale)
    ctx.close()


def test_moving_routines_match_oracle():
    """The per-routine face flux (roflux_b with the face speeds), spectral
    radii (eig_eul with the cell grid velocities) and BC fill (walls moving
    with their faces) against the oracle routines on a perturbed state."""
    case = _case(2)
    p = case.params
    S = 2 * p.nharms + 1
    O = oracle.OracleLevel(case.tables, p)
    ones = np.ones(O.n1)
    mo = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    ctx, m = _device(case)
    q = _state(case, 3)
    _bind(ctx, m, q)
    # BC fill on the primitive state
    qo = q.copy()
    O.cons2prim(qo)
    qg = ctx.alloc_p3().upload(qo)
    assert O.bc(qo, mo["si"], mo["sj"], mo["sk"]) == 0
    ctx.bc(1, qg, m["si"], m["sj"], m["sk"])
    np.testing.assert_allclose(qg.download(), qo, rtol=1e-12, atol=1e-14)
    # spectral radii
    lo = O.p3()
    O.lambda_(qo, mo["si"], mo["sj"], mo["sk"], lo)
    lg = ctx.alloc_p3()
    ctx.lambda_(1, qg, m["si"], m["sj"], m["sk"], m["vol"], lg)
    a, b = lg.download(), lo
    assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()
    # face fluxes of the three families from random face states
    rng = np.random.default_rng(8)
    for idir, (sk_, sg) in enumerate(((mo["si"], m["si"]), (mo["sj"], m["sj"]), (mo["sk"], m["sk"])), start=1):
        qr = qo * (1 + 0.01 * rng.standard_normal(qo.size))
        ql = qo * (1 + 0.01 * rng.standard_normal(qo.size))
        fo = O.f0()
        O.roflux(idir, qr, ql, fo, sk_)
        fg = ctx.alloc_f0()
        ctx.roflux(idir, 1, ctx.alloc_p3().upload(qr), ctx.alloc_p3().upload(ql), fg, sg)
        a = fg.download()
        assert np.abs(a - fo).max() <= 1e-12 * np.abs(fo).max(), idir
    ctx.close()


@pytest.mark.parametrize("nharms", [1, 2, 3])
def test_pitching_hb_cycles_match_oracle(nharms):
    """Fused harmonic-balance RK cycles on the moving grid (face-split
    schedule with the face speeds, moving walls, time-spectral source)."""
    case = _case(nharms)
    p = case.params
    S = 2 * p.nharms + 1
    O = oracle.OracleLevel(case.tables, p)
    ones = np.ones(O.n1)
    mo = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    q = _state(case, 7 + nharms)
    qo = q.copy()
    ncyc = 5
    hist_o, st_o = oracle.smooth_hb(O, qo, mo["si"], mo["sj"], mo["sk"], mo["vol"], ncyc, rms_every=1)
    assert st_o == 0
    ctx, m = _device(case)
    dq = _bind(ctx, m, q)
    hist_g, st = ctx.smooth(1, ncyc, 1, 1)
    assert st == 0
    assert _rel(dq.download(), qo, case.tables, S) <= TOL
    np.testing.assert_allclose(hist_g, hist_o, rtol=1e-9)
    # per-snapshot forces with the moment centre carried by the body
    co = oracle.force(O, qo, mo["x"], mo["y"], mo["z"], mo["si"], mo["sj"], mo["sk"], None, lngth=(1.0, 0.1, 1.0))
    cg = ctx.force(1, dq, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], lngth=(1.0, 0.1, 1.0))
    assert np.abs(cg - co).max() <= 1e-10 * np.abs(co).max()
    ctx.close()


def test_pitching_mixed_precision_close_to_fp64():
    """Mixed precision on the moving grid stays within 1e-6 of FP64 after 20
    cycles, and its CL(t) harmonics within 1e-6 of FP64's."""
    out, cls = [], []
    for prec in (0, PREC_MIXED):
        case = _case(2)
        ctx, m = _device(case, prec)
        dq = _bind(ctx, m, _state(case, 4))
        _, st = ctx.smooth(1, 20, 1, 20)
        assert st == 0
        out.append(dq.download())
        c = ctx.force(1, dq, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], lngth=(1.0, 0.1, 1.0))
        cls.append(hb_harmonics(c[:, 0], case.params.nharms, case.params.omegas))
        ctx.close()
    S = 5
    err = _rel(out[1], out[0], case.tables, S)
    assert 0 < err < 1e-6, err
    assert np.abs(cls[1] - cls[0]).max() < 1e-6


@pytest.mark.parametrize("nharms", [1, 2])
def test_laminar_pitching_hb_cycles_match_oracle(nharms):
    """Laminar harmonic balance on the pitching grid: the face inverse
    metrics of every node snapshot, the no-slip wall moving with the body,
    the grid velocity in the viscous time step, and the skin friction from
    the velocity relative to the grid."""
    case = cases.naca_pitching(nharms=nharms, blocks=(16, 16, 16, 16), nj=16, rfar=12.0, h1=5e-3, model="laminar")
    p = case.params
    S = 2 * p.nharms + 1
    O = oracle.OracleLevel(case.tables, p)
    ones = np.ones(O.n1)
    mo = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    vmo = oracle.viscous_setup(O, mo["x"], mo["y"], mo["z"], mo["vol"])
    q = _state(case, 31 + nharms)
    qo = q.copy()
    ncyc = 5
    hist_o, st_o = oracle.smooth_ns(O, qo, mo["si"], mo["sj"], mo["sk"], mo["vol"], vmo, ncyc, rms_every=1)
    assert st_o == 0
    ctx, m = _device(case)
    vm = ctx.alloc_vm(1)
    ctx.viscous_setup(1, m["x"], m["y"], m["z"], m["vol"], vm)
    assert np.abs(vm.download() - vmo).max() <= 1e-12 * np.abs(vmo).max()
    dq = _bind(ctx, m, q)
    hist_g, st = ctx.smooth(1, ncyc, 1, 1)
    assert st == 0
    assert _rel(dq.download(), qo, case.tables, S) <= TOL
    np.testing.assert_allclose(hist_g, hist_o, rtol=1e-9)
    co = oracle.force(O, qo, mo["x"], mo["y"], mo["z"], mo["si"], mo["sj"], mo["sk"], vmo, lngth=(1.0, 0.1, 1.0))
    cg = ctx.force(1, dq, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], vm=vm, lngth=(1.0, 0.1, 1.0))
    assert np.abs(cg - co).max() <= 1e-10 * np.abs(co).max()
    assert np.abs(co[:, 6:]).max() > 0
    ctx.close()
