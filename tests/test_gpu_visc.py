"""Parity of the laminar viscous path (sm_100a, through the C-ABI) with the
oracle's restatement of src/grid.f90, src/flux.f90, src/bc.f90 and
src/cosa.f90.

* set-up: coordex/cutman_x, volex/cutman_v and vmetrix (node and volume
  halos, the nine face inverse metrics) -- the metrics round their
  products separately on the device, so they match to the last bit in
  practice; the bar is 1e-14 relative;
* the per-routine entry points q_face, q_der, vflux, lambda_ns, deltat_ns
  against the oracle routines on the same inputs (1e-12 relative to the
  largest value of each variable: the device contracts multiply-adds);
* the fused viscous smooth (viscous face fluxes + the tile kernel) against
  the oracle's smooth with the viscous residual: state 1e-12, residual
  norms 1e-9; with implicit residual smoothing (irsop 6: the viscous floor of
  the coefficients) and in mixed precision (1e-6).
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p1_views, p3_views, vm_views
from cosa_b200.params import PREC_MIXED

import casekit

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = {
    "laminar": lambda: cases.laminar_channel(40, 20, 3),
    "laminar_partitioned": lambda: cases.partitioned_laminar_channel(40, 20, 3, isplit=(16,), jsplit=(8,)),
}


def _oracle_setup(oracle_mod, case):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    si, sj, sk, vol = O.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O, x, y, z, vol)
    return O, (x, y, z), (si, sj, sk), vol, vm


def _gpu_setup(case, params=None):
    ctx = gpu.Context([case.tables], params or case.params)
    X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
    m = [ctx.alloc_p2() for _ in range(3)]
    vol = ctx.alloc_p1()
    ctx.imetrix(1, X, Y, Z, *m)
    ctx.vols(1, X, Y, Z, vol)
    vm = ctx.alloc_vm()
    ctx.viscous_setup(1, X, Y, Z, vol, vm)
    return ctx, (X, Y, Z), m, vol, vm


def _relmax(a, b):
    s = np.abs(b).max() + 1e-300
    return float(np.abs(a - b).max() / s)


@pytest.mark.parametrize("which", list(CASES))
def test_viscous_setup_matches_oracle(oracle_mod, which):
    case = CASES[which]()
    O, (x, y, z), _, vol, vm = _oracle_setup(oracle_mod, case)
    ctx, (X, Y, Z), _, gvol, gvm = _gpu_setup(case)
    for g, o in ((X, x), (Y, y), (Z, z)):
        assert np.array_equal(g.download(), o)
    assert _relmax(gvol.download(), vol) <= 1e-14
    a = gvm.download()
    for vb_g, vb_o in zip(vm_views(case.tables, a), vm_views(case.tables, vm)):
        for d in range(3):
            for m in range(3):
                sc = np.abs(vb_o[d][m]).max() + 1e-300
                assert np.abs(vb_g[d][m] - vb_o[d][m]).max() <= 1e-14 * sc
    ctx.close()


def _prim_state(oracle_mod, O, case, si, sj, sk, seed):
    """A perturbed primitive state with BC/cut halos and q_edges, as the
    viscous residual sees it."""
    q = cases.perturbed_state(case, amp=0.05, seed=seed)
    O.cons2prim(q)
    assert O.bc(q, si, sj, sk) == 0
    O.cutman_q(q)
    oracle_mod.q_edges(O, q)
    return q


@pytest.mark.parametrize("which", list(CASES))
def test_face_routines_match_oracle(oracle_mod, which):
    case = CASES[which]()
    O, _, (si, sj, sk), vol, vm = _oracle_setup(oracle_mod, case)
    q = _prim_state(oracle_mod, O, case, si, sj, sk, seed=7)
    ctx, _, m, gvol, gvm = _gpu_setup(case)
    dq_ = ctx.alloc_p3().upload(q)
    for d, s_o, s_g in ((1, si, m[0]), (2, sj, m[1]), (3, sk, m[2])):
        qf_o = O.p3()
        g_o = [O.p3() for _ in range(3)]
        oracle_mod.q_face(O, d, q, qf_o)
        oracle_mod.q_der(O, d, q, *g_o)
        qf_g = ctx.alloc_p3()
        g_g = [ctx.alloc_p3() for _ in range(3)]
        ctx.q_face(d, 1, dq_, qf_g)
        ctx.q_der(d, 1, dq_, *g_g)
        # the face range of family d, per block
        for a, b in [(qf_g, qf_o)] + list(zip(g_g, g_o)):
            A = a.download()
            for vg, vo in zip(p3_views(case.tables, A, 5, 1), p3_views(case.tables, b, 5, 1)):
                sl = [slice(2, -2)] * 3
                sl[d - 1] = slice(2, -1)
                sc = np.abs(vo[tuple(sl)]).reshape(-1, 5).max(axis=0) + 1e-300
                assert (np.abs(vg[tuple(sl)] - vo[tuple(sl)]) / sc[None, None, None, :, None]).max() <= TOL
        # vflux from the oracle's inputs on both sides
        ins = [ctx.alloc_p3().upload(a) for a in [qf_o] + g_o]
        f_o, f_g = O.f0(), ctx.alloc_f0()
        oracle_mod.vflux(O, d, qf_o, *g_o, vm, s_o, f_o)
        ctx.vflux(d, 1, *ins, gvm, s_g, f_g)
        F = f_g.download()
        for vg, vo in zip(cases.f0_views(case.tables, F, 5), cases.f0_views(case.tables, f_o, 5)):
            ni, nj, nk = (vg.shape[0] - (d != 1), vg.shape[1] - (d != 2), vg.shape[2] - (d != 3))
            a, b = vg[:ni, :nj, :nk], vo[:ni, :nj, :nk]
            sc = np.abs(b).reshape(-1, 5).max(axis=0) + 1e-300
            assert (np.abs(a - b) / sc[None, None, None, :, None]).max() <= TOL
    # viscous spectral radii and time step (irsop 6: the viscous IRS floor)
    p = case.params
    p.irsop, p.rat, p.psirs = 6, float(np.sqrt(1 + 4 * 0.6)), 0.125
    ctx.set_params(p)
    O.p = p
    lam_o, lamv_o = O.p3(), O.p3()
    oracle_mod.lambda_ns(O, q, si, sj, sk, vol, lam_o, lamv_o)
    lam_g, lamv_g = ctx.alloc_p3(), ctx.alloc_p3()
    ctx.lambda_ns(1, dq_, m[0], m[1], m[2], gvol, lam_g, lamv_g)
    assert _rel3(case, lam_g.download(), lam_o) <= TOL
    assert _rel3(case, lamv_g.download(), lamv_o) <= TOL
    outs_o = [O.p1() for _ in range(4)]
    oracle_mod.deltat_ns(O, outs_o[0], lam_o, lamv_o, *outs_o[1:])
    outs_g = [ctx.alloc_p1() for _ in range(4)]
    ctx.deltat_ns(1, outs_g[0], lam_g, lamv_g, *outs_g[1:])
    for g, o in zip(outs_g, outs_o):
        np.testing.assert_allclose(g.download(), o, rtol=1e-11, atol=1e-300)
    ctx.close()


def _rel3(case, a, b):
    A = casekit.interior_cells(case, a, 5)[:, :3]
    B = casekit.interior_cells(case, b, 5)[:, :3]
    sc = np.abs(B).reshape(-1, 3).max(axis=0) + 1e-300
    return float((np.abs(A - B) / sc[None, :, None]).max())


def _smooth_pair(oracle_mod, case, ncyc, seed, params=None, schedule=0):
    p = params or case.params
    O, _, (si, sj, sk), vol, vm = _oracle_setup(oracle_mod, case)
    O.p = p
    q = cases.perturbed_state(case, amp=0.02, seed=seed)
    qo = q.copy()
    hist_o, st_o = oracle_mod.smooth_ns(O, qo, si, sj, sk, vol, vm, ncyc, rms_every=2)
    assert st_o == 0
    ctx, _, m, gvol, gvm = _gpu_setup(case, p)
    dq_ = ctx.alloc_p3().upload(q)
    betas = [ctx.alloc_p1() for _ in range(3)]
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2], vol=gvol,
                   betaxi=betas[0], betaeta=betas[1], betazeta=betas[2])
    ctx.set_schedule(1, schedule)
    hist_g, st = ctx.smooth(1, ncyc, 1, 2)
    assert st == 0
    out = dq_.download()
    ctx.close()
    return qo, hist_o, out, hist_g


def _state_err(case, a, b):
    A = casekit.interior_cells(case, a, 5)
    B = casekit.interior_cells(case, b, 5)
    sc = np.abs(B).reshape(-1, 5).max(axis=0)
    d = np.abs(A - B) / sc[None, :, None]
    return float(np.inf if not np.isfinite(d).all() else d.max())


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("which", list(CASES))
def test_fused_viscous_smooth_matches_oracle(oracle_mod, which, schedule):
    case = CASES[which]()
    qo, hist_o, qg, hist_g = _smooth_pair(oracle_mod, case, 6, seed=5, schedule=schedule)
    assert _state_err(case, qg, qo) <= TOL
    rows = ~np.isnan(hist_o[:, 0])
    assert np.array_equal(rows, ~np.isnan(hist_g[:, 0]))
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)


def test_fused_viscous_smooth_with_irs(oracle_mod):
    case = CASES["laminar_partitioned"]()
    p = case.params
    p.irsop, p.cutcirs, p.psirs = 6, 1, 0.125
    p.rat = float(np.sqrt(1 + 4 * 0.6))
    p.cfl = 1.5 * p.rat
    qo, hist_o, qg, hist_g = _smooth_pair(oracle_mod, case, 4, seed=6, params=p)
    assert _state_err(case, qg, qo) <= TOL
    rows = ~np.isnan(hist_o[:, 0])
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)


def test_viscous_mixed_precision_close_to_fp64(oracle_mod):
    case = CASES["laminar"]()
    p = case.params
    p.precision = PREC_MIXED
    qo, hist_o, qg, hist_g = _smooth_pair(oracle_mod, case, 10, seed=8, params=p)
    err = _state_err(case, qg, qo)
    assert 0 < err < 1e-6, err
