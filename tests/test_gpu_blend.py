"""Parity of the BSL and SST k-omega variants (sm_100a, through the C-ABI)
with the oracle's restatement of src/update.f90 (update_ttrm, tur_vis_sst),
src/src.f90 (srckw_sst), src/flux.f90 (vflux's BSL/SST branch, q_der_c of
k and omega) and src/grid.f90 (facedist): per routine on the same inputs
(1e-12 relative to the largest value of each variable), RK cycles with and
without IRS, and two- and three-level multigrid cycles (the coarse-level SST
eddy viscosity of the first visit included).  States 1e-12, norms 1e-9.
"""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p3_views, f0_views
from cosa_b200.params import CosaParams

import casekit
import test_gpu_kom as K

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _variant(p, which):
    q = CosaParams.from_buffer_copy(p)
    q.kom, q.kom_bsl, q.kom_sst = 0, int(which == "bsl"), int(which == "sst")
    return q


def _case(which):
    case = cases.partitioned_turbulent_channel(40, 20, 3, isplit=(16,), jsplit=(8,))
    case.params = _variant(case.params, which)
    case.q0 = cases._freestream_state(case.tables, case.params)
    return case


@pytest.mark.parametrize("which", ["bsl", "sst"])
def test_blend_routines_match_oracle(oracle_mod, which):
    case = _case(which)
    O, A = K._oracle(oracle_mod, case)
    q = K._initial(oracle_mod, O, A, case, seed=9)
    ctx, m, gvol, gvm, gdist = K._gpu(case)
    # face distances
    fd_o = np.zeros(3 * O.n0)
    oracle_mod.facedist(O, A.dist, fd_o)
    fd_g = [ctx.alloc_f0s() for _ in range(3)]
    ctx.facedist(1, gdist, *fd_g)
    for d in range(3):
        got, ref = fd_g[d].download(), fd_o[d * O.n0:(d + 1) * O.n0]
        for vg, vo in zip(f0_views(case.tables, got, 1), f0_views(case.tables, ref, 1)):
            ni, nj, nk = (vg.shape[0] - (d != 0), vg.shape[1] - (d != 1), vg.shape[2] - (d != 2))
            assert np.array_equal(vg[:ni, :nj, :nk], vo[:ni, :nj, :nk])
    qp_ = K._prim(oracle_mod, O, A, case, q)
    dq_ = ctx.alloc_p3().upload(qp_)
    ms = (A.si, A.sj, A.sk)
    # the blended k-omega face fluxes
    for d in (1, 2, 3):
        qf_o, g_o = O.p3(), [O.p3() for _ in range(3)]
        oracle_mod.q_face(O, d, qp_, qf_o)
        oracle_mod.q_der(O, d, qp_, *g_o)
        fm_o = O.f0()
        oracle_mod.q_face_mut(O, d, A.mut, fm_o)
        fm_g = ctx.alloc_f0().upload(fm_o)
        ins = [ctx.alloc_p3().upload(a) for a in [qf_o] + g_o]
        tau_o = O.p3()
        oracle_mod.rtst(O, d, qf_o, *g_o, A.vm, tau_o, fm_o)
        tau_g = ctx.alloc_p3().upload(tau_o)
        fdo = fd_o[(d - 1) * O.n0:d * O.n0].copy()
        oracle_mod.vflux_kom(O, d, qf_o, *g_o, tau_o, A.vm, ms[d - 1], fm_o, fdo)
        ctx.vflux_kom(d, 1, *ins, tau_g, gvm, m[d - 1], fm_g, fd_g[d - 1])
        F = fm_g.download()
        for vg, vo in zip(f0_views(case.tables, F, 7), f0_views(case.tables, fm_o, 7)):
            ni, nj, nk = (vg.shape[0] - (d != 1), vg.shape[1] - (d != 2), vg.shape[2] - (d != 3))
            x, y = vg[:ni, :nj, :nk], vo[:ni, :nj, :nk]
            sc = np.abs(y).reshape(-1, 7).max(axis=0) + 1e-300
            assert (np.abs(x - y) / sc[None, None, None, :, None]).max() <= TOL
    # cell-centred differences of u, v, w, k, omega
    dc_o = [O.p3() for _ in range(3)]
    dc_g = [ctx.alloc_p3() for _ in range(3)]
    for d in (1, 2, 3):
        qf_o = O.p3()
        oracle_mod.q_face(O, d, qp_, qf_o)
        oracle_mod.q_der_c(O, d, qf_o, dc_o[d - 1])
        ctx.q_der_c(d, 1, ctx.alloc_p3().upload(qf_o), dc_g[d - 1])
        for v in (slice(1, 4), slice(5, 7)):
            sl = (slice(2, -2), slice(2, -2), slice(2, -2), v)
            for vg, vo in zip(p3_views(case.tables, dc_g[d - 1].download(), 7, 1),
                              p3_views(case.tables, dc_o[d - 1], 7, 1)):
                assert np.abs(vg[sl] - vo[sl]).max() <= TOL * np.abs(vo[sl]).max()
    dcg = [ctx.alloc_p3().upload(a) for a in dc_o]
    # ttrm
    tt_o = np.zeros(O.n3 * 3)
    oracle_mod.update_ttrm(O, qp_, *dc_o, A.vm, tt_o, A.dist)
    tt_g = ctx.alloc_p3(nvar=3)
    ctx.update_ttrm(1, dq_, *dcg, gvm, tt_g, gdist)
    tg = casekit.interior_cells(case, tt_g.download(), 3)
    to = casekit.interior_cells(case, tt_o, 3)
    for c in range(3):
        assert np.abs(tg[:, c] - to[:, c]).max() <= 1e-11 * np.abs(to[:, c]).max(), c
    # SST / BSL sources
    n3s = O.n3 * O.S
    prd_o, dv_o, dp_o = (np.zeros(n3s) for _ in range(3))
    oracle_mod.turprod(O, qp_, *dc_o, A.vm, prd_o, dv_o, dp_o)
    res_o = cases.perturbed_state(case, amp=0.5, seed=3) * 1e-3
    res_g = ctx.alloc_p3().upload(res_o)
    mut = ctx.alloc_p3s().upload(A.mut)
    oracle_mod.srckw_sst(O, 1, qp_, A.mut, prd_o, dv_o, res_o, tt_o, A.vol)
    ctx.srckw_sst(1, dq_, ctx.alloc_p3s().upload(prd_o), ctx.alloc_p3s().upload(dv_o), res_g, mut,
                  ctx.alloc_p3(nvar=3).upload(tt_o), gvol)
    K._cmp_p3(case, res_g.download(), res_o)
    # update with the blended gamma and beta
    qn_o, qold = q.copy(), cases.perturbed_state(case, amp=0.01, seed=4)
    dtt = np.abs(cases.perturbed_state(case, amp=0.3, seed=5)[:O.n1]) * 1e-2 + 1e-3
    qn_g = ctx.alloc_p3().upload(q)
    oracle_mod.update_kom(O, res_o, qn_o, qold, A.vol, dtt, dp_o, prd_o, 0.5, tt_o)
    ctx.update_kom(1, ctx.alloc_p3().upload(res_o), qn_g, ctx.alloc_p3().upload(qold), gvol,
                   ctx.alloc_p1().upload(dtt), ctx.alloc_p3s().upload(dp_o), ctx.alloc_p3s().upload(prd_o), 0.5,
                   ctx.alloc_p3(nvar=3).upload(tt_o))
    K._cmp_p3(case, qn_g.download(), qn_o)
    if which == "sst":
        mo = A.mut.copy()
        oracle_mod.tur_vis_sst(O, q, mo, *dc_o, A.vm, A.dist)
        mg_ = ctx.alloc_p3s().upload(A.mut)
        ctx.tur_vis_sst(1, ctx.alloc_p3().upload(q), mg_, *dcg, gvm, gdist)
        a, b = mg_.download(), mo
        for va, vb in zip(p3_views(case.tables, a, 1, 1), p3_views(case.tables, b, 1, 1)):
            x, y = va[1:-1, 1:-1, 1:-1], vb[1:-1, 1:-1, 1:-1]  # cells 0..imax incl. the face halos
            assert np.abs(x - y).max() <= 1e-11 * np.abs(y).max()
    ctx.close()


def _smooth_pair(oracle_mod, case, ncyc, seed):
    O, A = K._oracle(oracle_mod, case)
    q = K._initial(oracle_mod, O, A, case, seed)
    mut0 = A.mut.copy()
    hist_o, st = oracle_mod.smooth_rans(O, A, ncyc, rms_every=2)
    assert st == 0
    ctx, m, gvol, gvm, gdist = K._gpu(case)
    arr = {k: ctx.alloc_p3() for k in ("q", "qold", "res", "qp", "qm", "dq", "dqp", "dqm")}
    arr["q"].upload(q)
    betas = [ctx.alloc_p1() for _ in range(3)]
    mut = ctx.alloc_p3s().upload(mut0)
    ctx.bind_level(1, q=arr["q"], qold=arr["qold"], res=arr["res"], dtvol=ctx.alloc_p1(), dtvolt=ctx.alloc_p1(),
                   si=m[0], sj=m[1], sk=m[2], vol=gvol, qp=arr["qp"], qm=arr["qm"], dq=arr["dq"], dqp=arr["dqp"],
                   dqm=arr["dqm"], flux=ctx.alloc_f0(), betaxi=betas[0], betaeta=betas[1], betazeta=betas[2],
                   mut=mut, dist=gdist)
    hist_g, st = ctx.smooth(1, ncyc, 1, 2)
    assert st == 0
    out, mut_g = arr["q"].download(), mut.download()
    ctx.close()
    return A.q, A.mut, hist_o, out, mut_g, hist_g


@pytest.mark.parametrize("which,irsop", [("bsl", 0), ("sst", 0), ("sst", 6)])
def test_blend_smooth_matches_oracle(oracle_mod, which, irsop):
    case = _case(which)
    p = case.params
    if irsop:
        p.irsop, p.cutcirs, p.psirs = irsop, 1, 0.125
        p.rat = p.ratt = float(np.sqrt(1 + 4 * 0.6))
        p.cfl = p.cflt = 1.5 * p.rat
    qo, muo, ho, qg, mug, hg = _smooth_pair(oracle_mod, case, 4, seed=5)
    assert K._state_err(case, qg, qo) <= TOL
    mo, mg_ = casekit.interior_cells(case, muo, 1), casekit.interior_cells(case, mug, 1)
    assert np.abs(mo - mg_).max() <= TOL * np.abs(mo).max()
    rows = ~np.isnan(ho[:, 0])
    assert np.array_equal(rows, ~np.isnan(hg[:, 0]))
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9)


@pytest.mark.parametrize("which,nlevel", [("bsl", 2), ("sst", 2), ("sst", 3)])
def test_blend_mg_cycles_match_oracle(oracle_mod, which, nlevel):
    import test_gpu_mg as M
    case = cases.turbulent_channel(32, 16, 8)
    p = _variant(case.params, which)
    case.params = p
    case.q0 = cases._freestream_state(case.tables, p)
    p.nlevel = nlevel
    p.nstart = p.npre = p.npost = p.ncrs = 1
    p.bln_prol = 1
    p.cfl = p.cflt = 1.0
    lv, Os, As = casekit.mg_rans_oracle(case, nlevel, p, oracle_mod)
    ctx, D = M._gpu_levels_rans(lv, p, As)
    ncyc = 4
    ho, st = oracle_mod.mg_rans(Os, As, 1, ncyc, ncyc, rms_every=2)
    hg, stg = ctx.mg(1, ncyc, ncyc, rms_every=2)
    assert st == 0 and stg == 0
    for nl in range(nlevel):
        t = lv[nl][0]
        a = np.concatenate([cases.interior(v).reshape(-1, 7) for v in p3_views(t, D[nl]["q"].download(), 7, 1)])
        b = np.concatenate([cases.interior(v).reshape(-1, 7) for v in p3_views(t, As[nl].q, 7, 1)])
        sc = np.abs(b).max(axis=0)
        sc[3] = max(sc[3], sc[1:3].max())  # rho w is rounding noise in these 2D flows
        err = float((np.abs(a - b) / sc[None, :]).max())
        assert err <= TOL * (10 if nl else 1), (nl, err)
    rows = ~np.isnan(ho[:, 0])
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9, atol=1e-15)
    ctx.close()
