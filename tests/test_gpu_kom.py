"""Parity of the Wilcox k-omega path (sm_100a, through the C-ABI) with the
oracle's restatement of src/flux.f90 (roflux turbulence fluxes, q_face with
mut, rtst, vflux, q_der_c), src/src.f90 (turprod, srckw), src/update.f90
(update_b), src/bc.f90 (bc_walvis_15, cutman_mut) and src/cosa.f90
(lambda, deltat, smooth).

Routines are compared on the same inputs (1e-12 relative to the largest
value of each variable; the device contracts multiply-adds), the RK cycles
of cosa_gpu_smooth against the oracle's driver (state 1e-12, residual norms
1e-9), with and without implicit residual smoothing.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p1_views, p3_views, f0_views

import casekit

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = {
    "turbulent": lambda: cases.turbulent_channel(40, 20, 3),
    "turbulent_partitioned": lambda: cases.partitioned_turbulent_channel(40, 20, 3, isplit=(16,), jsplit=(8,)),
}


def _oracle(oracle_mod, case):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    A = oracle_mod.RansArrays(O)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    A.si, A.sj, A.sk, A.vol = O.metrics(x, y, z)
    A.vm = oracle_mod.viscous_setup(O, x, y, z, A.vol)
    A.dist[:] = cases.wall_distance(case)
    return O, A


def _initial(oracle_mod, O, A, case, seed):
    """Perturbed state (k, omega kept positive) and its turbulent viscosity."""
    q = cases.perturbed_state(case, amp=0.02, seed=seed)
    for v in p3_views(case.tables, q, 7, 1):
        v[..., 5, :] = np.abs(v[..., 5, :]) + 1e-4 * v[..., 0, :]
        v[..., 6, :] = np.abs(v[..., 6, :]) + 0.5 * v[..., 0, :]
    A.q[:] = q
    qq = q.copy()
    O.cons2prim(qq)
    assert oracle_mod.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist) == 0
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle_mod.tur_vis(O, qq, A.mut)
    oracle_mod.cutman_mut(O, A.mut)
    return q


def _gpu(case, params=None):
    ctx = gpu.Context([case.tables], params or case.params)
    X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
    m = [ctx.alloc_p2() for _ in range(3)]
    vol = ctx.alloc_p1()
    ctx.imetrix(1, X, Y, Z, *m)
    ctx.vols(1, X, Y, Z, vol)
    vm = ctx.alloc_vm()
    ctx.viscous_setup(1, X, Y, Z, vol, vm)
    dist = ctx.alloc_p1().upload(cases.wall_distance(case))
    return ctx, m, vol, vm, dist


def _cmp_p3(case, a, b, nvar=7, sl=None, tol=TOL):
    for va, vb in zip(p3_views(case.tables, a, nvar, 1), p3_views(case.tables, b, nvar, 1)):
        s = sl or (slice(2, -2), slice(2, -2), slice(2, -2))
        x, y = va[s], vb[s]
        sc = np.abs(y).reshape(-1, nvar).max(axis=0) + 1e-300
        err = (np.abs(x - y) / sc[None, None, None, :, None]).max()
        assert err <= tol, err


def _prim(oracle_mod, O, A, case, q):
    a = q.copy()
    O.cons2prim(a)
    assert oracle_mod.bc_dist(O, a, A.si, A.sj, A.sk, A.dist) == 0
    O.cutman_q(a)
    oracle_mod.q_edges(O, a, A.mut)
    return a


@pytest.mark.parametrize("which", list(CASES))
def test_kom_routines_match_oracle(oracle_mod, which):
    case = CASES[which]()
    O, A = _oracle(oracle_mod, case)
    q = _initial(oracle_mod, O, A, case, seed=9)
    ctx, m, gvol, gvm, gdist = _gpu(case)
    # bc with the k-omega wall (halos included)
    a_o = q.copy()
    O.cons2prim(a_o)
    assert oracle_mod.bc_dist(O, a_o, A.si, A.sj, A.sk, A.dist) == 0
    a_g = ctx.alloc_p3().upload(q)
    ctx.cons2prim(1, a_g)
    ctx.bc_dist(1, a_g, m[0], m[1], m[2], gdist)
    _cmp_p3(case, a_g.download(), a_o, sl=(slice(None), slice(None), slice(2, -2)))
    # primitive state with halos, edges of q and mut
    qp_ = _prim(oracle_mod, O, A, case, q)
    dq_ = ctx.alloc_p3().upload(qp_)
    mut = ctx.alloc_p3s().upload(A.mut)
    ms = (A.si, A.sj, A.sk)
    for d in (1, 2, 3):
        # Roe fluxes incl. the turbulence fluxes
        b_o = [O.p3() for _ in range(5)]
        O.muscl(d, 1, qp_, *b_o)
        b_g = [ctx.alloc_p3().upload(a) for a in b_o]
        f_o, f_g = O.f0(), ctx.alloc_f0()
        O.roflux(d, b_o[0], b_o[1], f_o, ms[d - 1])
        ctx.roflux(d, 1, b_g[0], b_g[1], f_g, m[d - 1])
        F, Fo = f_g.download(), f_o
        for vg, vo in zip(f0_views(case.tables, F, 7), f0_views(case.tables, Fo, 7)):
            ni, nj, nk = (vg.shape[0] - (d != 1), vg.shape[1] - (d != 2), vg.shape[2] - (d != 3))
            x, y = vg[:ni, :nj, :nk], vo[:ni, :nj, :nk]
            sc = np.abs(y).reshape(-1, 7).max(axis=0) + 1e-300
            assert (np.abs(x - y) / sc[None, None, None, :, None]).max() <= TOL
        # face state / gradients / face mut / Reynolds stresses / viscous flux
        qf_o, g_o = O.p3(), [O.p3() for _ in range(3)]
        oracle_mod.q_face(O, d, qp_, qf_o)
        oracle_mod.q_der(O, d, qp_, *g_o)
        qf_g, g_g = ctx.alloc_p3(), [ctx.alloc_p3() for _ in range(3)]
        ctx.q_face(d, 1, dq_, qf_g)
        ctx.q_der(d, 1, dq_, *g_g)
        fsl = [slice(2, -2)] * 3
        fsl[d - 1] = slice(2, -1)
        _cmp_p3(case, qf_g.download(), qf_o, sl=tuple(fsl))
        for a, b in zip(g_g, g_o):
            _cmp_p3(case, a.download(), b, sl=tuple(fsl))
        fm_o, fm_g = O.f0(), ctx.alloc_f0()
        oracle_mod.q_face_mut(O, d, A.mut, fm_o)
        ctx.q_face_mut(d, 1, mut, fm_g)
        ins = [ctx.alloc_p3().upload(a) for a in [qf_o] + g_o]
        tau_o, tau_g = O.p3(), ctx.alloc_p3()
        oracle_mod.rtst(O, d, qf_o, *g_o, A.vm, tau_o, fm_o)
        ctx.rtst(d, 1, *ins, gvm, fm_g, tau_g)
        _cmp_p3(case, tau_g.download(), tau_o, sl=tuple(fsl))
        oracle_mod.vflux_kom(O, d, qf_o, *g_o, tau_o, A.vm, ms[d - 1], fm_o)
        ctx.vflux_kom(d, 1, *ins, tau_g, gvm, m[d - 1], fm_g)
        F = fm_g.download()
        for vg, vo in zip(f0_views(case.tables, F, 7), f0_views(case.tables, fm_o, 7)):
            ni, nj, nk = (vg.shape[0] - (d != 1), vg.shape[1] - (d != 2), vg.shape[2] - (d != 3))
            x, y = vg[:ni, :nj, :nk], vo[:ni, :nj, :nk]
            sc = np.abs(y).reshape(-1, 7).max(axis=0) + 1e-300
            assert (np.abs(x - y) / sc[None, None, None, :, None]).max() <= TOL
    # cell gradients, production, sources, update
    dc_o = [O.p3() for _ in range(3)]
    dc_g = [ctx.alloc_p3() for _ in range(3)]
    for d in (1, 2, 3):
        qf_o = O.p3()
        oracle_mod.q_face(O, d, qp_, qf_o)
        oracle_mod.q_der_c(O, d, qf_o, dc_o[d - 1])
        ctx.q_der_c(d, 1, ctx.alloc_p3().upload(qf_o), dc_g[d - 1])
        sl = (slice(2, -2), slice(2, -2), slice(2, -2), slice(1, 4))
        for vg, vo in zip(p3_views(case.tables, dc_g[d - 1].download(), 7, 1), p3_views(case.tables, dc_o[d - 1], 7, 1)):
            assert np.abs(vg[sl] - vo[sl]).max() <= TOL * np.abs(vo[sl]).max()
    n3s = O.n3 * O.S
    prd_o, dv_o, dp_o = (np.zeros(n3s) for _ in range(3))
    oracle_mod.turprod(O, qp_, *dc_o, A.vm, prd_o, dv_o, dp_o)
    prd_g, dv_g, dp_g = (ctx.alloc_p3s() for _ in range(3))
    ctx.turprod(1, *[ctx.alloc_p3().upload(a) for a in dc_o], gvm, prd_g, dv_g, dp_g)
    for g_, o_ in ((prd_g, prd_o), (dv_g, dv_o), (dp_g, dp_o)):
        gg = casekit.interior_cells(case, g_.download(), 1)
        oo = casekit.interior_cells(case, o_, 1)
        assert np.abs(gg - oo).max() <= TOL * (np.abs(oo).max() + 1e-300)
    res_o = cases.perturbed_state(case, amp=0.5, seed=3) * 1e-3
    res_g = ctx.alloc_p3().upload(res_o)
    oracle_mod.srckw(O, 1, qp_, A.mut, prd_o, dv_o, res_o, A.vol)
    ctx.srckw(1, dq_, mut, prd_g, dv_g, res_g, gvol)
    _cmp_p3(case, res_g.download(), res_o)
    qn_o, qold = q.copy(), cases.perturbed_state(case, amp=0.01, seed=4)
    dtt = np.abs(cases.perturbed_state(case, amp=0.3, seed=5)[:O.n1]) * 1e-2 + 1e-3
    qn_g = ctx.alloc_p3().upload(q)
    oracle_mod.update_kom(O, res_o, qn_o, qold, A.vol, dtt, dp_o, prd_o, 0.5)
    ctx.update_kom(1, res_g, qn_g, ctx.alloc_p3().upload(qold), gvol, ctx.alloc_p1().upload(dtt), dp_g, prd_g, 0.5)
    _cmp_p3(case, qn_g.download(), qn_o)
    # spectral radii with mut, time steps with dtvolt and the turbulence IRS coefficients
    p = case.params
    p.irsop, p.rat, p.ratt, p.psirs = 6, float(np.sqrt(1 + 4 * 0.6)), float(np.sqrt(1 + 4 * 0.4)), 0.125
    ctx.set_params(p)
    lam_o, lamv_o = O.p3(), O.p3()
    oracle_mod.lambda_ns(O, qp_, A.si, A.sj, A.sk, A.vol, lam_o, lamv_o, A.mut)
    lam_g, lamv_g = ctx.alloc_p3(), ctx.alloc_p3()
    ctx.lambda_ns(1, dq_, m[0], m[1], m[2], gvol, lam_g, lamv_g, mut)
    sl3 = (slice(2, -2), slice(2, -2), slice(2, -2), slice(0, 3))
    for a, b in ((lam_g, lam_o), (lamv_g, lamv_o)):
        for vg, vo in zip(p3_views(case.tables, a.download(), 7, 1), p3_views(case.tables, b, 7, 1)):
            assert np.abs(vg[sl3] - vo[sl3]).max() <= TOL * np.abs(vo[sl3]).max()
    outs_o = [O.p1(O.S) for _ in range(8)]
    oracle_mod.deltat_ns_full(O, outs_o[0], lam_o, lamv_o, *outs_o[1:])
    outs_g = [ctx.alloc_p1() for _ in range(8)]
    ctx.deltat_ns(1, outs_g[0], lam_g, lamv_g, *outs_g[1:])
    for g_, o_ in zip(outs_g, outs_o):
        np.testing.assert_allclose(g_.download(), o_, rtol=1e-11, atol=1e-300)
    # cutman_mut
    mu2 = A.mut.copy()
    mu2[:] = np.arange(mu2.size) * 1e-3
    mg = ctx.alloc_p3s().upload(mu2)
    oracle_mod.cutman_mut(O, mu2)
    ctx.cutman_mut(1, mg)
    assert np.array_equal(mg.download(), mu2)
    ctx.close()


def _smooth_pair(oracle_mod, case, ncyc, seed):
    O, A = _oracle(oracle_mod, case)
    q = _initial(oracle_mod, O, A, case, seed)
    mut0 = A.mut.copy()
    hist_o, st = oracle_mod.smooth_rans(O, A, ncyc, rms_every=2)
    assert st == 0
    ctx, m, gvol, gvm, gdist = _gpu(case)
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


def _state_err(case, a, b):
    A = casekit.interior_cells(case, a, 7)
    B = casekit.interior_cells(case, b, 7)
    sc = np.abs(B).reshape(-1, 7).max(axis=0)
    d = np.abs(A - B) / sc[None, :, None]
    return float(np.inf if not np.isfinite(d).all() else d.max())


@pytest.mark.parametrize("which", list(CASES))
def test_rans_smooth_matches_oracle(oracle_mod, which):
    case = CASES[which]()
    qo, muo, ho, qg, mug, hg = _smooth_pair(oracle_mod, case, 4, seed=5)
    assert _state_err(case, qg, qo) <= TOL
    mo, mg_ = casekit.interior_cells(case, muo, 1), casekit.interior_cells(case, mug, 1)
    assert np.abs(mo - mg_).max() <= TOL * np.abs(mo).max()
    rows = ~np.isnan(ho[:, 0])
    assert np.array_equal(rows, ~np.isnan(hg[:, 0]))
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9)


@pytest.mark.parametrize("irsop,cutcirs", [(1, 0), (6, 1)])
def test_rans_smooth_with_irs_matches_oracle(oracle_mod, irsop, cutcirs):
    case = CASES["turbulent_partitioned"]()
    p = case.params
    p.irsop, p.cutcirs, p.psirs = irsop, cutcirs, 0.125
    p.rat = float(np.sqrt(1 + 4 * 0.6))
    p.ratt = p.rat
    p.cfl = 1.5 * p.rat
    p.cflt = p.cfl
    qo, muo, ho, qg, mug, hg = _smooth_pair(oracle_mod, case, 3, seed=6)
    assert _state_err(case, qg, qo) <= TOL
    rows = ~np.isnan(ho[:, 0])
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9)

