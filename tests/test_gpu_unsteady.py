"""Parity of the time-accurate paths (sm_100a, through the C-ABI) with the
oracle: src_uns / rhs_uns per routine; dual time stepping (physical steps of
pseudo-time multigrid cycles, the first one first order) for the Euler path
explicit, with the physical-time term implicit (rkimp) with and without IRS,
on one and two levels, and for the k-omega path; rkuns for Euler and laminar
flow.  States 1e-12 of the largest value of each variable, norms 1e-9.
"""
import numpy as np
import pytest

from cosa_b200 import cases, unsteady
from cosa_b200.params import CosaParams

import casekit
import test_gpu_mg as M

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _dual(p, dt, rkimp=0):
    q = CosaParams.from_buffer_copy(p)
    q.dualt, q.rkimp, q.dt, q.bdf1 = 1, rkimp, dt, 1
    return q


def _oracle_dual(oracle_mod, mg_fn, Os, As, p, ntime, ncycle):
    """The physical-time loop of the reference's main program on the oracle."""
    O, A = Os[0], As[0]
    q1, q2 = O.p3(), O.p3()
    hist = []
    for itime in range(1, ntime + 1):
        p.bdf1 = 1 if itime == 1 else 0
        oracle_mod.copy_interior(O, q1, A.q)
        oracle_mod.rhs_uns(O, A.rhs, q1, q2, A.vol)
        h, st = mg_fn(Os, As, 1, ncycle, ncycle, rms_every=1)
        assert st == 0
        oracle_mod.copy_interior(O, q2, q1)
        hist.append(h)
    return hist


def test_src_rhs_uns_match_oracle(oracle_mod):
    case = casekit.small_partitioned(32, 16, 4)
    p = _dual(case.params, 0.05)
    O = oracle_mod.OracleLevel(case.tables, p)
    _, _, _, vol = O.metrics(case.x, case.y, case.z)
    rng = np.random.default_rng(2)
    q, q1, q2, r0 = (rng.uniform(0.5, 1.5, O.n3 * 5) for _ in range(4))
    from cosa_b200 import gpu
    ctx = gpu.Context([case.tables], p)
    g = {k: ctx.alloc_p3().upload(a) for k, a in (("q", q), ("q1", q1), ("q2", q2), ("r", r0), ("h", r0))}
    gvol = ctx.alloc_p1().upload(vol)
    for bdf1 in (1, 0):
        p.bdf1 = bdf1
        ctx.set_params(p)
        ro, ho = r0.copy(), r0.copy()
        oracle_mod.src_uns(O, q, vol, ro)
        oracle_mod.rhs_uns(O, ho, q1, q2, vol)
        g["r"].upload(r0)
        ctx.src_uns(1, g["q"], gvol, g["r"])
        ctx.rhs_uns(1, g["h"], g["q1"], g["q2"], gvol)
        for a, b in ((g["r"].download(), ro), (g["h"].download(), ho)):
            A, B = casekit.interior_cells(case, a, 5), casekit.interior_cells(case, b, 5)
            assert np.abs(A - B).max() <= TOL * np.abs(B).max()
    ctx.close()


@pytest.mark.parametrize("nlevel,rkimp,irsop", [(2, 0, 0), (2, 1, 0), (1, 1, 0), (2, 1, 1)])
def test_dual_time_matches_oracle(oracle_mod, nlevel, rkimp, irsop):
    case = casekit.small_channel(32, 16, 4)
    p = _dual(case.params, 0.2, rkimp)
    p.nlevel, p.cfl = nlevel, 1.0
    if irsop:
        p.irsop, p.rat = irsop, float(np.sqrt(1 + 4 * 0.6))
        p.cfl = 1.0 * p.rat
    q = cases.perturbed_state(case, amp=0.01, seed=4)
    lv, Os, As = casekit.mg_oracle(case, nlevel, p, oracle_mod, q_fine=q)
    ctx, D = M._gpu_levels(lv, p, As)
    ho = _oracle_dual(oracle_mod, oracle_mod.mg, Os, As, p, 3, 4)
    p.bdf1 = 1
    ctx.set_params(p)
    hg = unsteady.dual_time(ctx, D[0]["q"], D[0]["rhs"], D[0]["vol"], 3, 4)
    for nl in range(nlevel):
        err = M._interior_rel(D[nl]["q"].download(), As[nl].q, lv[nl][0], 5, 1)
        assert err <= TOL * (10 if nl else 1), (nl, err)
    for a, b in zip(hg, ho):
        np.testing.assert_allclose(a, b, rtol=1e-9)
    ctx.close()


@pytest.mark.parametrize("rkimp", [0, 1])
def test_kom_dual_time_matches_oracle(oracle_mod, rkimp):
    case = cases.turbulent_channel(32, 16, 4)
    p = _dual(case.params, 0.2, rkimp)
    p.nlevel, p.cfl, p.cflt = 2, 1.0, 1.0
    p.nstart = p.npre = p.npost = p.ncrs = 1
    lv, Os, As = casekit.mg_rans_oracle(case, 2, p, oracle_mod)
    ctx, D = M._gpu_levels_rans(lv, p, As)
    ho = _oracle_dual(oracle_mod, oracle_mod.mg_rans, Os, As, p, 2, 3)
    p.bdf1 = 1
    ctx.set_params(p)
    hg = unsteady.dual_time(ctx, D[0]["q"], D[0]["rhs"], D[0]["vol"], 2, 3)
    from cosa_b200.cases import p3_views
    for nl in range(2):
        t = lv[nl][0]
        a = np.concatenate([cases.interior(v).reshape(-1, 7) for v in p3_views(t, D[nl]["q"].download(), 7, 1)])
        b = np.concatenate([cases.interior(v).reshape(-1, 7) for v in p3_views(t, As[nl].q, 7, 1)])
        sc = np.abs(b).max(axis=0)
        sc[3] = max(sc[3], sc[1:3].max())
        assert float((np.abs(a - b) / sc[None, :]).max()) <= TOL * (10 if nl else 1), nl
    for a, b in zip(hg, ho):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-15)
    ctx.close()


@pytest.mark.parametrize("model", ["euler", "laminar"])
def test_rkuns_matches_oracle(oracle_mod, model):
    import test_gpu_visc as V
    case = casekit.small_partitioned(32, 16, 4) if model == "euler" else V.CASES["laminar_partitioned"]()
    p = CosaParams.from_buffer_copy(case.params)
    p.rgkuns, p.dt = 1, 0.004
    q = cases.perturbed_state(case, amp=0.01, seed=9)
    if model == "euler":
        O = oracle_mod.OracleLevel(case.tables, p)
        A = oracle_mod.LevelArrays(O)
        A.si, A.sj, A.sk, A.vol = O.metrics(case.x, case.y, case.z)
        vm = None
    else:
        O, _, (si, sj, sk), vol, vm = V._oracle_setup(oracle_mod, case)
        O.p = p
        A = oracle_mod.LevelArrays(O)
        A.si, A.sj, A.sk, A.vol = si, sj, sk, vol
    A.q[:] = q
    ho, st = oracle_mod.rkuns(O, A, 6, iprint=2, vm=vm)
    assert st == 0
    if model == "euler":
        from cosa_b200 import gpu
        ctx = gpu.Context([case.tables], p)
        m = [ctx.alloc_p2().upload(a) for a in (A.si, A.sj, A.sk)]
        gvol = ctx.alloc_p1().upload(A.vol)
    else:
        ctx, _, m, gvol, gvm = V._gpu_setup(case, p)
    dq = ctx.alloc_p3().upload(q)
    ctx.bind_level(1, q=dq, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2], vol=gvol)
    hg = unsteady.rkuns(ctx, 6, iprint=2)
    err = M._interior_rel(dq.download(), A.q, case.tables, 5, 1)
    assert err <= TOL, err
    rows = ~np.isnan(ho[:, 0])
    assert np.array_equal(rows, ~np.isnan(hg[:, 0]))
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9)
    ctx.close()
