"""Known-answer tests of the oracle's time-accurate paths (src/src.f90
src_uns / rhs_uns, src/update.f90 update_b with rkimp, src/cosa.f90 dual
time stepping and rkuns):

* src_uns and rhs_uns follow their BDF1 / BDF2 closed forms;
* with an enormous physical time step the dual-time pseudo iteration is the
  steady iteration (the BDF terms vanish to rounding);
* explicit and rkimp (physical-time term implicit) pseudo iterations converge
  to the same solution of one physical step, with and without multigrid;
* a one-stage rkuns step is forward Euler, q - dt / V res(q);
* rkuns keeps the norm of the last stage on printed steps only.
"""
import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p1_views, p3_views
from cosa_b200.params import CosaParams

import casekit


def _dual(p, dt, rkimp=0):
    q = CosaParams.from_buffer_copy(p)
    q.dualt, q.rkimp, q.dt, q.bdf1 = 1, rkimp, dt, 1
    return q


def test_src_and_rhs_uns_closed_form(oracle_mod):
    case = casekit.small_channel(12, 6, 2)
    p = _dual(case.params, 0.05)
    O = oracle_mod.OracleLevel(case.tables, p)
    _, _, _, vol = O.metrics(case.x, case.y, case.z)
    rng = np.random.default_rng(1)
    q, q1, q2 = (rng.uniform(0.5, 1.5, O.n3 * 5) for _ in range(3))
    V = np.concatenate([v[1:-1, 1:-1, 1:-1, 0].ravel(order="F") for v in p1_views(case.tables, vol, 1)])
    for bdf1 in (1, 0):
        p.bdf1 = bdf1
        res = np.zeros(O.n3 * 5)
        oracle_mod.src_uns(O, q, vol, res)
        rhs = np.zeros(O.n3 * 5)
        oracle_mod.rhs_uns(O, rhs, q1, q2, vol)
        R = casekit.interior_cells(case, res, 5)[..., 0]
        H = casekit.interior_cells(case, rhs, 5)[..., 0]
        Q, Q1, Q2 = (casekit.interior_cells(case, a, 5)[..., 0] for a in (q, q1, q2))
        fact = 1.0 if bdf1 else 1.5
        np.testing.assert_allclose(R, fact * Q * V[:, None] / p.dt, rtol=1e-14)
        ref = (Q1 if bdf1 else 2 * Q1 - Q2 / 2) * V[:, None] / p.dt
        np.testing.assert_allclose(H, ref, rtol=1e-14)


def _mg_run(oracle_mod, case, p, nlevel, ncyc, q):
    p.nlevel = nlevel
    lv, Os, As = casekit.mg_oracle(case, nlevel, p, oracle_mod, q_fine=q)
    h, st = oracle_mod.mg(Os, As, 1, ncyc, ncyc, rms_every=1)
    return As, Os, h, st


def test_dual_with_huge_dt_is_steady(oracle_mod):
    case = casekit.small_partitioned(32, 16, 4)
    ps = case.params
    ps.cfl = 1.0
    q = cases.perturbed_state(case, amp=0.01, seed=3)
    As_s, _, hs, st = _mg_run(oracle_mod, case, ps, 2, 4, q)
    assert st == 0
    pd = _dual(ps, 1.0e30)
    As_d, _, hd, st = _mg_run(oracle_mod, case, pd, 2, 4, q)
    assert st == 0
    np.testing.assert_allclose(As_d[0].q, As_s[0].q, rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(hd, hs, rtol=1e-10)


def _physical_step(oracle_mod, case, p, nlevel, ncyc, q0):
    """One BDF1 physical step from q0: q1 = q0, rhs = q1 V / dt, ncyc cycles."""
    p.nlevel = nlevel
    lv, Os, As = casekit.mg_oracle(case, nlevel, p, oracle_mod, q_fine=q0)
    A, O = As[0], Os[0]
    q1 = q0.copy()
    oracle_mod.rhs_uns(O, A.rhs, q1, q1, A.vol)
    h, st = oracle_mod.mg(Os, As, 1, ncyc, ncyc, rms_every=ncyc)
    assert st == 0
    return A.q, h


def test_explicit_and_implicit_pseudo_iterations_agree(oracle_mod):
    """(Coarse blocks two cells thick: one-cell-thick coarse blocks read stale
    opposite-face halos in the reference's BCs, which stalls multigrid.)"""
    case = casekit.small_channel(24, 12, 4)
    p = case.params
    p.cfl = 1.0
    q0 = cases.perturbed_state(case, amp=0.01, seed=5)
    dt = 0.2
    out = {}
    for nlevel in (1, 2):
        for rkimp in (0, 1):
            qd, h = _physical_step(oracle_mod, case, _dual(p, dt, rkimp), nlevel, 300, q0)
            rows = h[~np.isnan(h[:, 0])]
            assert rows[-1, 0] < 1e-10 * rows[0, 0], (nlevel, rkimp, rows[:, 0])
            out[(nlevel, rkimp)] = qd
    a = casekit.interior_cells(case, out[(1, 0)], 5)
    for key, qd in out.items():
        b = casekit.interior_cells(case, qd, 5)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max(), key
    # the step moved the state
    assert np.abs(a - casekit.interior_cells(case, q0, 5)).max() > 1e-5


def test_one_stage_rkuns_is_forward_euler(oracle_mod):
    case = casekit.small_channel(12, 6, 2)
    p = CosaParams.from_buffer_copy(case.params)
    p.rgkuns, p.dt, p.nstage = 1, 0.01, 1
    p.alphas[0] = 1.0
    O = oracle_mod.OracleLevel(case.tables, p)
    A = oracle_mod.LevelArrays(O)
    A.si, A.sj, A.sk, A.vol = O.metrics(case.x, case.y, case.z)
    q = cases.perturbed_state(case, amp=0.01, seed=7)
    A.q[:] = q
    h, st = oracle_mod.rkuns(O, A, 1)
    assert st == 0
    qr = q.copy()
    res, _, _ = _residual(oracle_mod, O, A, qr)
    V = p1_views(case.tables, A.vol, 1)
    for vq, v0, vr, vv in zip(p3_views(case.tables, A.q, 5, 1), p3_views(case.tables, q, 5, 1),
                              p3_views(case.tables, res, 5, 1), V):
        ref = cases.interior(v0) - p.dt / vv[1:-1, 1:-1, 1:-1, 0][:, :, :, None, None] * cases.interior(vr)
        np.testing.assert_allclose(cases.interior(vq), ref, rtol=1e-13, atol=1e-15)


def _residual(oracle_mod, O, A, q):
    res = O.p3()
    w = [O.p3() for _ in range(5)]
    flux = O.f0()
    dtv = O.p1()
    st = oracle_mod.lib().orc_residual(O.h, oracle_mod._par(O.p), 1, oracle_mod._p(q), oracle_mod._p(A.si),
                                       oracle_mod._p(A.sj), oracle_mod._p(A.sk), oracle_mod._p(res),
                                       *[oracle_mod._p(a) for a in w], oracle_mod._p(flux), oracle_mod._p(dtv), 0)
    return res, st, dtv


def test_rkuns_history_rows(oracle_mod):
    case = casekit.small_channel(12, 6, 2)
    p = CosaParams.from_buffer_copy(case.params)
    p.rgkuns, p.dt = 1, 0.005
    O = oracle_mod.OracleLevel(case.tables, p)
    A = oracle_mod.LevelArrays(O)
    A.si, A.sj, A.sk, A.vol = O.metrics(case.x, case.y, case.z)
    A.q[:] = cases.perturbed_state(case, amp=0.01, seed=8)
    h, st = oracle_mod.rkuns(O, A, 7, iprint=3)
    assert st == 0
    printed = ~np.isnan(h[:, 0])
    assert list(np.nonzero(printed)[0]) == [2, 5, 6]
    assert np.isfinite(A.q).all()


def test_kom_dual_with_huge_dt_is_steady_and_implicit_converges(oracle_mod):
    """The k-omega stage with the BDF terms: an enormous physical step gives
    the steady cycles; a physical step of dt = 0.2 converges with the
    physical-time term implicit (rkimp) on two levels."""
    case = cases.turbulent_channel(24, 12, 4)
    ps = case.params
    ps.cfl = ps.cflt = 1.0
    ps.nlevel = 2
    lv, Os, As = casekit.mg_rans_oracle(case, 2, ps, oracle_mod)
    hs, st = oracle_mod.mg_rans(Os, As, 1, 3, 3)
    assert st == 0
    pd = _dual(ps, 1.0e30)
    pd.nlevel = 2
    lv, Os2, As2 = casekit.mg_rans_oracle(case, 2, pd, oracle_mod)
    hd, st = oracle_mod.mg_rans(Os2, As2, 1, 3, 3)
    assert st == 0
    a, b = casekit.interior_cells(case, As2[0].q, 7), casekit.interior_cells(case, As[0].q, 7)
    sc = np.abs(b).max(axis=(0, 2))
    assert (np.abs(a - b) / sc[None, :, None]).max() <= 1e-12
    np.testing.assert_allclose(hd, hs, rtol=1e-9)
    pi = _dual(ps, 0.2, rkimp=1)
    pi.nlevel = 2
    lv, Os3, As3 = casekit.mg_rans_oracle(case, 2, pi, oracle_mod)
    q1 = As3[0].q.copy()
    oracle_mod.rhs_uns(Os3[0], As3[0].rhs, q1, q1, As3[0].vol)
    h, st = oracle_mod.mg_rans(Os3, As3, 1, 60, 60, rms_every=20)
    assert st == 0
    rows = h[~np.isnan(h[:, 0])]
    assert np.isfinite(As3[0].q).all() and rows[-1, 0] < 1e-3 * rows[0, 0], rows[:, 0]
