"""Parity of low-speed preconditioning (sm_100a, through the C-ABI) with the
oracle: the per-routine entries (lm_cutoff_pg, lm_viscoff, rest3, proflux,
the preconditioned spectral radii, lsp, precres), multigrid cycles of the
preconditioned Euler stage on a low-Mach bump channel (cut-off types 1, 2
and 3, with IRS) and single-level laminar cycles with the viscous cut-off.
Routines 1e-13 of the largest value, states 1e-12 of the largest value of
each variable, norms 1e-9, cut-offs 1e-12.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p3_views
from cosa_b200.params import CosaParams, set_low_speed

import casekit
import test_gpu_mg as M
import test_gpu_visc as V

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _low_mach_channel(ni=32, nj=16, nk=4, mach=0.1, partitioned=False):
    if partitioned:
        return cases.partitioned_channel(ni, nj, nk, isplit=(ni // 2 - 4,), jsplit=(nj // 2,), permute_last=True,
                                         mach=mach)
    return cases.bump_channel(ni, nj, nk, mach=mach)


def _random_prim(O, seed):
    """A primitive state of low-Mach values in every cell (halos included)."""
    rng = np.random.default_rng(seed)
    q = O.p3()
    lo = (0.9, 0.02, -0.03, -0.01, 0.69)
    hi = (1.1, 0.12, 0.03, 0.01, 0.74)
    for v in p3_views(O.t, q, 5, O.S):
        for m in range(5):
            v[..., m, :] = rng.uniform(lo[m], hi[m], v[..., m, :].shape)
    return q


def _rel(a, b):
    return float(np.abs(a - b).max() / (np.abs(b).max() + 1e-300))


def test_lsp_routines_match_oracle(oracle_mod):
    case = casekit.small_partitioned(24, 12, 2)
    p = set_low_speed(CosaParams.from_buffer_copy(case.params), cutoff_type=2, epsp=(0.03,))
    p.machfs = 0.1
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = _random_prim(O, 1)
    ctx = gpu.Context([case.tables], p)
    d = {k: ctx.alloc_p2().upload(a) for k, a in (("si", si), ("sj", sj), ("sk", sk))}
    dq = ctx.alloc_p3().upload(q)
    # pressure-gradient cut-off
    cpg = oracle_mod.m1(O)
    oracle_mod.lm_cutoff_pg(O, q, cpg)
    gpg = ctx.alloc_m1()
    ctx.lm_cutoff_pg(1, dq, gpg)
    assert _rel(gpg.download(), cpg) <= 1e-14
    cvs = np.random.default_rng(3).uniform(0, 2e-3, cpg.size)
    gvs = ctx.alloc_m1().upload(cvs)
    # preconditioned spectral radii (inviscid)
    lam = O.p3()
    oracle_mod.lambda_p(O, 1, q, si, sj, sk, lam, cpg, cvs)
    glam = ctx.alloc_p3()
    ctx.lambda_p(1, dq, d["si"], d["sj"], d["sk"], glam, gpg, gvs)
    a, b = casekit.interior_cells(case, glam.download(), 5), casekit.interior_cells(case, lam, 5)
    assert _rel(a[:, :3], b[:, :3]) <= 1e-13
    # preconditioned Roe flux of each family from random face states
    qr, ql = _random_prim(O, 4), _random_prim(O, 5)
    gqr, gql = ctx.alloc_p3().upload(qr), ctx.alloc_p3().upload(ql)
    for idir, s in ((1, si), (2, sj), (3, sk)):
        f = O.f0()
        oracle_mod.proflux(O, idir, 1, qr, ql, f, s, cpg, cvs)
        gf = ctx.alloc_f0()
        ctx.proflux(idir, 1, gqr, gql, gf, d[("si", "sj", "sk")[idir - 1]], gpg, gvs)
        assert _rel(gf.download(), f) <= 1e-13, idir
    # preconditioner from a conservative state and its product with res
    qc = cases.perturbed_state(case, amp=0.02, seed=6)
    prec = oracle_mod.lsp_prec(O, 1, qc, cpg, cvs)
    gprec = ctx.alloc_m1(nvar=25)
    ctx.lsp(1, ctx.alloc_p3().upload(qc), gpg, gvs, gprec)
    assert _rel(gprec.download(), prec) <= 1e-14
    res = np.random.default_rng(7).normal(size=q.size)
    ro = res.copy()
    oracle_mod.precres(O, ro, prec)
    gres = ctx.alloc_p3().upload(res)
    ctx.precres(1, gres, gprec)
    assert _rel(casekit.interior_cells(case, gres.download(), 5), casekit.interior_cells(case, ro, 5)) <= 1e-13
    ctx.close()


def test_viscous_cutoff_and_rest3_match_oracle(oracle_mod):
    case = V.CASES["laminar_partitioned"]()
    p = set_low_speed(CosaParams.from_buffer_copy(case.params), cutoff_type=3, visprec=True, epsp=(0.05, 0.05))
    O, _, (si, sj, sk), vol, vm = V._oracle_setup(oracle_mod, case)
    O.p = p
    q = V._prim_state(oracle_mod, O, case, si, sj, sk, seed=3)
    ctx, _, m, gvol, gvm = V._gpu_setup(case, p)
    cvo = oracle_mod.m1(O)
    oracle_mod.lm_viscoff(O, q, si, sj, sk, cvo)
    gcv = ctx.alloc_m1()
    ctx.lm_viscoff(1, ctx.alloc_p3().upload(q), m[0], m[1], m[2], gcv)
    assert _rel(gcv.download(), cvo) <= 1e-12
    ctx.close()
    # rest3 on a two-level set-up of the low-Mach channel
    c = _low_mach_channel(32, 16, 4)
    lv = cases.mg_levels(c, 2)
    Os = [oracle_mod.OracleLevel(t, p) for (t, _, _, _) in lv]
    vols = [Oi.metrics(x, y, z)[3] for Oi, (t, x, y, z) in zip(Os, lv)]
    c1 = np.random.default_rng(2).uniform(0, 1, Os[0].nm1)
    c2 = oracle_mod.m1(Os[1])
    oracle_mod.rest3(Os[0], Os[1], c1, c2, vols[0], vols[1])
    ctx = gpu.Context([t for (t, _, _, _) in lv], p)
    g2 = ctx.alloc_m1(2)
    ctx.rest3(1, ctx.alloc_m1(1).upload(c1), g2, ctx.alloc_p1(1).upload(vols[0]), ctx.alloc_p1(2).upload(vols[1]))
    assert _rel(g2.download(), c2) <= 1e-14
    ctx.close()


def _gpu_lsp_levels(lv, p, As):
    """M._gpu_levels plus the lambda scratch and residual the preconditioned
    stage uses."""
    ctx = gpu.Context([t for (t, _, _, _) in lv], p)
    D = []
    for nl, A in enumerate(As, start=1):
        d = {
            "q": ctx.alloc_p3(nl).upload(A.q), "qold": ctx.alloc_p3(nl), "res": ctx.alloc_p3(nl),
            "rhs": ctx.alloc_p3(nl).upload(A.rhs), "dtvol": ctx.alloc_p1(nl, ctx.S),
            "si": ctx.alloc_p2(nl).upload(A.si), "sj": ctx.alloc_p2(nl).upload(A.sj),
            "sk": ctx.alloc_p2(nl).upload(A.sk), "vol": ctx.alloc_p1(nl).upload(A.vol),
            "qp": ctx.alloc_p3(nl), "dq": ctx.alloc_p3(nl),
        }
        if p.irsop >= 2:
            for k in ("betaxi", "betaeta", "betazeta"):
                d[k] = ctx.alloc_p1(nl, ctx.S)
        ctx.bind_level(nl, **d)
        D.append(d)
    return ctx, D


@pytest.mark.parametrize("ctype,nlevel,irsop,epsp", [(2, 1, 0, (0.1,)), (2, 2, 0, (0.1, 0.2)), (3, 2, 0, (0.1, 0.2)),
                                                      (1, 2, 1, (0.1, 0.03)), (3, 2, 2, (0.1, 0.03)), (2, 1, 2, (0.1,))])
def test_lsp_cycles_match_oracle(oracle_mod, ctype, nlevel, irsop, epsp):
    case = _low_mach_channel(32, 16, 4, mach=0.1, partitioned=True)
    p = CosaParams.from_buffer_copy(case.params)
    p.nlevel, p.cfl = nlevel, 1.5
    set_low_speed(p, cutoff_type=ctype, epsp=epsp)
    if irsop:
        p.irsop, p.rat = irsop, float(np.sqrt(1 + 4 * 0.6))
        p.cfl = 1.5 * p.rat
    q = cases.perturbed_state(case, amp=0.01, seed=8)
    lv, Os, As = casekit.mg_oracle(case, nlevel, p, oracle_mod, q_fine=q)
    ctx, D = _gpu_lsp_levels(lv, p, As)
    ncyc = 4
    ho, st = oracle_mod.mg(Os, As, 1, ncyc, ncyc)
    assert st == 0
    hg, stg = ctx.mg(1, ncyc, ncyc)
    assert stg == 0
    for nl in range(nlevel):
        err = M._interior_rel(D[nl]["q"].download(), As[nl].q, lv[nl][0], 5, 1)
        assert err <= TOL * (10 if nl else 1), (nl, err)
    np.testing.assert_allclose(hg, ho, rtol=1e-9)
    # the level's own cut-offs (restricted from the fine level with type 3)
    for nl in range(nlevel):
        pg, vs = ctx.lsp_cutoffs(nl + 1)
        po, vo = oracle_mod.get_cutoffs(Os[nl])
        assert _rel(pg, po) <= 1e-12 if np.abs(po).max() > 0 else np.abs(pg).max() == 0.0
    ctx.close()


def test_laminar_lsp_cycles_with_viscous_cutoff(oracle_mod):
    case = V.CASES["laminar_partitioned"]()
    p = set_low_speed(CosaParams.from_buffer_copy(case.params), cutoff_type=2, visprec=True, epsp=(0.05,))
    O, _, (si, sj, sk), vol, vm = V._oracle_setup(oracle_mod, case)
    O.p = p
    q = cases.perturbed_state(case, amp=0.02, seed=5)
    qo = q.copy()
    ncyc = 5
    hist_o, st_o = oracle_mod.smooth_ns(O, qo, si, sj, sk, vol, vm, ncyc, rms_every=1)
    assert st_o == 0
    ctx, _, m, gvol, gvm = V._gpu_setup(case, p)
    dq_ = ctx.alloc_p3().upload(q)
    ctx.bind_level(1, q=dq_, qold=ctx.alloc_p3(), res=ctx.alloc_p3(), qp=ctx.alloc_p3(), dq=ctx.alloc_p3(),
                   dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2], vol=gvol)
    hist_g, st = ctx.smooth(1, ncyc, 1, 1)
    assert st == 0
    assert V._state_err(case, dq_.download(), qo) <= TOL
    np.testing.assert_allclose(hist_g, hist_o, rtol=1e-9)
    ctx.close()
