"""Parity of k-omega harmonic balance (sm_100a, through the C-ABI) with the
oracle: the routine-by-routine k-omega stage with all snapshots (src_bhb on
the seven equations, the snapshot-averaged norm), explicit and with the
implicit time-spectral update of update_bhb (its k-omega part: rho omega and
rho k snapshots coupled per cell), with IRS, and two-level multigrid cycles
(lim_res_ome_bhb on the residual pass).  States 1e-12 of the largest value
of each variable (coarse levels 1e-11), norms 1e-9.
"""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p3_views
from cosa_b200.params import CosaParams, set_harmonic_balance

import casekit
import test_gpu_mg as M

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("nharms,nlevel,rkimp,irsop", [(1, 1, 0, 0), (1, 1, 1, 0), (1, 1, 1, 1), (2, 2, 0, 0),
                                                       (1, 2, 1, 0)])
def test_kom_hb_cycles_match_oracle(oracle_mod, nharms, nlevel, rkimp, irsop):
    base = cases.turbulent_channel(32, 16, 4)
    p = CosaParams.from_buffer_copy(base.params)
    set_harmonic_balance(p, nharms, 0.16)
    S = 2 * nharms + 1
    p.rkimp, p.nlevel = rkimp, nlevel
    p.cfl = p.cflt = 1.0
    p.nstart = p.npre = p.npost = p.ncrs = 1
    p.bln_prol = 1
    if irsop:
        p.irsop, p.rat, p.ratt = irsop, float(np.sqrt(1 + 4 * 0.6)), float(np.sqrt(1 + 4 * 0.6))
        p.cfl = p.cflt = 1.0 * p.rat
    case = cases.turbulent_channel(32, 16, 4)
    case.params = p
    q = np.zeros(base.q0.size * S)
    for vo, vi in zip(p3_views(case.tables, q, 7, S), p3_views(case.tables, base.q0, 7, 1)):
        I = np.arange(vo.shape[0])[:, None, None]
        for n in range(S):
            vo[..., n] = vi[..., 0]
            vo[..., 1, n] *= 1 + 0.03 * np.sin(0.3 * I + 2 * np.pi * n / S)
    case.q0 = q
    lv, Os, As = casekit.mg_rans_oracle(case, nlevel, p, oracle_mod)
    ctx, D = M._gpu_levels_rans(lv, p, As)
    ncyc = 3
    ho, st = oracle_mod.mg_rans(Os, As, 1, ncyc, ncyc, rms_every=1)
    hg, stg = ctx.mg(1, ncyc, ncyc, rms_every=1)
    assert st == 0 and stg == 0
    for nl in range(nlevel):
        t = lv[nl][0]
        a = np.concatenate([cases.interior(v).reshape(-1, 7, S) for v in p3_views(t, D[nl]["q"].download(), 7, S)])
        b = np.concatenate([cases.interior(v).reshape(-1, 7, S) for v in p3_views(t, As[nl].q, 7, S)])
        sc = np.abs(b).max(axis=(0, 2))
        sc[3] = max(sc[3], sc[1:3].max())
        err = float((np.abs(a - b) / sc[None, :, None]).max())
        assert err <= TOL * (10 if nl else 1), (nl, err)
    np.testing.assert_allclose(hg, ho, rtol=1e-9, atol=1e-15)
    ctx.close()
