"""Known-answer tests of the oracle's k-omega harmonic balance
(src/update.f90 update_bhb with its k-omega part, lim_res_ome_bhb;
src/src.f90 src_bhb on all seven equations):

* with every snapshot equal the time-spectral term vanishes, so the
  harmonic-balance cycles (explicit, and rkimp with the snapshots coupled per
  cell) reproduce the steady k-omega cycles of one snapshot;
* with snapshot-dependent states the explicit and rkimp cycles, on one level
  and on two, run and differ on the way.
"""
import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p3_views
from cosa_b200.params import CosaParams, set_harmonic_balance

import casekit


def _hb_params(p, nharms, rkimp, nlevel):
    q = CosaParams.from_buffer_copy(p)
    set_harmonic_balance(q, nharms, 0.16)
    q.rkimp, q.nlevel = rkimp, nlevel
    return q


def _replicate(case, q1, S):
    """A one-snapshot state copied into every snapshot."""
    out = np.zeros(q1.size * S)
    for vo, vi in zip(p3_views(case.tables, out, 7, S), p3_views(case.tables, q1, 7, 1)):
        for n in range(S):
            vo[..., n] = vi[..., 0]
    return out


def _run(oracle_mod, case, p, ncyc, q_fine=None):
    lv, Os, As = casekit.mg_rans_oracle(case, p.nlevel, p, oracle_mod)
    if q_fine is not None:
        As[0].q[:] = q_fine
    h, st = oracle_mod.mg_rans(Os, As, 1, ncyc, ncyc, rms_every=1)
    return As, h, st


def test_equal_snapshots_reduce_to_steady(oracle_mod):
    case = cases.turbulent_channel(24, 12, 4)
    ps = case.params
    ps.cfl = ps.cflt = 1.0
    ps.nlevel = 1
    As, hs, st = _run(oracle_mod, case, ps, 4)
    assert st == 0
    qs = As[0].q
    S = 3
    for rkimp in (0, 1):
        p = _hb_params(ps, 1, rkimp, 1)
        hcase = cases.turbulent_channel(24, 12, 4)
        hcase.params = p
        hcase.q0 = _replicate(case, case.q0, S)
        Ah, hh, st = _run(oracle_mod, hcase, p, 4)
        assert st == 0
        for v_h, v_s in zip(p3_views(case.tables, Ah[0].q, 7, S), p3_views(case.tables, qs, 7, 1)):
            a, b = cases.interior(v_h), cases.interior(v_s)
            sc = np.abs(b).reshape(-1, 7).max(axis=0)
            sc[3] = max(sc[3], sc[1:3].max())
            for n in range(S):
                err = (np.abs(a[..., n] - b[..., 0]) / sc[None, None, None, :]).max()
                assert err <= 1e-10, (rkimp, n, err)
        np.testing.assert_allclose(hh[:, 0], hs[:, 0], rtol=1e-8)


def test_snapshot_dependent_cycles_run(oracle_mod):
    case = cases.turbulent_channel(24, 12, 4)
    S = 3
    out = {}
    for nlevel in (1, 2):
        for rkimp in (0, 1):
            p = _hb_params(case.params, 1, rkimp, nlevel)
            p.cfl = p.cflt = 1.0
            p.nstart = p.npre = p.npost = p.ncrs = 1
            hcase = cases.turbulent_channel(24, 12, 4)
            hcase.params = p
            q = _replicate(case, case.q0, S)
            for v in p3_views(hcase.tables, q, 7, S):
                I = np.arange(v.shape[0])[:, None, None]
                for n in range(S):
                    v[..., 1, n] *= 1 + 0.03 * np.sin(0.3 * I + 2 * np.pi * n / S)
            hcase.q0 = q
            Ah, h, st = _run(oracle_mod, hcase, p, 30)
            assert st == 0, (nlevel, rkimp)
            assert np.isfinite(Ah[0].q).all()
            out[(nlevel, rkimp)] = Ah[0].q.copy()
    assert np.abs(out[(1, 1)] - out[(1, 0)]).max() > 1e-8
