"""Known-answer tests of the oracle's multigrid pieces (src/cosa.f90:2672-3889,
src/flux.f90:3132-4263): exactness of the edge/corner extrapolation and of
the transfer operators on fields they must reproduce, and the FAS identity
that an unsmoothed coarse level prolongs a zero correction."""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p3_views

import casekit


def _linear_fill(O, q, coef):
    """q(i,j,k,v,n) = c0 + c1 i + c2 j + c3 k (+ v, n offsets) on every cell."""
    for v in p3_views(O.t, q, O.p.npde, O.S):
        I, J, K = v.shape[:3]
        i = np.arange(-1, I - 1)[:, None, None]
        j = np.arange(-1, J - 1)[None, :, None]
        k = np.arange(-1, K - 1)[None, None, :]
        for var in range(O.p.npde):
            for n in range(O.S):
                v[..., var, n] = coef[0] + var + 0.5 * n + coef[1] * i + coef[2] * j + coef[3] * k


def _edge_corner_mask(dims):
    im, jm, km = dims
    i = np.arange(-1, im + 2)[:, None, None]
    j = np.arange(-1, jm + 2)[None, :, None]
    k = np.arange(-1, km + 2)[None, None, :]
    oi = (i == 0) | (i == im)
    oj = (j == 0) | (j == jm)
    ok = (k == 0) | (k == km)
    ii = (i >= 1) & (i <= im - 1)
    jj = (j >= 1) & (j <= jm - 1)
    kk = (k >= 1) & (k <= km - 1)
    edges = (oi & oj & kk) | (oi & jj & ok) | (ii & oj & ok)
    corners = oi & oj & ok
    return edges, corners


@pytest.mark.parametrize("with_mut", [False, True])
def test_edges_corners_reproduce_linear_fields(oracle_mod, with_mut):
    """A plane through neighbours reproduces any field linear in (i,j,k)."""
    case = casekit.small_partitioned(permute=True)
    p = case.params
    O = oracle_mod.OracleLevel(case.tables, p)
    q = O.p3()
    coef = (1.0, 0.03, -0.07, 0.11)
    _linear_fill(O, q, coef)
    ref = q.copy()
    mut = None
    if with_mut:
        mut = np.zeros(O.n3 * O.S)
        off, _ = case.tables.offsets()
        for b, (im, jm, km) in enumerate(case.tables.dims):
            n = (im + 3) * (jm + 3) * (km + 3)
            for s in range(O.S):
                v = mut[off["p3"][b] * O.S + s * n: off["p3"][b] * O.S + (s + 1) * n].reshape(
                    (im + 3, jm + 3, km + 3), order="F")
                v[:] = 2.0 + 0.01 * np.arange(-1, im + 2)[:, None, None] + 0.02 * np.arange(-1, km + 2)[None, None, :]
        mref = mut.copy()
    # spoil every edge and corner cell
    for v, (im, jm, km) in zip(p3_views(case.tables, q, p.npde, O.S), case.tables.dims):
        e, c = _edge_corner_mask((im, jm, km))
        v[e | c] = -77.0
    oracle_mod.q_edges(O, q, mut)
    oracle_mod.q_corns(O, q, mut)
    for v, r, (im, jm, km) in zip(p3_views(case.tables, q, p.npde, O.S), p3_views(case.tables, ref, p.npde, O.S),
                                  case.tables.dims):
        e, c = _edge_corner_mask((im, jm, km))
        np.testing.assert_allclose(v[e | c], r[e | c], rtol=0, atol=1e-12)
    if with_mut:
        np.testing.assert_allclose(mut, mref, rtol=0, atol=1e-12)


def _two_levels(oracle_mod, case, nlevel=2):
    p = case.params
    lv = cases.mg_levels(case, nlevel)
    Os = [oracle_mod.OracleLevel(t, p) for (t, _, _, _) in lv]
    return lv, Os


def test_rest1_rest2_values(oracle_mod):
    case = casekit.small_channel(32, 16, 4)
    lv, (Of, Oc) = _two_levels(oracle_mod, case)
    rng = np.random.default_rng(3)
    q1 = rng.uniform(0.5, 2.0, Of.p3().size)
    v1 = rng.uniform(0.5, 1.5, Of.p1().size)
    v2 = rng.uniform(4.0, 12.0, Oc.p1().size)
    q2 = Oc.p3()
    oracle_mod.rest1(Of, Oc, q1, q2, v1, v2)
    rhs2 = Oc.p3()
    oracle_mod.rest2(Of, Oc, rhs2, q1)
    p = case.params
    F = p3_views(lv[0][0], q1, p.npde, 1)[0]
    C = p3_views(lv[1][0], q2, p.npde, 1)[0]
    R = p3_views(lv[1][0], rhs2, p.npde, 1)[0]
    V1 = cases.p1_views(lv[0][0], v1)[0][..., 0]
    V2 = cases.p1_views(lv[1][0], v2)[0][..., 0]
    im2, jm2, km2 = lv[1][0].dims[0]
    for i2 in range(1, im2):
        for j2 in range(1, jm2):
            for k2 in range(1, km2):
                sl = (slice(2 * i2 - 1 + 1, 2 * i2 + 1 + 1), slice(2 * j2 - 1 + 1, 2 * j2 + 1 + 1),
                      slice(2 * k2 - 1 + 1, 2 * k2 + 1 + 1))
                vs = V1[2 * i2 - 1:2 * i2 + 1, 2 * j2 - 1:2 * j2 + 1, 2 * k2 - 1:2 * k2 + 1]
                for var in range(p.npde):
                    f = F[sl + (var, 0)]
                    np.testing.assert_allclose(C[i2 + 1, j2 + 1, k2 + 1, var, 0], (vs * f).sum() / V2[i2, j2, k2],
                                               rtol=1e-14)
                    np.testing.assert_allclose(R[i2 + 1, j2 + 1, k2 + 1, var, 0], -f.sum(), rtol=1e-14)


def test_rest2_ho_weights(oracle_mod):
    """rest2_ho_b (src/cosa.f90:2871-2954): the 27/9/3/1 weights sum to 512,
    so a constant residual c restricts to -8 c like rest2_lo; the stencil is
    symmetric about the centre of the 2x2x2 fine cells, so a field linear in
    the cell indices (halos included) restricts to -8 x its value there."""
    case = casekit.small_channel(32, 16, 8)
    lv, (Of, Oc) = _two_levels(oracle_mod, case)
    p = case.params
    for kind in ("const", "linear"):
        r1 = Of.p3()
        for v in p3_views(lv[0][0], r1, p.npde, 1):
            ii, jj, kk = np.meshgrid(*(np.arange(n) - 1.0 for n in v.shape[:3]), indexing="ij")
            for var in range(p.npde):
                v[..., var, 0] = 0.7 + var if kind == "const" else 0.3 + 0.11 * ii - 0.07 * jj + 0.05 * kk + var
        rhs2 = Oc.p3()
        oracle_mod.rest2_ho(Of, Oc, rhs2, r1)
        R = p3_views(lv[1][0], rhs2, p.npde, 1)[0]
        im2, jm2, km2 = lv[1][0].dims[0]
        for i2 in range(1, im2):
            for j2 in range(1, jm2):
                for k2 in range(1, km2):
                    ic, jc, kc = 2 * i2 - 0.5, 2 * j2 - 0.5, 2 * k2 - 0.5
                    for var in range(p.npde):
                        want = 0.7 + var if kind == "const" else 0.3 + 0.11 * ic - 0.07 * jc + 0.05 * kc + var
                        np.testing.assert_allclose(R[i2 + 1, j2 + 1, k2 + 1, var, 0], -8 * want, rtol=1e-13)


def test_bc_res_first_layer(oracle_mod):
    """bc_res (src/bc.f90:2802-2995): the first halo layer of every patch is
    the first interior cell, negated on 15xx walls; nothing else changes."""
    case = cases.duct3d(segs=cases.duct_segments(seed=5, lo=20_000, hi=60_000, choices=tuple(range(8, 33, 8))),
                        wall=cases.VISCOUS_WALL)
    p = case.params
    O = oracle_mod.OracleLevel(case.tables, p)
    rng = np.random.default_rng(4)
    r = rng.standard_normal(O.p3().size)
    r0 = r.copy()
    oracle_mod.bc_res(O, r)
    t = case.tables
    off = 0
    changed = np.zeros(r.size, dtype=bool)
    for b, (v, v0) in enumerate(zip(p3_views(t, r, p.npde, 1), p3_views(t, r0, p.npde, 1))):
        for rec in t.bctopo[t.nbcs[:b].sum():t.nbcs[:b + 1].sum()]:
            typ, idir, inrout = rec[0], rec[1], rec[2]
            lo = [rec[3], rec[5], rec[7]]
            hi = [rec[4], rec[6], rec[8]]
            pm = -1.0 if typ // 100 == 15 else 1.0
            dims = t.dims[b]
            sl_h, sl_c = [], []
            for d in range(3):
                if d == idir - 1:
                    h = 0 if inrout == 1 else dims[d]
                    c = 1 if inrout == 1 else dims[d] - 1
                    sl_h.append(slice(h + 1, h + 2)); sl_c.append(slice(c + 1, c + 2))
                else:
                    sl_h.append(slice(lo[d] + 1, hi[d] + 2)); sl_c.append(slice(lo[d] + 1, hi[d] + 2))
            np.testing.assert_array_equal(v[tuple(sl_h)], pm * v0[tuple(sl_c)])
    # interior cells untouched
    for v, v0 in zip(p3_views(t, r, p.npde, 1), p3_views(t, r0, p.npde, 1)):
        np.testing.assert_array_equal(cases.interior(v), cases.interior(v0))


def test_prol_bln_reproduces_linear_corrections(oracle_mod):
    """27/9/3/1 weights: constant corrections pass unchanged and corrections
    linear in the coarse index reproduce the line through the fine centres."""
    case = casekit.small_channel(32, 16, 4)
    lv, (Of, Oc) = _two_levels(oracle_mod, case)
    p = case.params
    q2 = Oc.p3()
    a, b, c = 0.1, -0.05, 0.02
    C = p3_views(lv[1][0], q2, p.npde, 1)[0]
    i2 = np.arange(-1, C.shape[0] - 1)[:, None, None]
    j2 = np.arange(-1, C.shape[1] - 1)[None, :, None]
    k2 = np.arange(-1, C.shape[2] - 1)[None, None, :]
    for var in range(p.npde):
        C[..., var, 0] = 1.0 + var + a * i2 + b * j2 + c * k2
    q1 = Of.p3()
    oracle_mod.prol_bln(Of, Oc, q1, q2)
    F = p3_views(lv[0][0], q1, p.npde, 1)[0]
    im1, jm1, km1 = lv[0][0].dims[0]
    # coarse cell i2 spans fine cells 2 i2 - 1, 2 i2: centre at fine 2 i2 - 1/2
    i1 = np.arange(0, im1 + 1)[:, None, None]
    j1 = np.arange(0, jm1 + 1)[None, :, None]
    k1 = np.arange(0, km1 + 1)[None, None, :]
    for var in range(p.npde):
        want = 1.0 + var + a * (i1 + 0.5) / 2 + b * (j1 + 0.5) / 2 + c * (k1 + 0.5) / 2
        np.testing.assert_allclose(F[1:im1 + 2, 1:jm1 + 2, 1:km1 + 2, var, 0], want, rtol=0, atol=1e-13)


def test_prol_lin_constant_correction(oracle_mod):
    case = casekit.small_channel(32, 16, 4)
    lv, (Of, Oc) = _two_levels(oracle_mod, case)
    p = case.params
    q2 = Oc.p3() + 0.25
    q1 = Of.p3()
    vol1 = np.random.default_rng(2).uniform(0.5, 2.0, Of.p1().size)
    oracle_mod.prol_lin(Of, Oc, q1, q2, vol1)
    F = p3_views(lv[0][0], q1, p.npde, 1)[0]
    im1, jm1, km1 = lv[0][0].dims[0]
    np.testing.assert_allclose(F[1:im1 + 2, 1:jm1 + 2, 1:km1 + 2], 0.25, rtol=0, atol=1e-15)


@pytest.mark.parametrize("which", ["channel", "partitioned"])
def test_fas_zero_correction(oracle_mod, which):
    """restrict then prolong with no coarse smoothing leaves the fine state
    unchanged: q2 and qold2 are the same restriction through the same BCs."""
    case = casekit.small_channel(32, 16, 4) if which == "channel" else casekit.small_partitioned(32, 16, 4)
    p = case.params
    p.nlevel = 2
    q = cases.perturbed_state(case, amp=0.01, seed=4)
    lv, Os, As = casekit.mg_oracle(case, 2, p, oracle_mod, q_fine=q)
    Of, Oc = Os
    row, st = oracle_mod.smooth_level(Of, 1, As[0], 1, False, True)
    assert st == 0
    assert oracle_mod.restrict(Of, Oc, As[0], As[1]) == 0
    before = As[0].q.copy()
    assert oracle_mod.prolong(Of, Oc, As[0], As[1]) == 0
    F0 = casekit.interior_cells(case, before, p.npde)
    F1 = casekit.interior_cells(case, As[0].q, p.npde)
    np.testing.assert_array_equal(F1, F0)


def test_mg_beats_single_grid(oracle_mod):
    """Three-level V-cycles reduce the residual further than as many
    single-grid cycles (bump channel, CFL 1)."""
    case = casekit.small_channel(32, 16, 4)
    p = case.params
    p.cfl = 1.0
    p.nlevel = 3
    lv, Os, As = casekit.mg_oracle(case, 3, p, oracle_mod)
    h3, st = oracle_mod.mg(Os, As, 1, 40, 40)
    assert st == 0
    p1 = cases.channel_params()
    p1.cfl = 1.0
    O1 = oracle_mod.OracleLevel(case.tables, p1)
    si, sj, sk, vol = O1.metrics(case.x, case.y, case.z)
    q = case.q0.copy()
    h1, st1 = O1.smooth(q, si, sj, sk, 40)
    assert st1 == 0
    assert np.isfinite(h3[-1, -1])
    assert h3[-1, -1] < 0.7 * h1[-1, -1], (h3[-1, -1], h1[-1, -1])


def test_lu_solve_matches_numpy(oracle_mod):
    """The partial-pivot LU of update_bhb (DGETF2/DGETRS order) solves random
    systems, pivoting included, to rounding."""
    rng = np.random.default_rng(3)
    for n in (3, 5, 7, 15):
        a = rng.standard_normal((n, n))
        b = rng.standard_normal((n, 5))
        x = oracle_mod.lu_solve(a, b)
        np.testing.assert_allclose(a @ x, b, rtol=0, atol=1e-12 * np.abs(b).max() * n)


def test_implicit_hb_update(oracle_mod):
    """rkimp (no IRS, one level): with every snapshot equal the time-spectral
    term vanishes and the implicit update equals the explicit one; with
    snapshot-dependent states both converge and differ on the way."""
    from cosa_b200.params import set_harmonic_balance
    case = casekit.small_partitioned()
    p = set_harmonic_balance(case.params, 1, 0.16)
    case.q0 = cases._freestream_state(case.tables, p)
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    out = {}
    for imp in (0, 1):
        p.rkimp = imp
        q = cases.perturbed_state(case, seed=4)  # the same perturbation in every snapshot
        h, st = oracle_mod.smooth_hb(O, q, si, sj, sk, vol, 5, rms_every=1)
        assert st == 0
        out[imp] = (q, h)
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=0, atol=1e-12)
    np.testing.assert_allclose(out[1][1], out[0][1], rtol=1e-10)
    qs = {}
    for imp in (0, 1):
        p.rkimp = imp
        q = cases.perturbed_state(case, seed=4)
        for v in cases.p3_views(case.tables, q, 5, 3):
            for n in range(3):
                v[..., 1, n] *= 1 + 0.05 * np.sin(2 * np.pi * n / 3)
        h, st = oracle_mod.smooth_hb(O, q, si, sj, sk, vol, 300, rms_every=100)
        rows = h[~np.isnan(h[:, 0])]
        assert st == 0 and rows[-1, 0] < 0.5 * rows[0, 0]
        qs[imp] = q
    assert np.abs(qs[1] - qs[0]).max() > 1e-6


def test_implicit_hb_update_irs_branch(oracle_mod):
    """rkimp with IRS (src/update.f90:1771-1836): src_hb's term enters the
    residual and update_bhb takes it out again.  With a smoothing
    coefficient of zero (rat = 1) IRS is the identity, so the IRS branch must
    reproduce the branch without IRS to rounding; with rat > 1 both converge
    and differ on the way."""
    from cosa_b200.params import set_harmonic_balance
    case = casekit.small_partitioned()
    p = set_harmonic_balance(case.params, 1, 0.16)
    p.rkimp = 1
    case.q0 = cases._freestream_state(case.tables, p)
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)

    def state():
        q = cases.perturbed_state(case, seed=4)
        for v in cases.p3_views(case.tables, q, 5, 3):
            for n in range(3):
                v[..., 1, n] *= 1 + 0.05 * np.sin(2 * np.pi * n / 3)
        return q

    out = {}
    for irsop, rat in ((0, 1.0), (1, 1.0), (1, 1.6)):
        p.irsop, p.rat, p.cutcirs = irsop, rat, 0
        q = state()
        h, st = oracle_mod.smooth_hb(O, q, si, sj, sk, vol, 40, rms_every=10)
        assert st == 0
        out[(irsop, rat)] = (q, h)
    q0, h0 = out[(0, 1.0)]
    q1, h1 = out[(1, 1.0)]
    np.testing.assert_allclose(q1, q0, rtol=0, atol=1e-12)
    rows = ~np.isnan(h0[:, 0])
    # the norms differ by design: without IRS the term is added back to the
    # unsmoothed residual, with IRS the residual already holds it
    np.testing.assert_allclose(h1[rows], h0[rows], rtol=1e-8)
    q2, h2 = out[(1, 1.6)]
    assert np.isfinite(q2).all() and np.abs(q2 - q0).max() > 1e-8
    r2 = h2[~np.isnan(h2[:, 0])]
    assert r2[-1, 0] < r2[0, 0]
