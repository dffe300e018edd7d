"""Known-answer tests of the oracle's BSL and SST k-omega variants
(src/update.f90 update_ttrm_b / tur_vis_sst_b, src/src.f90 srckw_sst_b,
src/flux.f90 vflux BSL/SST branch, src/grid.f90 facedist_b):

* the face distances follow facedist_b's averages and boundary copies;
* ttrm (the blended gamma, beta and cross diffusion) and F1 follow their
  closed forms for linear k and omega fields on a uniform box;
* the SST eddy viscosity of a simple shear follows a1 rho k / max(a1 omega,
  |du/dy| F2);
* the SST omega source adds the cross-diffusion term;
* with F1 = 1 everywhere (zero wall distance, no viscous walls) the BSL
  constants reduce to Wilcox's, so BSL cycles equal Wilcox k-omega cycles
  bit for bit;
* BSL and SST cycles on the viscous channel stay finite; SST converges.
"""
import math

import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p1_views, p3_views, f0_views
from cosa_b200.params import CosaParams

from test_oracle_kom import DX, DY, DZ, _box, _setup


def _variant(p, which):
    q = CosaParams.from_buffer_copy(p)
    q.kom, q.kom_bsl, q.kom_sst = (1, 0, 0) if which == "wilcox" else (0, int(which == "bsl"), int(which == "sst"))
    return q


def _blend(p, sst):
    bstr, kap = 0.09, p.kappa
    c = dict(sigk1=0.85 if sst else 0.5, sigk2=1.0, sigw1=0.5, sigw2=0.856, b1=3.0 / 40.0, b2=0.0828, a1=0.31)
    c["g1"] = c["b1"] / bstr - c["sigw1"] * kap * kap / math.sqrt(bstr)
    c["g2"] = c["b2"] / bstr - c["sigw2"] * kap * kap / math.sqrt(bstr)
    return c


def _tanh(a):
    return (np.exp(2 * a) - 1) / (np.exp(2 * a) + 1)


def test_facedist(oracle_mod):
    case = _box(_variant(cases.kom_params(), "bsl"))
    O, A = _setup(oracle_mod, case)
    rng = np.random.default_rng(3)
    A.dist[:] = rng.uniform(0.1, 1.0, A.dist.size)
    fd = np.zeros(3 * O.n0)
    oracle_mod.facedist(O, A.dist, fd)
    d = p1_views(case.tables, A.dist, 1)[0][..., 0]
    (im, jm, km), = case.tables.dims
    F = [fd[m * O.n0:(m + 1) * O.n0].reshape((im, jm, km), order="F") for m in range(3)]
    # family 1 at interior j, k: boundary faces copy the halo cell, inner faces average
    np.testing.assert_array_equal(F[0][0, :jm - 1, :km - 1], d[0, 1:jm, 1:km])
    np.testing.assert_array_equal(F[0][im - 1, :jm - 1, :km - 1], d[im, 1:jm, 1:km])
    np.testing.assert_allclose(F[0][1:im - 1, :jm - 1, :km - 1], (d[1:im - 1, 1:jm, 1:km] + d[2:im, 1:jm, 1:km]) / 2,
                               rtol=1e-15)
    np.testing.assert_allclose(F[1][:im - 1, 1:jm - 1, :km - 1], (d[1:im, 1:jm - 1, 1:km] + d[1:im, 2:jm, 1:km]) / 2,
                               rtol=1e-15)
    np.testing.assert_array_equal(F[2][:im - 1, :jm - 1, km - 1], d[1:im, 1:jm, km])


def _linear_kw_state(case, O, rho=1.1, pr=0.7, k0=2e-3, kx=1e-3, ky=5e-3, w0=3.0, wx=-0.5, wy=2.0):
    """Primitive state with k and omega linear in x and y (cell centres)."""
    q = O.p3()
    for v in p3_views(case.tables, q, 7, 1):
        I = (np.arange(v.shape[0]) - 1.5) * DX
        J = (np.arange(v.shape[1]) - 1.5) * DY
        v[..., 0, 0] = rho
        v[..., 4, 0] = pr
        v[..., 5, 0] = k0 + kx * I[:, None, None] + ky * J[None, :, None]
        v[..., 6, 0] = w0 + wx * I[:, None, None] + wy * J[None, :, None]
    return q


def test_update_ttrm_closed_form(oracle_mod):
    for which in ("bsl", "sst"):
        case = _box(_variant(cases.kom_params(), which))
        p = case.params
        O, A = _setup(oracle_mod, case)
        rng = np.random.default_rng(4)
        A.dist[:] = rng.uniform(0.01, 0.5, A.dist.size)
        q = _linear_kw_state(case, O)
        grads = []
        for d in (1, 2, 3):
            qf, dc = O.p3(), O.p3()
            oracle_mod.q_face(O, d, q, qf)
            oracle_mod.q_der_c(O, d, qf, dc)
            grads.append(dc)
        ttrm = np.zeros(O.n3 * 3)
        oracle_mod.update_ttrm(O, q, *grads, A.vm, ttrm, A.dist)
        (im, jm, km), = case.tables.dims
        c = _blend(p, which == "sst")
        # interior cells away from the box faces (q_face keeps halo values there)
        sl = (slice(2, im - 1), slice(2, jm - 1), slice(1, km))
        v = p3_views(case.tables, q, 7, 1)[0]
        rho, pr = v[..., 0, 0][3:-3, 3:-3, 2:-2], v[..., 4, 0][3:-3, 3:-3, 2:-2]
        tke, ome = v[..., 5, 0][3:-3, 3:-3, 2:-2], v[..., 6, 0][3:-3, 3:-3, 2:-2]
        dd = p1_views(case.tables, A.dist, 1)[0][..., 0][sl] + p.epst
        t = p.gamma * pr / rho
        mu = (p.stemp + 1) / (t + p.stemp) * t ** 1.5
        dkdx, dkdy, dwdx, dwdy = 1e-3, 5e-3, -0.5, 2.0
        arg1 = np.maximum(np.sqrt(tke) / 0.09 / ome / dd, 500 * mu / rho / ome / dd ** 2 * p.machfs / p.reyno)
        cdt = 2 * rho * c["sigw2"] / ome * (dkdx * dwdx + dkdy * dwdy)
        arg1 = np.minimum(arg1, 4 * rho * c["sigw2"] * tke / np.maximum(cdt, 1e-20) / dd ** 2)
        f1 = _tanh(np.minimum(arg1 ** 4, 100.0))
        T = ttrm.reshape(3, km + 3, jm + 3, im + 3).transpose(3, 2, 1, 0)[3:-3, 3:-3, 2:-2]
        np.testing.assert_allclose(T[..., 1], f1 * c["g1"] + (1 - f1) * c["g2"], rtol=1e-10)
        np.testing.assert_allclose(T[..., 2], f1 * c["b1"] + (1 - f1) * c["b2"], rtol=1e-10)
        np.testing.assert_allclose(T[..., 0], cdt * (1 - f1), rtol=1e-9, atol=1e-14)
        assert ((f1 > 0.05) & (f1 < 0.95)).sum() > 10  # the blend is exercised, not saturated


def test_tur_vis_sst_of_a_shear(oracle_mod):
    case = _box(_variant(cases.kom_params(), "sst"))
    p = case.params
    O, A = _setup(oracle_mod, case)
    rng = np.random.default_rng(5)
    A.dist[:] = rng.uniform(0.01, 0.5, A.dist.size)
    cs = 40.0
    rho, k, w, e = 1.2, 3e-3, 2.0, 2.5
    q = O.p3()
    for v in p3_views(case.tables, q, 7, 1):
        J = (np.arange(v.shape[1]) - 1.5) * DY
        v[..., 0, 0] = 1.0
        v[..., 1, 0] = cs * J[None, :, None]
    grads = []
    for d in (1, 2, 3):
        qf, dc = O.p3(), O.p3()
        oracle_mod.q_face(O, d, q, qf)
        oracle_mod.q_der_c(O, d, qf, dc)
        grads.append(dc)
    qc = O.p3()  # conservative state of the eddy-viscosity evaluation
    for v in p3_views(case.tables, qc, 7, 1):
        v[..., 0, 0] = rho
        v[..., 4, 0] = e
        v[..., 5, 0] = rho * k
        v[..., 6, 0] = rho * w
    mut = np.zeros(O.n3)
    oracle_mod.tur_vis_sst(O, qc, mut, *grads, A.vm, A.dist)
    (im, jm, km), = case.tables.dims
    c = _blend(p, True)
    sl = (slice(2, im - 1), slice(2, jm - 1), slice(1, km))
    dd = p1_views(case.tables, A.dist, 1)[0][..., 0][sl] + p.epst
    pr = (p.gamma - 1) * (e - rho * k)
    t = p.gamma * pr / rho
    mu = (p.stemp + 1) / (t + p.stemp) * t ** 1.5
    arg2 = np.maximum(2 * math.sqrt(k) / 0.09 / w / dd, 500 * mu / rho / w / dd ** 2 * p.machfs / p.reyno)
    f2 = _tanh(np.minimum(arg2 ** 2, 100.0))
    ref = c["a1"] * rho * k / np.maximum(c["a1"] * w, cs * f2) * p.reyno / p.machfs
    M = mut.reshape(km + 3, jm + 3, im + 3).T
    np.testing.assert_allclose(M[3:-3, 3:-3, 2:-2], ref, rtol=1e-11)
    assert (cs * f2 > c["a1"] * w).any()  # the limiter is active somewhere
    # the face halos copy the adjacent cell
    np.testing.assert_array_equal(M[2:-2, 1, 2:-2], M[2:-2, 2, 2:-2])


def test_srckw_sst_closed_form(oracle_mod):
    case = _box(_variant(cases.kom_params(), "sst"))
    p = case.params
    O, A = _setup(oracle_mod, case)
    rho, k, w, mut, prod, cdif, gav, bav = 1.2, 2e-3, 3.0, 5.0, 0.4, 0.07, 0.5, 0.08
    q = O.p3()
    for v in p3_views(case.tables, q, 7, 1):
        v[..., 0, 0] = rho
        v[..., 4, 0] = 0.7
        v[..., 5, 0] = k
        v[..., 6, 0] = w
    ttrm = np.zeros(O.n3 * 3)
    T = ttrm.reshape(3, O.n3)
    T[0], T[1], T[2] = cdif, gav, bav
    res = O.p3()
    oracle_mod.srckw_sst(O, 1, q, np.full(O.n3, mut), np.full(O.n3, prod), np.zeros(O.n3), res, ttrm, A.vol)
    mor = p.machfs / p.reyno
    V = DX * DY * DZ
    r = p3_views(case.tables, res, 7, 1)[0][2:-2, 2:-2, 2:-2]
    np.testing.assert_allclose(r[..., 5, 0], -V * (mor * mut * prod - p.bstrkw * rho * k * w), rtol=1e-12)
    np.testing.assert_allclose(r[..., 6, 0], -V * (gav * p.cmu * rho * prod - bav * rho * w * w + cdif), rtol=1e-12)


def _kw_channel(params):
    """The partitioned channel with slip walls (no wall-distance terms in the
    BCs) and a perturbed k-omega state."""
    case = cases.partitioned_channel(24, 12, 2, isplit=(10,), jsplit=(5,), kface_bc=4, wall=14, params=params)
    q = case.q0.copy()
    for v in p3_views(case.tables, q, 7, 1):
        I = np.arange(v.shape[0])[:, None, None]
        J = np.arange(v.shape[1])[None, :, None]
        v[..., 1, 0] *= 1 + 0.05 * np.sin(0.4 * I + 0.7 * J)
        v[..., 5, 0] *= 1 + 0.3 * np.sin(0.4 * I - 0.2 * J)
        v[..., 6, 0] *= 1 + 0.2 * np.cos(0.3 * I + 0.5 * J)
    return case, q


def _run(oracle_mod, case, q, ncyc, dist=None):
    O, A = _setup(oracle_mod, case)
    if dist is not None:
        A.dist[:] = dist
    A.q[:] = q
    qq = A.q.copy()
    O.cons2prim(qq)
    oracle_mod.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist)
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle_mod.tur_vis(O, qq, A.mut)
    oracle_mod.cutman_mut(O, A.mut)
    hist, st = oracle_mod.smooth_rans(O, A, ncyc, rms_every=max(1, ncyc // 4))
    return A, hist, st


def test_bsl_with_unit_blending_is_wilcox(oracle_mod):
    pw = cases.kom_params(reyno=1.0e5)
    out = {}
    for which in ("wilcox", "bsl"):
        case, q = _kw_channel(_variant(pw, which))
        A, hist, st = _run(oracle_mod, case, q, 6, dist=0.0)
        assert st == 0
        out[which] = (A.q.copy(), A.mut.copy(), hist)
    np.testing.assert_array_equal(out["bsl"][0], out["wilcox"][0])
    np.testing.assert_array_equal(out["bsl"][1], out["wilcox"][1])


def test_bsl_and_sst_channel_cycles(oracle_mod):
    """The viscous channel with the wall distance: BSL and SST stay finite
    over 100 cycles, and SST drops its residual tenfold in 400 (Wilcox and
    BSL lose positivity on this grid at CFL 1 after a few hundred cycles)."""
    for which, ncyc in (("bsl", 100), ("sst", 400)):
        case = cases.turbulent_channel(24, 12, 2)
        case.params = _variant(case.params, which)
        case.params.cfl = case.params.cflt = 1.0
        A, hist, st = _run(oracle_mod, case, case.q0.copy(), ncyc, dist=cases.wall_distance(case))
        assert st == 0
        rows = hist[~np.isnan(hist[:, 0])]
        assert np.isfinite(A.q).all() and np.isfinite(A.mut).all()
        if which == "sst":
            assert rows[-1, 0] < 0.1 * rows[0, 0], rows[:, 0]
