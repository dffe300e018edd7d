"""Known-answer tests of the oracle's low-speed preconditioning (lomach):
the cut-offs of src/losp.f90, blsp's preconditioner and prec_bres, the
preconditioned Roe flux proflux_b (src/flux.f90:390-830), the preconditioned
spectral radii (eig_eul_p, src/cosa.f90:4300-4372) and the lomach branches of
bc_far1 / bc_insub (src/bc.f90):

* with the constant cut-off epsp = 1 the preconditioned Mach number is 1:
  the preconditioner is the identity, proflux is roflux, the preconditioned
  spectral radii and the boundary characteristics are the plain ones, so
  two-level multigrid cycles match the unpreconditioned cycles to rounding;
* prec times the inverse the reference writes out in blsp's debug branch
  (src/losp.f90:196-300) is the identity;
* the pressure-gradient cut-off of a uniform state is zero and of a single
  pressure jump is the jump over rho a^2; rest3 keeps a constant field;
* with equal face states proflux is the physical flux, and its dissipation
  is P^-1 |P A| (q_R - q_L) with P blsp's preconditioner and A the flux
  Jacobian, both at the Roe-averaged state (the preconditioned Roe scheme);
* a low-Mach channel is driven further down by the preconditioned cycles.
"""
import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p3_views
from cosa_b200.params import CosaParams, set_low_speed

import casekit


def _lsp(p, **kw):
    q = CosaParams.from_buffer_copy(p)
    return set_low_speed(q, **kw)


def test_unit_cutoff_matches_plain_cycles(oracle_mod):
    case = casekit.small_channel(32, 16, 4)
    q0 = cases.perturbed_state(case, amp=0.01, seed=3)
    out = {}
    for lsp in (0, 1):
        p = CosaParams.from_buffer_copy(case.params)
        p.nlevel, p.cfl = 2, 1.0
        if lsp:
            set_low_speed(p, cutoff_type=2, epsp=(1.0, 1.0, 1.0))
        lv, Os, As = casekit.mg_oracle(case, 2, p, oracle_mod, q_fine=q0)
        h, st = oracle_mod.mg(Os, As, 1, 5, 5)
        assert st == 0
        out[lsp] = (As[0].q.copy(), h)
    (qa, ha), (qb, hb) = out[0], out[1]
    assert np.abs(qa - qb).max() <= 1e-13 * np.abs(qa).max()
    np.testing.assert_allclose(hb, ha, rtol=1e-11)


def _preci(q, mp2, g, kom=False):
    """The inverse preconditioner as blsp's debug branch writes it."""
    n = 7 if kom else 5
    rho, u, v, w = q[0], q[1] / q[0], q[2] / q[0], q[3] / q[0]
    q2, e0 = u * u + v * v + w * w, q[4] / rho
    tke = q[5] / rho if kom else 0.0
    p = (g - 1) * (e0 - 0.5 * q2 - tke) * rho
    a2 = g * p / rho
    m1, g1 = mp2 - 1, g - 1
    vel = [u, v, w]
    P = np.zeros((n, n))
    P[0, 0] = -g1 * m1 * q2 / 2 / a2 / mp2 + 1
    for c in range(3):
        P[0, c + 1] = vel[c] * m1 * g1 / a2 / mp2
    P[0, 4] = -m1 * g1 / a2 / mp2
    for r in range(3):
        P[r + 1, 0] = -vel[r] * g1 * m1 * q2 / 2 / a2 / mp2
        for c in range(3):
            P[r + 1, c + 1] = (1 if r == c else 0) + vel[r] * vel[c] * m1 * g1 / a2 / mp2
        P[r + 1, 4] = -vel[r] * m1 * g1 / a2 / mp2
    h = 2 * a2 + g1 * (q2 + 2 * tke)
    P[4, 0] = -q2 * m1 * h / 4 / a2 / mp2
    for c in range(3):
        P[4, c + 1] = vel[c] * m1 * h / 2 / a2 / mp2
    P[4, 4] = -g1 * (q2 / 2 + tke) * m1 / a2 / mp2 + 1 / mp2
    if kom:
        ome = q[6] / rho
        P[0, 5] = m1 * g1 / a2 / mp2
        for r in range(3):
            P[r + 1, 5] = vel[r] * m1 * g1 / a2 / mp2
        P[4, 5] = 1 - 1 / mp2 + (q2 / 2 + tke) * m1 * g1 / a2 / mp2
        for r, t in ((5, tke), (6, ome)):
            P[r, 0] = -t * g1 * m1 * q2 / 2 / a2 / mp2
            for c in range(3):
                P[r, c + 1] = vel[c] * t * m1 * g1 / a2 / mp2
            P[r, 4] = -t * m1 * g1 / a2 / mp2
        P[5, 5] = 1 + tke * m1 * g1 / a2 / mp2
        P[6, 5] = ome * m1 * g1 / a2 / mp2
        P[6, 6] = 1
    return P


def test_prec_times_reference_inverse_is_identity(oracle_mod):
    case = casekit.small_channel(16, 8, 2)
    p = _lsp(case.params, cutoff_type=1, epsp=(1e-3,))
    p.machfs = 0.05
    O = oracle_mod.OracleLevel(case.tables, p)
    rng = np.random.default_rng(4)
    q = O.p3()
    for v in p3_views(case.tables, q, 5, 1):
        v[..., 0, 0] = rng.uniform(0.9, 1.1, v.shape[:3])
        v[..., 1, 0] = v[..., 0, 0] * rng.uniform(-0.05, 0.05, v.shape[:3])
        v[..., 2, 0] = v[..., 0, 0] * rng.uniform(-0.05, 0.05, v.shape[:3])
        v[..., 3, 0] = 0.0
        v[..., 4, 0] = 1 / 0.4 / 1.4 + 0.5 * (v[..., 1, 0] ** 2 + v[..., 2, 0] ** 2) / v[..., 0, 0]
    zero = oracle_mod.m1(O)
    prec = oracle_mod.lsp_prec(O, 1, q, zero, zero)
    t = case.tables
    nc = (t.dims[0, 0] - 1) * (t.dims[0, 1] - 1) * (t.dims[0, 2] - 1)
    P = prec.reshape(5, 5, nc)  # (col, row, cell) in Fortran order
    cell = next(iter(p3_views(t, q, 5, 1)))
    qi = cases.interior(cell)[..., 0].reshape(-1, 5, order="F")
    for c in range(0, nc, 7):
        rho, u, v = qi[c, 0], qi[c, 1] / qi[c, 0], qi[c, 2] / qi[c, 0]
        pr = 0.4 * (qi[c, 4] - 0.5 * rho * (u * u + v * v))
        mp2 = min(1.0, max((u * u + v * v) / (1.4 * pr / rho), 1e-6))
        A = P[:, :, c].T
        np.testing.assert_allclose(A @ _preci(qi[c], mp2, 1.4), np.eye(5), atol=1e-11)


def test_pressure_cutoff_and_rest3(oracle_mod):
    case = casekit.small_channel(16, 8, 2)
    p = _lsp(case.params)
    O = oracle_mod.OracleLevel(case.tables, p)
    q = O.p3()
    for v in p3_views(case.tables, q, 5, 1):
        v[..., 0, 0], v[..., 4, 0] = 1.2, 0.9
    cut = oracle_mod.m1(O)
    oracle_mod.lm_cutoff_pg(O, q, cut)
    assert np.abs(cut).max() == 0.0
    v0 = next(iter(p3_views(case.tables, q, 5, 1)))
    v0[4, 3, 2, 4, 0] = 1.0  # primitive p of cell (3, 2, 1) raised by 0.1 (views start at index -1)
    oracle_mod.lm_cutoff_pg(O, q, cut)
    t = case.tables
    I, J, K = t.dims[0, 0] - 1, t.dims[0, 1] - 1, t.dims[0, 2] - 1
    c = cut.reshape(K, J, I)
    assert np.isclose(c[0, 1, 2], 0.1 / 1.2 / (1.4 * 1.0 / 1.2), rtol=1e-14)  # the raised cell
    for kk, jj, ii in ((0, 1, 3), (0, 1, 1), (0, 2, 2), (0, 0, 2), (1, 1, 2)):
        assert np.isclose(c[kk, jj, ii], 0.1 / 1.2 / (1.4 * 0.9 / 1.2), rtol=1e-12)
    assert np.count_nonzero(c) == 6  # the cell and its five interior neighbours
    # rest3: each coarse cell the volume-weighted sum of its eight fine cells
    # over the coarse cell's own volume
    lv = cases.mg_levels(case, 2)
    O1, O2 = (oracle_mod.OracleLevel(tt, p) for tt, *_ in lv)
    v1, v2 = (Oi.metrics(x, y, z)[3] for Oi, (tt, x, y, z) in zip((O1, O2), lv))
    c1, c2 = np.random.default_rng(1).uniform(0, 1, O1.nm1), oracle_mod.m1(O2)
    oracle_mod.rest3(O1, O2, c1, c2, v1, v2)
    d1, d2 = lv[0][0].dims[0], lv[1][0].dims[0]
    V1 = v1.reshape(d1[2] + 1, d1[1] + 1, d1[0] + 1)[1:-1, 1:-1, 1:-1]
    V2 = v2.reshape(d2[2] + 1, d2[1] + 1, d2[0] + 1)[1:-1, 1:-1, 1:-1]
    C1 = c1.reshape(d1[2] - 1, d1[1] - 1, d1[0] - 1)
    W = (V1 * C1).reshape(V2.shape[0], 2, V2.shape[1], 2, V2.shape[2], 2).sum(axis=(1, 3, 5))
    np.testing.assert_allclose(c2.reshape(V2.shape), W / V2, rtol=1e-14)


def test_proflux_of_equal_states_is_physical(oracle_mod):
    case = casekit.small_channel(16, 8, 2)
    p = _lsp(case.params, cutoff_type=2, epsp=(1e-2,))
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = O.p3()
    for v in p3_views(case.tables, q, 5, 1):
        v[..., 0, 0], v[..., 1, 0], v[..., 2, 0], v[..., 3, 0], v[..., 4, 0] = 1.1, 0.03, -0.02, 0.0, 0.7
    flux = O.f0()
    zero = oracle_mod.m1(O)
    oracle_mod.proflux(O, 1, 1, q, q.copy(), flux, si, zero, zero)
    t = case.tables
    im, jm, km = t.dims[0]
    F = flux[:im * jm * km * 5].reshape(5, km, jm, im)
    s = si.reshape(-1)[: 4 * (im + 2) * (jm + 2) * (km + 2)].reshape(km + 2, jm + 2, im + 2, 4)
    kx, ky, kz, ds = (s[1, 1:jm, 1:im + 1, c] for c in range(4))
    un = 0.03 * kx - 0.02 * ky
    h0 = 1.4 / 0.4 * 0.7 / 1.1 + (0.03 ** 2 + 0.02 ** 2) / 2
    np.testing.assert_allclose(F[0, 0, :jm - 1, :], 1.1 * un * ds, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(F[1, 0, :jm - 1, :], (1.1 * 0.03 * un + 0.7 * kx) * ds, rtol=1e-13, atol=1e-16)
    np.testing.assert_allclose(F[4, 0, :jm - 1, :], 1.1 * h0 * un * ds, rtol=1e-13, atol=1e-16)


def _cons(w, g=1.4):
    r, u, v, ww, p = w
    return np.array([r, r * u, r * v, r * ww, p / (g - 1) + 0.5 * r * (u * u + v * v + ww * ww)])


def _flux(Q, n, g=1.4):
    r = Q[0]
    u, v, w = Q[1:4] / r
    p = (g - 1) * (Q[4] - 0.5 * r * (u * u + v * v + w * w))
    U = u * n[0] + v * n[1] + w * n[2]
    return np.array([r * U, r * u * U + p * n[0], r * v * U + p * n[1], r * w * U + p * n[2], (Q[4] + p) * U])


def test_proflux_dissipation_is_preconditioned_roe(oracle_mod):
    case = casekit.small_channel(4, 4, 2)
    p = _lsp(case.params, cutoff_type=1, epsp=(0.02,))
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    wr, wl = np.array([1.02, 0.05, 0.01, 0.0, 0.716]), np.array([0.99, 0.04, -0.01, 0.0, 0.713])
    qr, ql = O.p3(), O.p3()
    for m in range(5):
        qr[m * O.n3:(m + 1) * O.n3], ql[m * O.n3:(m + 1) * O.n3] = wr[m], wl[m]
    f, zero = O.f0(), oracle_mod.m1(O)
    oracle_mod.proflux(O, 1, 1, qr, ql, f, si, zero, zero)
    im, jm, km = case.tables.dims[0]
    F = f[:im * jm * km * 5].reshape(5, km, jm, im)[:, 0, 1, 2]  # face (3, 2, 1)
    s = si.reshape(-1)[:4 * (im + 2) * (jm + 2) * (km + 2)].reshape(km + 2, jm + 2, im + 2, 4)[1, 2, 3]
    n, ds = s[:3], s[3]
    QR, QL = _cons(wr), _cons(wl)
    df = _flux(QR, n) + _flux(QL, n) - 2 * F / ds
    rl, rr = np.sqrt(wl[0]), np.sqrt(wr[0])
    u = (rl * wl[1:4] + rr * wr[1:4]) / (rl + rr)
    h0 = (rl * (3.5 * wl[4] / wl[0] + 0.5 * wl[1:4] @ wl[1:4]) + rr * (3.5 * wr[4] / wr[0] + 0.5 * wr[1:4] @ wr[1:4]))
    h0 /= rl + rr
    a2 = 0.4 * (h0 - 0.5 * u @ u)
    Q = _cons(np.array([rl * rr, *u, rl * rr * a2 / 1.4]))
    A = np.zeros((5, 5))
    for c in range(5):
        dq = np.zeros(5)
        dq[c] = 1e-7 * max(1.0, abs(Q[c]))
        A[:, c] = (_flux(Q + dq, n) - _flux(Q - dq, n)) / (2 * dq[c])
    mp2 = min(1.0, max(u @ u / a2, 0.02 ** 2))
    P = np.linalg.inv(_preci(Q, mp2, 1.4))
    ev, R = np.linalg.eig(P @ A)
    D = np.linalg.inv(P) @ (R @ np.diag(np.abs(ev)) @ np.linalg.inv(R)).real @ (QR - QL)
    np.testing.assert_allclose(df, D, rtol=1e-7, atol=1e-9 * np.abs(D).max())


def test_low_mach_cycles_converge_further(oracle_mod):
    drops = {}
    for lsp in (0, 1):
        c = cases.bump_channel(64, 32, 2, mach=0.05)
        p = CosaParams.from_buffer_copy(c.params)
        p.cfl = 1.5
        if lsp:
            set_low_speed(p, cutoff_type=2, epsp=(0.05,))
        lv, Os, As = casekit.mg_oracle(c, 1, p, oracle_mod)
        h, st = oracle_mod.mg(Os, As, 1, 600, 600, rms_every=600)
        assert st == 0
        r = h[~np.isnan(h[:, 0]), 0]
        drops[lsp] = r[-1] / r[0]
    assert drops[1] < 0.9 * drops[0], drops
