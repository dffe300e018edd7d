"""Known-answer tests of the CPU oracle (the checker of the GPU path).

COSA ships no tests or golden data, so the oracle is pinned by properties
that follow from the reference's mathematics (src/flux.f90, src/cosa.f90):
Roe consistency and upwinding, limiter values, free-stream preservation,
telescoping conservation, multi-block equivalence through cut_q.
"""
import math

import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p3_views
from cosa_b200.params import default_params

import casekit


def _phys_flux(q, n, g=1.4):
    rho, u, v, w, p = q
    un = u * n[0] + v * n[1] + w * n[2]
    h0 = g / (g - 1) * p / rho + (u * u + v * v + w * w) / 2
    return np.array([rho * un, rho * u * un + p * n[0], rho * v * un + p * n[1], rho * w * un + p * n[2],
                     rho * h0 * un]) * n[3]


def test_roe_consistency(oracle_mod):
    """F_roe(q, q) equals the physical flux (src/flux.f90:117-243)."""
    p = default_params()
    rng = np.random.default_rng(1)
    for _ in range(50):
        q = np.array([rng.uniform(0.5, 2), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1),
                      rng.uniform(0.3, 2)])
        nv = rng.standard_normal(3)
        nv /= np.linalg.norm(nv)
        n = np.array([*nv, rng.uniform(0.1, 3)])
        f = oracle_mod.roe_face(p, n, q, q)
        np.testing.assert_allclose(f, _phys_flux(q, n), rtol=1e-14, atol=1e-14)


def test_roe_supersonic_upwind(oracle_mod):
    """With all Roe eigenvalues positive the flux is the left physical flux."""
    p = default_params()
    ql = np.array([1.0, 3.0, 0.1, 0.0, 1 / 1.4])
    qr = np.array([1.05, 3.1, 0.12, 0.01, 1.02 / 1.4])
    n = np.array([1.0, 0.0, 0.0, 1.0])
    f = oracle_mod.roe_face(p, n, qr, ql)
    np.testing.assert_allclose(f, _phys_flux(ql, n), rtol=1e-12, atol=1e-13)


def _limit_ref(ilim, eps, rkap, d):
    """Direct transcription of limit_i's formulas (src/flux.f90:3472-3620)
    over one line of differences d[0..n+1]; returns dqp, dqm on faces 1..n."""
    n = len(d) - 2
    dqp = np.zeros(n + 2)
    dqm = np.zeros(n + 2)
    if ilim in (0, 1):
        for i in range(1, n + 1):
            if ilim == 0:
                rkp, rkm = 1 + rkap, 1 - rkap
                dqp[i] = -(rkp * d[i] + rkm * d[i + 1]) / 4
                dqm[i] = (rkm * d[i - 1] + rkp * d[i]) / 4
            else:
                s = (2 * d[i + 1] * d[i] + eps) / (d[i + 1] ** 2 + d[i] ** 2 + eps)
                dqp[i] = -s * ((1 + rkap * s) * d[i] + (1 - rkap * s) * d[i + 1]) / 4
                s = (2 * d[i] * d[i - 1] + eps) / (d[i] ** 2 + d[i - 1] ** 2 + eps)
                dqm[i] = s * ((1 - rkap * s) * d[i - 1] + (1 + rkap * s) * d[i]) / 4
    else:
        for i in range(0, n + 1):
            d1, d2 = d[i + 1], d[i]
            if ilim == 2:
                b = (3 - rkap) / (1 - rkap)
                sg = lambda x: math.copysign(1.0, x)
                mx = (sg(d2) + sg(d1)) / 2 * min(abs(d2), abs(d1) * b)
                px = (sg(d1) + sg(d2)) / 2 * min(abs(d1), abs(d2) * b)
                dqp[i] = -((1 + rkap) * mx + (1 - rkap) * px) / 4
                dqm[i + 1] = ((1 - rkap) * mx + (1 + rkap) * px) / 4
            elif ilim == 3:
                e2 = eps * eps
                mx = (d1 * (d2 ** 2 + 2 * e2) + d2 * (2 * d1 ** 2 + e2)) / (2 * d1 ** 2 - d1 * d2 + 2 * d2 ** 2 + 3 * e2)
                px = (d2 * (d1 ** 2 + 2 * e2) + d1 * (2 * d2 ** 2 + e2)) / (2 * d2 ** 2 - d2 * d1 + 2 * d1 ** 2 + 3 * e2)
                dqp[i] = -px / 2
                dqm[i + 1] = mx / 2
            else:
                e2 = eps * eps
                mx = (d1 * (d2 ** 2 + e2) + d2 * (d1 ** 2 + e2)) / (d1 ** 2 + d2 ** 2 + 2 * e2)
                dqp[i] = -mx / 2
                dqm[i + 1] = mx / 2
    return dqp[1:n + 1], dqm[1:n + 1]


@pytest.mark.parametrize("ilim", [0, 1, 2, 3, 4])
def test_limiters_match_formulas(oracle_mod, ilim):
    """muscl_bi + limit_i on a line: oracle dqp/dqm vs the transcribed formulas,
    including the hand values of a uniform slope (dqp = -1/2, dqm = +1/2)."""
    case = cases.bump_channel(12, 4, 2)
    p = case.params
    p.ilimf = ilim
    p.epslimf = 1e-3
    O = oracle_mod.OracleLevel(case.tables, p)
    q = O.p3()
    rng = np.random.default_rng(ilim)
    v = p3_views(case.tables, q, 5, 1)[0]
    prof = np.cumsum(rng.standard_normal(v.shape[0])) * 0.2
    for var in range(5):
        v[:, :, :, var, 0] = 1.0 + prof[:, None, None] * (var + 1)
    qp, qm, dq, dqp, dqm = (O.p3() for _ in range(5))
    O.muscl(1, 1, q, qp, qm, dq, dqp, dqm)
    d = np.diff(v[:, 2, 2, 0, 0])  # dq(i) = q(i)-q(i-1) for i = 0..imax+1
    ref_p, ref_m = _limit_ref(ilim, p.epslimf, p.rkap, d)
    vp = p3_views(case.tables, dqp, 5, 1)[0][:, 2, 2, 0, 0]
    vm = p3_views(case.tables, dqm, 5, 1)[0][:, 2, 2, 0, 0]
    imax = case.tables.dims[0, 0]
    # faces 2..imax-1 (faces 1 and imax carry the inlet/outlet, not strong BCs)
    np.testing.assert_allclose(vp[3:imax + 1], ref_p[1:imax - 1], rtol=1e-13, atol=1e-15)
    np.testing.assert_allclose(vm[3:imax + 1], ref_m[1:imax - 1], rtol=1e-13, atol=1e-15)
    # uniform slope: exact linear reconstruction
    v[:, :, :, 0, 0] = 1.0 + 0.1 * np.arange(v.shape[0])[:, None, None]
    O.muscl(1, 1, q, qp, qm, dq, dqp, dqm)
    vp = p3_views(case.tables, dqp, 5, 1)[0][:, 2, 2, 0, 0]
    np.testing.assert_allclose(vp[4:imax], -0.05, rtol=1e-9)


def _allfar(case):
    """Same grid with every BC replaced by the far field (30)."""
    t = case.tables
    t.bctopo[:, 0] = np.where(t.bctopo[:, 0] == 80, 80, 30)
    p = case.params
    p.machfs = 0.5
    return case


def test_freestream_preservation(oracle_mod):
    """Uniform free stream on a curved grid with far-field BCs: R ~ 0."""
    case = _allfar(cases.bump_channel(32, 16, 2))
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = case.q0.copy()
    res, dt, st = O.residual(q, si, sj, sk)
    assert st == 0
    r = casekit.interior_cells(case, res, 5)
    assert np.abs(r).max() < 1e-13


def test_multiblock_equals_single_block(oracle_mod):
    """The channel as 1 block and as 4 blocks (one with permuted indices):
    cut_q halos make the stage-1 residuals agree (src/bc.f90:1894-2141)."""
    one = cases.bump_channel(48, 24, 2, kface_bc=4)
    four = cases.partitioned_channel(48, 24, 2, isplit=(20,), jsplit=(10,), permute_last=True)
    q1 = cases.perturbed_state(one, seed=3)
    # build the same physical state on the 4-block layout
    v1 = p3_views(one.tables, q1, 5, 1)[0]
    q4 = four.q0.copy()
    views = p3_views(four.tables, q4, 5, 1)
    ib, jb = [0, 20, 48], [0, 10, 24]
    b = 0
    for bj in range(2):
        for bi in range(2):
            src = v1[ib[bi]:ib[bi + 1] + 4, jb[bj]:jb[bj + 1] + 4]
            if bi == 1 and bj == 1:
                src = np.transpose(src, (1, 2, 0, 3, 4))
            views[b][...] = src
            b += 1
    O1 = oracle_mod.OracleLevel(one.tables, one.params)
    O4 = oracle_mod.OracleLevel(four.tables, four.params)
    m1 = O1.metrics(one.x, one.y, one.z)
    m4 = O4.metrics(four.x, four.y, four.z)
    r1, dt1, _ = O1.residual(q1, *m1[:3])
    r4, dt4, _ = O4.residual(q4, *m4[:3])
    R1 = p3_views(one.tables, r1, 5, 1)[0][2:-2, 2:-2, 2:-2]
    R4 = p3_views(four.tables, r4, 5, 1)
    scale = np.abs(R1).max()
    b = 0
    for bj in range(2):
        for bi in range(2):
            part = R1[ib[bi]:ib[bi + 1], jb[bj]:jb[bj + 1]]
            got = R4[b][2:-2, 2:-2, 2:-2]
            if bi == 1 and bj == 1:
                got = np.transpose(got, (2, 0, 1, 3, 4))
            assert np.abs(got - part).max() <= 1e-12 * scale, b
            b += 1


def test_conservation_telescopes(oracle_mod):
    """Sum of the residual over a block = net flux through its boundary faces."""
    case = casekit.small_channel(24, 12, 2)
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = cases.perturbed_state(case, seed=7)
    O.cons2prim(q)
    O.bc(q, si, sj, sk)
    res = O.p3()
    O.zero_res(res)
    boundary = np.zeros(5)
    imax, jmax, kmax = case.tables.dims[0]
    for d, s in ((1, si), (2, sj), (3, sk)):
        qp, qm, dq, dqp, dqm = (O.p3() for _ in range(5))
        flux = O.f0()
        O.muscl(d, 1, q, qp, qm, dq, dqp, dqm)
        O.roflux(d, qp, qm, flux, s)
        O.resid(d, flux, res)
        F = flux.reshape((5, kmax, jmax, imax))  # (v, k, j, i) C-order of the F0 block
        if d == 1:
            boundary += F[:, :kmax - 1, :jmax - 1, imax - 1].sum(axis=(1, 2)) - F[:, :kmax - 1, :jmax - 1, 0].sum(axis=(1, 2))
        elif d == 2:
            boundary += F[:, :kmax - 1, jmax - 1, :imax - 1].sum(axis=(1, 2)) - F[:, :kmax - 1, 0, :imax - 1].sum(axis=(1, 2))
        else:
            boundary += F[:, kmax - 1, :jmax - 1, :imax - 1].sum(axis=(1, 2)) - F[:, 0, :jmax - 1, :imax - 1].sum(axis=(1, 2))
    total = casekit.interior_cells(case, res, 5).sum(axis=0)[:, 0]
    np.testing.assert_allclose(total, boundary, rtol=1e-10, atol=1e-12)


def test_smooth_converges(oracle_mod):
    """The single-level RK driver reduces the residual on the bump channel."""
    case = cases.bump_channel(32, 16, 2)
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = case.q0.copy()
    hist, st = O.smooth(q, si, sj, sk, 400, rms_every=50)
    assert st == 0
    first, last = hist[0, 5], hist[-1, 5]
    assert np.isfinite(last) and last < 0.2 * first


def test_prtest_flags_negative_pressure(oracle_mod):
    case = cases.bump_channel(16, 8, 2)
    O = oracle_mod.OracleLevel(case.tables, case.params)
    q = case.q0.copy()
    O.cons2prim(q)
    v = p3_views(case.tables, q, 5, 1)[0]
    v[5, 3, 2, 4, 0] = -1.0
    assert O.prtest(q) & 0x1


@pytest.mark.parametrize("nharms", [1, 2, 3])
def test_hb_operator_differentiates_harmonics(nharms):
    """omega * D u(t_n) = du/dt(t_n) exactly for every harmonic up to nharms,
    and D annihilates constants, so a steady state has src_hb = 0
    (mathb, src/input.f90:5206-5284)."""
    from cosa_b200.params import hb_matrix
    omega = 0.08 * 2 / 0.5 * 0.5  # reduced frequency 0.08 at M = 0.5, c = 1
    D = hb_matrix(nharms, omega)
    S = 2 * nharms + 1
    t = np.arange(S) * 2 * np.pi / omega / S
    np.testing.assert_allclose(D @ np.ones(S), 0.0, atol=1e-13)
    for k in range(1, nharms + 1):
        np.testing.assert_allclose(omega * D @ np.cos(k * omega * t), -k * omega * np.sin(k * omega * t), atol=1e-12)
        np.testing.assert_allclose(omega * D @ np.sin(k * omega * t), k * omega * np.cos(k * omega * t), atol=1e-12)


def test_src_hb_vanishes_on_identical_snapshots(oracle_mod):
    from cosa_b200.params import set_harmonic_balance
    case = cases.bump_channel(16, 8, 2)
    p = set_harmonic_balance(case.params, 2, 0.16)
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = cases._freestream_state(case.tables, p)
    res = O.p3()
    oracle_mod.src_hb(O, q, vol, res)
    assert np.abs(res).max() < 1e-14


def test_far_field_bc_far1_keeps_the_free_stream(oracle_mod):
    """bc_far1 (type 31) with the free stream inside writes the free stream
    into both halo layers (unb = q_inf . n, pb = p_inf, rho from the
    isentrope through p_inf), at inflow and outflow faces alike."""
    p = cases.naca_params("euler", mach=0.5, alpha_deg=3.0, eps_irs=0.0)
    case = cases.naca0012_ogrid(blocks=(8, 12, 12, 8), nj=8, nk=2, rfar=10.0, h1=5e-3, params=p, wall=14, far=31)
    O = oracle_mod.OracleLevel(case.tables, p)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = case.q0.copy()
    O.cons2prim(q)
    assert O.bc(q, si, sj, sk) == 0
    fs = np.array([p.rhoinf, p.machfs * np.cos(p.alpha), p.machfs * np.sin(p.alpha), 0.0, p.pinf])
    for v in p3_views(case.tables, q, 5, 1):
        jm = v.shape[1] - 3
        h = v[2:-2, jm + 1:jm + 3, 2:-2, :, 0]   # far-field halo layers j = jmax, jmax+1
        np.testing.assert_allclose(h, np.broadcast_to(fs, h.shape), rtol=1e-13, atol=1e-15)
