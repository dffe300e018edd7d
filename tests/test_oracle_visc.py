"""Known-answer tests of the oracle's laminar viscous path.

The restatement follows src/grid.f90 (coordex, volex, cut_x, cut_v,
vmetrix), src/flux.f90 (q_face, q_der, vflux), src/bc.f90 (bc_walvis_15)
and src/cosa.f90 (lambdab/eig_ns, deltat).  COSA ships no data for these,
so they are pinned by properties of the mathematics:

* on a Cartesian grid the face inverse metrics are exactly 1/dx, 1/dy, 1/dz
  on every face, boundary faces included (the doubled one-sided
  differences where a ghost node repeats its node);
* cut_x supplies the neighbour block's nodes: the metrics of a partitioned
  grid equal the single-block ones face for face;
* face gradients of a field linear in the cell index are exact;
* the viscous flux of a Couette shear / a conduction profile matches the
  closed-form stress and heat flux;
* the viscous residual is linear in 1/Re and vanishes as Re -> infinity,
  where the convective residual of the inviscid path is recovered.
"""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p1_views, p2_views, p3_views, f0_views, vm_views
from cosa_b200.tables import BlockSpec


DX, DY, DZ = 0.1, 0.05, 0.2


def _box(ni=6, nj=5, nk=4, bcs=None):
    xs, ys, zs = DX * np.arange(ni + 1), DY * np.arange(nj + 1), DZ * np.arange(nk + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    types = bcs or {"imin": 4, "imax": 4, "jmin": cases.VISCOUS_WALL, "jmax": cases.VISCOUS_WALL, "kmin": 80,
                    "kmax": 80}
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, cases._face_bcs(ni + 1, nj + 1, nk + 1, types))
    return cases._assemble("box", [(X.copy(), Y.copy(), Z.copy())], [spec], [], cases.laminar_params())


def _setup(oracle_mod, case):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    si, sj, sk, vol = O.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O, x, y, z, vol)
    return O, (x, y, z), (si, sj, sk), vol, vm


def test_vmetrix_cartesian_exact(oracle_mod):
    case = _box()
    O, _, _, vol, vm = _setup(oracle_mod, case)
    (im, jm, km), = case.tables.dims
    v = vm_views(case.tables, vm)[0]
    inv = np.diag([1 / DX, 1 / DY, 1 / DZ])
    for d in range(3):
        ni, nj, nk = im - (d != 0), jm - (d != 1), km - (d != 2)
        for m in range(3):
            a = v[d][m][:, :ni, :nj, :nk]
            for c in range(3):
                np.testing.assert_allclose(a[c], inv[m, c], rtol=1e-13, atol=1e-12)
    # volex: face halos repeat the first interior cell
    V = p1_views(case.tables, vol)[0][..., 0]
    np.testing.assert_array_equal(V[0, 1:jm, 1:km], V[1, 1:jm, 1:km])
    np.testing.assert_array_equal(V[im, 1:jm, 1:km], V[im - 1, 1:jm, 1:km])
    np.testing.assert_array_equal(V[1:im, 0, 1:km], V[1:im, 1, 1:km])
    np.testing.assert_array_equal(V[1:im, 1:jm, km], V[1:im, 1:jm, km - 1])


def test_vmetrix_partitioned_equals_single_block(oracle_mod):
    """cut_x / cut_v give every block the neighbour's nodes and volumes, so
    each face's metrics equal the single-block grid's bit for bit."""
    ni, nj, nk, isp, jsp = 24, 12, 2, 10, 5
    one = cases.laminar_channel(ni, nj, nk)
    part = cases.partitioned_laminar_channel(ni, nj, nk, isplit=(isp,), jsplit=(jsp,), permute_last=False)
    _, _, _, _, vm1 = _setup(oracle_mod, one)
    _, _, _, _, vm4 = _setup(oracle_mod, part)
    full = vm_views(one.tables, vm1)[0]
    origin = {0: (0, 0), 1: (isp, 0), 2: (0, jsp), 3: (isp, jsp)}
    for b, vb in enumerate(vm_views(part.tables, vm4)):
        im, jm, km = part.tables.dims[b]
        i0, j0 = origin[b]
        for d in range(3):
            ni_, nj_, nk_ = im - (d != 0), jm - (d != 1), km - (d != 2)
            for m in range(3):
                got = vb[d][m][:, :ni_, :nj_, :nk_]
                ref = full[d][m][:, i0:i0 + ni_, j0:j0 + nj_, :nk_]
                np.testing.assert_array_equal(got, ref)


def _linear_prim(case, coef):
    """Primitive state linear in the cell index over the whole P3 array."""
    q = np.zeros(case.q0.size)
    for v in p3_views(case.tables, q, 5, 1):
        I, J, K = np.meshgrid(*(np.arange(s) - 1.0 for s in v.shape[:3]), indexing="ij")
        for m in range(5):
            v[..., m, 0] = coef[m][0] + coef[m][1] * I + coef[m][2] * J + coef[m][3] * K
    return q


def test_q_der_linear_exact_and_wall_formula(oracle_mod):
    case = _box()
    O = oracle_mod.OracleLevel(case.tables, case.params)
    coef = [(1.0, 0.01, 0.02, 0.03), (0.3, 0.1, -0.2, 0.05), (0.1, -0.05, 0.3, 0.0), (0.0, 0.02, 0.01, -0.1),
            (0.7, 0.0, 0.04, 0.02)]
    q = _linear_prim(case, coef)
    (im, jm, km), = case.tables.dims
    qv = p3_views(case.tables, q, 5, 1)[0]
    for d in (1, 2, 3):
        g = [O.p3() for _ in range(3)]
        oracle_mod.q_der(O, d, q, *g)
        qf = O.p3()
        oracle_mod.q_face(O, d, q, qf)
        gv = [p3_views(case.tables, a, 5, 1)[0] for a in g]
        fv = p3_views(case.tables, qf, 5, 1)[0]
        rng = [range(1, im), range(1, jm), range(1, km)]
        rng[d - 1] = range(1, (im, jm, km)[d - 1] + 1)
        for i in rng[0]:
            for j in rng[1]:
                for k in rng[2]:
                    on_wall = d == 2 and j in (1, jm)
                    for m in range(5):
                        for t in range(3):
                            got = gv[t][i + 1, j + 1, k + 1, m, 0]
                            if not on_wall:
                                assert abs(got - coef[m][t + 1]) < 1e-13
                        if not on_wall:
                            cm = (i - (d == 1), j - (d == 2), k - (d == 3))
                            avg = (qv[cm[0] + 1, cm[1] + 1, cm[2] + 1, m, 0] + qv[i + 1, j + 1, k + 1, m, 0]) / 2
                            assert fv[i + 1, j + 1, k + 1, m, 0] == avg
        if d == 2:
            # strong boundary (wall) faces: halo value, 3-point normal
            # derivative, tangential derivatives along the halo line
            for j, aux, in1, in2, sg in ((1, 0, 1, 2, 1.0), (jm, jm, jm - 1, jm - 2, -1.0)):
                for i in range(1, im):
                    for k in range(1, km):
                        for m in range(5):
                            Q = lambda a, b, c: qv[a + 1, b + 1, c + 1, m, 0]
                            assert fv[i + 1, j + 1, k + 1, m, 0] == Q(i, aux, k)
                            nrm = sg / 3 * (-Q(i, aux, k) * 8 + Q(i, in1, k) * 9 - Q(i, in2, k))
                            assert gv[1][i + 1, j + 1, k + 1, m, 0] == nrm
                            if i == 1:
                                ex = (Q(i, aux, k) + Q(i + 1, aux, k)) / 2 - (Q(i, aux, k) * 3 - Q(i + 1, aux, k)) / 2
                            elif i == im - 1:
                                ex = (Q(i, aux, k) * 3 - Q(i - 1, aux, k)) / 2 - (Q(i, aux, k) + Q(i - 1, aux, k)) / 2
                            else:
                                ex = (Q(i, aux, k) + Q(i + 1, aux, k)) / 2 - (Q(i - 1, aux, k) + Q(i, aux, k)) / 2
                            assert gv[0][i + 1, j + 1, k + 1, m, 0] == ex


def _sutherland(t, stemp):
    return (stemp + 1) / (t + stemp) * t ** 1.5


def test_vflux_couette_and_conduction(oracle_mod):
    """j-faces of a Cartesian box with a uniform face state, a shear du/deta
    and a pressure gradient dp/deta (temperature gradient at fixed rho)."""
    case = _box()
    p = case.params
    O, _, (si, sj, sk), vol, vm = _setup(oracle_mod, case)
    (im, jm, km), = case.tables.dims
    rho, u, pr = 1.1, 0.3, 0.8
    du, dp = 0.02, 0.01
    qf, dx_, de_, dz_ = (O.p3() for _ in range(4))
    for v in p3_views(case.tables, qf, 5, 1):
        v[..., 0, 0] = rho
        v[..., 1, 0] = u
        v[..., 4, 0] = pr
    for v in p3_views(case.tables, de_, 5, 1):
        v[..., 1, 0] = du
        v[..., 4, 0] = dp
    flux = O.f0()
    oracle_mod.vflux(O, 2, qf, dx_, de_, dz_, vm, sj, flux)
    f = f0_views(case.tables, flux, 5)[0][..., 0]
    g = p.gamma
    t = g * pr / rho
    mu = _sutherland(t, p.stemp)
    mr = p.machfs / p.reyno
    txy = mr * mu * (du / DY)
    dtdy = t * (dp / pr) / DY
    qy = -mr * (mu / p.pranl) / (g - 1) * dtdy
    ds = DX * DZ
    np.testing.assert_allclose(f[:im - 1, :jm, :km - 1, 0], 0.0, atol=0)
    np.testing.assert_allclose(f[:im - 1, :jm, :km - 1, 1], -txy * ds, rtol=1e-12)
    np.testing.assert_allclose(f[:im - 1, :jm, :km - 1, 2], 0.0, atol=1e-18)
    np.testing.assert_allclose(f[:im - 1, :jm, :km - 1, 4], -(u * txy) * ds + qy * ds, rtol=1e-12)


def test_viscous_lambda_uniform_state(oracle_mod):
    case = _box()
    p = case.params
    O, _, (si, sj, sk), vol, vm = _setup(oracle_mod, case)
    q = case.q0.copy()
    O.cons2prim(q)
    assert O.bc(q, si, sj, sk) == 0  # primitive halos (uniform temperature)
    lam, lamv = O.p3(), O.p3()
    oracle_mod.lambda_ns(O, q, si, sj, sk, vol, lam, lamv)
    (im, jm, km), = case.tables.dims
    lv = p3_views(case.tables, lamv, 5, 1)[0][2:im + 1, 2:jm + 1, 2:km + 1, :3, 0]
    rho = p.rhoinf
    t = p.gamma * (1 / p.gamma) / rho
    mu = _sutherland(t, p.stemp)
    V = DX * DY * DZ
    for c, area in enumerate((DY * DZ, DX * DZ, DX * DY)):
        ref = p.cdff * area * area * p.gamma * p.machfs / p.reyno * (mu / p.pranl) / (rho * V)
        np.testing.assert_allclose(lv[..., c], ref, rtol=1e-13)
    # the time step adds the viscous lambdas (irsop = 0)
    dt = O.p1(1)
    oracle_mod.deltat_ns(O, dt, lam, lamv)
    lm = p3_views(case.tables, lam, 5, 1)[0][2:im + 1, 2:jm + 1, 2:km + 1, :3, 0]
    d = p1_views(case.tables, dt, 1)[0][1:im, 1:jm, 1:km, 0]
    np.testing.assert_allclose(d, p.cfl / (lm.sum(-1) + lv.sum(-1)), rtol=1e-14)


def _residual(oracle_mod, case, reyno, viscous, q):
    p = cases.laminar_params(case.params.machfs, reyno)
    p.viscous = viscous
    O = oracle_mod.OracleLevel(case.tables, p)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    si, sj, sk, vol = O.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O, x, y, z, vol)
    qq = q.copy()
    if viscous:
        res, dt, st = oracle_mod.residual_ns(O, qq, si, sj, sk, vol, vm, want_dt=False)
    else:
        res, dt, st = O.residual(qq, si, sj, sk, want_dt=False)
    assert st == 0
    return casekit.interior_cells(case, res, 5)


import casekit  # noqa: E402


def test_viscous_residual_linear_in_inverse_reynolds(oracle_mod):
    case = cases.partitioned_laminar_channel(24, 12, 2, isplit=(10,), jsplit=(5,))
    q = cases.perturbed_state(case, amp=0.05, seed=3)
    r0 = _residual(oracle_mod, case, 500.0, 0, q)
    r_inf = _residual(oracle_mod, case, 1e300, 1, q)
    scale = np.abs(r0).reshape(-1, 5).max(axis=0)
    assert (np.abs(r_inf - r0) / scale[None, :, None]).max() < 1e-15
    r1 = _residual(oracle_mod, case, 200.0, 1, q)
    r2 = _residual(oracle_mod, case, 2000.0, 1, q)
    v1, v2 = (r1 - r0) * 200.0, (r2 - r0) * 2000.0
    vs = np.abs(v1).reshape(-1, 5).max(axis=0)
    assert vs[1] > 0 and vs[4] > 0
    assert (np.abs(v1 - v2) / np.maximum(vs, 1e-300)[None, :, None]).max() < 1e-9


def test_laminar_smooth_runs_and_walls_hold(oracle_mod):
    """A few viscous RK cycles: status 0, finite norms, and the wall halo
    carries zero velocity and the extrapolated pressure."""
    case = cases.laminar_channel(24, 12, 2)
    O, _, (si, sj, sk), vol, vm = _setup(oracle_mod, case)
    q = case.q0.copy()
    hist, st = oracle_mod.smooth_ns(O, q, si, sj, sk, vol, vm, 5)
    assert st == 0 and np.isfinite(hist).all()
    # one more residual leaves q primitive-consistent; check the wall halo
    qq = q.copy()
    O.cons2prim(qq)
    O.bc(qq, si, sj, sk)
    v = p3_views(case.tables, qq, 5, 1)[0]
    (im, jm, km), = case.tables.dims
    assert np.all(v[2:im + 1, 1, 2:km + 1, 1:4, 0] == 0.0)
    p1, p2 = v[2:im + 1, 2, 2:km + 1, 4, 0], v[2:im + 1, 3, 2:km + 1, 4, 0]
    np.testing.assert_array_equal(v[2:im + 1, 1, 2:km + 1, 4, 0], 0.5 * (3 * p1 - p2))
    np.testing.assert_array_equal(v[2:im + 1, 0, 2:km + 1, :, 0], v[2:im + 1, 1, 2:km + 1, :, 0])
