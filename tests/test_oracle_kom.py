"""Known-answer tests of the oracle's Wilcox k-omega path (src/src.f90
turprod/srckw, src/flux.f90 rtst/vflux/q_der_c, src/update.f90 update_b,
src/bc.f90 bc_walvis_15):

* production of a simple shear u = c y is c^2, div u = delta+ = 0;
* the k and omega sources and the point-implicit update follow their
  closed forms for a uniform state;
* the Reynolds stress of a shear adds mut to mu in the face momentum flux;
* with k = 0 and mut = 0 the mean-flow residual of the k-omega path equals
  the laminar one to rounding (the model only adds terms; the k terms of
  the BCs and cons2prim round differently in the last bit);
* the omega wall value follows Menter's formula 60 mu / (beta rho d^2).
"""
import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p1_views, p3_views, f0_views
from cosa_b200.tables import BlockSpec

DX, DY, DZ = 0.1, 0.05, 0.2


def _box(params, ni=6, nj=5, nk=4):
    xs, ys, zs = DX * np.arange(ni + 1), DY * np.arange(nj + 1), DZ * np.arange(nk + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    types = {"imin": 4, "imax": 4, "jmin": cases.VISCOUS_WALL, "jmax": cases.VISCOUS_WALL, "kmin": 80, "kmax": 80}
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, cases._face_bcs(ni + 1, nj + 1, nk + 1, types))
    return cases._assemble("box", [(X.copy(), Y.copy(), Z.copy())], [spec], [], params)


def _setup(oracle_mod, case):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    A = oracle_mod.RansArrays(O)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    A.si, A.sj, A.sk, A.vol = O.metrics(x, y, z)
    A.vm = oracle_mod.viscous_setup(O, x, y, z, A.vol)
    A.dist[:] = cases.wall_distance(case)
    return O, A


def test_production_of_simple_shear(oracle_mod):
    case = _box(cases.kom_params())
    O, A = _setup(oracle_mod, case)
    c = 0.7
    q = O.p3()
    for v in p3_views(case.tables, q, 7, 1):
        J = np.arange(v.shape[1]) - 1.0
        v[..., 0, 0] = 1.0
        v[..., 1, 0] = c * DY * J[None, :, None]   # u at cell centre j: c * y
        v[..., 4, 0] = 0.7
        v[..., 5, 0] = 1e-3
        v[..., 6, 0] = 1.0
    grads = []
    for d in (1, 2, 3):
        qf, dc = O.p3(), O.p3()
        oracle_mod.q_face(O, d, q, qf)
        oracle_mod.q_der_c(O, d, qf, dc)
        grads.append(dc)
    prd, dv, dp = (np.zeros(O.n3 * O.S) for _ in range(3))
    oracle_mod.turprod(O, q, *grads, A.vm, prd, dv, dp)
    (im, jm, km), = case.tables.dims
    # interior away from the walls, where q_face keeps the halo values
    P = prd.reshape(km + 3, jm + 3, im + 3)[3:-3, 3:-3, 2:-2]
    np.testing.assert_allclose(P, c * c, rtol=1e-12)
    assert np.abs(dv).max() < 1e-12 and np.abs(dp).max() < 1e-12


def test_sources_and_point_implicit_update_closed_form(oracle_mod):
    case = _box(cases.kom_params())
    p = case.params
    O, A = _setup(oracle_mod, case)
    rho, k, w, mut, prod = 1.2, 2e-3, 3.0, 5.0, 0.4
    q = O.p3()
    for v in p3_views(case.tables, q, 7, 1):
        v[..., 0, 0] = rho
        v[..., 4, 0] = 0.7
        v[..., 5, 0] = k
        v[..., 6, 0] = w
    muta = np.full(O.n3, mut)
    prd = np.full(O.n3, prod)
    dv = np.zeros(O.n3)
    res = O.p3()
    oracle_mod.srckw(O, 1, q, muta, prd, dv, res, A.vol)
    mor = p.machfs / p.reyno
    V = DX * DY * DZ
    r = p3_views(case.tables, res, 7, 1)[0][2:-2, 2:-2, 2:-2]
    np.testing.assert_allclose(r[..., 5, 0], -V * (mor * mut * prod - p.bstrkw * rho * k * w), rtol=1e-12)
    np.testing.assert_allclose(r[..., 6, 0], -V * (p.gkw * p.cmu * rho * prod - p.bkw * rho * w * w), rtol=1e-12)
    # update: conservative q, res and delta+ zero, dtvolt set
    qc = O.p3()
    for v in p3_views(case.tables, qc, 7, 1):
        v[..., 0, 0] = rho
        v[..., 5, 0] = rho * k
        v[..., 6, 0] = rho * w
    qold = qc.copy()
    dtt = np.full(O.n1, 0.01)
    zero = O.p3()
    oracle_mod.update_kom(O, zero, qc, qold, A.vol, dtt, np.zeros(O.n3), np.zeros(O.n3), 0.5)
    ar, dtau = 0.5, 0.01 * V
    rw = (rho * w + ar * dtau * rho * w * (2 * p.bkw * w)) / (1 + ar * dtau * (2 * p.bkw * w))
    rk = (rho * k + ar * dtau * rho * k * (p.bstrkw * w) - ar * dtau * p.bstrkw * k * (rw - rho * w)) / \
        (1 + ar * dtau * (p.bstrkw * w))
    u = p3_views(case.tables, qc, 7, 1)[0][2:-2, 2:-2, 2:-2]
    np.testing.assert_allclose(u[..., 6, 0], rw, rtol=1e-13)
    np.testing.assert_allclose(u[..., 5, 0], rk, rtol=1e-13)


def test_reynolds_stress_adds_eddy_viscosity(oracle_mod):
    """j-faces, uniform face state with k = 0 and a shear du/deta: the k-omega
    face flux of u-momentum is -(mu + mut) M/Re du/dy ds."""
    case = _box(cases.kom_params())
    p = case.params
    O, A = _setup(oracle_mod, case)
    rho, u, pr, du, mut = 1.1, 0.3, 0.8, 0.02, 7.0
    qf, gx, ge, gz, tau = (O.p3() for _ in range(5))
    for v in p3_views(case.tables, qf, 7, 1):
        v[..., 0, 0] = rho
        v[..., 1, 0] = u
        v[..., 4, 0] = pr
        v[..., 6, 0] = 1.0
    for v in p3_views(case.tables, ge, 7, 1):
        v[..., 1, 0] = du
    flux = O.f0()
    f = f0_views(case.tables, flux, 7)[0]
    f[..., 0, 0] = mut
    oracle_mod.rtst(O, 2, qf, gx, ge, gz, A.vm, tau, flux)
    oracle_mod.vflux_kom(O, 2, qf, gx, ge, gz, tau, A.vm, A.sj, flux)
    (im, jm, km), = case.tables.dims
    t = p.gamma * pr / rho
    mu = (p.stemp + 1) / (t + p.stemp) * t ** 1.5
    ref = -(p.machfs / p.reyno * (mu + mut) * (du / DY)) * (DX * DZ)
    np.testing.assert_allclose(f[:im - 1, :jm, :km - 1, 1, 0], ref, rtol=1e-12)
    assert np.abs(f[:im - 1, :jm, :km - 1, 0, 0]).max() == 0.0


def test_mean_flow_residual_equals_laminar_without_turbulence(oracle_mod):
    case7 = cases.partitioned_turbulent_channel(24, 12, 2, isplit=(10,), jsplit=(5,), reyno=500.0)
    case5 = cases.partitioned_laminar_channel(24, 12, 2, isplit=(10,), jsplit=(5,), reyno=500.0)
    q5 = cases.perturbed_state(case5, amp=0.05, seed=2)
    case7.params.tkefar = 0.0  # no k in the inlet halo either
    O7, A7 = _setup(oracle_mod, case7)
    q7 = A7.q
    for v7, v5 in zip(p3_views(case7.tables, q7, 7, 1), p3_views(case5.tables, q5, 5, 1)):
        v7[..., :5, :] = v5
        v7[..., 5, :] = 0.0
        v7[..., 6, :] = 1.0
    A7.mut[:] = 0.0
    st = oracle_mod.residual_rans(O7, A7, want_dt=False)
    assert st == 0
    O5 = oracle_mod.OracleLevel(case5.tables, case5.params)
    x, y, z = case5.x.copy(), case5.y.copy(), case5.z.copy()
    si, sj, sk, vol = O5.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O5, x, y, z, vol)
    res5, _, st5 = oracle_mod.residual_ns(O5, q5.copy(), si, sj, sk, vol, vm, want_dt=False)
    assert st5 == 0
    for r7, r5 in zip(p3_views(case7.tables, A7.res, 7, 1), p3_views(case5.tables, res5, 5, 1)):
        a, b = r7[2:-2, 2:-2, 2:-2, :5], r5[2:-2, 2:-2, 2:-2, :5]
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()  # the residual is a sum of O(1) fluxes


def test_menter_wall_omega(oracle_mod):
    case = cases.turbulent_channel(16, 8, 2)
    p = case.params
    O, A = _setup(oracle_mod, case)
    q = case.q0.copy()
    O.cons2prim(q)
    assert oracle_mod.bc_dist(O, q, A.si, A.sj, A.sk, A.dist) == 0
    v = p3_views(case.tables, q, 7, 1)[0]
    d = p1_views(case.tables, A.dist, 1)[0][..., 0]
    (im, jm, km), = case.tables.dims
    rhow, pw = v[2:im + 1, 1, 2:km + 1, 0, 0], v[2:im + 1, 1, 2:km + 1, 4, 0]
    tw = pw * p.gamma / rhow
    muw = (p.stemp + 1) / (tw + p.stemp) * tw ** 1.5
    dd = d[1:im, 1, 1:km]
    omew = 60.0 * muw / (p.bkw * rhow * dd * dd + 1e-24) * p.machfs / p.reyno
    np.testing.assert_allclose(v[2:im + 1, 1, 2:km + 1, 6, 0], omew, rtol=1e-13)
    assert np.all(v[2:im + 1, 1, 2:km + 1, 5, 0] == 0.0)
    np.testing.assert_array_equal(v[2:im + 1, 0, 2:km + 1, 5:, 0], v[2:im + 1, 1, 2:km + 1, 5:, 0])


def test_rans_smooth_runs(oracle_mod):
    case = cases.turbulent_channel(24, 12, 2)
    O, A = _setup(oracle_mod, case)
    A.q[:] = case.q0
    qq = A.q.copy()
    O.cons2prim(qq)
    oracle_mod.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist)
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle_mod.tur_vis(O, qq, A.mut)
    oracle_mod.cutman_mut(O, A.mut)
    hist, st = oracle_mod.smooth_rans(O, A, 10, rms_every=5)
    assert st == 0
    rows = hist[~np.isnan(hist[:, 0])]
    assert np.isfinite(rows).all() and (rows[:, [0, 1, 4, 5, 6]] > 0).all()


def test_rest4_and_omega_residual_limiter(oracle_mod):
    """rest4 restricts a constant to itself; lim_res_ome rewrites the omega
    residual exactly where the point-implicit update would undercut
    gkw cmu rho sqrt(prd), to the value that lands on that floor."""
    case = cases.turbulent_channel(16, 8, 4)
    p = case.params
    lv = cases.mg_levels(case, 2)
    Of, Oc = (oracle_mod.OracleLevel(t, p) for (t, _, _, _) in lv)
    vf = np.random.default_rng(1).uniform(0.5, 2.0, Of.p1().size)
    vc = np.zeros(Oc.p1().size)
    # coarse volumes = sums of their 8 fine volumes, so a constant survives
    for bf, bc in zip(p1_views(lv[0][0], vf, 1), p1_views(lv[1][0], vc, 1)):
        f = bf[1:-1, 1:-1, 1:-1, 0]
        bc[1:-1, 1:-1, 1:-1, 0] = (f[0::2, 0::2, 0::2] + f[1::2, 0::2, 0::2] + f[0::2, 1::2, 0::2] +
                                   f[1::2, 1::2, 0::2] + f[0::2, 0::2, 1::2] + f[1::2, 0::2, 1::2] +
                                   f[0::2, 1::2, 1::2] + f[1::2, 1::2, 1::2])
    f1 = np.full(Of.n3 * Of.S, 3.25)
    f2 = np.zeros(Oc.n3 * Oc.S)
    oracle_mod.rest4(Of, Oc, f1, f2, vf, vc)
    (im, jm, km), = lv[1][0].dims
    f2v = f2.reshape(km + 3, jm + 3, im + 3)[2:-2, 2:-2, 2:-2]
    np.testing.assert_allclose(f2v, 3.25, rtol=1e-14)
    # lim_res_ome on a uniform conservative state
    O = Of
    rho, rk, rw = 1.1, 2e-4, 0.4
    q = O.p3()
    for v in p3_views(lv[0][0], q, 7, 1):
        v[..., 0, 0] = rho
        v[..., 5, 0] = rk
        v[..., 6, 0] = rw
    dtt = np.full(O.n1, 0.02)
    vol = np.full(O.n1, 0.5)
    dpl = np.zeros(O.n3)
    prd = np.full(O.n3, 0.09)
    res = O.p3()
    r = p3_views(lv[0][0], res, 7, 1)[0]
    r[..., 6, 0] = 100.0          # large positive residual: rho omega would drop below the floor
    r[2:-2, 2:-2, 2, 6, 0] = -1.0  # negative residual on one k plane: untouched
    ar = 0.25
    oracle_mod.lim_res_ome(O, res, q, vol, dtt, dpl, prd, ar)
    dtau = 0.02 * 0.5
    den1 = 1 + ar * dtau * (2 * p.bkw * rw / rho)
    floor = p.gkw * p.cmu * rho * np.sqrt(0.09)
    assert rw - ar * 100.0 * 0.02 / den1 < floor
    np.testing.assert_allclose(r[2:-2, 2:-2, 3:-2, 6, 0], den1 * (rw - floor) / 0.02 / ar, rtol=1e-13)
    assert np.all(r[2:-2, 2:-2, 2, 6, 0] == -1.0)


def test_kom_multigrid_accelerates(oracle_mod):
    """Three-level k-omega V-cycles (forcing, restricted production terms,
    lim_res_ome) reduce the density residual faster than single-grid
    cycles from the same start."""
    import casekit
    out = {}
    for nlevel in (1, 3):
        p = cases.kom_params(0.3, 1e5)
        p.cfl = p.cflt = 1.5
        p.nlevel = nlevel
        p.nstart = p.npre = p.npost = p.ncrs = 1
        p.bln_prol = 1
        case = cases.turbulent_channel(32, 16, 8)
        lv, Os, As = casekit.mg_rans_oracle(case, nlevel, p, oracle_mod)
        h, st = oracle_mod.mg_rans(Os, As, 1, 30, 30, rms_every=10)
        assert st == 0
        rows = h[~np.isnan(h[:, 0])]
        assert np.isfinite(rows).all()
        out[nlevel] = rows[-1, 0] / rows[0, 0]
    assert out[3] < 0.5 * out[1], out


def test_cfl_ramps():
    """bdeltat's k-omega CFL ramps (src/cosa.f90:4763-4815): mode 1 holds its
    value between cycle 1 and every 100th cycle and grows cubically then
    linearly; mode 2 is piecewise linear; both are continuous at the
    segment ends and reach the final CFL."""
    from cosa_b200.params import cfl_ramp
    nc, c, t = (0, 100, 600, 1200), (0.5, 1.5, 3.0), (0.4, 1.0, 2.0)
    cur = None
    seen = []
    for m in range(1, 1401):
        cur = cfl_ramp(m, 1, nc, c, t, cur)
        seen.append(cur)
    assert seen[0] == (0.5, 0.4) and seen[1399] == (3.0, 2.0)
    assert seen[149] == seen[100]                       # held between updates (cycles 101..199)
    np.testing.assert_allclose(cfl_ramp(600, 1, nc, c, t), (1.5, 1.0), rtol=1e-12)
    np.testing.assert_allclose(cfl_ramp(900, 1, nc, c, t), (2.25, 1.5), rtol=1e-12)
    nc2 = (50, 150, 300, 500)
    np.testing.assert_allclose(cfl_ramp(50, 2, nc2, c, t), (0.5, 0.4))
    np.testing.assert_allclose(cfl_ramp(100, 2, nc2, c, t), (1.0, 0.7), rtol=1e-12)
    np.testing.assert_allclose(cfl_ramp(200, 2, nc2, c, t), (1.5, 1.0))
    np.testing.assert_allclose(cfl_ramp(400, 2, nc2, c, t), (2.25, 1.5), rtol=1e-12)
    np.testing.assert_allclose(cfl_ramp(600, 2, nc2, c, t), (3.0, 2.0))
