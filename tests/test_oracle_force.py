"""Known-answer tests of the oracle's wall-force integration (force_b,
src/output.f90:4388-4900, summed over blocks as force(), 4283-4320):

* a uniform state on the closed NACA 0012 contour gives no net pressure
  force and no skin friction; its pitching moment is only the offset of
  the reference's moment arm (the face's first node, not its centroid);
* a linear pressure p0 + a y, set at the face centroids, gives the force
  -a V (V the volume of the discrete body), split into lift and drag by
  the incidence;
* a linear shear u = c y over the flat wall of a box gives the skin
  friction M/Re mu_w c per unit area (the three-point wall derivative is
  exact for it) and the pressure force -p A;
* the NACA O-grid generator makes positive volumes and a closed seam.
"""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p2_views, p3_views
from cosa_b200.tables import BlockSpec


def _naca_small(model="euler", alpha_deg=4.0):
    p = cases.naca_params(model, mach=0.5, alpha_deg=alpha_deg, reyno=1.0e4, eps_irs=0.0)
    return cases.naca0012_ogrid(blocks=(12, 20, 20, 12), nj=12, nk=2, rfar=20.0, h1=1e-3, params=p)


def _geometry(oracle_mod, case):
    O = oracle_mod.OracleLevel(case.tables, case.params)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    si, sj, sk, vol = O.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O, x, y, z, vol)
    return O, x, y, z, si, sj, sk, vol, vm


def test_naca_grid_volumes_positive_and_seam_closed(oracle_mod):
    case = cases.naca0012_ogrid(blocks=(24, 40, 40, 24), nj=32, nk=2, h1=1e-4)
    O, x, y, z, si, sj, sk, vol, vm = _geometry(oracle_mod, case)
    from cosa_b200.cases import p1_views
    for v in p1_views(case.tables, vol, 1):
        assert (v[1:-1, 1:-1, 1:-1, 0] > 0).all()
    gx = p2_views(case.tables, case.x)
    gy = p2_views(case.tables, case.y)
    # trailing-edge seam: last block's imax plane is the first block's imin plane
    np.testing.assert_array_equal(gx[-1][-2, 1:-1, 1:-1], gx[0][1, 1:-1, 1:-1])
    np.testing.assert_array_equal(gy[-1][-2, 1:-1, 1:-1], gy[0][1, 1:-1, 1:-1])
    # wall nodes on the aerofoil contour
    X, Y = gx[1][1:-1, 1, 1], gy[1][1:-1, 1, 1]
    np.testing.assert_allclose(np.abs(Y), cases.naca0012_thickness(X), atol=1e-15)


def test_uniform_state_gives_no_force(oracle_mod):
    case = _naca_small("laminar")
    O, x, y, z, si, sj, sk, vol, vm = _geometry(oracle_mod, case)
    q = case.q0.copy()  # conservative free stream, halos included
    xm = (0.25, 0.0, 0.0)
    c = oracle_mod.force(O, q, x, y, z, si, sj, sk, vm, 1, xmom=xm, lngth=(1.0, 0.1, 1.0))
    assert c.shape == (1, 12)
    assert np.abs(c[0, :5]).max() < 1e-12
    assert np.abs(c[0, 6:]).max() < 1e-15  # (-8u + 9u - u)/3 rounds to O(eps u)
    # the moment arm is the face's first node, not its centroid: a uniform
    # pressure leaves sum_f ((r_node - r_face) x k ds)_z, which the closed
    # contour does not cancel
    pw = 1 / case.params.gamma / case.params.rhoinf
    mz = 0.0
    for X, Y, SJ in zip(p2_views(case.tables, x), p2_views(case.tables, y), p2_views(case.tables, sj, 4)):
        for k in (1, 2):
            xn, yn = X[1:-2, 1, k], Y[1:-2, 1, k]
            xf = 0.25 * (X[1:-2, 1, k] + X[2:-1, 1, k] + X[1:-2, 1, k + 1] + X[2:-1, 1, k + 1])
            yf = 0.25 * (Y[1:-2, 1, k] + Y[2:-1, 1, k] + Y[1:-2, 1, k + 1] + Y[2:-1, 1, k + 1])
            kx, ky, ds = SJ[0, 1:-2, 1, k], SJ[1, 1:-2, 1, k], SJ[3, 1:-2, 1, k]
            mz += np.sum((kx * (yn - yf) - ky * (xn - xf)) * pw * ds)
    cmf = 2 / (1.0 * 0.1 * 1.0 * case.params.machfs ** 2)
    np.testing.assert_allclose(c[0, 5], mz * cmf, rtol=1e-10)


def test_linear_pressure_gives_body_volume(oracle_mod):
    alpha = 4.0
    case = _naca_small("euler", alpha)
    p = case.params
    O, x, y, z, si, sj, sk, vol, vm = _geometry(oracle_mod, case)
    p0, a = 0.7, 0.3
    q = case.q0.copy()
    gx, gy = p2_views(case.tables, x), p2_views(case.tables, y)
    for v, X, Y in zip(p3_views(case.tables, q, 5, 1), gx, gy):
        # wall faces (i, 1, k): centroid of the planar face = mean of its 4 nodes
        yc = 0.25 * (Y[1:-2, 1, 1:-2] + Y[2:-1, 1, 1:-2] + Y[1:-2, 1, 2:-1] + Y[2:-1, 1, 2:-1])
        v[2:-2, 1, 2:-2, 0, 0] = 1.0
        v[2:-2, 1, 2:-2, 1:4, 0] = 0.0
        v[2:-2, 1, 2:-2, 4, 0] = (p0 + a * yc) / (p.gamma - 1)
    span = 0.1
    c = oracle_mod.force(O, q, x, y, z, si, sj, sk, None, 1, lngth=(1.0, span, 1.0))
    # body volume: shoelace area of the wall polygon times the span
    xs = np.concatenate([X[1:-2, 1, 1] for X in gx])
    ys = np.concatenate([Y[1:-2, 1, 1] for Y in gy])
    area = 0.5 * abs(np.dot(xs, np.roll(ys, -1)) - np.dot(ys, np.roll(xs, -1)))
    fy, fx = -a * area * span, 0.0
    cf = 2 / (1.0 * span * p.machfs ** 2)
    al = np.deg2rad(alpha)
    np.testing.assert_allclose(c[0, 0], (-np.sin(al) * fx + np.cos(al) * fy) * cf, rtol=1e-11)
    np.testing.assert_allclose(c[0, 1], (np.cos(al) * fx + np.sin(al) * fy) * cf, rtol=1e-11, atol=1e-14)


def test_linear_shear_wall_friction(oracle_mod):
    p = cases.laminar_params(0.3, 500.0)
    ni, nj, nk, DX, DY, DZ = 6, 5, 3, 0.1, 0.05, 0.2
    xs, ys, zs = DX * np.arange(ni + 1), DY * np.arange(nj + 1), DZ * np.arange(nk + 1)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    types = {"imin": 4, "imax": 4, "jmin": 1500, "jmax": 1501, "kmin": 80, "kmax": 80}
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, cases._face_bcs(ni + 1, nj + 1, nk + 1, types))
    case = cases._assemble("box", [(X.copy(), Y.copy(), Z.copy())], [spec], [], p)
    O, x, y, z, si, sj, sk, vol, vm = _geometry(oracle_mod, case)
    c_sh, rho, pr = 0.8, 1.1, 0.9
    q = O.p3()
    v = p3_views(case.tables, q, 5, 1)[0]
    J = np.arange(v.shape[1]) - 1           # P3 j index
    ycell = DY * (J - 0.5)                  # cell-centre height; the wall halo j = 0 holds the wall value
    u = np.where(J >= 1, c_sh * ycell, 0.0)
    v[..., 0, 0] = rho
    v[..., 1, 0] = rho * u[None, :, None]
    v[..., 4, 0] = pr / (p.gamma - 1) + 0.5 * rho * u[None, :, None] ** 2
    c = oracle_mod.force(O, q, x, y, z, si, sj, sk, vm, 1, lngth=(1.0, 1.0, 1.0))
    A = ni * DX * nk * DZ
    tw = pr * p.gamma / rho
    muw = (p.stemp + 1) / (tw + p.stemp) * tw ** 1.5
    cf = 2 / p.machfs ** 2
    np.testing.assert_allclose(c[0, 7], p.machfs / p.reyno * muw * c_sh * A * cf, rtol=1e-12)  # cd_v
    np.testing.assert_allclose(c[0, 6], 0.0, atol=1e-15)                                       # cl_v
    np.testing.assert_allclose(c[0, 0], -pr * A * cf, rtol=1e-12)                              # cl_p
    np.testing.assert_allclose(c[0, 1], 0.0, atol=1e-15)                                       # cd_p
