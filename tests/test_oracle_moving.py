"""Known-answer tests of the oracle's moving-grid pieces (harmonic balance of
a rigidly pitching body): pitch/movegrid (src/grid.f90:1783-1966), the face
velocities of imetrix_b (src/grid.f90:1024-1062), vert2cell_bg
(src/output.f90:3276-3480) and the face speed in roflux_b
(src/flux.f90:110-189)."""
import numpy as np
import pytest

from cosa_b200 import cases
from cosa_b200.cases import p2_views

import oracle


def _case(nharms=1):
    return cases.naca_pitching(nharms=nharms, blocks=(8, 8, 8, 8), nj=8, rfar=10.0, h1=2e-2)


def _setup(case):
    O = oracle.OracleLevel(case.tables, case.params)
    ones = np.ones(O.n1)
    m = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    return O, m


def _snap(tables, a, S):
    """Per-block node views (I2, J2, K2, S) of a snapshot-resolved node array."""
    off, _ = tables.offsets()
    out = []
    for b, (im, jm, km) in enumerate(tables.dims):
        n = (im + 2) * (jm + 2) * (km + 2)
        out.append(a[off["p2"][b] * S:off["p2"][b] * S + n * S].reshape((im + 2, jm + 2, km + 2, S), order="F"))
    return out


@pytest.mark.parametrize("nharms", [1, 2])
def test_pitch_is_a_rigid_rotation(nharms):
    """With unit displacement scales every node of snapshot n is x0 rotated
    by theta_n about the hinge, and its velocity is theta'_n e_z x (x - x_h)
    with theta'_n = dtheta0 omegas cos(omegas t_n)."""
    case = _case(nharms)
    p = case.params
    O, m = _setup(case)
    S = O.S
    zeit, dth = oracle.hb_motion(p, S)
    np.testing.assert_allclose(dth, p.dtheta0 * np.sin(p.omegas * zeit), rtol=0, atol=1e-16)
    X0 = p2_views(case.tables, case.x, 1)
    Y0 = p2_views(case.tables, case.y, 1)
    xs, ys = _snap(case.tables, m["x"], S), _snap(case.tables, m["y"], S)
    for b in range(case.tables.nblocks):
        for n in range(S):
            c, s = np.cos(dth[n]), np.sin(dth[n])
            rx, ry = X0[b] - p.xh, Y0[b] - p.yh
            np.testing.assert_allclose(xs[b][..., n], p.xh + c * rx - s * ry, rtol=0, atol=1e-13)
            np.testing.assert_allclose(ys[b][..., n], p.yh + s * rx + c * ry, rtol=0, atol=1e-13)


def test_face_velocity_of_a_rotation():
    """A rigid rotation's velocity is linear in position, so the mean of a
    face's four node velocities is the rotation velocity at the mean of its
    four nodes."""
    case = _case(2)
    p = case.params
    O, m = _setup(case)
    S = O.S
    zeit, dth = oracle.hb_motion(p, S)
    om = p.dtheta0 * p.omegas * np.cos(p.omegas * zeit)
    xs, ys = _snap(case.tables, m["x"], S), _snap(case.tables, m["y"], S)
    for b, (im, jm, km) in enumerate(case.tables.dims):
        f = m["fvi"][case.tables.offsets()[0]["p2"][b] * 3 * S:][:(im + 2) * (jm + 2) * (km + 2) * 3 * S]
        f = f.reshape((3, im + 2, jm + 2, km + 2, S), order="F")
        for n in range(S):
            X, Y = xs[b][..., n], ys[b][..., n]
            for k in range(1, km):
                for j in range(1, jm):
                    for i in range(1, im + 1):
                        xc = (X[i, j + 1, k + 1] + X[i, j + 1, k] + X[i, j, k + 1] + X[i, j, k]) / 4
                        yc = (Y[i, j + 1, k + 1] + Y[i, j + 1, k] + Y[i, j, k + 1] + Y[i, j, k]) / 4
                        np.testing.assert_allclose(f[0, i, j, k, n], -om[n] * (yc - p.yh), rtol=0, atol=1e-14)
                        np.testing.assert_allclose(f[1, i, j, k, n], om[n] * (xc - p.xh), rtol=0, atol=1e-14)
                        assert f[2, i, j, k, n] == 0.0


def test_vert2cell_of_a_linear_field():
    """Interior cells take the mean of their 8 nodes: exact for a field
    linear in the node indices at the cell's index centre; bounding-face
    cells the mean of the 4 face nodes, edges of 2, vertices the node."""
    case = _case(1)
    O, m = _setup(case)
    S = O.S
    w = np.zeros(O.n2 * S)
    for v in _snap(case.tables, w, S):
        I, J, K = np.meshgrid(*(np.arange(n, dtype=float) for n in v.shape[:3]), indexing="ij")
        for n in range(S):
            v[..., n] = 0.5 + 0.3 * I - 0.2 * J + 0.7 * K + n
    oracle.lib().orc_vert2cell(O.h, oracle._p(w))
    for (im, jm, km), v in zip(case.tables.dims, _snap(case.tables, w, S)):
        def node(i, j, k, n):
            return 0.5 + 0.3 * i - 0.2 * j + 0.7 * k + n
        for n in range(S):
            for (i, j, k) in [(2, 3, 1), (1, 1, 1), (im - 1, jm - 1, km - 1)]:
                assert abs(v[i, j, k, n] - node(i + 0.5, j + 0.5, k + 0.5, n)) < 1e-13
            # a bounding face (k = 0): mean of the 4 nodes at k = 1
            assert abs(v[2, 3, 0, n] - node(2.5, 3.5, 1, n)) < 1e-13
            # an edge (j = 0, k = kmax): mean of 2 nodes along i
            assert abs(v[3, 0, km, n] - node(3.5, 1, km, n)) < 1e-13
            # a vertex
            assert abs(v[im, jm, 0, n] - node(im, jm, 1, n)) < 1e-13


def test_roe_flux_on_a_moving_face():
    """roflux_b with a face moving at normal speed ubn: equal states give the
    flux relative to the face, F(q) - ubn q (mass, momentum) and
    (rho h0)(u.n - ubn) + p ubn (energy); supersonic motion of the face is
    still upwinded consistently (F(q, q) does not depend on the limiter)."""
    p = cases.naca_params("euler", mach=0.5)
    g = p.gamma
    rng = np.random.default_rng(3)
    for _ in range(20):
        nrm = rng.standard_normal(3)
        nrm /= np.linalg.norm(nrm)
        ds, ubn = rng.uniform(0.5, 2.0), rng.uniform(-0.8, 0.8)
        q = np.array([rng.uniform(0.5, 1.5), *rng.uniform(-0.5, 0.5, 3), rng.uniform(0.5, 1.0)])
        f = oracle.roe_face(p, np.array([*nrm, ds, ubn]), q, q)
        rho, u, pr = q[0], q[1:4], q[4]
        un = u @ nrm - ubn
        h0 = g / (g - 1) * pr / rho + u @ u / 2
        want = np.array([rho * un, *(rho * u * un + pr * nrm), rho * h0 * un + pr * ubn]) * ds
        np.testing.assert_allclose(f, want, rtol=1e-13, atol=1e-15)
