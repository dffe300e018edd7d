"""Wall forces on the device (cosa_gpu_force, through the C-ABI) against the
oracle's restatement of force_b (src/output.f90:4388-4900) summed over
blocks as force() does (src/output.f90:4283-4320):

* the 12 coefficients of a perturbed conservative state on a four-block
  NACA 0012 O-grid (laminar, so the skin-friction part runs too), one
  surface and a second, empty one; 1e-11 relative (the device sums the
  faces of a block as a tree, the reference in patch order);
* the k-omega smooth on the NACA O-grid (trailing-edge seam cut, far field,
  1500 walls with the Menter omega value) against the oracle's, then the
  forces of both final states.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.params import PREC_MIXED

import casekit

pytestmark = pytest.mark.gpu


def _naca(model, mach=0.5, reyno=1.0e4):
    p = cases.naca_params(model, mach=mach, alpha_deg=4.0, reyno=reyno, eps_irs=0.0)
    p.cfl = 1.0
    p.cflt = 1.0
    return cases.naca0012_ogrid(blocks=(12, 20, 20, 12), nj=16, nk=2, rfar=20.0, h1=2e-3, params=p)


def _geometry_gpu(ctx, case):
    X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
    m = [ctx.alloc_p2() for _ in range(3)]
    vol = ctx.alloc_p1()
    ctx.imetrix(1, X, Y, Z, *m)
    ctx.vols(1, X, Y, Z, vol)
    vm = ctx.alloc_vm()
    ctx.viscous_setup(1, X, Y, Z, vol, vm)
    return (X, Y, Z), m, vol, vm


def test_force_matches_oracle(oracle_mod):
    case = _naca("laminar")
    O = oracle_mod.OracleLevel(case.tables, case.params)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    si, sj, sk, vol = O.metrics(x, y, z)
    vm = oracle_mod.viscous_setup(O, x, y, z, vol)
    q = cases.perturbed_state(case, amp=0.05, seed=11)
    xm, ln = (0.25, 0.01, 0.0), (1.0, 0.1, 1.0)
    co = oracle_mod.force(O, q, x, y, z, si, sj, sk, vm, 1, xmom=xm, lngth=ln)
    ctx = gpu.Context([case.tables], case.params)
    (X, Y, Z), m, gvol, gvm = _geometry_gpu(ctx, case)
    gq = ctx.alloc_p3().upload(q)
    cg = ctx.force(1, gq, X, Y, Z, *m, vm=gvm, isurf=1, xmom=xm, lngth=ln)
    assert np.abs(co).max() > 1e-3 and np.abs(co[0, 6:]).max() > 0
    np.testing.assert_allclose(cg, co, rtol=1e-11, atol=1e-13)
    # no 1501 patch: surface 2 is empty
    c2 = ctx.force(1, gq, X, Y, Z, *m, vm=gvm, isurf=2, xmom=xm, lngth=ln)
    assert np.all(c2 == 0.0)
    ctx.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_rans_naca_smooth_and_forces_match_oracle(oracle_mod, precision):
    """FP64: state 1e-12, norms 1e-9, forces 1e-10.  Mixed (MUSCL slopes and
    Roe dissipation in FP32 on FP64 differences): state within 1e-6 of each
    variable's scale, force coefficients within 1e-7, and not identical."""
    case = _naca("kom", mach=0.5, reyno=1.0e5)
    mixed = precision == "mixed"
    O = oracle_mod.OracleLevel(case.tables, case.params)
    A = oracle_mod.RansArrays(O)
    x, y, z = case.x.copy(), case.y.copy(), case.z.copy()
    A.si, A.sj, A.sk, A.vol = O.metrics(x, y, z)
    A.vm = oracle_mod.viscous_setup(O, x, y, z, A.vol)
    dist = cases.wall_distance(case)
    A.dist[:] = dist
    q = case.q0.copy()  # impulsive start: free stream against the no-slip wall
    A.q[:] = q
    qq = q.copy()
    O.cons2prim(qq)
    assert oracle_mod.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist) == 0
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle_mod.tur_vis(O, qq, A.mut)
    oracle_mod.cutman_mut(O, A.mut)
    mut0 = A.mut.copy()
    ncyc = 6
    hist_o, st = oracle_mod.smooth_rans(O, A, ncyc, rms_every=2)
    assert st == 0

    pg = case.params
    if mixed:
        pg = cases.naca_params("kom", mach=0.5, alpha_deg=4.0, reyno=1.0e5, eps_irs=0.0)
        pg.cfl = pg.cflt = case.params.cfl
        pg.precision = PREC_MIXED
    ctx = gpu.Context([case.tables], pg)
    (X, Y, Z), m, gvol, gvm = _geometry_gpu(ctx, case)
    gdist = ctx.alloc_p1().upload(dist)
    arr = {k: ctx.alloc_p3() for k in ("q", "qold", "res", "qp", "qm", "dq", "dqp", "dqm")}
    arr["q"].upload(q)
    betas = [ctx.alloc_p1() for _ in range(3)]
    mut = ctx.alloc_p3s().upload(mut0)
    ctx.bind_level(1, q=arr["q"], qold=arr["qold"], res=arr["res"], dtvol=ctx.alloc_p1(), dtvolt=ctx.alloc_p1(),
                   si=m[0], sj=m[1], sk=m[2], vol=gvol, qp=arr["qp"], qm=arr["qm"], dq=arr["dq"], dqp=arr["dqp"],
                   dqm=arr["dqm"], flux=ctx.alloc_f0(), betaxi=betas[0], betaeta=betas[1], betazeta=betas[2],
                   mut=mut, dist=gdist)
    hist_g, st = ctx.smooth(1, ncyc, 1, 2)
    assert st == 0
    qg = arr["q"].download()
    A_ = casekit.interior_cells(case, qg, 7)
    B_ = casekit.interior_cells(case, A.q, 7)
    sc = np.abs(B_).reshape(-1, 7).max(axis=0)
    sc[3] = sc[1:3].max()  # rho w is rounding noise in this 2D flow: momentum scale
    err = (np.abs(A_ - B_) / sc[None, :, None]).max()
    tol = 1e-6 if mixed else 1e-12
    assert err <= tol, err
    # the face halos of both states (the wall halos feed the forces)
    for vg, vo in zip(cases.p3_views(case.tables, qg, 7, 1), cases.p3_views(case.tables, A.q, 7, 1)):
        hg, ho = vg[2:-2, 1, 2:-2, :5, 0], vo[2:-2, 1, 2:-2, :5, 0]
        assert np.isfinite(hg).all()
        assert np.abs(hg - ho).max() <= tol * np.abs(ho).max()
    rows = ~np.isnan(hist_o[:, 0])
    # the rho w norm is rounding noise (1e-16) on both sides
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-5 if mixed else 1e-9, atol=1e-15)
    xm, ln = (0.25, 0.0, 0.0), (1.0, 0.1, 1.0)
    co = oracle_mod.force(O, A.q, x, y, z, A.si, A.sj, A.sk, A.vm, 1, xmom=xm, lngth=ln)
    cg = ctx.force(1, arr["q"], X, Y, Z, *m, vm=gvm, isurf=1, xmom=xm, lngth=ln)
    if mixed:
        assert err > 0
        assert np.abs(cg - co).max() <= 1e-7, np.abs(cg - co).max()
    else:
        np.testing.assert_allclose(cg, co, rtol=1e-10, atol=1e-12)
    ctx.close()
