"""k-omega RANS harmonic balance of a rigidly pitching NACA 0012 on the
device against the oracle, through the C-ABI: the viscous set-up of every
node snapshot (coordex, cut_x and vmetrix per snapshot), the fused k-omega
stage with the face speeds in the mean-flow and turbulence Roe fluxes, the
grid velocity in the viscous spectral radii, the 1500 wall moving with the
body (Wilcox's wall omega from the velocity relative to the wall), and the
per-snapshot pressure and skin-friction forces with the wall derivative of
the velocity relative to the grid.

States 1e-12 relative to the largest value of each variable, residual norms
1e-9, forces 1e-10 of the largest coefficient."""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p3_views
from cosa_b200.params import PREC_MIXED

import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _case(nharms, **kw):
    return cases.naca_pitching(nharms=nharms, blocks=(16, 16, 16, 16), nj=16, rfar=12.0, h1=5e-3, model="kom",
                               **kw)


def _state(case, seed):
    """A snapshot-dependent perturbation of the mean flow over the free
    stream; k and omega stay at their free-stream values."""
    S = 2 * case.params.nharms + 1
    q = case.q0.copy()
    rng = np.random.default_rng(seed)
    for v in p3_views(case.tables, q, 7, S):
        I, J, K = v.shape[:3]
        ii = np.arange(I)[:, None, None] / max(I - 1, 1)
        jj = np.arange(J)[None, :, None] / max(J - 1, 1)
        for var in range(5):
            a, ph = rng.uniform(0.5, 1.5, 2), rng.uniform(0, 2 * np.pi, 2)
            f = np.sin(2 * np.pi * a[0] * ii + ph[0]) * np.cos(2 * np.pi * a[1] * jj + ph[1])
            scale = 0.01 * (abs(v[..., var, 0]).mean() + 0.1)
            for n in range(S):
                v[..., var, n] = v[..., var, n] + scale * f * (1.0 + 0.5 * np.sin(2 * np.pi * n / S + 0.3))
    return q


def _rel(a, b, tables, S):
    worst = 0.0
    for va, vb in zip(p3_views(tables, a, 7, S), p3_views(tables, b, 7, S)):
        ia, ib = cases.interior(va), cases.interior(vb)
        sc = np.abs(ib).reshape(-1, 7, S).max(axis=(0, 2))
        sc[1:4] = max(sc[1:4].max(), 1e-300)  # momentum components share one scale
        worst = max(worst, float((np.abs(ia - ib) / sc[None, None, None, :, None]).max()))
    return worst


def _oracle_setup(case, q):
    p = case.params
    O = oracle.OracleLevel(case.tables, p)
    A = oracle.RansArrays(O)
    ones = np.ones(O.n1)
    mo = oracle.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    A.si, A.sj, A.sk, A.vol = mo["si"], mo["sj"], mo["sk"], mo["vol"]
    A.vm = oracle.viscous_setup(O, mo["x"], mo["y"], mo["z"], A.vol)
    # rigid motion: the wall distance of every snapshot is that of the grid at rest
    A.dist[:] = cases.wall_distance(case)
    A.q[:] = q
    qq = A.q.copy()
    O.cons2prim(qq)
    oracle.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist)
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle.tur_vis(O, qq, A.mut)
    oracle.cutman_mut(O, A.mut)
    return O, A, mo


def _device_setup(case, A):
    p = case.params
    ctx = gpu.Context([case.tables], p)
    m = ctx.pitching_setup(1, case)
    vm = ctx.alloc_vm(1)
    ctx.viscous_setup(1, m["x"], m["y"], m["z"], m["vol"], vm)
    d = {
        "q": ctx.alloc_p3().upload(A.q), "qold": ctx.alloc_p3(), "res": ctx.alloc_p3(), "rhs": ctx.alloc_p3(),
        "dtvol": ctx.alloc_p1(nsnap=ctx.S), "dtvolt": ctx.alloc_p1(nsnap=ctx.S),
        "si": m["si"], "sj": m["sj"], "sk": m["sk"], "vol": m["vol"],
        "qp": ctx.alloc_p3(), "qm": ctx.alloc_p3(), "dq": ctx.alloc_p3(), "dqp": ctx.alloc_p3(),
        "dqm": ctx.alloc_p3(), "flux": ctx.alloc_f0(),
        "mut": ctx.alloc_p3s().upload(A.mut), "dist": ctx.alloc_p1().upload(A.dist),
        "xdot": m["xdot"], "ydot": m["ydot"], "zdot": m["zdot"], "fvi": m["fvi"], "fvj": m["fvj"], "fvk": m["fvk"],
    }
    ctx.bind_level(1, **d)
    return ctx, m, vm, d


def test_moving_viscous_setup_matches_oracle():
    """coordex, cut_x and the face inverse metrics of every node snapshot."""
    case = _case(2)
    O, A, mo = _oracle_setup(case, case.q0)
    ctx, m, vm, _ = _device_setup(case, A)
    for k in ("x", "y", "z", "vol"):
        a, b = m[k].download(), mo[k]
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max(), k
    a = vm.download()
    assert a.size == A.vm.size
    assert np.abs(a - A.vm).max() <= 1e-12 * np.abs(A.vm).max()
    ctx.close()


@pytest.mark.parametrize("nharms,model", [(1, "kom"), (2, "kom"), (1, "sst")])
def test_kom_pitching_hb_cycles_match_oracle(nharms, model):
    case = _case(nharms)
    p = case.params
    if model == "sst":
        p.kom, p.kom_sst = 0, 1
    S = 2 * p.nharms + 1
    q = _state(case, 11 + nharms)
    O, A, mo = _oracle_setup(case, q)
    ctx, m, vm, d = _device_setup(case, A)
    ncyc = 4
    ho, st = oracle.mg_rans([O], [A], 1, ncyc, ncyc, rms_every=1)
    assert st == 0
    hg, stg = ctx.mg(1, ncyc, ncyc, rms_every=1)
    assert stg == 0
    assert _rel(d["q"].download(), A.q, case.tables, S) <= TOL
    np.testing.assert_allclose(hg, ho, rtol=1e-9, atol=1e-15)
    # per-snapshot pressure and skin-friction forces on the moving wall
    co = oracle.force(O, A.q, mo["x"], mo["y"], mo["z"], A.si, A.sj, A.sk, A.vm, lngth=(1.0, 0.1, 1.0))
    cg = ctx.force(1, d["q"], m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], vm=vm, lngth=(1.0, 0.1, 1.0))
    assert np.abs(cg - co).max() <= 1e-10 * np.abs(co).max()
    assert np.abs(co[:, 6:]).max() > 0  # the skin-friction part is present
    ctx.close()


def test_mixed_precision_moving_kom_close_to_fp64():
    """FP32 reconstruction and Roe dissipation (the face speed in both) on
    the pitching grid: 20 cycles of k-omega HB (S = 3) against the FP64
    device path, states within 1e-6 of the largest value of each variable
    and the per-snapshot force and moment coefficients within 1e-6."""
    out = {}
    for prec in (0, PREC_MIXED):
        case = _case(1)
        case.params.precision = prec
        q = _state(case, 21)
        O, A, mo = _oracle_setup(case, q)
        ctx, m, vm, d = _device_setup(case, A)
        hg, st = ctx.smooth(1, 20, 1, 20)
        assert st == 0
        c = ctx.force(1, d["q"], m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], vm=vm, lngth=(1.0, 0.1, 1.0))
        out[prec] = (d["q"].download(), c, case.tables)
        ctx.close()
    (q64, c64, t), (q32, c32, _) = out[0], out[PREC_MIXED]
    err = _rel(q32, q64, t, 3)
    assert 0 < err <= 1e-6, err
    assert np.abs(c32 - c64).max() <= 1e-6, np.abs(c32 - c64).max()
