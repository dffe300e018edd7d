"""Parity with the oracle at the benchmark configurations' own sizes, through
the C-ABI, with the error measured per cell:

  - the bump channel, 128 x 64 x 2 cells, 2000 RK iterations from the free
    stream, the residual history every 100 iterations;
  - one RK cycle of the 30.7 M-cell, 24-block duct;
  - Wilcox k-omega on the 512 x 128 x 2 NACA 0012 O-grid with implicit
    residual smoothing, three cycles;
  - harmonic balance with S = 5 snapshots on the pitching 256 x 64 x 2
    NACA 0012 O-grid, twenty cycles.

Per cell: |gpu - oracle| / |oracle| for rho and rho E (never near zero);
besides, the normwise bound of the other parity tests (largest difference
over the largest value of the variable).  The device contracts
multiply-adds and takes Newton-Raphson reciprocals where the oracle keeps
the reference's operation order, so the two differ by rounding, which 2000
iterations of a converging solve do not amplify beyond the bounds below.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu
from cosa_b200.cases import p3_views

import casekit

pytestmark = pytest.mark.gpu


def _errors(case, a, b, nvar, nsnap=1):
    """(per-cell relative error of rho and rho E, normwise error of every
    variable with the momentum components on one scale)."""
    A = np.concatenate([cases.interior(v).reshape(-1, nvar, nsnap, order="F")
                        for v in p3_views(case.tables, a, nvar, nsnap)], axis=0)
    B = np.concatenate([cases.interior(v).reshape(-1, nvar, nsnap, order="F")
                        for v in p3_views(case.tables, b, nvar, nsnap)], axis=0)
    if not (np.isfinite(A).all() and np.isfinite(B).all()):
        return np.inf, np.inf
    d = np.abs(A - B)
    per_cell = float(max((d[:, 0] / np.abs(B[:, 0])).max(), (d[:, 4] / np.abs(B[:, 4])).max()))
    sc = np.abs(B).max(axis=(0, 2))
    sc[1:4] = sc[1:4].max()
    norm = float((d / sc[None, :, None]).max())
    return per_cell, norm


def test_bump_channel_2000_iterations_with_history(oracle_mod):
    case = cases.bump_channel()  # 128 x 64 x 2, CFL 2, M 0.5 inlet
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    qo = case.q0.copy()
    hist_o, st = O.smooth(qo, si, sj, sk, 2000, rms_every=100)
    assert st == 0
    ctx = gpu.Context([case.tables], case.params)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    q = ctx.alloc_p3().upload(case.q0)
    ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    hist_g, st = ctx.smooth(1, 2000, 1, 100)
    assert st == 0
    per_cell, norm = _errors(case, q.download(), qo, 5)
    print(f"bump channel 2000 it: per-cell {per_cell:.2e}, normwise {norm:.2e}")
    assert per_cell <= 1e-10 and norm <= 1e-11
    rows = ~np.isnan(hist_o[:, 0])
    assert rows.sum() == 21 and np.array_equal(rows, ~np.isnan(hist_g[:, 0]))
    # the w-momentum residual of a two-dimensional flow is zero in the oracle
    # and rounding-sized on the device
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-8, atol=1e-15)
    ctx.close()


def test_duct_30m_one_cycle(oracle_mod):
    case = cases.duct3d()  # 30.7 M cells, 24 blocks, seed 3
    assert case.ncells > 27_000_000
    O = oracle_mod.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    qo = case.q0.copy()
    hist_o, st = O.smooth(qo, si, sj, sk, 1, rms_every=1)
    assert st == 0
    ctx = gpu.Context([case.tables], case.params)
    m = [ctx.alloc_p2().upload(a) for a in (si, sj, sk)]
    del si, sj, sk
    q = ctx.alloc_p3().upload(case.q0)
    ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=m[0], sj=m[1], sk=m[2])
    ctx.autotune(1, 1)  # whichever stage schedule the bench would run
    q.upload(case.q0)
    hist_g, st = ctx.smooth(1, 1, 1, 1)
    assert st == 0
    per_cell, norm = _errors(case, q.download(), qo, 5)
    print(f"30.7M duct 1 cycle: per-cell {per_cell:.2e}, normwise {norm:.2e}")
    assert per_cell <= 1e-12 and norm <= 1e-12
    np.testing.assert_allclose(hist_g, hist_o, rtol=1e-9)
    ctx.close()


def test_kom_naca_512x128_irs_cycles(oracle_mod):
    import test_gpu_kom as K
    p = cases.naca_params("kom", mach=0.3, alpha_deg=4.0, reyno=6.0e6, cfl=3.0, eps_irs=0.6)
    case = cases.naca0012_ogrid(params=p)  # 512 x 128 x 2 in blocks 96/160/160/96
    qo, muo, ho, qg, mug, hg = K._smooth_pair(oracle_mod, case, 3, seed=2)
    per_cell, norm = _errors(case, qg, qo, 7)
    print(f"k-omega NACA 512x128x2 3 cycles: per-cell {per_cell:.2e}, normwise {norm:.2e}")
    assert per_cell <= 1e-11 and K._state_err(case, qg, qo) <= 1e-11
    mo, mg_ = casekit.interior_cells(case, muo, 1), casekit.interior_cells(case, mug, 1)
    assert np.abs(mo - mg_).max() <= 1e-11 * np.abs(mo).max()
    rows = ~np.isnan(ho[:, 0])
    np.testing.assert_allclose(hg[rows], ho[rows], rtol=1e-9)


def test_pitching_hb_s5_full_grid(oracle_mod):
    import test_gpu_pitching as T
    case = cases.naca_pitching(nharms=2)  # 256 x 64 x 2, S = 5
    p = case.params
    S = 5
    O = oracle_mod.OracleLevel(case.tables, p)
    ones = np.ones(O.n1)
    mo = oracle_mod.moving_setup(O, case.x, case.y, case.z, ones, ones, ones)
    q = T._state(case, 11)
    qo = q.copy()
    hist_o, st = oracle_mod.smooth_hb(O, qo, mo["si"], mo["sj"], mo["sk"], mo["vol"], 20, rms_every=5)
    assert st == 0
    ctx, m = T._device(case)
    dq = T._bind(ctx, m, q)
    hist_g, st = ctx.smooth(1, 20, 1, 5)
    assert st == 0
    per_cell, norm = _errors(case, dq.download(), qo, 5, S)
    print(f"pitching HB S=5 256x64x2 20 cycles: per-cell {per_cell:.2e}, normwise {norm:.2e}")
    assert per_cell <= 1e-11 and norm <= 1e-12
    rows = ~np.isnan(hist_o[:, 0])
    np.testing.assert_allclose(hist_g[rows], hist_o[rows], rtol=1e-9)
    ctx.close()
