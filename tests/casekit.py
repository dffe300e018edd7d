"""Test helpers: small cases, oracle metrics, and error measures."""
from __future__ import annotations

import numpy as np

from cosa_b200 import cases
from cosa_b200.cases import p3_views, interior


def small_channel(ni=48, nj=24, nk=2):
    return cases.bump_channel(ni, nj, nk)


def small_partitioned(ni=48, nj=24, nk=2, permute=True):
    return cases.partitioned_channel(ni, nj, nk, isplit=(20,), jsplit=(10,), permute_last=permute)


def small_duct(seed=5):
    # 2x3x4 partition with small segments (same generator as the 30M-cell case)
    segs = cases.duct_segments(seed=seed, lo=20_000, hi=60_000, choices=tuple(range(8, 33, 8)))
    return cases.duct3d(segs=segs)


def interior_cells(case, arr, nvar, nsnap=1):
    """Concatenated interior cells of every block: (ncells_total, nvar, nsnap)."""
    out = []
    for v in p3_views(case.tables, arr, nvar, nsnap):
        iv = interior(v)
        out.append(iv.reshape(-1, nvar, nsnap, order="F"))
    return np.concatenate(out, axis=0)


def scaled_err(gpu, ref, scale):
    """max |gpu - ref| / scale (scale per variable, broadcast on axis 1)."""
    d = np.abs(gpu - ref)
    return float((d / scale[None, :, None]).max())


def mg_oracle(case, nlevel, params, oracle_mod, q_fine=None):
    """Oracle levels + LevelArrays of an nlevel multigrid set-up of `case`;
    coarse states start at the free stream (init2fs on every level)."""
    lv = cases.mg_levels(case, nlevel)
    Os, As = [], []
    for i, (t, x, y, z) in enumerate(lv):
        O = oracle_mod.OracleLevel(t, params)
        A = oracle_mod.LevelArrays(O)
        A.si, A.sj, A.sk, A.vol = O.metrics(x, y, z)
        A.q[:] = case.q0 if i == 0 else cases._freestream_state(t, params)
        Os.append(O)
        As.append(A)
    if q_fine is not None:
        As[0].q[:] = q_fine
    return lv, Os, As


def mg_rans_oracle(case, nlevel, params, oracle_mod):
    """Oracle levels + RansArrays of an nlevel k-omega multigrid set-up of
    `case`: metrics, viscous set-up and wall distance on every level, the
    free stream on every level, the fine level's mut from its state after
    the BCs (coarse mut is set by the first cycle's visit)."""
    lv = cases.mg_levels(case, nlevel)
    Os, As = [], []
    for i, (t, x, y, z) in enumerate(lv):
        O = oracle_mod.OracleLevel(t, params)
        A = oracle_mod.RansArrays(O)
        x, y, z = x.copy(), y.copy(), z.copy()
        A.si, A.sj, A.sk, A.vol = O.metrics(x, y, z)
        A.vm = oracle_mod.viscous_setup(O, x, y, z, A.vol)
        A.dist[:] = cases.wall_distance(cases.Case("level", t, params, x, y, z, None))
        A.q[:] = case.q0 if i == 0 else cases._freestream_state(t, params)
        Os.append(O)
        As.append(A)
    O, A = Os[0], As[0]
    qq = A.q.copy()
    O.cons2prim(qq)
    oracle_mod.bc_dist(O, qq, A.si, A.sj, A.sk, A.dist)
    O.cutman_q(qq)
    O.prim2cons(qq)
    oracle_mod.tur_vis(O, qq, A.mut)
    oracle_mod.cutman_mut(O, A.mut)
    return lv, Os, As
