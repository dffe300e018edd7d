"""Synthetic multiblock cases in COSA's layout (grid, tables, parameters, state).

COSA ships no meshes or inputs, so every case is generated from formulas:

* ``bump_channel`` -- single-block quasi-2D channel with a 10%-thick
  circular-arc bump (radius 1.3 through (0,0), (0.5,0.1), (1,0)) on the lower
  wall; x uniform on [-1.5, 2.5], y linear between the wall and y=1, z two
  cells of width 0.1.  BCs 21 (inlet) / 91 (outlet) / 14 (walls) / 80
  (symmetry in z).
* ``duct3d`` -- 3D duct x in [-1,2], y in [0,1], z in [-1,1] with the floor
  bump h(x,z) = 0.1 sin^2(pi x) cos^2(pi z / 2) for x in [0,1]; a 2x3x4
  tensor partition into 24 blocks whose segment lengths are drawn (seeded)
  from {24, 32, ..., 160} until the cell count lies in a target window;
  1-to-1 cuts between neighbours.
* ``partitioned_channel`` -- the bump channel cut into several blocks, one of
  them stored with cyclically permuted indices, to exercise cut_q's iord.
* ``naca0012_ogrid`` -- O-grid around the NACA 0012 (4-digit formula, closed
  trailing edge), 512 x 128 x 2 cells in four blocks of 96/160/160/96 cells
  along the contour, far field 50 chords, first spacing of y+ ~ 1 at Re 6e6;
  BCs 1500 (wall, force surface 1) / 30 (far field) / 80 (k faces).

Arrays are flat float64 in the reference layout (column-major per block,
blocks concatenated with setoffs offsets).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .params import CosaParams, default_params, subsonic_inlet_total_state
from .tables import BlockSpec, LevelTables, build_tables, coarsen


@dataclass
class Case:
    name: str
    tables: LevelTables
    params: CosaParams
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    q0: np.ndarray  # conservative initial state (P3 * npde * S)

    @property
    def ncells(self) -> int:
        return self.tables.ncells()


# ---- layout helpers -------------------------------------------------------------
def p3_views(tables: LevelTables, arr: np.ndarray, npde: int, nsnap: int):
    """Per-block views (I3,J3,K3,npde,S) Fortran-ordered into a flat P3 array."""
    off, _ = tables.offsets()
    views = []
    for b, (im, jm, km) in enumerate(tables.dims):
        n = (im + 3) * (jm + 3) * (km + 3) * npde * nsnap
        s = off["p3"][b] * npde * nsnap
        views.append(arr[s:s + n].reshape((im + 3, jm + 3, km + 3, npde, nsnap), order="F"))
    return views


def p2_views(tables: LevelTables, arr: np.ndarray, ncomp: int = 1):
    off, _ = tables.offsets()
    views = []
    for b, (im, jm, km) in enumerate(tables.dims):
        n = (im + 2) * (jm + 2) * (km + 2) * ncomp
        s = off["p2"][b] * ncomp
        if ncomp == 1:
            views.append(arr[s:s + n].reshape((im + 2, jm + 2, km + 2), order="F"))
        else:
            views.append(arr[s:s + n].reshape((ncomp, im + 2, jm + 2, km + 2), order="F"))
    return views


def p1_views(tables: LevelTables, arr: np.ndarray, nsnap: int = 1):
    off, _ = tables.offsets()
    views = []
    for b, (im, jm, km) in enumerate(tables.dims):
        n = (im + 1) * (jm + 1) * (km + 1) * nsnap
        s = off["p1"][b] * nsnap
        views.append(arr[s:s + n].reshape((im + 1, jm + 1, km + 1, nsnap), order="F"))
    return views


def f0_views(tables: LevelTables, arr: np.ndarray, npde: int, nsnap: int = 1):
    """Per-block views (im, jm, km, npde, S) of a face-flux (F0) array."""
    off, _ = tables.offsets()
    views = []
    for b, (im, jm, km) in enumerate(tables.dims):
        n = im * jm * km * npde * nsnap
        s = off["f0"][b] * npde * nsnap
        views.append(arr[s:s + n].reshape((im, jm, km, npde, nsnap), order="F"))
    return views


def vm_views(tables: LevelTables, vm: np.ndarray):
    """Per-block views of the face inverse metrics: vm[b][d-1][m] is the
    (3, im, jm, km) array of the derivatives of xi (m=0), eta (1), zeta (2)
    on the faces of family d; array (d, m) starts at ((d-1)*3 + m)*3*n0."""
    off, tot = tables.offsets()
    n0 = tot["f0"]
    out = []
    for b, (im, jm, km) in enumerate(tables.dims):
        per = []
        for d in range(3):
            row = []
            for m in range(3):
                s = (d * 3 + m) * 3 * n0 + off["f0"][b] * 3
                row.append(vm[s:s + 3 * im * jm * km].reshape((3, im, jm, km), order="F"))
            per.append(row)
        out.append(per)
    return out


def interior(v: np.ndarray) -> np.ndarray:
    """Interior cells (1..imax-1, ...) of a P3 block view."""
    return v[2:-2, 2:-2, 2:-2]


def _embed_grid(nodes: np.ndarray, dst: np.ndarray):
    """nodes (ni,nj,nk) at 1..imax -> dst (0:imax+1) with linear halo extrapolation."""
    dst[1:-1, 1:-1, 1:-1] = nodes
    dst[0, :, :] = 2 * dst[1, :, :] - dst[2, :, :]
    dst[-1, :, :] = 2 * dst[-2, :, :] - dst[-3, :, :]
    dst[:, 0, :] = 2 * dst[:, 1, :] - dst[:, 2, :]
    dst[:, -1, :] = 2 * dst[:, -2, :] - dst[:, -3, :]
    dst[:, :, 0] = 2 * dst[:, :, 1] - dst[:, :, 2]
    dst[:, :, -1] = 2 * dst[:, :, -2] - dst[:, :, -3]


def _freestream_state(tables: LevelTables, p: CosaParams) -> np.ndarray:
    """init2fs (src/input.f90:4741-4775): conservative free stream everywhere."""
    _, tot = tables.offsets()
    S = 2 * p.nharms + 1
    q = np.zeros(tot["p3"] * p.npde * S)
    ca, sa = np.cos(p.alpha), np.sin(p.alpha)
    cb, sb = np.cos(p.beta), np.sin(p.beta)
    for v in p3_views(tables, q, p.npde, S):
        v[..., 0, :] = p.rhoinf
        v[..., 1, :] = p.rhoinf * p.machfs * ca * cb
        v[..., 2, :] = p.rhoinf * p.machfs * sa * cb
        v[..., 3, :] = p.rhoinf * p.machfs * sb
        v[..., 4, :] = 1 / p.rhoinf / p.gamma / (p.gamma - 1) + 0.5 * p.machfs ** 2
        if p.kom or p.kom_bsl or p.kom_sst:
            # interior cells only (src/input.f90:4826-4836)
            v[2:-2, 2:-2, 2:-2, 5, :] = p.rhoinf * p.tkefar
            v[2:-2, 2:-2, 2:-2, 6, :] = p.rhoinf * p.omefar
    return q


def _assemble(name, blocks_nodes, specs, cuts, params) -> Case:
    tables = build_tables(specs, cuts)
    _, tot = tables.offsets()
    x = np.zeros(tot["p2"]); y = np.zeros(tot["p2"]); z = np.zeros(tot["p2"])
    for (X, Y, Z), vx, vy, vz in zip(blocks_nodes, p2_views(tables, x), p2_views(tables, y), p2_views(tables, z)):
        _embed_grid(X, vx); _embed_grid(Y, vy); _embed_grid(Z, vz)
    q0 = _freestream_state(tables, params)
    return Case(name, tables, params, x, y, z, q0)


def _face_bcs(ni, nj, nk, types):
    """BC lines for the six faces of a block (node counts ni,nj,nk); types is
    a dict face->bctype with faces 'imin','imax','jmin','jmax','kmin','kmax'."""
    out = []
    f = {
        "imin": ((1, 1, 1), (1, nj, nk)), "imax": ((ni, 1, 1), (ni, nj, nk)),
        "jmin": ((1, 1, 1), (ni, 1, nk)), "jmax": ((1, nj, 1), (ni, nj, nk)),
        "kmin": ((1, 1, 1), (ni, nj, 1)), "kmax": ((1, 1, nk), (ni, nj, nk)),
    }
    for face in ("imin", "imax", "jmin", "jmax", "kmin", "kmax"):
        if face in types:
            s, e = f[face]
            out.append((s, e, types[face]))
    return out


def mg_levels(case: Case, nlevel: int):
    """[(tables, x, y, z)] of levels 1..nlevel: the coarsen() tables and the
    grid of every other node (coarsen_b, src/cosa.f90:2609-2670), halo nodes
    extrapolated as on the fine level."""
    out = [(case.tables, case.x, case.y, case.z)]
    for nl in range(2, nlevel + 1):
        f = 2 ** (nl - 1)
        if ((case.tables.dims - 1) % f).any():
            raise ValueError(f"cell counts not divisible by {f} for {nlevel} levels")
        t = coarsen(case.tables, nl)
        _, tot = t.offsets()
        grids = []
        for a in (case.x, case.y, case.z):
            dst = np.zeros(tot["p2"])
            for vf, vc in zip(p2_views(case.tables, a), p2_views(t, dst)):
                _embed_grid(vf[1:-1:f, 1:-1:f, 1:-1:f], vc)
            grids.append(dst)
        out.append((t, *grids))
    return out


# ---- configuration 1: bump channel ------------------------------------------------
def bump_wall(x: np.ndarray) -> np.ndarray:
    r = 1.3
    yb = np.sqrt(np.maximum(r * r - (x - 0.5) ** 2, 0.0)) - (r - 0.1)
    return np.where((x >= 0.0) & (x <= 1.0), yb, 0.0)


def channel_nodes(ni: int, nj: int, nk: int):
    """Node coordinates (ni+1, nj+1, nk+1) of the bump channel."""
    xs = -1.5 + 4.0 * np.arange(ni + 1) / ni
    eta = np.arange(nj + 1) / nj
    zs = 0.1 * np.arange(nk + 1)
    X = np.broadcast_to(xs[:, None, None], (ni + 1, nj + 1, nk + 1)).copy()
    yb = bump_wall(xs)[:, None, None]
    Y = np.broadcast_to(yb + (1.0 - yb) * eta[None, :, None], (ni + 1, nj + 1, nk + 1)).copy()
    Z = np.broadcast_to(zs[None, None, :], (ni + 1, nj + 1, nk + 1)).copy()
    return X, Y, Z


def channel_params(mach: float = 0.5) -> CosaParams:
    p = default_params()
    p.machfs = mach
    p.alpha = 0.0
    p.beta = 0.0
    t0, p0 = subsonic_inlet_total_state(p.gamma, mach)
    p.inlet_t0 = t0
    p.inlet_p0 = p0
    p.cfl = 2.0
    p.irsop = 0
    p.nstage = 4
    return p


def bump_channel(ni: int = 128, nj: int = 64, nk: int = 2, mach: float = 0.5, kface_bc: int = 80) -> Case:
    X, Y, Z = channel_nodes(ni, nj, nk)
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, _face_bcs(ni + 1, nj + 1, nk + 1, {
        "imin": 21, "imax": 91, "jmin": 14, "jmax": 14, "kmin": kface_bc, "kmax": kface_bc}))
    return _assemble(f"bump_channel_{ni}x{nj}x{nk}", [(X, Y, Z)], [spec], [], channel_params(mach))


def _permute_block(X, Y, Z):
    """Store a block with cyclically permuted indices: new (i,j,k) = old (j,k,i)."""
    return tuple(np.ascontiguousarray(np.transpose(A, (1, 2, 0))) for A in (X, Y, Z))


def partitioned_channel(ni: int = 48, nj: int = 24, nk: int = 2, isplit=(20,), jsplit=(10,),
                        permute_last: bool = True, mach: float = 0.5, kface_bc: int = 4, wall: int = 14,
                        params: CosaParams = None) -> Case:
    """Bump channel split at node planes isplit (i) and jsplit (j); the last
    block is stored with permuted indices when permute_last.  The z faces
    default to extrapolation (4): the reference's symmetry BC (80) reflects
    the velocity component of the block's own index direction
    (src/bc.f90:2684-2687), which is only the plane normal on blocks whose
    axes follow x, y, z."""
    X, Y, Z = channel_nodes(ni, nj, nk)
    ib = [0] + list(isplit) + [ni]
    jb = [0] + list(jsplit) + [nj]
    nbi, nbj = len(ib) - 1, len(jb) - 1
    nodes, specs, ids = [], [], {}
    perm = {}
    for bj in range(nbj):
        for bi in range(nbi):
            i0, i1, j0, j1 = ib[bi], ib[bi + 1], jb[bj], jb[bj + 1]
            Xb, Yb, Zb = (A[i0:i1 + 1, j0:j1 + 1, :] for A in (X, Y, Z))
            n = len(nodes)
            ids[(bi, bj)] = n + 1
            last = (bi == nbi - 1 and bj == nbj - 1)
            ni_b, nj_b, nk_b = i1 - i0 + 1, j1 - j0 + 1, nk + 1
            types = {}
            if bi == 0: types["imin"] = 21
            if bi == nbi - 1: types["imax"] = 91
            if bj == 0: types["jmin"] = wall
            if bj == nbj - 1: types["jmax"] = wall
            types["kmin"] = kface_bc
            types["kmax"] = kface_bc
            if permute_last and last and (nbi * nbj > 1):
                Xb, Yb, Zb = _permute_block(Xb, Yb, Zb)
                # old face -> new face under new(i,j,k) = old(j,k,i)
                fmap = {"imin": "kmin", "imax": "kmax", "jmin": "imin", "jmax": "imax",
                        "kmin": "jmin", "kmax": "jmax"}
                types = {fmap[f]: t for f, t in types.items()}
                dims = (nj_b, nk_b, ni_b)
                perm[n + 1] = True
            else:
                dims = (ni_b, nj_b, nk_b)
            nodes.append((Xb, Yb, Zb))
            specs.append(BlockSpec(*dims, _face_bcs(*dims, types)))
    cuts = []

    def face_nodes(b, face):
        """input.dat node range of a face of block b, in b's own indices."""
        ni_b, nj_b, nk_b = specs[b - 1].imax, specs[b - 1].jmax, specs[b - 1].kmax
        if b in perm:
            face = {"imin": "kmin", "imax": "kmax", "jmin": "imin", "jmax": "imax"}[face]
        return {
            "imin": ((1, 1, 1), (1, nj_b, nk_b)), "imax": ((ni_b, 1, 1), (ni_b, nj_b, nk_b)),
            "jmin": ((1, 1, 1), (ni_b, 1, nk_b)), "jmax": ((1, nj_b, 1), (ni_b, nj_b, nk_b)),
            "kmin": ((1, 1, 1), (ni_b, nj_b, 1)), "kmax": ((1, 1, nk_b), (ni_b, nj_b, nk_b)),
        }[face]

    def iord(b1, b2):
        # index of block 2 matching index l of block 1 (both in own storage)
        p1, p2 = b1 in perm, b2 in perm
        # storage axis of the "physical" (i,j,k) of the unpermuted channel
        ax = lambda p: (3, 1, 2) if p else (1, 2, 3)   # physical l -> storage axis
        inv = lambda p: (2, 3, 1) if p else (1, 2, 3)  # storage axis -> physical
        a1, a2 = inv(p1), ax(p2)
        return tuple(a2[a1[l] - 1] for l in range(3))

    for bj in range(nbj):
        for bi in range(nbi):
            b = ids[(bi, bj)]
            if bi + 1 < nbi:
                o = ids[(bi + 1, bj)]
                s1, e1 = face_nodes(b, "imax")
                s2, e2 = face_nodes(o, "imin")
                cuts.append((b, s1, e1, o, s2, e2, iord(b, o)))
            if bj + 1 < nbj:
                o = ids[(bi, bj + 1)]
                s1, e1 = face_nodes(b, "jmax")
                s2, e2 = face_nodes(o, "jmin")
                cuts.append((b, s1, e1, o, s2, e2, iord(b, o)))
    return _assemble(f"partitioned_channel_{ni}x{nj}x{nk}", nodes, specs, cuts,
                     params if params is not None else channel_params(mach))


# ---- laminar channel: viscous walls (bctyp 15xx) on the bump channel -----------------
VISCOUS_WALL = 1500


def laminar_params(mach: float = 0.3, reyno: float = 500.0) -> CosaParams:
    """Channel scheme with the laminar Navier-Stokes terms (viscous = .true.,
    no turbulence model) at Reynolds number reyno."""
    p = channel_params(mach)
    p.viscous = 1
    p.reyno = reyno
    p.cfl = 1.5
    return p


def laminar_channel(ni: int = 48, nj: int = 24, nk: int = 2, mach: float = 0.3, reyno: float = 500.0,
                    kface_bc: int = 80) -> Case:
    """The bump channel with no-slip adiabatic walls at j = 1 and j = jmax."""
    X, Y, Z = channel_nodes(ni, nj, nk)
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, _face_bcs(ni + 1, nj + 1, nk + 1, {
        "imin": 21, "imax": 91, "jmin": VISCOUS_WALL, "jmax": VISCOUS_WALL, "kmin": kface_bc, "kmax": kface_bc}))
    return _assemble(f"laminar_channel_{ni}x{nj}x{nk}", [(X, Y, Z)], [spec], [], laminar_params(mach, reyno))


def partitioned_laminar_channel(ni: int = 48, nj: int = 24, nk: int = 2, isplit=(20,), jsplit=(10,),
                                permute_last: bool = True, mach: float = 0.3, reyno: float = 500.0) -> Case:
    """laminar_channel split into blocks joined by cuts (the last block stored
    with permuted indices), z faces extrapolated."""
    return partitioned_channel(ni, nj, nk, isplit, jsplit, permute_last, mach, kface_bc=4, wall=VISCOUS_WALL,
                               params=laminar_params(mach, reyno))


# ---- turbulent channel: Wilcox k-omega on the bump channel with viscous walls ---------
def kom_params(mach: float = 0.3, reyno: float = 1.0e5, tu2: float = 1.0e-6, mutfar: float = 1.0,
               wall: str = "menter", roughk: float = 0.0) -> CosaParams:
    """laminar_params plus the Wilcox k-omega model (npde = 7): far-field
    k and omega from the turbulence intensity squared tu2 and the viscosity
    ratio mutfar (src/input.f90:2696-2720), omega wall value after Menter
    or Wilcox (rough wall, roughk)."""
    p = laminar_params(mach, reyno)
    p.npde = 7
    p.kom = 1
    p.mutfar = mutfar
    p.tkefar = tu2 * mach ** 2
    p.omefar = p.cmu * p.rhoinf * p.tkefar / mutfar * p.reyno / p.machfs
    p.wallwilc = 1 if wall == "wilcox" else 0
    p.roughk = roughk
    p.turcmp = 1.0
    p.lim_prodtke = 0
    p.lim_prodomega = 0
    p.prdlim = 20.0
    p.ifixq = 1
    p.cflt = p.cfl
    p.ratt = p.rat
    return p


def turbulent_channel(ni: int = 48, nj: int = 24, nk: int = 2, mach: float = 0.3, reyno: float = 1.0e5,
                      wall: str = "menter", kface_bc: int = 80) -> Case:
    """laminar_channel with the k-omega model (npde = 7)."""
    X, Y, Z = channel_nodes(ni, nj, nk)
    spec = BlockSpec(ni + 1, nj + 1, nk + 1, _face_bcs(ni + 1, nj + 1, nk + 1, {
        "imin": 21, "imax": 91, "jmin": VISCOUS_WALL, "jmax": VISCOUS_WALL, "kmin": kface_bc, "kmax": kface_bc}))
    return _assemble(f"turbulent_channel_{ni}x{nj}x{nk}", [(X, Y, Z)], [spec], [],
                     kom_params(mach, reyno, wall=wall))


def partitioned_turbulent_channel(ni: int = 48, nj: int = 24, nk: int = 2, isplit=(20,), jsplit=(10,),
                                  permute_last: bool = True, mach: float = 0.3, reyno: float = 1.0e5,
                                  wall: str = "menter") -> Case:
    return partitioned_channel(ni, nj, nk, isplit, jsplit, permute_last, mach, kface_bc=4, wall=VISCOUS_WALL,
                               params=kom_params(mach, reyno, wall=wall))


def wall_distance(case: Case) -> np.ndarray:
    """Wall distance of every cell (P1 array): the distance of each grid
    node to the nearest node of a viscous-wall (15xx) patch, averaged over
    the cell's eight nodes; halo cells repeat their neighbour.  Stands in for
    the solver's set-up routine dist2wall (outside the hot path) in the test
    cases."""
    t = case.tables
    gx, gy, gz = (p2_views(t, a) for a in (case.x, case.y, case.z))
    walls = []
    rows = t.bctopo
    ob = np.concatenate([[0], np.cumsum(t.nbcs)[:-1]])
    for b, (im, jm, km) in enumerate(t.dims):
        for r in rows[ob[b]:ob[b] + t.nbcs[b]]:
            if r[0] // 100 != 15:
                continue
            d, inrout = r[1], r[2]
            sl = [slice(r[3], r[4] + 2), slice(r[5], r[6] + 2), slice(r[7], r[8] + 2)]
            sl[d - 1] = slice(1, 2) if inrout == 1 else slice((im, jm, km)[d - 1], (im, jm, km)[d - 1] + 1)
            walls.append(np.stack([gx[b][tuple(sl)].ravel(), gy[b][tuple(sl)].ravel(), gz[b][tuple(sl)].ravel()], 1))
    W = np.concatenate(walls, 0) if walls else np.zeros((0, 3))
    _, tot = t.offsets()
    out = np.zeros(tot["p1"])
    for b, (v, X, Y, Z) in enumerate(zip(p1_views(t, out, 1), gx, gy, gz)):
        N = np.stack([X[1:-1, 1:-1, 1:-1].ravel(order="F"), Y[1:-1, 1:-1, 1:-1].ravel(order="F"),
                      Z[1:-1, 1:-1, 1:-1].ravel(order="F")], 1)
        if len(W):
            from scipy.spatial import cKDTree
            dn, _ = cKDTree(W).query(N, workers=-1)
        else:
            dn = np.full(len(N), 1e20)
        dn = np.asarray(dn).reshape(X[1:-1, 1:-1, 1:-1].shape, order="F")
        cell = (dn[:-1, :-1, :-1] + dn[1:, :-1, :-1] + dn[:-1, 1:, :-1] + dn[1:, 1:, :-1] +
                dn[:-1, :-1, 1:] + dn[1:, :-1, 1:] + dn[:-1, 1:, 1:] + dn[1:, 1:, 1:]) / 8
        V = v[..., 0]
        V[1:-1, 1:-1, 1:-1] = cell
        V[0, :, :] = V[1, :, :]; V[-1, :, :] = V[-2, :, :]
        V[:, 0, :] = V[:, 1, :]; V[:, -1, :] = V[:, -2, :]
        V[:, :, 0] = V[:, :, 1]; V[:, :, -1] = V[:, :, -2]
    return out


# ---- configuration 3: 3D bump duct --------------------------------------------------
def duct_segments(seed: int = 3, lo: int = 27_000_000, hi: int = 33_000_000, parts=(2, 3, 4),
                  choices=tuple(range(24, 161, 8)), max_draws: int = 100000):
    """Seeded draw of the tensor-partition segment lengths (cells) with
    lo <= N <= hi."""
    rng = np.random.default_rng(seed)
    for _ in range(max_draws):
        segs = [rng.choice(choices, size=n) for n in parts]
        n = int(np.prod([s.sum() for s in segs]))
        if lo <= n <= hi:
            return [list(map(int, s)) for s in segs]
    raise RuntimeError("no partition in the window")


def duct_params(mach: float = 0.6) -> CosaParams:
    return channel_params(mach)


def duct3d(segs=None, seed: int = 3, lo: int = 27_000_000, hi: int = 33_000_000,
           mach: float = 0.6, grid: bool = True, wall: int = 14, params: CosaParams = None) -> Case:
    if segs is None:
        segs = duct_segments(seed, lo, hi)
    si, sj, sk = segs
    NI, NJ, NK = sum(si), sum(sj), sum(sk)
    xs = -1.0 + 3.0 * np.arange(NI + 1) / NI
    eta = np.arange(NJ + 1) / NJ
    zs = -1.0 + 2.0 * np.arange(NK + 1) / NK
    ib = np.concatenate([[0], np.cumsum(si)]); jb = np.concatenate([[0], np.cumsum(sj)])
    kb = np.concatenate([[0], np.cumsum(sk)])
    nodes, specs, ids = [], [], {}
    for bk in range(len(sk)):
        for bj in range(len(sj)):
            for bi in range(len(si)):
                i0, i1, j0, j1, k0, k1 = ib[bi], ib[bi + 1], jb[bj], jb[bj + 1], kb[bk], kb[bk + 1]
                ids[(bi, bj, bk)] = len(specs) + 1
                types = {}
                if bi == 0: types["imin"] = 21
                if bi == len(si) - 1: types["imax"] = 91
                if bj == 0: types["jmin"] = wall
                if bj == len(sj) - 1: types["jmax"] = wall
                if bk == 0: types["kmin"] = wall
                if bk == len(sk) - 1: types["kmax"] = wall
                dims = (i1 - i0 + 1, j1 - j0 + 1, k1 - k0 + 1)
                specs.append(BlockSpec(*dims, _face_bcs(*dims, types)))
                if grid:
                    x = xs[i0:i1 + 1][:, None, None]
                    z = zs[k0:k1 + 1][None, None, :]
                    h = np.where((x >= 0) & (x <= 1), 0.1 * np.sin(np.pi * x) ** 2 * np.cos(np.pi * z / 2) ** 2, 0.0)
                    e = eta[j0:j1 + 1][None, :, None]
                    shp = (dims[0], dims[1], dims[2])
                    X = np.broadcast_to(x, shp).copy()
                    Y = np.broadcast_to(h + (1.0 - h) * e, shp).copy()
                    Z = np.broadcast_to(z, shp).copy()
                    nodes.append((X, Y, Z))
    cuts = []
    for (bi, bj, bk), b in ids.items():
        d = specs[b - 1]
        for axis, nb in ((0, (bi + 1, bj, bk)), (1, (bi, bj + 1, bk)), (2, (bi, bj, bk + 1))):
            if nb not in ids:
                continue
            o = ids[nb]
            od = specs[o - 1]
            if axis == 0:
                s1, e1 = (d.imax, 1, 1), (d.imax, d.jmax, d.kmax)
                s2, e2 = (1, 1, 1), (1, od.jmax, od.kmax)
            elif axis == 1:
                s1, e1 = (1, d.jmax, 1), (d.imax, d.jmax, d.kmax)
                s2, e2 = (1, 1, 1), (od.imax, 1, od.kmax)
            else:
                s1, e1 = (1, 1, d.kmax), (d.imax, d.jmax, d.kmax)
                s2, e2 = (1, 1, 1), (od.imax, od.jmax, 1)
            cuts.append((b, s1, e1, o, s2, e2, (1, 2, 3)))
    p = params if params is not None else duct_params(mach)
    if not grid:
        tables = build_tables(specs, cuts)
        return Case(f"duct3d_{NI}x{NJ}x{NK}", tables, p, None, None, None, None)
    return _assemble(f"duct3d_{NI}x{NJ}x{NK}", nodes, specs, cuts, p)



# ---- configuration 2/4: NACA 0012 O-grid --------------------------------------------
FAR_FIELD = 30


def naca0012_thickness(x: np.ndarray) -> np.ndarray:
    """Half thickness of the NACA 0012 from the 4-digit formula with the
    closed-trailing-edge last coefficient (-0.1036), chord 1."""
    x = np.clip(x, 0.0, 1.0)
    return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def _geometric_distances(n: int, h1: float, total: float) -> np.ndarray:
    """n+1 distances 0, h1, h1(1+r), ... ending at total (ratio r by bisection)."""
    lo, hi = 1.0 + 1e-12, 2.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if h1 * (r ** n - 1) / (r - 1) > total:
            hi = r
        else:
            lo = r
    r = 0.5 * (lo + hi)
    d = np.concatenate([[0.0], h1 * np.cumsum(r ** np.arange(n))])
    return d * (total / d[-1])


def naca0012_nodes(ni: int = 512, nj: int = 128, nk: int = 2, rfar: float = 50.0, h1: float = 4.5e-6,
                   span: float = 0.1, blend: float = 1.0):
    """Node coordinates (ni+1, nj+1, nk+1) of an O-grid around the NACA 0012.

    i runs clockwise from the trailing edge (i = 0 and i = ni coincide) over
    the lower surface, the leading edge (i = ni/2) and the upper surface,
    with cosine clustering at both edges; j runs from the wall to a circle of
    radius rfar about mid-chord with first spacing h1 (geometric); k spans
    z in [0, span].  Grid line i leaves the wall along the surface normal and
    bends over a length ~blend (chords) to the radial direction of its
    far-field point."""
    beta = 2 * np.pi * np.arange(ni + 1) / ni
    xs = 0.5 * (1 + np.cos(beta))
    ys = np.where(beta < np.pi, -1.0, 1.0) * naca0012_thickness(xs)
    ys[0] = ys[-1] = 0.0
    ys[ni // 2] = 0.0
    P = np.stack([xs, ys], 1)
    # outward normal of the clockwise contour: the tangent turned by +90 deg
    Pp = np.roll(P[:-1], -1, 0); Pm = np.roll(P[:-1], 1, 0)
    t = Pp - Pm
    t = np.concatenate([t, t[:1]], 0)
    Nrm = np.stack([-t[:, 1], t[:, 0]], 1)
    Nrm /= np.linalg.norm(Nrm, axis=1, keepdims=True)
    c = np.array([0.5, 0.0])
    R = P - c
    U0 = R / np.linalg.norm(R, axis=1, keepdims=True)
    Cfar = c + rfar * U0
    L = np.linalg.norm(Cfar - P, axis=1)
    U = (Cfar - P) / L[:, None]
    d = _geometric_distances(nj, h1, rfar)
    s = d / d[-1]
    w = 1.0 - np.exp(-d / blend)
    D = (1 - w)[None, :, None] * Nrm[:, None, :] + w[None, :, None] * U[:, None, :]
    D /= np.linalg.norm(D, axis=2, keepdims=True)
    XY = P[:, None, :] + (s[None, :, None] * L[:, None, None]) * D
    XY[:, -1, :] = Cfar
    zs = span * np.arange(nk + 1) / nk
    X = np.repeat(XY[:, :, 0:1], nk + 1, axis=2)
    Y = np.repeat(XY[:, :, 1:2], nk + 1, axis=2)
    Z = np.broadcast_to(zs[None, None, :], X.shape).copy()
    return X, Y, Z


def naca_params(model: str = "kom", mach: float = 0.3, alpha_deg: float = 4.0, reyno: float = 6.0e6,
                cfl: float = 3.0, eps_irs: float = 0.6, nlevel: int = 1) -> CosaParams:
    """Free stream at incidence alpha for the aerofoil cases: model "euler",
    "laminar" or "kom"; constant-coefficient IRS (irsop 1) with smoothing
    coefficient eps_irs (rat = sqrt(1 + 4 eps)) when eps_irs > 0."""
    if model == "kom":
        p = kom_params(mach, reyno)
    elif model == "laminar":
        p = laminar_params(mach, reyno)
    else:
        p = channel_params(mach)
    p.alpha = np.deg2rad(alpha_deg)
    p.beta = 0.0
    p.aircraft = 1
    p.cfl = cfl
    p.cflt = cfl
    p.nlevel = nlevel
    if nlevel > 1:
        # one pre-, post- and coarsest-level iteration, bilinear prolongation
        p.nstart = p.npre = p.npost = p.ncrs = 1
        p.bln_prol = 1
    if eps_irs > 0:
        p.irsop = 1
        p.rat = float(np.sqrt(1 + 4 * eps_irs))
        p.ratt = p.rat
    return p


def naca0012_ogrid(blocks=(96, 160, 160, 96), nj: int = 128, nk: int = 2, rfar: float = 50.0,
                   h1: float = 4.5e-6, span: float = 0.1, params: CosaParams = None,
                   wall: int = VISCOUS_WALL, kface_bc: int = 80, far: int = FAR_FIELD) -> Case:
    """NACA 0012 O-grid split along i into len(blocks) blocks of the given
    cell counts (default 96/160/160/96, 512 x nj x nk cells), 1-to-1 cuts
    between consecutive blocks and across the trailing-edge seam (last block
    imax to first block imin).  BCs: wall (default 1500, the force surface)
    on jmin, far field `far` (30, or 31 for bc_far1) on jmax, kface_bc on
    the k faces.  h1 = 4.5e-6
    chords is the first spacing of y+ ~ 1 at Re = 6e6 (flat-plate skin
    friction)."""
    ni = int(sum(blocks))
    X, Y, Z = naca0012_nodes(ni, nj, nk, rfar, h1, span)
    ib = np.concatenate([[0], np.cumsum(blocks)])
    nodes, specs = [], []
    for b in range(len(blocks)):
        i0, i1 = ib[b], ib[b + 1]
        nodes.append(tuple(A[i0:i1 + 1].copy() for A in (X, Y, Z)))
        dims = (i1 - i0 + 1, nj + 1, nk + 1)
        specs.append(BlockSpec(*dims, _face_bcs(*dims, {
            "jmin": wall, "jmax": far, "kmin": kface_bc, "kmax": kface_bc})))
    cuts = []
    nb = len(blocks)
    for b in range(nb):
        o = (b + 1) % nb
        d, od = specs[b], specs[o]
        cuts.append((b + 1, (d.imax, 1, 1), (d.imax, d.jmax, d.kmax), o + 1, (1, 1, 1), (1, od.jmax, od.kmax),
                     (1, 2, 3)))
    p = params if params is not None else naca_params()
    return _assemble(f"naca0012_{ni}x{nj}x{nk}", nodes, specs, cuts, p)

def naca_pitching(nharms: int = 1, blocks=(64, 64, 64, 64), nj: int = 64, nk: int = 2, mach: float = 0.5,
                  alpha_deg: float = 0.0, amp_deg: float = 2.5, kred: float = 0.08, xh: float = 0.25,
                  rfar: float = 30.0, h1: float = 2.0e-3, cfl: float = 1.0, model: str = "euler") -> Case:
    """Harmonic balance of a NACA 0012 pitching about the quarter chord:
    theta(t) = amp sin(omega t), omega = 2 kred M (chord 1, a_inf = 1), the
    O-grid of naca0012_ogrid (default 256 x 64 x 2 cells in 4 blocks), every
    snapshot on its own rotated grid.  The inviscid run keeps the 1500 wall
    (force surface 1): its halo holds the wall velocity, and the strong
    boundary face carries no mass flux.  Explicit 4-stage RK, no IRS, CFL 1
    (at CFL 2 the explicit time-spectral cycles of this grid lose
    positivity, in the oracle as on the device)."""
    from .params import set_pitching
    p = naca_params(model, mach=mach, alpha_deg=alpha_deg, reyno=1.0e6, cfl=cfl, eps_irs=0.0)
    set_pitching(p, nharms, amp_deg, kred, xh, 0.0)
    case = naca0012_ogrid(blocks=blocks, nj=nj, nk=nk, rfar=rfar, h1=h1, params=p)
    case.q0 = _freestream_state(case.tables, p)
    return case


def perturbed_state(case: Case, amp: float = 0.02, seed: int = 0) -> np.ndarray:
    """Free stream plus a smooth seeded perturbation of every conservative
    variable (keeps rho, p > 0); used to exercise limiters and all BC branches."""
    rng = np.random.default_rng(seed)
    q = case.q0.copy()
    p = case.params
    S = 2 * p.nharms + 1
    for v in p3_views(case.tables, q, p.npde, S):
        I, J, K = v.shape[:3]
        ii = np.arange(I)[:, None, None] / max(I - 1, 1)
        jj = np.arange(J)[None, :, None] / max(J - 1, 1)
        kk = np.arange(K)[None, None, :] / max(K - 1, 1)
        for var in range(p.npde):
            a = rng.uniform(0.5, 1.5, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            f = (np.sin(2 * np.pi * a[0] * ii + ph[0]) * np.cos(2 * np.pi * a[1] * jj + ph[1]) *
                 (1.0 + 0.5 * np.sin(2 * np.pi * a[2] * kk + ph[2])))
            noise = rng.standard_normal((I, J, K)) * 0.1
            scale = amp * (abs(v[..., var, 0]).mean() + 0.1)
            for n in range(S):
                v[..., var, n] = v[..., var, n] + scale * (f + noise)
    return q
