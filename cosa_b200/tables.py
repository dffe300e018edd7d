"""Block, boundary-condition and cut tables in COSA's own encoding.

input() turns each ``input.dat`` BC line ``istrt(1:3) iend(1:3) bctype``
(node indices) into a ``bcdata(10)`` record and each cut line pair into two
``cutdata(21)`` records (src/input.f90:3830-4000); setdim_bbc / setdimcut
(src/input.f90:5136-5200, 5285-5344) derive the coarse-level tables.  This
module reproduces that encoding so that the tables handed to the C-ABI are
exactly what the Fortran driver would pass.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Sequence, Tuple

import numpy as np


def _cyc(idir: int, m: int) -> int:
    # cyc = reshape((/1,2,3,2,3,1,3,1,2/),(/3,3/)) (src/input.f90:2409):
    # cyc(idir,1:3) is the cyclic order starting at idir
    return ((1, 2, 3), (2, 3, 1), (3, 1, 2))[idir - 1][m - 1]


def bc_record(istrt: Sequence[int], iend: Sequence[int], bctype: int) -> List[int]:
    """bcdata(1:10) of one BC line (src/input.f90:3846-3871)."""
    s = list(istrt)
    e = list(iend)
    idir = 0
    for i in range(3):
        if s[i] == e[i]:
            idir = i + 1
    if idir < 1:
        raise ValueError("error in reading bc data: no constant index")
    for i in range(3):
        if i + 1 != idir:
            e[i] -= 1
    return [bctype, idir, s[idir - 1], s[0], e[0], s[1], e[1], s[2], e[2], 0]


def _cut_face(istrt, iend):
    s = list(istrt)
    e = list(iend)
    idir = 0
    for l in range(3):
        if s[l] == e[l]:
            idir = l + 1
    if idir < 1:
        raise ValueError("error in reading cut data: no constant index")
    for l in range(3):
        if l + 1 != idir:
            if e[l] > s[l]:
                e[l] -= 1
            else:
                s[l] -= 1
    return idir, s, e


def cut_records(blk1: int, s1, e1, blk2: int, s2, e2, iord) -> Tuple[List[int], List[int]]:
    """The two cutdata(21) records of one input cut (src/input.f90:3903-4000).

    Blocks are 1-based as in input.dat.  Record 1 fills block 1's halo from
    block 2, record 2 the reverse.
    """
    c1 = [0] * 21
    c2 = [0] * 21
    idir, s, e = _cut_face(s1, e1)
    c1[0:9] = [blk1, idir, s[idir - 1], s[0], e[0], s[1], e[1], s[2], e[2]]
    c2[9:18] = [blk1, idir, s[idir - 1], s[0], e[0], s[1], e[1], s[2], e[2]]
    for l in iord:
        if l < 1 or l > 3:
            raise ValueError("error in reading cut data (iord)")
    idir, s, e = _cut_face(s2, e2)
    c1[9:18] = [blk2, idir, s[idir - 1], s[0], e[0], s[1], e[1], s[2], e[2]]
    c1[18:21] = list(iord)
    c2[0:9] = [blk2, idir, s[idir - 1], s[0], e[0], s[1], e[1], s[2], e[2]]
    if iord[0] == 2 and iord[1] == 3:
        m = 2
    elif iord[0] == 3 and iord[1] == 1:
        m = 3
    else:
        m = 1
    c2[18:21] = [_cyc(iord[0], m), _cyc(iord[1], m), _cyc(iord[2], m)]
    return c1, c2


@dataclass
class LevelTables:
    dims: np.ndarray            # (nblocks, 3) int32 node counts
    nbcs: np.ndarray            # (nblocks,) int32
    bctopo: np.ndarray          # (sum nbcs, 10) int32
    cutopo: np.ndarray          # (ncuts, 21) int32

    @property
    def nblocks(self) -> int:
        return int(self.dims.shape[0])

    @property
    def ncuts(self) -> int:
        return int(self.cutopo.shape[0])

    def offsets(self):
        """Per-block offsets (in cells) of the P3/P2/P1/F0/M1 arrays, as
        setoffs() computes them (src/input.f90:5502-5585), plus totals."""
        im, jm, km = self.dims[:, 0].astype(np.int64), self.dims[:, 1].astype(np.int64), self.dims[:, 2].astype(np.int64)
        sz = {
            "p3": (im + 3) * (jm + 3) * (km + 3),
            "p2": (im + 2) * (jm + 2) * (km + 2),
            "p1": (im + 1) * (jm + 1) * (km + 1),
            "f0": im * jm * km,
            "m1": (im - 1) * (jm - 1) * (km - 1),
        }
        off = {k: np.concatenate([[0], np.cumsum(v)[:-1]]) for k, v in sz.items()}
        tot = {k: int(v.sum()) for k, v in sz.items()}
        return off, tot

    def ncells(self) -> int:
        d = self.dims.astype(np.int64)
        return int(((d[:, 0] - 1) * (d[:, 1] - 1) * (d[:, 2] - 1)).sum())


def coarsen(fine: LevelTables, nl: int) -> LevelTables:
    """Level-nl tables from the fine ones (src/input.f90:4426-4432,
    5136-5200, 5285-5344)."""
    f = 2 ** (nl - 1)
    dims = (fine.dims - 1) // f + 1
    bct = fine.bctopo.copy()
    if nl > 1:
        bct[:, 2] = fine.bctopo[:, 2] // f + 1
        bct[:, 3:9] = (fine.bctopo[:, 3:9] - 1) // f + 1
    cut = fine.cutopo.copy()
    if nl > 1:
        cut[:, 2] = fine.cutopo[:, 2] // f + 1
        cut[:, 3:9] = (fine.cutopo[:, 3:9] - 1) // f + 1
        cut[:, 11] = fine.cutopo[:, 11] // f + 1
        cut[:, 12:18] = (fine.cutopo[:, 12:18] - 1) // f + 1
    return LevelTables(dims.astype(np.int32), fine.nbcs.copy(), bct.astype(np.int32), cut.astype(np.int32))


@dataclass
class BlockSpec:
    """input.dat-style description of one block: node counts and BC lines."""
    imax: int
    jmax: int
    kmax: int
    bcs: List[Tuple[Tuple[int, int, int], Tuple[int, int, int], int]] = field(default_factory=list)


def build_tables(blocks: List[BlockSpec], cuts) -> LevelTables:
    dims = np.array([[b.imax, b.jmax, b.kmax] for b in blocks], dtype=np.int32)
    nbcs = np.array([len(b.bcs) for b in blocks], dtype=np.int32)
    rows = [bc_record(s, e, t) for b in blocks for (s, e, t) in b.bcs]
    bct = np.array(rows, dtype=np.int32).reshape(-1, 10)
    crows = []
    for (b1, s1, e1, b2, s2, e2, iord) in cuts:
        c1, c2 = cut_records(b1, s1, e1, b2, s2, e2, iord)
        crows += [c1, c2]
    cut = np.array(crows, dtype=np.int32).reshape(-1, 21)
    return LevelTables(dims, nbcs, bct, cut)
