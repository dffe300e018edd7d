"""Single-level steady driver over the C-ABI: the part of COSA's main program
(src/cosa.f90:300-322 viscous set-up, 780-840 the iteration loop of a
one-level mg(), src/output.f90:4960-4990 the force output) that a solve of
one synthetic case needs.

    s = SteadySolver(case)            # geometry, metrics, viscous set-up, wall distance
    hist = s.run(2000, rms_every=100) # resrms rows of the printed iterations
    c = s.forces()                    # (S, 12) force/moment coefficients of surface 1

Every array lives on the device; the state is read back only by state()
and forces() (12 doubles per snapshot).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import cases, gpu
from .params import CosaParams


class SteadySolver:
    def __init__(self, case: "cases.Case", params: Optional[CosaParams] = None, device: int = 0,
                 q0: Optional[np.ndarray] = None):
        self.case = case
        self.p = params if params is not None else case.params
        p = self.p
        self.viscous = bool(p.viscous)
        self.kom = bool(p.kom)
        ctx = gpu.Context([case.tables], p, device=device)
        self.ctx = ctx
        self.X, self.Y, self.Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
        self.si, self.sj, self.sk = (ctx.alloc_p2() for _ in range(3))
        self.vol = ctx.alloc_p1()
        ctx.imetrix(1, self.X, self.Y, self.Z, self.si, self.sj, self.sk)
        ctx.vols(1, self.X, self.Y, self.Z, self.vol)
        self.vm = None
        if self.viscous:
            self.vm = ctx.alloc_vm()
            ctx.viscous_setup(1, self.X, self.Y, self.Z, self.vol, self.vm)
        self.q = ctx.alloc_p3().upload(case.q0 if q0 is None else q0)
        arrays = dict(q=self.q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=self.si, sj=self.sj, sk=self.sk,
                      vol=self.vol)
        if p.irsop > 0:
            arrays.update(betaxi=ctx.alloc_p1(), betaeta=ctx.alloc_p1(), betazeta=ctx.alloc_p1())
        self.mut = None
        if self.kom:
            self.mut = ctx.alloc_p3s()
            self.dist = ctx.alloc_p1().upload(cases.wall_distance(case))
            arrays.update(res=ctx.alloc_p3(), dtvolt=ctx.alloc_p1(), qp=ctx.alloc_p3(), qm=ctx.alloc_p3(),
                          dq=ctx.alloc_p3(), dqp=ctx.alloc_p3(), dqm=ctx.alloc_p3(), flux=ctx.alloc_f0(),
                          mut=self.mut, dist=self.dist)
            # the initial turbulent viscosity: tur_vis of the state after the
            # BCs (src/cosa.f90:560-600), halos of the cuts copied
            qq = ctx.alloc_p3()
            qq.upload(self.q.download())
            ctx.cons2prim(1, qq)
            ctx.bc_dist(1, qq, self.si, self.sj, self.sk, self.dist)
            ctx.cutman_q(1, qq)
            ctx.prim2cons(1, qq)
            ctx.tur_vis(1, qq, self.mut)
            ctx.cutman_mut(1, self.mut)
        ctx.bind_level(1, **arrays)
        self.arrays = arrays
        self.it = 0

    def run(self, niter: int, rms_every: int = 10, want_hist: bool = True):
        """niter iterations (one-level mg cycles); returns the resrms rows of
        the printed iterations (NaN rows elsewhere) and the status word."""
        hist, st = self.ctx.smooth(1, niter, self.it + 1, rms_every, want_hist=want_hist)
        self.it += niter
        return hist, st

    def forces(self, isurf: int = 1, xmom=(0.25, 0.0, 0.0), lngth=(1.0, None, 1.0)) -> np.ndarray:
        """(S, 12) coefficients of wall surface isurf; lngth[1] defaults to
        the z extent of the grid (per-span coefficients of a quasi-2D case)."""
        ln = list(lngth)
        if ln[1] is None:
            ln[1] = float(self.case.z.max() - self.case.z.min())
        return self.ctx.force(1, self.q, self.X, self.Y, self.Z, self.si, self.sj, self.sk, vm=self.vm,
                              isurf=isurf, xmom=xmom, lngth=tuple(ln))

    def state(self) -> np.ndarray:
        return self.q.download()

    def close(self):
        self.ctx.close()
