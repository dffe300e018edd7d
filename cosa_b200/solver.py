"""Steady driver over the C-ABI: the part of COSA's main program
(src/cosa.f90:300-322 viscous set-up, 780-930 the iteration loop of mg(),
src/output.f90:4960-4990 the force output) that a solve of one synthetic
case needs, on one level or on params.nlevel multigrid levels.

    s = SteadySolver(case)            # geometry, metrics, viscous set-up, wall distance
    hist = s.run(2000, rms_every=100) # resrms rows of the printed cycles
    c = s.forces()                    # (S, 12) force/moment coefficients of surface 1

With params.nlevel > 1 every level gets its own coarsened grid (every other
node), metrics, face inverse metrics and wall distance, its state starts at
the free stream like the fine one (init2fs on every level), and run() calls
cosa_gpu_mg.  Every array lives on the device; the state is read back only
by state() and forces() (12 doubles per snapshot).
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from . import cases, gpu
from .params import CosaParams


class SteadySolver:
    def __init__(self, case: "cases.Case", params: Optional[CosaParams] = None, device: int = 0,
                 q0: Optional[np.ndarray] = None, ncycle: Optional[int] = None, ramp: Optional[dict] = None):
        self.case = case
        self.p = params if params is not None else case.params
        p = self.p
        self.nlevel = max(1, int(p.nlevel))
        self.ncycle = ncycle
        # k-omega CFL ramp of bdeltat: dict(mode=1|2, ncycr=(n0..n3), vcfli=(3), vcflit=(3))
        self.ramp = ramp if (ramp and (p.kom or p.kom_bsl or p.kom_sst)) else None
        self._cfl = None
        self.viscous = bool(p.viscous)
        self.kom = bool(p.kom or p.kom_bsl or p.kom_sst)
        lv = cases.mg_levels(case, self.nlevel) if self.nlevel > 1 else [(case.tables, case.x, case.y, case.z)]
        ctx = gpu.Context([t for (t, _, _, _) in lv], p, device=device)
        self.ctx = ctx
        self.levels = []
        for nl, (t, x, y, z) in enumerate(lv, start=1):
            L = {}
            L["X"], L["Y"], L["Z"] = (ctx.alloc_p2(nl, ncomp=1).upload(a) for a in (x, y, z))
            si, sj, sk = (ctx.alloc_p2(nl) for _ in range(3))
            vol = ctx.alloc_p1(nl)
            ctx.imetrix(nl, L["X"], L["Y"], L["Z"], si, sj, sk)
            ctx.vols(nl, L["X"], L["Y"], L["Z"], vol)
            vm = None
            if self.viscous:
                vm = ctx.alloc_vm(nl)
                ctx.viscous_setup(nl, L["X"], L["Y"], L["Z"], vol, vm)
            if nl == 1:
                qinit = case.q0 if q0 is None else q0
            else:
                qinit = cases._freestream_state(t, p)
            q = ctx.alloc_p3(nl).upload(qinit)
            arrays = dict(q=q, qold=ctx.alloc_p3(nl), dtvol=ctx.alloc_p1(nl, ctx.S), si=si, sj=sj, sk=sk, vol=vol)
            if self.nlevel > 1:
                arrays.update(res=ctx.alloc_p3(nl), rhs=ctx.alloc_p3(nl))
            if p.irsop > 0:
                arrays.update(betaxi=ctx.alloc_p1(nl, ctx.S), betaeta=ctx.alloc_p1(nl, ctx.S),
                              betazeta=ctx.alloc_p1(nl, ctx.S))
            if self.kom:
                dist = cases.wall_distance(cases.Case("level", t, p, x, y, z, None))
                if "res" not in arrays:
                    arrays["res"] = ctx.alloc_p3(nl)
                arrays.update(dtvolt=ctx.alloc_p1(nl, ctx.S), qp=ctx.alloc_p3(nl), qm=ctx.alloc_p3(nl), dq=ctx.alloc_p3(nl), dqp=ctx.alloc_p3(nl),
                              dqm=ctx.alloc_p3(nl), flux=ctx.alloc_f0(nl), mut=ctx.alloc_p3s(nl),
                              dist=ctx.alloc_p1(nl).upload(dist))
            ctx.bind_level(nl, **arrays)
            L.update(arrays)
            L["vm"] = vm
            self.levels.append(L)
        fine = self.levels[0]
        self.q, self.X, self.Y, self.Z = fine["q"], fine["X"], fine["Y"], fine["Z"]
        self.si, self.sj, self.sk, self.vol, self.vm = fine["si"], fine["sj"], fine["sk"], fine["vol"], fine["vm"]
        self.mut = fine.get("mut")
        if self.kom:
            # the initial turbulent viscosity: tur_vis of the fine state after
            # the BCs (src/cosa.f90:560-600), halos of the cuts copied; the
            # coarse levels' mut is set by the first cycle's visit
            qq = ctx.alloc_p3()
            qq.upload(self.q.download())
            ctx.cons2prim(1, qq)
            ctx.bc_dist(1, qq, self.si, self.sj, self.sk, fine["dist"])
            ctx.cutman_q(1, qq)
            ctx.prim2cons(1, qq)
            ctx.tur_vis(1, qq, self.mut)
            ctx.cutman_mut(1, self.mut)
        self.it = 0

    def run(self, niter: int, rms_every: int = 10, want_hist: bool = True):
        """niter cycles of mg() (one-level: RK iterations); returns the resrms
        rows of the printed cycles (NaN rows elsewhere) and the status word.
        The solve's last cycle (ncycle, when given at construction) adds the
        fine-level post-smoothing of mg()."""
        if self.ramp:
            return self._run_ramped(niter, rms_every, want_hist)
        hist, st = self._cycles(niter, rms_every, want_hist)
        self.it += niter
        return hist, st

    def _cycles(self, niter, rms_every, want_hist):
        if self.nlevel == 1:
            return self.ctx.smooth(1, niter, self.it + 1, rms_every, want_hist=want_hist)
        ncycle = self.ncycle if self.ncycle is not None else 2 ** 30
        return self.ctx.mg(self.it + 1, niter, ncycle, rms_every, want_hist=want_hist)

    def _run_ramped(self, niter, rms_every, want_hist):
        """Cycles in runs of constant CFL: the parameters are uploaded where
        the ramp changes cfl/cflt (cycle 1 and every 100th for mode 1, every
        cycle of a ramp segment for mode 2)."""
        from .params import cfl_ramp
        r = self.ramp
        rows, st = [], 0
        end = self.it + niter
        while self.it < end:
            mgit = self.it + 1
            c = cfl_ramp(mgit, r["mode"], r["ncycr"], r["vcfli"], r["vcflit"], self._cfl)
            if c != self._cfl:
                self._cfl = c
                self.p.cfl, self.p.cflt = c
                self.ctx.set_params(self.p)
            # run until the next cycle where the ramp may change the CFL
            n = 1
            while self.it + n < end:
                nxt = cfl_ramp(self.it + n + 1, r["mode"], r["ncycr"], r["vcfli"], r["vcflit"], c)
                if nxt != c:
                    break
                n += 1
            h, s_ = self._cycles(n, rms_every, want_hist)
            st |= s_
            if h is not None:
                rows.append(h[:n])
            self.it += n
            if s_:
                break
        hist = np.concatenate(rows, axis=0) if rows else None
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
