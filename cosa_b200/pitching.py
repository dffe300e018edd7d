"""Harmonic balance of a pitching NACA 0012 (the benchmark's
harmonic-balance configuration, Euler or k-omega RANS): the O-grid of
naca0012_ogrid, 256 x 64 x 2 cells by default, pitching theta(t) = 2.5 deg
sin(omega t) about the quarter chord at reduced frequency 0.08 and M = 0.5,
with NH harmonics (S = 2 NH + 1 snapshots, each on its own rotated grid)
solved together in one set of stage launches.  Reports the device-timed
throughput in cell-snapshot-stages per second, the residual history, the
per-snapshot lift and moment coefficients and their harmonics (mathb's E,
src/input.f90:5240-5251), FP64 and mixed precision side by side.  The
k-omega case (Re 1e6, no-slip wall with first spacing 2e-4 chords) adds the
viscous set-up of every snapshot, the wall distance and the initial eddy
viscosity; its coefficients include the skin friction.

    python -m cosa_b200.pitching --nharms 1 2 3 --cycles 4000 [--model kom]

Needs a GPU.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases, gpu
from .params import PREC_MIXED, hb_harmonics

LNGTH = (1.0, 0.1, 1.0)  # chord, span (z extent of the 2-cell O-grid), moment arm reference


def _bind_kom(ctx, case, m, q):
    """The k-omega arrays of a pitching level: the face inverse metrics of
    every snapshot, the wall distance (rigid motion: that of the grid at
    rest), the work arrays, and the initial eddy viscosity from the state
    after the BCs (tur_vis, cut halos copied); returns vm."""
    vm = ctx.alloc_vm(1)
    ctx.viscous_setup(1, m["x"], m["y"], m["z"], m["vol"], vm)
    dist = ctx.alloc_p1().upload(cases.wall_distance(case))
    mut = ctx.alloc_p3s()
    ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), res=ctx.alloc_p3(), dtvol=ctx.alloc_p1(nsnap=ctx.S),
                   dtvolt=ctx.alloc_p1(nsnap=ctx.S), si=m["si"], sj=m["sj"], sk=m["sk"], vol=m["vol"],
                   qp=ctx.alloc_p3(), qm=ctx.alloc_p3(), dq=ctx.alloc_p3(), dqp=ctx.alloc_p3(), dqm=ctx.alloc_p3(),
                   flux=ctx.alloc_f0(), mut=mut, dist=dist, xdot=m["xdot"], ydot=m["ydot"], zdot=m["zdot"],
                   fvi=m["fvi"], fvj=m["fvj"], fvk=m["fvk"])
    qq = ctx.alloc_p3().upload(q.download())
    ctx.cons2prim(1, qq)
    ctx.bc_dist(1, qq, m["si"], m["sj"], m["sk"], dist)
    ctx.cutman_q(1, qq)
    ctx.prim2cons(1, qq)
    ctx.tur_vis(1, qq, mut)
    ctx.cutman_mut(1, mut)
    return vm


class PitchingSolver:
    """A pitching harmonic-balance solve resident on the device, with the
    interface of solver.SteadySolver (run, state, close): the moving-grid
    set-up of every snapshot (and, for k-omega, the viscous set-up, wall
    distance and initial eddy viscosity), then run() advances it niter
    explicit cycles through cosa_gpu_smooth."""

    def __init__(self, case: "cases.Case", params=None, device: int = 0):
        p = params if params is not None else case.params
        self.case, self.p = case, p
        self.kom = bool(p.kom or p.kom_bsl or p.kom_sst)
        self.ctx = gpu.Context([case.tables], p, device=device)
        self.m = self.ctx.pitching_setup(1, case)
        self.q = self.ctx.alloc_p3().upload(case.q0)
        self.vm = None
        m = self.m
        if self.kom:
            self.vm = _bind_kom(self.ctx, case, m, self.q)
        else:
            self.ctx.bind_level(1, q=self.q, qold=self.ctx.alloc_p3(), dtvol=self.ctx.alloc_p1(nsnap=self.ctx.S),
                                si=m["si"], sj=m["sj"], sk=m["sk"], vol=m["vol"], xdot=m["xdot"], ydot=m["ydot"],
                                zdot=m["zdot"], fvi=m["fvi"], fvj=m["fvj"], fvk=m["fvk"])
        self.it = 0

    def run(self, niter: int, rms_every: int = 10, want_hist: bool = True):
        h, st = self.ctx.smooth(1, niter, self.it + 1, rms_every, want_hist=want_hist)
        self.it += niter
        return h, st

    def forces(self):
        m = self.m
        return self.ctx.force(1, self.q, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], vm=self.vm, lngth=LNGTH)

    def state(self):
        return self.q.download()

    def close(self):
        self.ctx.close()


def run(nharms=1, precision=0, cycles=2000, chunk=500, blocks=(64, 64, 64, 64), nj=64, device=0, model="euler"):
    """One pitching solve on the device: returns a dict with the throughput
    (Mcell-snapshot-stage/s, CUDA events on the library's stream), the
    residual drop of rho, the per-snapshot CL and CM and their harmonics."""
    import torch
    kom = model == "kom"
    case = cases.naca_pitching(nharms=nharms, blocks=blocks, nj=nj, model=model, **({"h1": 2e-4} if kom else {}))
    p = case.params
    p.precision = precision
    ctx = gpu.Context([case.tables], p, device=device)
    m = ctx.pitching_setup(1, case)
    q = ctx.alloc_p3().upload(case.q0)
    vm = None
    if kom:
        vm = _bind_kom(ctx, case, m, q)
    else:
        ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(nsnap=ctx.S), si=m["si"], sj=m["sj"],
                       sk=m["sk"], vol=m["vol"], xdot=m["xdot"], ydot=m["ydot"], zdot=m["zdot"], fvi=m["fvi"],
                       fvj=m["fvj"], fvk=m["fvk"])
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    hist = []
    ms = 0.0
    done, st = 0, 0
    while done < cycles:
        n = min(chunk, cycles - done)
        ctx.sync()
        e0.record(stream)
        h, st = ctx.smooth(1, n, done + 1, n)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
        done += n
        hist.append(h[~np.isnan(h[:, 0])])
        if st:
            break
    hist = np.concatenate(hist, axis=0)
    coef = ctx.force(1, q, m["x"], m["y"], m["z"], m["si"], m["sj"], m["sk"], vm=vm, lngth=LNGTH)
    ctx.close()
    S = 2 * nharms + 1
    cl, cm = coef[:, 0] + coef[:, 6], coef[:, 5] + coef[:, 11]  # pressure + skin friction (0 for Euler)
    return {"nharms": nharms, "model": model, "snapshots": S, "precision": "mixed" if precision else "fp64",
            "cycles": done,
            "status": int(st), "cells": case.ncells,
            "mcell_snapshot_stage_s": case.ncells * S * p.nstage * done / (ms / 1e3) / 1e6,
            "ms_per_cycle": ms / max(done, 1),
            "drop_rho": float(hist[-1, 0] / hist[0, 0]) if len(hist) else None,
            "cl": cl.tolist(), "cm": cm.tolist(),
            "cl_harmonics": hb_harmonics(cl, nharms, p.omegas).tolist(),
            "cm_harmonics": hb_harmonics(cm, nharms, p.omegas).tolist()}


def compare(nharms=1, cycles=2000, **kw):
    """FP64 and mixed precision on the same case: both results and the
    largest differences of their CL and CM harmonics."""
    a = run(nharms, 0, cycles, **kw)
    b = run(nharms, PREC_MIXED, cycles, **kw)
    dcl = float(np.abs(np.array(a["cl_harmonics"]) - np.array(b["cl_harmonics"])).max())
    dcm = float(np.abs(np.array(a["cm_harmonics"]) - np.array(b["cm_harmonics"])).max())
    return {"fp64": a, "mixed": b, "max_dcl_harmonic": dcl, "max_dcm_harmonic": dcm,
            "mixed_speedup": b["mcell_snapshot_stage_s"] / a["mcell_snapshot_stage_s"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nharms", type=int, nargs="+", default=[1, 2, 3])
    ap.add_argument("--cycles", type=int, default=2000)
    ap.add_argument("--chunk", type=int, default=500)
    ap.add_argument("--model", choices=("euler", "kom"), default="euler")
    a = ap.parse_args()
    for nh in a.nharms:
        t = time.time()
        r = compare(nh, a.cycles, chunk=a.chunk, model=a.model)
        r["seconds"] = time.time() - t
        print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
