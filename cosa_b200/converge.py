"""FP64 against mixed precision to convergence: the same case solved twice
(FP64, then FP32 slopes and Roe dissipation on FP64 differences) until the
stage-1 residual norm of rho has dropped by `drop` (or max_cycles), then
the cycles and seconds each took and the L2 difference of the two
converged fields, relative to the L2 norm of the FP64 field, per variable.

    python -m cosa_b200.converge --case duct --cells 4e6 --nlevel 3 --drop 1e-8

Needs a GPU.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from .params import PREC_MIXED
from .solver import SteadySolver


def _case(kind: str, cells: float, seed: int):
    if kind == "duct":
        lo, hi = int(0.85 * cells), int(1.15 * cells)
        segs = cases.duct_segments(seed=seed, lo=lo, hi=hi, choices=tuple(range(24, 97, 8)))
        return cases.duct3d(segs=segs), f"bump duct {segs}"
    if kind == "channel":
        return cases.bump_channel(), "bump channel 128x64x2"
    raise ValueError(kind)


def run(kind="duct", cells=4e6, seed=3, nlevel=3, drop=1e-8, max_cycles=20000, chunk=100, verbose=True):
    out = {}
    fields = {}
    for prec in ("fp64", "mixed"):
        case, desc = _case(kind, cells, seed)
        p = case.params
        p.nlevel = nlevel
        if nlevel > 1:
            p.nstart = p.npre = p.npost = p.ncrs = 1
            p.bln_prol = 1
            p.nl_crs = 2  # first order on the coarse levels
        if prec == "mixed":
            p.precision = PREC_MIXED
        s = SteadySolver(case, ncycle=10 ** 9)
        r0, t0, last, st = None, time.time(), None, 0
        while s.it < max_cycles:
            h, st = s.run(chunk, rms_every=chunk)
            if r0 is None:
                r0 = h[0, 0]
            last = h[chunk - 1, 0] / r0  # the row of the chunk's last cycle
            if verbose:
                print(json.dumps({"prec": prec, "cycles": s.it, "drop": last, "status": st}), flush=True)
            if st or not np.isfinite(last) or last <= drop:
                break
        s.ctx.sync()
        fields[prec] = cases_interior(case, s.state())
        out[prec] = {"cycles": s.it, "drop": float(last), "seconds": time.time() - t0, "status": int(st),
                     "cells": case.ncells, "workload": desc, "nlevel": nlevel}
        s.close()
    a, b = fields["fp64"], fields["mixed"]
    # density, momentum (the vector: a component that is zero in a
    # quasi-2D flow is measured against the momentum norm) and energy
    groups = {"rho": [0], "momentum": [1, 2, 3], "rhoE": [4]}
    out["l2_rel_diff"] = {k: float(np.linalg.norm(b[:, g] - a[:, g]) / np.linalg.norm(a[:, g]))
                          for k, g in groups.items()}
    out["max_rel_diff"] = {k: float(np.abs(b[:, g] - a[:, g]).max() / np.abs(a[:, g]).max())
                           for k, g in groups.items()}
    return out


def cases_interior(case, q):
    vs = [cases.interior(v)[..., 0].reshape(-1, 5) for v in cases.p3_views(case.tables, q, 5, 1)]
    return np.concatenate(vs, axis=0)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="duct", choices=["duct", "channel"])
    ap.add_argument("--cells", type=float, default=4e6)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--nlevel", type=int, default=3)
    ap.add_argument("--drop", type=float, default=1e-8)
    ap.add_argument("--max-cycles", type=int, default=20000)
    ap.add_argument("--chunk", type=int, default=100)
    a = ap.parse_args()
    res = run(a.case, a.cells, a.seed, a.nlevel, a.drop, a.max_cycles, a.chunk)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
