"""FP64 against mixed precision on the NACA 0012 O-grid: the same number of
single-grid iterations from the free stream in each precision, force
coefficients of the 1500 wall every `chunk` iterations, and the final
differences |dCL|, |dCD|, |dCM|.

    python -m cosa_b200.naca_compare --model kom --niter 20000 --mach 0.3 \\
        --alpha 4 --reyno 6e6 --cfl 3 --out naca_kom.json

One JSON line per chunk and a final summary line on stdout; --out keeps the
histories.  Needs a GPU.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from .params import PREC_MIXED
from .solver import SteadySolver


def run(model="kom", niter=20000, chunk=2000, cfl=3.0, eps=0.6, reyno=6.0e6, mach=0.3, alpha=4.0, nj=128,
        h1=4.5e-6, nlevel=1, nk=2, ramp=None, verbose=True):
    res = {}
    for prec in ("fp64", "mixed"):
        p = cases.naca_params(model, mach=mach, alpha_deg=alpha, reyno=reyno, cfl=cfl, eps_irs=eps, nlevel=nlevel)
        if prec == "mixed":
            p.precision = PREC_MIXED
        case = cases.naca0012_ogrid(nj=nj, nk=nk, h1=h1, params=p)
        s = SteadySolver(case, ncycle=niter, ramp=ramp)
        hist, r0, t0 = [], None, time.time()
        for _ in range(0, niter, chunk):
            h, st = s.run(chunk, rms_every=chunk)
            rows = h[~np.isnan(h[:, 0])]
            if r0 is None and len(rows):
                r0 = rows[0, 0]
            c = s.forces()[0]
            line = dict(prec=prec, it=s.it, st=int(st), r1=float(rows[-1, 0]) if len(rows) else None,
                        drop=float(rows[-1, 0] / r0) if len(rows) else None, cl=float(c[0] + c[6]),
                        cd=float(c[1] + c[7]), cm=float(c[5] + c[11]))
            if verbose:
                print(json.dumps(line), flush=True)
            hist.append(line)
            if st != 0 or not len(rows):
                break
        s.ctx.sync()
        res[prec] = dict(hist=hist, sec=time.time() - t0)
        s.close()
    f, m = res["fp64"]["hist"][-1], res["mixed"]["hist"][-1]
    res["final"] = {k: abs(f[k] - m[k]) for k in ("cl", "cd", "cm")}
    return res


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--model", default="kom", choices=["kom", "laminar"])
    ap.add_argument("--niter", type=int, default=20000)
    ap.add_argument("--chunk", type=int, default=2000)
    ap.add_argument("--cfl", type=float, default=3.0)
    ap.add_argument("--eps", type=float, default=0.6, help="IRS smoothing coefficient (irsop 1)")
    ap.add_argument("--reyno", type=float, default=6.0e6)
    ap.add_argument("--mach", type=float, default=0.3)
    ap.add_argument("--alpha", type=float, default=4.0)
    ap.add_argument("--nj", type=int, default=128)
    ap.add_argument("--h1", type=float, default=4.5e-6, help="first wall spacing (chords)")
    ap.add_argument("--nlevel", type=int, default=1, help="multigrid levels (3 needs --nk 8)")
    ap.add_argument("--nk", type=int, default=2, help="cells in k (span 0.1)")
    ap.add_argument("--ramp", default=None,
                    help="k-omega CFL ramp 'mode:n0,n1,n2,n3:c1,c2' from c1 over c2 to --cfl (bdeltat ramping1/2)")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    ramp = None
    if a.ramp:
        mode, ns, cs = a.ramp.split(":")
        c1, c2 = (float(v) for v in cs.split(","))
        ramp = dict(mode=int(mode), ncycr=tuple(int(v) for v in ns.split(",")), vcfli=(c1, c2, a.cfl),
                    vcflit=(c1, c2, a.cfl))
    res = run(a.model, a.niter, a.chunk, a.cfl, a.eps, a.reyno, a.mach, a.alpha, a.nj, a.h1, a.nlevel, a.nk, ramp)
    print(json.dumps(dict(final=res["final"], fp64=res["fp64"]["hist"][-1], mixed=res["mixed"]["hist"][-1],
                          sec_fp64=res["fp64"]["sec"], sec_mixed=res["mixed"]["sec"])))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
