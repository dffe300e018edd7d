"""Serving sweep over the cosa_serve engine (continuous batching on one GPU).

A seeded Poisson stream of steady solves arrives; each request is the bump
channel at one of three in-plane scales with its own free-stream Mach
number (and the matching inlet total state), or an Euler NACA 0012 O-grid
at one of three scales with its own Mach number and incidence.  Requests are submitted when
they arrive, admitted by the engine as device memory allows, advanced
together with whatever else is on the GPU, and retired at convergence.
Reports throughput (solves per hour) and p50/p99 latency (arrival to
retirement).  The reference has no serving mode: each of its runs is one
solve; this is the batched counterpart of running those one after another.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import cases
from .gpu import Server
from .params import CosaParams, subsonic_inlet_total_state


@dataclass
class Request:
    scale: float
    mach: float
    arrival: float
    case: Optional[cases.Case] = None
    flow: Optional[CosaParams] = None
    alpha_deg: float = 0.0
    grid: str = "channel"


def channel_request(scale: float, mach: float, arrival: float = 0.0) -> Request:
    """Bump channel 128 x 64 x 2 cells scaled by `scale` in i and j, free
    stream and inlet total state at `mach`."""
    ni, nj = max(8, int(round(128 * scale))), max(4, int(round(64 * scale)))
    case = cases.bump_channel(ni, nj, 2, mach=mach)
    return Request(scale, mach, arrival, case, case.params)


def naca_request(scale: float, mach: float, alpha_deg: float, arrival: float = 0.0) -> Request:
    """Euler NACA 0012 O-grid of the harmonic-balance family, 256 x 64 x 2
    cells in four blocks (3/16, 5/16, 5/16, 3/16 of the contour) scaled by
    `scale` in i and j, slip wall (14), far field (30) at 20 chords, free
    stream at `mach` and incidence `alpha_deg`, CFL 1 (each solve's CFL
    number travels with its flow conditions)."""
    ni, nj = max(16, int(round(256 * scale)) // 16 * 16), max(8, int(round(64 * scale)))
    blocks = (3 * ni // 16, 5 * ni // 16, 5 * ni // 16, 3 * ni // 16)
    p = cases.channel_params(mach)
    p.alpha = float(np.deg2rad(alpha_deg))
    p.cfl = 1.0  # the O-grids' thin wall cells and closed trailing edge diverge at the channel's CFL 2
    case = cases.naca0012_ogrid(blocks=blocks, nj=nj, nk=2, rfar=20.0, h1=2e-3 / scale, params=p, wall=14)
    return Request(scale, mach, arrival, case, case.params, alpha_deg, "naca")


def engine_scheme() -> CosaParams:
    """The engine's scheme: Roe + MUSCL (kappa 1/3, smooth limiter), 4-stage
    RK at CFL 2; flow conditions come with each request."""
    return cases.channel_params(0.5)


def poisson_requests(n: int, rate: float, seed: int, scales=(0.5, 1.0, 2.0), mach_range=(0.3, 0.7),
                     naca_fraction: float = 0.0, alpha_range=(-4.0, 8.0)) -> List[Request]:
    """n arrivals at `rate` per second (seeded): the bump channel, or with
    probability naca_fraction the Euler NACA 0012 at an incidence drawn from
    alpha_range (degrees); scale and Mach number drawn uniformly."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    out = []
    for k in range(n):
        scale, mach = float(rng.choice(scales)), float(rng.uniform(*mach_range))
        if rng.uniform() < naca_fraction:
            out.append(naca_request(scale, mach, float(rng.uniform(*alpha_range)), float(t[k])))
        else:
            out.append(channel_request(scale, mach, float(t[k])))
    return out


@dataclass
class SweepResult:
    n: int
    wall_s: float
    solves_per_hour: float
    p50_s: float
    p99_s: float
    iters: List[int] = field(default_factory=list)
    states: List[str] = field(default_factory=list)
    latencies: List[float] = field(default_factory=list)
    cell_stages: float = 0.0

    def summary(self) -> Dict:
        return {"requests": self.n, "wall_s": self.wall_s, "solves_per_hour": self.solves_per_hour,
                "p50_latency_s": self.p50_s, "p99_latency_s": self.p99_s,
                "converged": sum(s == "converged" for s in self.states),
                "stopped": sum(s == "stopped" for s in self.states),
                "failed": sum(s == "failed" for s in self.states),
                "mean_iters": float(np.mean(self.iters)) if self.iters else 0.0,
                "mcell_stages_per_s": self.cell_stages / self.wall_s / 1e6 if self.wall_s else 0.0}


def run_sweep(requests: List[Request], budget_bytes: float = 150e9, tol: float = 1e-8, max_iter: int = 200_000,
              check_every: int = 10, iters_per_step: int = 50, device: int = 0, precision: int = 0) -> SweepResult:
    """Feed `requests` at their arrival times (seconds after the start) and
    run the engine (precision 0: FP64, 1: mixed) until every one has retired."""
    scheme = engine_scheme()
    scheme.precision = precision
    srv = Server(scheme, int(budget_bytes), device=device, check_every=check_every)
    try:
        ids: List[int] = []
        pending = sorted(range(len(requests)), key=lambda k: requests[k].arrival)
        order: Dict[int, int] = {}
        t0 = time.perf_counter()
        done = 0
        nxt = 0
        while done < len(requests):
            now = time.perf_counter() - t0
            while nxt < len(pending) and requests[pending[nxt]].arrival <= now:
                r = requests[pending[nxt]]
                rid = srv.submit(r.case.tables, r.case.x, r.case.y, r.case.z, r.case.q0, r.flow, tol, max_iter)
                order[rid] = pending[nxt]
                ids.append(rid)
                nxt += 1
            na, nq = srv.step(iters_per_step) if ids else (0, 0)
            done = sum(srv.result(rid)["state"] not in ("queued", "active") for rid in ids)
            if na == 0 and nq == 0 and nxt < len(pending) and done == len(ids):
                wait = requests[pending[nxt]].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
        wall = time.perf_counter() - t0
        res = [srv.result(rid) for rid in ids]
        lat = [r["t_done"] - r["t_submit"] for r in res]
        cs = 0.0
        for rid, r in zip(ids, res):
            cs += requests[order[rid]].case.ncells * 4 * r["iters"]
        return SweepResult(len(ids), wall, len(ids) / wall * 3600.0, float(np.percentile(lat, 50)),
                           float(np.percentile(lat, 99)), [r["iters"] for r in res], [r["state"] for r in res], lat,
                           cs)
    finally:
        srv.close()


def main():
    import argparse
    import json
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--requests", type=int, default=20)
    ap.add_argument("--rate", type=float, default=2.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--tol", type=float, default=0.1)
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--naca-fraction", type=float, default=0.5)
    a = ap.parse_args()
    reqs = poisson_requests(a.requests, a.rate, a.seed, naca_fraction=a.naca_fraction)
    print(json.dumps(run_sweep(reqs, a.budget_gb * 1e9, a.tol).summary()))


if __name__ == "__main__":
    main()


def batched_vs_plain(requests: List[Request], niter: int = 400, device: int = 0, precision: int = 1,
                     repeats: int = 3) -> Dict:
    """Throughput of the same solves two ways, `niter` RK cycles each:
    plain -- one after another through the single-solve FP64 path
    (cosa_gpu_smooth, one context per request);
    batched -- all resident in the serving engine at once in the given
    precision (1 = mixed), advanced by shared stage launches.
    Both arms are timed the same way: host wall clock around one
    synchronous library call per solve (plain) or per engine step of niter
    cycles (batched), after a warm-up that captures the graphs; the work is
    counted from the cycles each solve actually completed.  The median over
    `repeats` measurements of each arm, Mcell-stage/s of both and their
    ratio."""
    import torch
    from . import gpu as _gpu
    cells = [r.case.ncells for r in requests]

    def plain_once():
        secs, work = 0.0, 0
        for r, nc in zip(requests, cells):
            p = engine_scheme()
            for k in ("machfs", "alpha", "beta", "rhoinf", "pinf", "ainf", "tinf", "inlet_t0", "inlet_p0", "cfl"):
                setattr(p, k, getattr(r.flow, k))
            for i in range(3):
                p.inlet_dir[i] = r.flow.inlet_dir[i]
                p.outlet_p[i] = r.flow.outlet_p[i]
            ctx = _gpu.Context([r.case.tables], p, device=device)
            x, y, z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (r.case.x, r.case.y, r.case.z))
            si, sj, sk, vol = ctx.alloc_p2(), ctx.alloc_p2(), ctx.alloc_p2(), ctx.alloc_p1()
            ctx.imetrix(1, x, y, z, si, sj, sk)
            ctx.vols(1, x, y, z, vol)
            q = ctx.alloc_p3().upload(r.case.q0)
            ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=si, sj=sj, sk=sk, vol=vol)
            ctx.smooth(1, 5, 1, 10 ** 6, want_hist=False)  # warm-up and graph capture
            ctx.sync()
            t0 = time.perf_counter()
            _, st = ctx.smooth(1, niter, 6, 10 ** 6, want_hist=False)
            ctx.sync()
            secs += time.perf_counter() - t0
            work += nc * 4 * niter
            ctx.close()
        return work / secs / 1e6

    def batched_once():
        scheme = engine_scheme()
        scheme.precision = precision
        srv = Server(scheme, int(40e9), device=device, check_every=10 ** 6)
        try:
            ids = [srv.submit(r.case.tables, r.case.x, r.case.y, r.case.z, r.case.q0, r.flow, 0.0, niter + 10)
                   for r in requests]
            srv.step(5)  # admission, table build and graph capture
            before = [srv.result(i)["iters"] for i in ids]
            torch.cuda.synchronize(device)
            t0 = time.perf_counter()
            srv.step(niter)
            torch.cuda.synchronize(device)
            secs = time.perf_counter() - t0
            after = [srv.result(i)["iters"] for i in ids]
        finally:
            srv.close()
        work = sum(nc * 4 * (b - a) for nc, a, b in zip(cells, before, after))
        return work / secs / 1e6

    plains = sorted(plain_once() for _ in range(repeats))
    batches = sorted(batched_once() for _ in range(repeats))
    plain, batched = plains[len(plains) // 2], batches[len(batches) // 2]
    return {"requests": len(requests), "cells": int(sum(cells)), "cycles_each": niter, "repeats": repeats,
            "timing": "host wall clock around synchronous library calls, both arms; median of repeats",
            "plain_fp64_mcell_stage_s": plain, "batched_mcell_stage_s": batched,
            "batched_precision": "mixed" if precision == 1 else "fp64", "speedup": batched / plain}
