"""Serving sweep over the cosa_serve engine (continuous batching on one GPU).

A seeded Poisson stream of steady solves arrives; each request is the bump
channel at one of three in-plane scales with its own free-stream Mach
number (and the matching inlet total state), or a NACA 0012 O-grid at one of
three scales with its own Mach number and incidence, and is an Euler or a
k-omega RANS solve.  Requests are submitted when they arrive, admitted as
device memory allows, advanced together with whatever else is on the GPU,
and retired at convergence.  Reports throughput (solves per hour) and
p50/p99 latency (arrival to retirement).  The reference has no serving mode:
each of its runs is one solve; this is the batched counterpart of running
those one after another.

Steady single-grid Euler solves share the engine's merged level (one halo
and one stage launch per RK stage for all of them).  k-omega solves,
multigrid solves and harmonic-balance solves of a pitching aerofoil run in
the context lane (ContextLane): each is resident in its own context with
its own CUDA stream and advanced by a worker thread, so their launches
overlap on the device with one another and with the engine's; the library
call releases the interpreter lock.  The device budget is split between the engine's pools
and the lane.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
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


def kom_channel_request(scale: float, mach: float, arrival: float = 0.0, reyno: float = 1.0e5) -> Request:
    """k-omega (Wilcox, Menter wall omega) bump channel 128 x 64 x 2 cells
    scaled by `scale` in i and j, no-slip walls (1500) top and bottom, free
    stream and inlet total state at `mach`, Reynolds number reyno per unit
    length, CFL 1.5.  Short runs only: the uniform inflow meets the no-slip
    walls at the inlet corners, where k-omega production runs away (k
    reaches four times the free-stream kinetic energy near cycle 60, in the
    oracle as on the device; the production limiters only delay it), so
    poisson_requests draws its k-omega solves on the NACA grid."""
    ni, nj = max(8, int(round(128 * scale))), max(4, int(round(64 * scale)))
    case = cases.turbulent_channel(ni, nj, 2, mach=mach, reyno=reyno)
    case.params.cfl = case.params.cflt = 1.5
    return Request(scale, mach, arrival, case, case.params, 0.0, "channel_kom")


def kom_naca_request(scale: float, mach: float, alpha_deg: float, arrival: float = 0.0,
                     reyno: float = 1.0e6, model: str = "sst") -> Request:
    """k-omega NACA 0012 O-grid 256 x 64 x 2 cells in four blocks scaled by
    `scale` in i and j, no-slip wall (1500), far field (30) at 20 chords,
    first spacing 2e-4 chords at every scale (at 4e-4 on the 128 x 32 grid
    the trailing-edge cells' k runs away by cycle 300, in the oracle as on
    the device), free stream at `mach` and incidence `alpha_deg`, Reynolds
    number reyno, constant-coefficient IRS (0.6) at CFL 3.  model "sst"
    (Menter's SST, the default) or "wilcox": on the 512 x 128 grid at 5-7
    deg incidence and M 0.33-0.44 Wilcox's k and omega go non-finite after
    2400-3700 cycles (at CFL 3 and 2; the production limiters save one of
    two such requests), while SST runs them 20k cycles."""
    ni, nj = max(16, int(round(256 * scale)) // 16 * 16), max(8, int(round(64 * scale)))
    blocks = (3 * ni // 16, 5 * ni // 16, 5 * ni // 16, 3 * ni // 16)
    p = cases.naca_params("kom", mach=mach, alpha_deg=alpha_deg, reyno=reyno, cfl=3.0, eps_irs=0.6)
    if model == "sst":
        p.kom, p.kom_sst = 0, 1
    case = cases.naca0012_ogrid(blocks=blocks, nj=nj, nk=2, rfar=20.0, h1=2e-4, params=p)
    return Request(scale, mach, arrival, case, case.params, alpha_deg, "naca_kom")


def hb_request(scale: float, mach: float, alpha_deg: float, nharms: int = 1, arrival: float = 0.0,
               model: str = "euler") -> Request:
    """Harmonic balance of the NACA 0012 pitching 2.5 deg about the quarter
    chord at reduced frequency 0.08 (cases.naca_pitching) with nharms
    harmonics, mean incidence alpha_deg, on the 256 x 64 x 2 O-grid scaled by
    `scale` in i and j; Euler (slip wall) or k-omega (Re 1e6, first spacing
    2e-4 chords), CFL 1."""
    ni, nj = max(16, int(round(256 * scale)) // 16 * 16), max(8, int(round(64 * scale)))
    blocks = (ni // 4,) * 4
    kw = {"h1": 2e-4} if model == "kom" else {}
    case = cases.naca_pitching(nharms=nharms, blocks=blocks, nj=nj, mach=mach, alpha_deg=alpha_deg, rfar=20.0,
                               model=model, **kw)
    return Request(scale, mach, arrival, case, case.params, alpha_deg, "naca_hb" if model == "euler" else "naca_hb_kom")


def mg_request(scale: float, mach: float, arrival: float = 0.0, nlevel: int = 2) -> Request:
    """Euler bump channel (channel_request's grid, in-plane sizes rounded to
    multiples of 2^(nlevel-1)) solved with nlevel-level multigrid: one pre-,
    post- and coarsest-level iteration, bilinear prolongation, first order
    from level 2 on (the 2-cell-thick grid is one cell thick there)."""
    m = 2 ** (nlevel - 1)
    ni, nj = max(8 * m, int(round(128 * scale)) // m * m), max(4 * m, int(round(64 * scale)) // m * m)
    case = cases.bump_channel(ni, nj, 2, mach=mach)
    p = case.params
    p.nlevel = nlevel
    p.nstart = p.npre = p.npost = p.ncrs = 1
    p.bln_prol = 1
    p.nl_crs = 2
    return Request(scale, mach, arrival, case, p, 0.0, "channel_mg")


def is_kom(r: Request) -> bool:
    p = r.flow
    return bool(p.kom or p.kom_bsl or p.kom_sst)


def in_lane(r: Request) -> bool:
    """Solves the engine cannot merge: k-omega, harmonic balance and
    multigrid."""
    return is_kom(r) or r.flow.nharms > 0 or r.flow.nlevel > 1


def engine_scheme() -> CosaParams:
    """The engine's scheme: Roe + MUSCL (kappa 1/3, smooth limiter), 4-stage
    RK at CFL 2; flow conditions come with each request."""
    return cases.channel_params(0.5)


def poisson_requests(n: int, rate: float, seed: int, scales=(0.5, 1.0, 2.0), mach_range=(0.3, 0.7),
                     naca_fraction: float = 0.0, alpha_range=(-4.0, 8.0), kom_fraction: float = 0.0,
                     hb_fraction: float = 0.0, nharms_choices=(1, 2, 3)) -> List[Request]:
    """n arrivals at `rate` per second (seeded): with probability
    kom_fraction a k-omega RANS solve of the NACA 0012 (kom_naca_request),
    else an Euler solve of the bump channel or, with probability
    naca_fraction, of the NACA 0012; incidence drawn from alpha_range
    (degrees), scale and Mach number uniformly.  With probability
    hb_fraction (drawn only when it is > 0) the request is instead a pitching
    harmonic-balance solve (hb_request, Euler or k-omega as drawn) with
    nharms from nharms_choices."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t -= t[0]
    out = []
    for k in range(n):
        scale, mach = float(rng.choice(scales)), float(rng.uniform(*mach_range))
        naca = rng.uniform() < naca_fraction
        alpha = float(rng.uniform(*alpha_range))
        kom = rng.uniform() < kom_fraction
        if hb_fraction > 0 and rng.uniform() < hb_fraction:
            out.append(hb_request(scale, mach, alpha, int(rng.choice(nharms_choices)), float(t[k]),
                                  "kom" if kom else "euler"))
        elif kom:
            out.append(kom_naca_request(scale, mach, alpha, float(t[k])))
        elif naca:
            out.append(naca_request(scale, mach, alpha, float(t[k])))
        else:
            out.append(channel_request(scale, mach, float(t[k])))
    return out


def lane_solve_bytes(case: "cases.Case") -> int:
    """Device bytes of one solve in its own context, an upper estimate from
    the arrays its driver binds and the context's own work arrays, per P3
    cell and snapshot: k-omega 8 states, 7 face-flux planes (one of the
    caller, six of the fused stage), the IRS pivots (2 per variable) and
    about 30 scalar arrays (149 doubles), plus the face inverse metrics (27
    per face cell); Euler 4 states and 4 scalars (24 doubles); a pitching
    grid adds its per-snapshot metrics (12), nodes and node velocities (6)
    and face velocities (9); multigrid adds the residual and forcing states
    (10) and counts the coarser levels as half the finest (each level has at
    most a quarter of the cells of the one above it on these grids, halos
    included)."""
    p = case.params
    S = 2 * p.nharms + 1
    _, tot = case.tables.offsets()
    kom = bool(p.kom or p.kom_bsl or p.kom_sst)
    per, face = (8 * 7 + 7 * 7 + 2 * 7 + 30, 27) if kom else (4 * 5 + 4, 0)
    if p.moving:
        per += 12 + 6 + 9
    levels = 1.0
    if p.nlevel > 1:
        per += 10
        levels = 1.5
    return int(8 * S * levels * (per * tot["p3"] + face * tot["f0"]))


kom_solve_bytes = lane_solve_bytes


class ContextLane:
    """k-omega, multigrid and harmonic-balance solves next to the serving
    engine.  A
    submitted solve waits in a queue until its device bytes
    (lane_solve_bytes) fit the lane's budget and a worker is free; it then
    runs on a worker thread in its own context and stream (SteadySolver, or
    pitching.PitchingSolver on a pitching grid: metrics, viscous set-up,
    wall distance and the initial eddy viscosity on the device),
    check_every RK cycles per library call, with the same convergence rule as the engine: the total
    residual norm of its first cycle is the reference, the solve converges
    when the norm of a checked cycle falls below tol times it, stops at
    max_iter cycles and fails on a status bit or a non-finite norm.  A
    retired solve's context is closed at once, so its bytes go back to the
    lane.  result() gives the engine's fields."""

    def __init__(self, budget_bytes: float, device: int = 0, check_every: int = 10, precision: int = 0,
                 workers: int = 16):
        self.budget, self.used = float(budget_bytes), 0.0
        self.device, self.check_every, self.precision = device, check_every, precision
        self.solves: List[Dict] = []
        self.queue: deque = deque()
        self.lock = threading.Lock()
        self.running = 0
        self.workers = workers
        self.pool = ThreadPoolExecutor(max_workers=workers)
        self.t0 = time.perf_counter()

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, case: "cases.Case", flow: CosaParams, tol: float, max_iter: int) -> int:
        nbytes = lane_solve_bytes(case)
        if nbytes > self.budget:
            raise ValueError(f"a solve of {nbytes} bytes exceeds the lane's budget of {self.budget:.0f}")
        with self.lock:
            rid = len(self.solves)
            self.solves.append({"case": case, "flow": flow, "tol": tol, "max_iter": max_iter, "bytes": nbytes,
                                "state": "queued", "iters": 0, "drop": 0.0, "t_submit": self.now(),
                                "t_admit": 0.0, "t_done": 0.0, "status": 0, "result": None})
            self.queue.append(rid)
        self.admit()
        return rid

    def admit(self):
        """Start queued solves in arrival order while the head one fits."""
        with self.lock:
            while self.queue and self.running < self.workers:
                s = self.solves[self.queue[0]]
                if self.used + s["bytes"] > self.budget:
                    break
                rid = self.queue.popleft()
                self.used += s["bytes"]
                self.running += 1
                s["state"], s["t_admit"] = "active", self.now()
                self.pool.submit(self._run, rid)

    def _run(self, rid: int):
        from .solver import SteadySolver
        s = self.solves[rid]
        solver = None
        state = "failed"
        try:
            import torch
            torch.cuda.set_device(self.device)  # a new thread starts on device 0; the per-routine entries use the current one
            p = CosaParams.from_buffer_copy(s["flow"])
            p.precision = self.precision
            if p.moving:
                from .pitching import PitchingSolver
                solver = PitchingSolver(s["case"], params=p, device=self.device)
            else:
                solver = SteadySolver(s["case"], params=p, device=self.device)
            npde, rms0 = p.npde, None
            while True:
                n = min(self.check_every, s["max_iter"] - s["iters"])
                hist, st = solver.run(n, rms_every=n)
                s["iters"] += n
                if rms0 is None:
                    rms0 = float(hist[0, npde])
                rms = float(hist[n - 1, npde])
                s["drop"] = rms / rms0 if rms0 > 0 else 0.0
                if st or not np.isfinite(rms):
                    s["status"] = int(st)
                    break
                if rms0 > 0 and rms < s["tol"] * rms0:
                    state = "converged"
                    break
                if s["iters"] >= s["max_iter"]:
                    state = "stopped"
                    break
            if state != "failed":
                s["result"] = solver.state()
        except Exception as e:  # a set-up or library error retires the solve as failed
            s["error"] = repr(e)
        finally:
            if solver is not None:
                solver.close()
            with self.lock:
                s["state"], s["t_done"] = state, self.now()
                s["case"] = None
                self.used -= s["bytes"]
                self.running -= 1
        self.admit()

    def result(self, rid: int) -> Dict:
        s = self.solves[rid]
        out = {k: s[k] for k in ("state", "iters", "drop", "t_submit", "t_admit", "t_done", "status")}
        if "error" in s:
            out["error"] = s["error"]
        return out

    def counts(self):
        with self.lock:
            return self.running, len(self.queue)

    def close(self):
        self.pool.shutdown(wait=True)


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

    kinds: List[str] = field(default_factory=list)
    errors: List[str] = field(default_factory=list)

    def summary(self) -> Dict:
        out = {"requests": self.n, "wall_s": self.wall_s, "solves_per_hour": self.solves_per_hour,
               "p50_latency_s": self.p50_s, "p99_latency_s": self.p99_s,
               "converged": sum(s == "converged" for s in self.states),
               "stopped": sum(s == "stopped" for s in self.states),
               "failed": sum(s == "failed" for s in self.states),
               "mean_iters": float(np.mean(self.iters)) if self.iters else 0.0,
               "mcell_stages_per_s": self.cell_stages / self.wall_s / 1e6 if self.wall_s else 0.0}
        if self.errors:
            out["errors"] = sorted(set(self.errors))
        for kind in sorted(set(self.kinds)):
            sel = [i for i, k in enumerate(self.kinds) if k == kind]
            lat = [self.latencies[i] for i in sel]
            out[kind] = {"requests": len(sel), "converged": sum(self.states[i] == "converged" for i in sel),
                         "stopped": sum(self.states[i] == "stopped" for i in sel),
                         "failed": sum(self.states[i] == "failed" for i in sel),
                         "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99))}
        return out


def run_sweep(requests: List[Request], budget_bytes: float = 150e9, tol: float = 1e-8, max_iter: int = 200_000,
              check_every: int = 10, iters_per_step: int = 50, device: int = 0, precision: int = 0,
              kom_share: Optional[float] = None, kom_max_iter: Optional[int] = None) -> SweepResult:
    """Feed `requests` at their arrival times (seconds after the start) and
    run the engine and the context lane (precision 0: FP64, 1: mixed) until
    every one has retired.  kom_share is the lane's part of the device budget
    (default: the fraction of the requests the lane serves, 0 without any);
    kom_max_iter caps the lane solves' cycles (default max_iter)."""
    nkom = sum(in_lane(r) for r in requests)
    share = (nkom / max(len(requests), 1)) if kom_share is None else kom_share
    share = share if nkom else 0.0
    scheme = engine_scheme()
    scheme.precision = precision
    srv = Server(scheme, int(budget_bytes * (1.0 - share)), device=device, check_every=check_every) \
        if nkom < len(requests) else None
    lane = ContextLane(budget_bytes * share, device=device, check_every=check_every, precision=precision) \
        if nkom else None
    try:
        ids: List[tuple] = []  # ("engine" | "lane", id) in submission order
        pending = sorted(range(len(requests)), key=lambda k: requests[k].arrival)
        order: Dict[tuple, int] = {}
        t0 = time.perf_counter()
        done = 0
        nxt = 0

        def result(key):
            return srv.result(key[1]) if key[0] == "engine" else lane.result(key[1])

        while done < len(requests):
            now = time.perf_counter() - t0
            while nxt < len(pending) and requests[pending[nxt]].arrival <= now:
                r = requests[pending[nxt]]
                if in_lane(r):
                    key = ("lane", lane.submit(r.case, r.flow, tol, kom_max_iter or max_iter))
                else:
                    key = ("engine", srv.submit(r.case.tables, r.case.x, r.case.y, r.case.z, r.case.q0, r.flow, tol,
                                                max_iter))
                order[key] = pending[nxt]
                ids.append(key)
                nxt += 1
            na, nq = srv.step(iters_per_step) if srv is not None and any(k[0] == "engine" for k in ids) else (0, 0)
            done = sum(result(k)["state"] not in ("queued", "active") for k in ids)
            if na == 0 and nq == 0 and done < len(ids):
                time.sleep(0.005)  # only k-omega solves in flight: their worker threads drive the GPU
            elif na == 0 and nq == 0 and nxt < len(pending) and done == len(ids):
                wait = requests[pending[nxt]].arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
        wall = time.perf_counter() - t0
        res = [result(k) for k in ids]
        lat = [r["t_done"] - r["t_submit"] for r in res]
        cs = 0.0
        for key, r in zip(ids, res):
            rq = requests[order[key]]
            cs += rq.case.ncells * int(rq.flow.nstage) * r["iters"]
        out = SweepResult(len(ids), wall, len(ids) / wall * 3600.0, float(np.percentile(lat, 50)),
                          float(np.percentile(lat, 99)), [r["iters"] for r in res], [r["state"] for r in res], lat,
                          cs)
        out.kinds = [("hb_" if requests[order[k]].flow.nharms > 0 else "") +
                     ("kom" if is_kom(requests[order[k]]) else "euler") for k in ids]
        out.errors = [r["error"] for r in res if r.get("error")]
        return out
    finally:
        if srv is not None:
            srv.close()
        if lane is not None:
            lane.close()


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
    ap.add_argument("--kom-fraction", type=float, default=0.5)
    a = ap.parse_args()
    reqs = poisson_requests(a.requests, a.rate, a.seed, naca_fraction=a.naca_fraction, kom_fraction=a.kom_fraction)
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
