"""Benchmark of the B200 explicit residual-and-update path (one JSON line).

Workload (default): the batched multiblock 3D Euler bump duct -- about 30 M
cells in 24 blocks of uneven sizes (seeded 2x3x4 tensor partition with
segment lengths from {24, ..., 160}), M = 0.6, 4-stage RK, CFL 2, Roe + MUSCL
(kappa = 1/3, smooth limiter), FP64 state.  A step is one RK cycle (4 stages)
over all cells; the metric is Mcell-stage/s = cells * 4 * steps / time.

Our arm times cosa_gpu_smooth (halo fill, line-marching face kernels and the
cell pass of the face-split schedule, or the fused tile kernel, whichever the
autotuner picks, replayed from a CUDA graph with the state resident in HBM)
with CUDA events on the library's stream; the state (1.4 GB) is larger than
the 126 MB L2, so no flush is needed between steps.  It also reports the
mixed-precision path, the roofline of the dominant kernel and of the whole
stage against the algorithmic bytes of the ideally fused stage, an
end-to-end number through cosa_gpu_smooth_host (state copied from pinned
host memory and back every step), the laminar and k-omega legs, the
harmonic-balance pitching aerofoil (NH = 1..3, FP64 and mixed), the serving
sweep and the CPU oracle's throughput on 2 cycles of the same workload.

--impl reference times the CPU restatement of the reference (oracle/; COSA
itself is Fortran and cannot be built here) on the host cores, 2 RK cycles of
the same 30.7 M-cell duct.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic bytes per cell-stage of the ideally fused Euler stage (FP64):
# read q 40 + read q^n 40 + write q 40 + face metrics of the 3 owned faces 96
# + vol 8 + dt/V 8 + dt/V write amortised 2.  The roofline fractions below
# charge every kernel with these bytes, whatever it moves itself.
B_ALG_STAGE = 234
# harmonic balance of a pitching body, per cell-snapshot-stage: state 120 +
# metrics 3 x 7 x 8 = 168 + cell grid velocity 24 + vol 8 + dt/V 8 + 2
B_ALG_HB_MOVING = 330
# k-omega on the pitching grid: the k-omega stage's 960 B per cell-stage
# (7 variables, the face inverse metrics, mut and the k-omega work arrays)
# per snapshot
B_ALG_KOM_HB_MOVING = 960
# bytes the face-split schedule's face kernels (k_faces_line, i-face and
# marching launches) move per cell: state reads 3 x 40 (once per family) +
# face metrics 96 + face fluxes written 120
B_FACES_OWN = 336
# DRAM bytes (read + write) per cell of one stage's two k_faces_line
# launches in an ncu capture of the 4.2 M-cell duct (k_faces_line<fp64>,
# scaled by the cells of the launch)
FACES_TRAFFIC_B_PER_CELL = 311.7


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms in the background."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return out
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            os.unlink(self.path)
        except Exception:
            return out
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1])); mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                pass
        if sm:
            out = {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                   "samples": len(sm)}
        return out


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def build_case(args):
    from cosa_b200 import cases
    if args.workload == "duct30m":
        segs = cases.duct_segments(seed=args.seed)
        return cases.duct3d(segs=segs), f"config3 bump duct, 24 blocks, segments {segs}"
    if args.workload == "duct4m":
        segs = cases.duct_segments(seed=args.seed, lo=3_500_000, hi=4_500_000, choices=tuple(range(24, 97, 8)))
        return cases.duct3d(segs=segs), f"config3 generator, 4M-cell window (profiling size), segments {segs}"
    if args.workload == "channel":
        return cases.bump_channel(), "config1 bump channel 128x64x2 (1 block)"
    raise SystemExit(f"unknown workload {args.workload}")


def run_cpu_oracle(case, desc, steps: int, warmup: int):
    """The oracle (C++ restatement of the reference, OpenMP over blocks and
    k-planes) on the benchmark's own workload: `steps` RK cycles after
    `warmup`, wall-timed around the cycles only (set-up and metrics
    excluded).  Returns the cpu_baseline record and the seconds."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    O = oracle.OracleLevel(case.tables, case.params)
    si, sj, sk, vol = O.metrics(case.x, case.y, case.z)
    q = case.q0.copy()
    if warmup:
        O.smooth(q, si, sj, sk, warmup, rms_every=10 ** 6)
    t = time.perf_counter()
    O.smooth(q, si, sj, sk, steps, rms_every=10 ** 6, mgit0=warmup + 1)
    dt = time.perf_counter() - t
    val = case.ncells * case.params.nstage * steps / dt / 1e6
    return {"value": val, "unit": "Mcell-stage/s", "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{desc}: {steps} RK cycles of the full workload after {warmup} warm-up, {dt:.2f} s"}, dt


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    # a bounded sample of the same workload: 2 cycles of the full grid
    steps, warmup = max(1, min(args.steps, 2)), min(args.warmup, 1)
    case, desc = build_case(args)
    cb, dt = run_cpu_oracle(case, desc, steps, warmup)
    line = {"impl": "reference", "metric": "Mcell-stage/s", "value": cb["value"], "unit": "Mcell-stage/s",
            "n_gpus": ws, "steps": steps, "warmup": warmup, "ms_per_step": dt / steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": desc, "cells": case.ncells, "blocks": case.tables.nblocks,
                                            "stages_per_step": case.params.nstage},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Mcell-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def max_over_ranks(ms: float, dist, torch, device: str) -> float:
    """The slowest rank's device time: every rank takes part in the same
    all-reduce (MAX) in the same order."""
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world_size: int, cell_stages_per_rank: float, ms_max: float) -> float:
    """Whole-job Mcell-stage/s of `world_size` replicas that each did
    cell_stages_per_rank in at most ms_max milliseconds (weak scaling)."""
    return world_size * cell_stages_per_rank / (ms_max / 1e3) / 1e6


def time_smooth(ctx, steps: int, torch):
    """Device time of `steps` fused cycles with CUDA events on the library's stream."""
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.sync()
    e0.record(stream)
    hist, st = ctx.smooth(1, steps, 10 ** 6, 10 ** 6, want_hist=False)
    e1.record(stream)
    e1.synchronize()
    if st:
        raise RuntimeError(f"cosa_gpu_smooth status 0x{st:x}")
    return e0.elapsed_time(e1)


def viscous_leg(kind: str, steps: int, warmup: int, dev: int, torch, precision: str = "fp64"):
    """FP64 (or mixed) throughput of the laminar path (fused stage + viscous
    face kernels) on the duct generator with no-slip walls, or of the Wilcox
    k-omega path (routine by routine, IRS) on the NACA 0012 O-grid of the
    RANS configuration: Mcell-stage/s, device-timed like the main leg."""
    from cosa_b200 import cases, gpu
    from cosa_b200.params import PREC_MIXED
    if kind == "kom":
        from cosa_b200.solver import SteadySolver
        p = cases.naca_params("kom", mach=0.3, alpha_deg=4.0, reyno=6.0e6, cfl=3.0, eps_irs=0.6)
        if precision == "mixed":
            p.precision = PREC_MIXED
        case = cases.naca0012_ogrid(params=p)
        s = SteadySolver(case, device=dev)
        ctx = s.ctx
        workload = ("NACA 0012 O-grid 512x128x2 (blocks 96/160/160/96), Wilcox k-omega, M=0.3, alpha=4, Re=6e6, "
                    "CFL 3, IRS eps 0.6, single grid, " + precision.upper())
    else:
        segs = cases.duct_segments(seed=3, lo=3_500_000, hi=4_500_000, choices=tuple(range(24, 97, 8)))
        p = cases.laminar_params(0.6, 1.0e4)
        if precision == "mixed":
            p.precision = PREC_MIXED
        case = cases.duct3d(segs=segs, wall=cases.VISCOUS_WALL, params=p)
        ctx = gpu.Context([case.tables], p, device=dev)
        X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
        si, sj, sk = (ctx.alloc_p2() for _ in range(3))
        vol = ctx.alloc_p1()
        ctx.imetrix(1, X, Y, Z, si, sj, sk)
        ctx.vols(1, X, Y, Z, vol)
        vm = ctx.alloc_vm()
        ctx.viscous_setup(1, X, Y, Z, vol, vm)
        q = ctx.alloc_p3().upload(case.q0)
        ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=si, sj=sj, sk=sk, vol=vol)
        workload = f"bump duct, segments {segs}, no-slip walls (1500), laminar Re=1e4, M=0.6, " + precision.upper()
    ctx.smooth(1, warmup, 1, 10 ** 6, want_hist=False)
    ctx.launch_count(reset=True)
    ms = time_smooth(ctx, steps, torch)
    launches = ctx.launch_count(reset=True)
    ctx.close()
    return {"value": case.ncells * p.nstage * steps / (ms / 1e3) / 1e6, "unit": "Mcell-stage/s",
            "ms_per_step": ms / steps, "cells": case.ncells, "steps": steps, "gpu_launches": launches,
            "workload": workload}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="duct30m", choices=["duct30m", "duct4m", "channel"])
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the mixed, e2e and CPU legs (profiling runs)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sweep")
    ap.add_argument("--no-viscous", action="store_true", help="skip the laminar and k-omega legs")
    ap.add_argument("--no-hb", action="store_true", help="skip the pitching harmonic-balance leg")
    ap.add_argument("--hb-cycles", type=int, default=400, help="RK cycles of each harmonic-balance run")
    ap.add_argument("--schedule", type=int, default=0, choices=[0, 1, 2],
                    help="0: autotune the stage schedule, 1: fused tile kernel, 2: face-split")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of the main timed leg (profiling runs; the default line reports both)")
    ap.add_argument("--leg", default="all", choices=["all", "laminar", "kom"],
                    help="laminar / kom: time only that viscous leg and print its line (profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.leg != "all":
        import torch
        torch.cuda.set_device(0)
        r = viscous_leg(args.leg, args.steps, args.warmup, 0, torch, args.precision)
        print(json.dumps({"metric": "Mcell-stage/s", "leg": args.leg, "precision": args.precision, **r}), flush=True)
        return

    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    ws, rank, local = _dist()
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)

    from cosa_b200 import gpu
    from cosa_b200.params import PREC_MIXED

    case, desc = build_case(args)
    p = case.params
    if args.precision == "mixed":
        p.precision = PREC_MIXED
    ncells = case.ncells
    ctx = gpu.Context([case.tables], p, device=dev)
    X, Y, Z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (case.x, case.y, case.z))
    si, sj, sk = (ctx.alloc_p2() for _ in range(3))
    vol = ctx.alloc_p1()
    ctx.imetrix(1, X, Y, Z, si, sj, sk)
    ctx.vols(1, X, Y, Z, vol)
    q = ctx.alloc_p3().upload(case.q0)
    qold = ctx.alloc_p3()
    dtvol = ctx.alloc_p1()
    ctx.bind_level(1, q=q, qold=qold, dtvol=dtvol, si=si, sj=sj, sk=sk, vol=vol)
    nstage = p.nstage

    # ---- stage schedule: the autotuner times the fused tile kernel and the
    # face-split schedule on this grid and keeps the faster (state restored)
    sched_fp64 = ctx.autotune(1, 3) if not args.schedule else (None, None, args.schedule - 1)
    if args.schedule:
        ctx.set_schedule(1, args.schedule - 1)

    # ---- FP64 path: warm-up then the timed region -------------------------------
    ctx.smooth(1, args.warmup, 1, 10 ** 6, want_hist=False)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    ctx.launch_count(reset=True)
    clk = ClockSampler(dev)
    clk.start()
    ms = time_smooth(ctx, args.steps, torch)
    clocks = clk.stop()
    launches = ctx.launch_count(reset=True)
    torch.cuda.synchronize()
    ms_max = max_over_ranks(ms, pg, torch, f"cuda:{dev}") if pg else ms
    value = replica_throughput(ws, ncells * nstage * args.steps, ms_max)

    # ---- kernel roofline: event-timed pass right after the timed region ----------
    # the dominant kernel is charged the whole stage's algorithmic bytes
    kms, kcnt = ctx.profile(1, 3)
    peak, peak_kind = _peaks()
    split = sched_fp64[2] == 1
    alg_bytes = B_ALG_STAGE * ncells
    achieved = alg_bytes / (kms[1] / 1e3) / 1e9
    stage_gbs = B_ALG_STAGE * ncells * nstage * args.steps / (ms / 1e3) / 1e9

    if args.no_extras:
        if rank == 0:
            print(json.dumps({"metric": "Mcell-stage/s", "value": value, "unit": "Mcell-stage/s", "n_gpus": ws,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
                              "higher_is_better": True, "dtype": "f64", "config": {"workload": desc},
                              "main_kernel_ms": kms[1], "halo_ms": kms[0], "cells_kernel_ms": kms[3],
                              "schedule": sched_fp64, "gpu_launches": launches}), flush=True)
        ctx.close()
        return

    # ---- mixed precision path on the same arrays -------------------------------------
    from cosa_b200.params import CosaParams
    pm = CosaParams.from_buffer_copy(bytes(memoryview(p)))
    pm.precision = PREC_MIXED
    ctx.set_params(pm)
    q.upload(case.q0)
    sched_mixed = ctx.autotune(1, 3) if not args.schedule else (None, None, args.schedule - 1)
    ctx.smooth(1, args.warmup, 1, 10 ** 6, want_hist=False)
    ms_mixed = time_smooth(ctx, args.steps, torch)
    kms_m, _ = ctx.profile(1, 3)
    value_mixed = ws * ncells * nstage * args.steps / (ms_mixed / 1e3) / 1e6
    ctx.set_params(p)
    ctx.set_schedule(1, sched_fp64[2])

    # ---- end to end through the host-buffer entry point --------------------------------
    nq = q.n
    hostq = torch.empty(nq, dtype=torch.float64, pin_memory=True)
    hostq.numpy()[:] = case.q0
    stream = torch.cuda.ExternalStream(ctx.stream())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ctx.sync()
    import ctypes as C
    hist = np.zeros((1, p.npde + 1))
    e0.record(stream)
    t0 = time.perf_counter()
    for s in range(args.e2e_steps):
        st = gpu.load().cosa_gpu_smooth_host(ctx.h, 1, C.c_void_p(hostq.data_ptr()), 1, s + 1, 1,
                                             hist.ctypes.data_as(C.POINTER(C.c_double)))
        if st:
            raise RuntimeError(f"smooth_host status 0x{st:x}")
    e1.record(stream)
    e1.synchronize()
    wall = time.perf_counter() - t0
    e2e_ms = max(e0.elapsed_time(e1), wall * 1e3)
    e2e_val = ws * ncells * nstage * args.e2e_steps / (e2e_ms / 1e3) / 1e6
    state_bytes = nq * 8
    # the duct's device arrays and the pinned host copy are not needed by the
    # legs below: release them, so that the serving sweep's 150 GB budget fits
    # the device beside the other legs' contexts
    ctx.close()
    del hostq
    torch.cuda.empty_cache()

    viscous = {}
    if rank == 0 and ws == 1 and not args.no_viscous:
        for kind in ("laminar", "kom"):
            try:
                viscous[kind] = viscous_leg(kind, min(args.steps, 10), 3, dev, torch)
                viscous[kind]["mixed"] = viscous_leg(kind, min(args.steps, 10), 3, dev, torch, "mixed")["value"]
            except Exception as e:  # reported, not fatal
                viscous[kind] = {"error": str(e)}

    serving = None
    if rank == 0 and ws == 1 and not args.no_serve:
        # continuous batching: 20 Poisson arrivals at 2 req/s, half k-omega
        # RANS (NACA 0012) and half Euler (bump channel or NACA 0012, 50/50),
        # at three scales, random Mach numbers and incidences (U[-4, 8] deg),
        # each to a residual drop of 1e-8 or a cycle cap (Euler 60k, k-omega
        # 20k: single-grid explicit schemes), admission against 150 GB split
        # between the Euler engine and the context lane by the request mix,
        # FP64 and mixed precision, on this GPU after the duct runs
        from cosa_b200 import serve
        serving = {}
        reqs = serve.poisson_requests(20, 2.0, 0, naca_fraction=0.5, kom_fraction=0.5)
        for name, prec in (("fp64", 0), ("mixed", 1)):
            try:
                serving[name] = serve.run_sweep(reqs, 150e9, 1e-8, max_iter=60_000, device=dev, precision=prec,
                                                kom_max_iter=20_000).summary()
            except Exception as e:  # reported, not fatal
                serving[name] = {"error": str(e)}
        serving["workload"] = ("k-omega SST NACA 0012 256x64x2 (Re 1e6, IRS, CFL 3) / Euler (bump channel 128x64x2 at "
                               "CFL 2 or NACA 0012 256x64x2 at CFL 1) 50/50, x{0.5,1,2} in-plane, M~U[0.3,0.7], "
                               "alpha~U[-4,8] deg, Poisson 2 req/s, drop 1e-8 or 60k (Euler) / 20k (k-omega) cycles, "
                               "150 GB; Euler solves batched in the engine's merged level, k-omega solves each in "
                               "its own context and stream on a worker thread (the context lane)")
        # the same kind of solves batched in the engine (mixed precision)
        # against the plain single-solve FP64 path, 400 RK cycles each
        try:
            reqs = serve.poisson_requests(12, 2.0, 5, naca_fraction=0.5, alpha_range=(-4.0, 4.0))
            serving["batched_vs_plain"] = serve.batched_vs_plain(reqs, 400, device=dev)
        except Exception as e:  # reported, not fatal
            serving["batched_vs_plain"] = {"error": str(e)}

    hb = None
    if rank == 0 and ws == 1 and not args.no_hb:
        # harmonic balance of the pitching NACA 0012 (256 x 64 x 2, NH = 1..3),
        # FP64 and mixed: throughput, roofline and the CL/CM harmonics' gap
        from cosa_b200 import pitching
        hb = {}
        for model, bpc in (("euler", B_ALG_HB_MOVING), ("kom", B_ALG_KOM_HB_MOVING)):
            for nh in (1, 2, 3):
                key = f"nh{nh}" if model == "euler" else f"kom_nh{nh}"
                try:
                    r = pitching.compare(nh, cycles=args.hb_cycles, chunk=args.hb_cycles, device=dev, model=model)
                    f, mx = r["fp64"], r["mixed"]
                    gbs = bpc * f["mcell_snapshot_stage_s"] * 1e6 / 1e9
                    hb[key] = {"snapshots": f["snapshots"], "cells": f["cells"], "cycles": f["cycles"],
                               "fp64_mcell_snapshot_stage_s": f["mcell_snapshot_stage_s"],
                               "mixed_mcell_snapshot_stage_s": mx["mcell_snapshot_stage_s"],
                               "mixed_speedup": r["mixed_speedup"],
                               "fp64_stage_gbs_alg": gbs, "fp64_stage_frac": gbs / peak,
                               "drop_rho_fp64": f["drop_rho"],
                               "cl_harmonics_fp64": f["cl_harmonics"], "cm_harmonics_fp64": f["cm_harmonics"],
                               "max_dcl_harmonic_mixed": r["max_dcl_harmonic"],
                               "max_dcm_harmonic_mixed": r["max_dcm_harmonic"]}
                except Exception as e:  # reported, not fatal
                    hb[key] = {"error": str(e)}
        hb["workload"] = ("NACA 0012 O-grid 256x64x2 (4 blocks), M=0.5, pitching 2.5 deg about c/4 at k=0.08, "
                          "harmonic balance with one grid per snapshot, CFL 1, 4-stage RK; nh*: Euler; kom_nh*: "
                          "k-omega (Wilcox), Re 1e6, first spacing 2e-4 chords, CL/CM with skin friction")

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            cpu, _ = run_cpu_oracle(case, desc, 2, 0)
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "error": str(e)}

    if rank == 0:
        line = {
            "metric": "Mcell-stage/s", "value": value, "unit": "Mcell-stage/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "cells": ncells, "blocks": case.tables.nblocks, "stages_per_step": nstage,
                       "scheme": "Roe FDS + MUSCL kappa=1/3 smooth limiter, 4-stage RK, CFL 2, M=0.6",
                       "l2": "state 1.4 GB > L2 (126 MB): no flush needed",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": FACES_TRAFFIC_B_PER_CELL * ncells if split else None,
                         "traffic_source": "ncu dram read+write of k_faces_line (both launches of a stage) per "
                                           "cell on the 4.2 M-cell duct, x cells",
                         "kernel": "k_faces_line<fp64> (i-face + marching launches)" if split
                                   else "k_stage_tile<32,7,fp64>",
                         "kernel_ms": kms[1], "halo_ms": kms[0], "cells_kernel_ms": kms[3] if split else None,
                         "alg_bytes_per_cell": B_ALG_STAGE, "kernel_own_bytes_per_cell": B_FACES_OWN if split else None,
                         "peak_kind": peak_kind, "stage_gbs_alg": stage_gbs, "stage_frac": stage_gbs / peak},
            "schedule": {"fp64": {"tile_ms_per_step": sched_fp64[0], "split_ms_per_step": sched_fp64[1],
                                  "chosen": ["tile", "split"][sched_fp64[2]]},
                         "mixed": {"tile_ms_per_step": sched_mixed[0], "split_ms_per_step": sched_mixed[1],
                                   "chosen": ["tile", "split"][sched_mixed[2]]}},
            "mixed": {"value": value_mixed, "ms_per_step": ms_mixed / args.steps,
                      "speedup_vs_fp64": value_mixed / value if value else None,
                      "main_kernel_ms": kms_m[1], "cells_kernel_ms": kms_m[3]},
            "e2e": {"value": e2e_val, "unit": "Mcell-stage/s", "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes + 8 * (p.npde + 1)},
            "cpu_baseline": cpu,
            "viscous": viscous or None,
            "harmonic_balance": hb,
            "serving": serving,
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
