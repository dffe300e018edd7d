"""Time-accurate runs on the device, through the C-ABI.

dual_time mirrors the dual-time branch of the reference's main program
(src/cosa.f90:437-667): for each physical step q1 <- q, rhs_uns into the
fine level's rhs, ncycle pseudo-time multigrid cycles (mg(), whose stages add
src_uns and subtract rhs_uns), q2 <- q1; the first step of a run not started
from a dual-time restart is first order (bdf1).  rkuns is the explicit
time-accurate RK integration (src/cosa.f90:3890-4180).

The convergence test of the pseudo-time iteration (toler) is the caller's:
each physical step runs exactly ncycle cycles.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from . import gpu
from .params import CosaParams


def dual_time(ctx: "gpu.Context", q: "gpu.DevArray", rhs: "gpu.DevArray", vol: "gpu.DevArray", ntime: int,
              ncycle: int, q1: Optional["gpu.DevArray"] = None, q2: Optional["gpu.DevArray"] = None,
              restart_two_states: bool = False, rms_every: int = 1) -> List[np.ndarray]:
    """ntime physical steps of dual time stepping on a context whose levels
    are bound (q, rhs and vol of level 1 the arrays given here).  q1 / q2
    hold q^n / q^(n-1) (allocated when absent; with restart_two_states q2 must
    hold the restart's previous state and the first step is second order).
    Returns each step's residual history (ncycle rows)."""
    p = ctx.params
    if not p.dualt or p.dt <= 0:
        raise ValueError("dual_time needs params.dualt and params.dt > 0")
    q1 = q1 if q1 is not None else ctx.alloc_p3()
    q2 = q2 if q2 is not None else ctx.alloc_p3()
    hist = []
    for itime in range(1, ntime + 1):
        bdf1 = 1 if (itime == 1 and not restart_two_states) else 0
        if p.bdf1 != bdf1:
            p2 = CosaParams.from_buffer_copy(p)
            p2.bdf1 = bdf1
            ctx.set_params(p2)
            p = p2
        ctx.copy_interior(1, q1, q)
        ctx.rhs_uns(1, rhs, q1, q2, vol)
        h, st = ctx.mg(1, ncycle, ncycle, rms_every)
        if st:
            raise gpu.CosaError(st, "cosa_gpu_mg")
        ctx.copy_interior(1, q2, q1)
        hist.append(h)
    return hist


def rkuns(ctx: "gpu.Context", ntime: int, iprint: int = 1) -> np.ndarray:
    """ntime explicit RK steps of dt on level 1; the history of printed steps."""
    h, st = ctx.rkuns(ntime, iprint)
    if st:
        raise gpu.CosaError(st, "cosa_gpu_rkuns")
    return h
