"""The serving engine (cosa_serve): several solves resident on one GPU and
advanced by shared stage launches.

* a served solve follows the fused single-solve path iteration for
  iteration (1e-12 relative, the parity bound);
* a solve gives the same result alone and among others (bit for bit: its
  cells, its norm reduction and its convergence checks never see the other
  solves);
* admission waits for device memory and retirement gives it back;
* a short Poisson sweep converges every request and reports latencies.

The explicit single-grid scheme reduces the bump channel's residual slowly
(about 10x in 500 iterations, 100x in 6000), so these tests converge to a
residual drop of 0.2.
"""
import numpy as np
import pytest

from cosa_b200 import cases, gpu, serve

import casekit

pytestmark = pytest.mark.gpu


def _interior(case, q):
    return casekit.interior_cells(case, q, 5)


def test_served_solve_matches_fused_path():
    r = serve.channel_request(0.5, 0.45)
    n = 40
    srv = gpu.Server(serve.engine_scheme(), 2e9, check_every=7)
    rid = srv.submit(r.case.tables, r.case.x, r.case.y, r.case.z, r.case.q0, r.flow, 0.0, n)
    while srv.result(rid)["state"] in ("queued", "active"):
        srv.step(16)
    res = srv.result(rid, want_state=True)
    srv.close()
    assert res["state"] == "stopped" and res["iters"] == n
    # the single-solve fused path on the same case
    p = serve.engine_scheme()
    for k in ("machfs", "inlet_t0", "inlet_p0"):
        setattr(p, k, getattr(r.flow, k))
    ctx = gpu.Context([r.case.tables], p)
    x, y, z = (ctx.alloc_p2(ncomp=1).upload(a) for a in (r.case.x, r.case.y, r.case.z))
    si, sj, sk, vol = ctx.alloc_p2(), ctx.alloc_p2(), ctx.alloc_p2(), ctx.alloc_p1()
    ctx.imetrix(1, x, y, z, si, sj, sk)
    ctx.vols(1, x, y, z, vol)
    q = ctx.alloc_p3().upload(r.case.q0)
    ctx.bind_level(1, q=q, qold=ctx.alloc_p3(), dtvol=ctx.alloc_p1(), si=si, sj=sj, sk=sk, vol=vol)
    _, st = ctx.smooth(1, n, 1, 10 ** 6, want_hist=False)
    assert st == 0
    a, b = _interior(r.case, res["q"]), _interior(r.case, q.download())
    scale = np.abs(b).reshape(-1, 5).max(axis=0)
    assert (np.abs(a - b) / scale[None, :, None]).max() <= 1e-12
    ctx.close()


def _run(reqs, order, tol=0.2, max_iter=5000, budget=4e9, steps=25):
    srv = gpu.Server(serve.engine_scheme(), budget, check_every=10)
    ids = {}
    for k in order:
        r = reqs[k]
        ids[k] = srv.submit(r.case.tables, r.case.x, r.case.y, r.case.z, r.case.q0, r.flow, tol, max_iter)
        srv.step(steps)  # the next request arrives while the earlier ones run
    while any(srv.result(i)["state"] in ("queued", "active") for i in ids.values()):
        srv.step(steps)
    out = {k: srv.result(i, want_state=True) for k, i in ids.items()}
    srv.close()
    return out


def test_result_same_alone_and_in_the_mix():
    reqs = [serve.channel_request(0.5, 0.4), serve.channel_request(1.0, 0.6), serve.channel_request(0.5, 0.65)]
    alone = _run(reqs, [0])[0]
    mixed = _run(reqs, [1, 0, 2])
    m = mixed[0]
    assert alone["state"] == m["state"] == "converged"
    assert alone["iters"] == m["iters"]
    assert np.array_equal(_interior(reqs[0].case, alone["q"]), _interior(reqs[0].case, m["q"]))
    assert all(v["state"] == "converged" for v in mixed.values())


def test_admission_waits_for_memory():
    reqs = [serve.channel_request(1.0, 0.5), serve.channel_request(1.0, 0.55)]
    slots = sum((d[0] + 3) * (d[1] + 3) * (d[2] + 3) for d in reqs[0].case.tables.dims)
    budget = int(slots * 1.5) * (3 * 5 + 2 + 3 * 4) * 8  # room for one solve, not two
    srv = gpu.Server(serve.engine_scheme(), budget, check_every=10)
    free0 = srv.free_slots()
    a = srv.submit(reqs[0].case.tables, reqs[0].case.x, reqs[0].case.y, reqs[0].case.z, reqs[0].case.q0,
                   reqs[0].flow, 0.2, 5000)
    b = srv.submit(reqs[1].case.tables, reqs[1].case.x, reqs[1].case.y, reqs[1].case.z, reqs[1].case.q0,
                   reqs[1].flow, 0.2, 5000)
    na, nq = srv.step(5)
    assert (na, nq) == (1, 1)
    assert srv.result(b)["state"] == "queued"
    while srv.result(b)["state"] in ("queued", "active"):
        srv.step(50)
    ra, rb = srv.result(a), srv.result(b)
    assert ra["state"] == rb["state"] == "converged"
    assert rb["t_admit"] >= ra["t_done"]
    assert srv.free_slots() == free0
    srv.close()


def test_short_sweep_reports_latency():
    reqs = serve.poisson_requests(6, rate=20.0, seed=1, scales=(0.5, 1.0))
    res = serve.run_sweep(reqs, budget_bytes=8e9, tol=0.2, max_iter=20000, iters_per_step=25)
    s = res.summary()
    assert s["converged"] == 6
    assert 0 < s["p50_latency_s"] <= s["p99_latency_s"]
    assert s["solves_per_hour"] > 0


def test_naca_requests_in_the_mix():
    """Euler NACA 0012 requests (4 blocks with the trailing-edge seam cut,
    far field at their own incidence) served among bump channels: the same
    bits alone and in the mix, every request converged."""
    reqs = [serve.naca_request(0.5, 0.5, 6.0), serve.channel_request(0.5, 0.45), serve.naca_request(0.5, 0.65, -3.0)]
    alone = _run(reqs, [0], tol=0.3)[0]
    mixed = _run(reqs, [1, 0, 2], tol=0.3)
    m = mixed[0]
    assert alone["state"] == m["state"] == "converged"
    assert alone["iters"] == m["iters"]
    assert np.array_equal(_interior(reqs[0].case, alone["q"]), _interior(reqs[0].case, m["q"]))
    assert all(v["state"] == "converged" for v in mixed.values())


def test_failed_solve_is_isolated():
    """A request whose state loses positivity (Euler NACA at 7.7 deg on the
    finer grid run at CFL 2: the impulsive start drives p below qmin at the
    leading edge) is retired as failed; the requests beside it converge
    with the same bits as alone."""
    bad = serve.naca_request(1.0, 0.417, 7.68)
    bad.flow.cfl = 2.0
    reqs = [serve.channel_request(0.5, 0.45), bad, serve.naca_request(0.5, 0.5, 6.0)]
    alone = {k: _run(reqs, [k], tol=0.3)[k] for k in (0, 2)}
    assert _run(reqs, [1], tol=0.3)[1]["state"] == "failed"
    mixed = _run(reqs, [0, 1, 2], tol=0.3)
    assert mixed[1]["state"] == "failed"
    for k in (0, 2):
        assert mixed[k]["state"] == alone[k]["state"] == "converged"
        assert mixed[k]["iters"] == alone[k]["iters"]
        assert np.array_equal(_interior(reqs[k].case, alone[k]["q"]), _interior(reqs[k].case, mixed[k]["q"]))


def test_short_mixed_sweep_reports_latency():
    reqs = serve.poisson_requests(6, rate=20.0, seed=1, scales=(0.5, 1.0), naca_fraction=0.5, alpha_range=(-4.0, 4.0))
    assert {r.grid for r in reqs} == {"channel", "naca"}
    res = serve.run_sweep(reqs, budget_bytes=8e9, tol=0.3, max_iter=20000, iters_per_step=25)
    s = res.summary()
    assert s["requests"] == 6 and s["converged"] == 6, res.states
    assert 0 < s["p50_latency_s"] <= s["p99_latency_s"]


def _lane_run(reqs, n, budget=4e9, check_every=10):
    lane = serve.ContextLane(budget, check_every=check_every)
    try:
        ids = [lane.submit(r.case, r.flow, 0.0, n) for r in reqs]
        while any(lane.result(i)["state"] in ("queued", "active") for i in ids):
            import time
            time.sleep(0.01)
        return [dict(lane.result(i), q=lane.solves[i]["result"]) for i in ids]
    finally:
        lane.close()


def test_kom_lane_matches_plain_solver_alone_and_in_the_mix():
    """k-omega requests in the lane (each in its own context and stream,
    advanced by worker threads at the same time): every solve gives the
    bits of a plain SteadySolver run of the same cycles, alone and beside
    other k-omega solves."""
    from cosa_b200.solver import SteadySolver
    reqs = [serve.kom_channel_request(0.5, 0.45), serve.kom_naca_request(0.5, 0.5, 4.0),
            serve.kom_channel_request(0.5, 0.4)]
    n = 60
    mixed = _lane_run(reqs, n)
    alone = _lane_run(reqs[1:2], n)[0]
    s = SteadySolver(reqs[1].case)
    _, st = s.run(n, rms_every=10)
    assert st == 0
    plain = s.state()
    s.close()
    assert mixed[1]["state"] == alone["state"] == "stopped" and mixed[1]["iters"] == n
    for r in (alone, mixed[1]):
        assert np.array_equal(casekit.interior_cells(reqs[1].case, r["q"], 7),
                              casekit.interior_cells(reqs[1].case, plain, 7))
    assert all(m["state"] == "stopped" for m in mixed), [(m["state"], m["status"], m.get("error")) for m in mixed]


def test_kom_lane_admission_waits_for_memory():
    a, b = serve.kom_channel_request(0.5, 0.45), serve.kom_channel_request(0.5, 0.55)
    budget = serve.kom_solve_bytes(a.case) * 1.5  # room for one solve at a time
    ra, rb = _lane_run([a, b], 30, budget=budget)
    assert ra["state"] == rb["state"] == "stopped"
    assert rb["t_admit"] >= ra["t_done"]


def test_euler_and_kom_sweep_retires_every_request():
    reqs = serve.poisson_requests(8, rate=20.0, seed=3, scales=(0.5,), naca_fraction=0.5, alpha_range=(-4.0, 4.0),
                                  kom_fraction=0.5)
    assert any(serve.is_kom(r) for r in reqs) and not all(serve.is_kom(r) for r in reqs)
    res = serve.run_sweep(reqs, budget_bytes=8e9, tol=0.3, max_iter=20000, iters_per_step=25, kom_max_iter=400)
    s = res.summary()
    assert s["requests"] == 8 and s["failed"] == 0, res.states
    assert s["euler"]["converged"] == s["euler"]["requests"]
    assert s["kom"]["converged"] + s["kom"]["stopped"] == s["kom"]["requests"]
    assert 0 < s["p50_latency_s"] <= s["p99_latency_s"]


def test_harmonic_balance_requests_in_the_lane():
    """Pitching harmonic-balance requests (Euler S = 3 and k-omega S = 3) in
    the context lane beside a steady k-omega solve: each gives the bits of
    a plain PitchingSolver run of the same cycles."""
    from cosa_b200.pitching import PitchingSolver
    reqs = [serve.hb_request(0.25, 0.5, 1.0, 1), serve.hb_request(0.25, 0.5, 0.0, 1, model="kom"),
            serve.kom_channel_request(0.5, 0.4)]
    n = 40
    got = _lane_run(reqs, n)
    assert all(g["state"] == "stopped" and g["iters"] == n for g in got), got
    for k in (0, 1):
        s = PitchingSolver(reqs[k].case)
        _, st = s.run(n, rms_every=10)
        assert st == 0
        plain = s.state()
        s.close()
        npde = reqs[k].flow.npde
        assert np.array_equal(got[k]["q"], plain), k


def test_multigrid_requests_in_the_lane():
    """Two-level multigrid Euler requests in the context lane beside a
    single-grid k-omega solve: each gives the bits of a plain SteadySolver
    multigrid run of the same cycles."""
    from cosa_b200.solver import SteadySolver
    reqs = [serve.mg_request(0.5, 0.45), serve.kom_channel_request(0.5, 0.4), serve.mg_request(0.5, 0.6)]
    assert all(serve.in_lane(r) for r in reqs)
    n = 30
    got = _lane_run(reqs, n)
    assert all(g["state"] == "stopped" and g["iters"] == n for g in got), got
    for k in (0, 2):
        s = SteadySolver(reqs[k].case)
        _, st = s.run(n, rms_every=10)
        assert st == 0
        plain = s.state()
        s.close()
        assert np.array_equal(got[k]["q"], plain), k
