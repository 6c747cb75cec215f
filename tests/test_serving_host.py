"""Host logic of the serving loop (admission by budget, continuous batching,
cancellation, failures) against a simulated backend: no GPU, failures are made
on the host (a backend call that raises, a request that never fits)."""
import numpy as np
import pytest

from spns_b200.serving import Server, SolveRequest, box_args, summarize, synthetic_workload


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


class SimBackend:
    """Each run takes `cost(N)` simulated seconds per step; the clock advances
    whenever the loop polls, as a GPU would progress meanwhile."""

    def __init__(self, clock, fail_create=(), fail_step=(), bytes_per_mode=16):
        self.clock = clock
        self.fail_create = set(fail_create)
        self.fail_step = set(fail_step)
        self.bytes_per_mode = bytes_per_mode
        self.live = {}
        self.max_live_bytes = 0

    def device_bytes(self, req):
        if req.args.Nx < 2:
            raise ValueError("invalid sizes or length factors")
        return req.args.Nx ** 3 * self.bytes_per_mode

    def create(self, req, priority=0):
        if req.rid in self.fail_create:
            raise RuntimeError("device allocation failed")
        inst = {"req": req, "done_at": 0.0, "steps": 0, "pending": 0}
        self.live[req.rid] = inst
        self.max_live_bytes = max(self.max_live_bytes, sum(self.device_bytes(i["req"]) for i in self.live.values()))
        return inst

    def step_async(self, inst, n):
        inst["pending"] = n
        inst["done_at"] = self.clock.t + 1e-4 * n * (inst["req"].args.Nx / 32) ** 3

    def query(self, inst):
        self.clock.t += 1e-5
        return self.clock.t >= inst["done_at"]

    def synchronize(self, inst):
        if inst["req"].rid in self.fail_step and inst["steps"] > 0:
            raise RuntimeError("libspns status -5: non-finite velocity")
        inst["steps"] += inst["pending"]
        inst["pending"] = 0

    def result(self, inst):
        return np.array([0.0, float(inst["steps"])]), float(inst["steps"]), 1e-3 * inst["steps"]

    def close(self, inst):
        self.live.pop(inst["req"].rid, None)


def _reqs(sizes, steps=100, spacing=0.0):
    return [SolveRequest(i, box_args(n, nu=1e-2), steps, seed=i, arrival=i * spacing) for i, n in enumerate(sizes)]


def _server(backend, clock, budget, chunk=10):
    return Server(backend, budget, chunk=chunk, clock=clock, sleep=clock.sleep, idle_sleep=0.0)


def test_all_complete_with_the_right_step_count():
    clock = FakeClock()
    be = SimBackend(clock)
    res = _server(be, clock, budget=10 ** 12).run(_reqs([32, 64, 32, 48], steps=95))
    assert all(r.status == "done" for r in res.values())
    assert all(r.steps_done == 95 and r.ek_tot == 95.0 for r in res.values())
    assert not be.live


def test_budget_is_never_exceeded_and_smaller_runs_pass_a_big_one():
    clock = FakeClock()
    be = SimBackend(clock)
    budget = 64 ** 3 * 16 + 2 * 32 ** 3 * 16        # one 64 box and two 32 boxes
    srv = _server(be, clock, budget)
    res = srv.run(_reqs([64, 64, 32, 32, 32]))
    assert all(r.status == "done" for r in res.values())
    assert be.max_live_bytes <= budget and srv.peak_used <= budget
    # the second 64 box waits for the first; the 32 boxes behind it are admitted meanwhile
    assert res[2].admitted < res[1].admitted and res[3].admitted < res[1].admitted


def test_request_larger_than_the_budget_is_rejected_not_blocking():
    clock = FakeClock()
    be = SimBackend(clock)
    res = _server(be, clock, budget=32 ** 3 * 16 * 2).run(_reqs([128, 32, 32]))
    assert res[0].status == "rejected" and "budget" in res[0].error
    assert res[1].status == res[2].status == "done"


def test_invalid_request_and_failing_runs_do_not_affect_the_others():
    clock = FakeClock()
    be = SimBackend(clock, fail_create={1}, fail_step={2})
    reqs = _reqs([32, 32, 32, 32])
    reqs.append(SolveRequest(9, _bad_args(), 10))
    srv = _server(be, clock, budget=10 ** 12)
    res = srv.run(reqs)
    assert res[1].status == "failed" and "allocation" in res[1].error
    assert res[2].status == "failed" and "non-finite" in res[2].error
    assert res[9].status == "rejected"
    assert res[0].status == res[3].status == "done"
    assert srv.used == 0 and not be.live


def _bad_args():
    import dataclasses
    return dataclasses.replace(box_args(32, nu=1e-2), Nx=1)


def test_cancellation_releases_the_run():
    clock = FakeClock()
    be = SimBackend(clock)
    srv = _server(be, clock, budget=10 ** 12)
    srv.cancel(1)
    res = srv.run(_reqs([32, 64, 32], steps=200))
    assert res[1].status == "cancelled"
    assert res[0].status == res[2].status == "done"
    assert srv.used == 0 and not be.live


def test_arrivals_are_admitted_while_others_run():
    clock = FakeClock()
    be = SimBackend(clock)
    res = _server(be, clock, budget=10 ** 12).run(_reqs([64, 32, 32], steps=400, spacing=0.01))
    # the later arrivals start before the first run has finished (continuous batching)
    assert res[1].admitted < res[0].finished and res[2].admitted < res[0].finished
    s = summarize(res, max(r.finished for r in res.values()))
    assert s["done"] == 3 and s["p99_latency_s"] >= s["p50_latency_s"] > 0


def test_idle_server_waits_for_late_arrivals():
    clock = FakeClock()
    be = SimBackend(clock)
    reqs = _reqs([32, 32], steps=20)
    reqs[1].arrival = 5.0                      # arrives long after the first has finished
    res = _server(be, clock, budget=10 ** 12).run(reqs)
    assert res[0].status == res[1].status == "done"
    assert res[1].admitted >= 5.0 and res[0].finished < 5.0


def test_synthetic_workload_matches_the_served_mix():
    reqs = synthetic_workload(400, rate=20.0, seed=1)
    sizes = np.array([r.args.Nx for r in reqs])
    assert set(sizes) <= {32, 64, 128, 256}
    assert abs(np.mean(sizes == 32) - 0.4) < 0.08 and abs(np.mean(sizes == 256) - 0.1) < 0.05
    steps = np.array([r.nsteps for r in reqs])
    assert steps.min() >= 200 and steps.max() <= 2000
    gaps = np.diff([0.0] + [r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 20.0) < 0.01
    assert any(r.args.isLES for r in reqs) and any(not r.args.isLES for r in reqs)


def test_shorter_runs_get_higher_stream_priority():
    clock = FakeClock()
    srv = _server(SimBackend(clock), clock, budget=10 ** 12)
    small = SolveRequest(0, box_args(32, nu=1e-2), 200)
    big = SolveRequest(1, box_args(256, nu=1e-2), 2000)
    p_small = srv._priority(small, 32 ** 3 * 1000)
    p_big = srv._priority(big, 256 ** 3 * 1000)
    assert p_small < p_big <= 0
