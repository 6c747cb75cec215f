"""Serving loop: continuous batching of solver runs on one GPU.

There is no counterpart in the reference, which runs one box per MPI job
(src/MAIN.cpp:325).  A request asks for ``nsteps`` steps of one box (DNS or
LES, any compiled size, FP64 or the compensated FP32 form) from a seeded
initial field, and returns the energy spectrum E(K) of the final state.

Runs are admitted as device memory frees up, against an HBM budget, first come
first served.  A request that does not fit yet does not hold back smaller ones
behind it.  Each admitted run keeps its fields resident and is advanced in
chunks of asynchronous steps on its own CUDA stream.  The loop re-issues work
to a run as soon as its previous chunk has finished, so the steps of all
admitted runs overlap on the device and new requests join between chunks.

A run's result does not depend on what else is on the GPU: its kernels touch
only its own buffers, and the step sequence is the same as stepping it alone.
(Runs that start from a seeded field carry the one source of run-to-run
variation: the shell sums that normalise the seeded spectrum add with
floating-point atomics, so two seedings of the same request can differ in the
last bit; a request that resumes from a checkpoint starts from an exact state.)

The loop is written against a small backend interface (``create``,
``device_bytes``, ``step_async``, ``query``, ``synchronize``, ``result``,
``close``).  The GPU backend drives libspns; the tests drive the host logic
(admission, budget, cancellation, failures) with a simulated backend.
"""
from __future__ import annotations

import dataclasses
import time
from collections import deque
from typing import Callable, Dict, List, Optional

import numpy as np

from .params import HitArgs


@dataclasses.dataclass
class SolveRequest:
    rid: int
    args: HitArgs
    nsteps: int
    seed: int = 0
    kp: float = 3.0
    urms: float = 1.0
    precision: int = 1            # SPNS_FP32_HILO
    arrival: float = 0.0          # seconds after the start of the run
    init: Optional[bytes] = None  # checkpoint to resume from instead of a seeded field


@dataclasses.dataclass
class SolveResult:
    rid: int
    status: str                   # "done", "rejected", "failed" or "cancelled"
    arrival: float
    admitted: Optional[float] = None
    finished: Optional[float] = None
    steps_done: int = 0
    ek: Optional[np.ndarray] = None
    ek_tot: Optional[float] = None
    time: Optional[float] = None  # simulated time of the final state
    error: str = ""

    @property
    def latency(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.arrival


class GpuBackend:
    """libspns handles: one per admitted run."""

    def __init__(self, device: int = 0, autotune: bool = True):
        self.device = device
        self.autotune = autotune

    def device_bytes(self, req: SolveRequest) -> int:
        from .hit import estimate_device_bytes
        return estimate_device_bytes(req.args, precision=req.precision, device=self.device)

    def create(self, req: SolveRequest, priority: int = 0):
        from .hit import HIT
        # the state comes from the checkpoint or the seed: no host-side K41 draw at creation
        h = HIT(req.args, precision=req.precision, device=self.device, stream_priority=priority, k41_ranks=-1)
        if req.init is not None:
            h.checkpoint_load(req.init)
        else:
            h.seed_field(req.seed, req.kp, req.urms)
        if self.autotune:
            h.autotune(steps=2)       # timed on the first run of a box class, cached after
        return h

    def step_async(self, inst, n: int):
        inst.step_async(n)

    def query(self, inst) -> bool:
        return inst.query()

    def synchronize(self, inst):
        inst.synchronize()

    def result(self, inst):
        ek = inst.Recalculate_Energy_Cascade()
        return ek, float(ek.sum()), inst.gettime()

    def close(self, inst):
        inst.close()


@dataclasses.dataclass
class _Run:
    req: SolveRequest
    inst: object
    nbytes: int
    remaining: int
    in_flight: int = 0


class Server:
    """Admits requests by HBM budget and advances all admitted runs concurrently."""

    def __init__(self, backend, budget_bytes: int, chunk: int = 25, max_active: int = 256,
                 clock: Callable[[], float] = time.monotonic, sleep: Callable[[float], None] = time.sleep,
                 idle_sleep: float = 2e-4, prioritize: bool = True, levels: int = 6):
        self.backend = backend
        self.prioritize = prioritize
        self.levels = levels
        self.budget = int(budget_bytes)
        self.chunk = int(chunk)
        self.max_active = int(max_active)
        self.clock = clock
        self.sleep = sleep
        self.idle_sleep = idle_sleep
        self.used = 0
        self.peak_used = 0
        self._cancel = set()

    def _priority(self, req: SolveRequest, nbytes: int) -> int:
        """Stream priority by expected work (steps x bytes): shorter runs get
        precedence on the device (lower value = higher priority), so small
        requests are not held behind large ones that share the GPU."""
        if not self.prioritize:
            return 0
        work = max(1.0, float(req.nsteps) * float(nbytes))
        # one level per factor 2^2.5 of work above 2^30 byte-steps; the largest runs get 0 (lowest)
        level = max(0, min(self.levels - 1, int((np.log2(work) - 30.0) / 2.5)))
        return -(self.levels - 1 - level)

    def cancel(self, rid: int):
        """Stops a queued or running request at its next chunk boundary."""
        self._cancel.add(rid)

    def run(self, requests: List[SolveRequest]) -> Dict[int, SolveResult]:
        t0 = self.clock()
        now = lambda: self.clock() - t0  # noqa: E731
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        queue: deque = deque()
        active: Dict[int, _Run] = {}
        results: Dict[int, SolveResult] = {}
        nbytes_cache: Dict[int, int] = {}

        def finish(run: _Run, status: str, error: str = ""):
            res = results[run.req.rid]
            res.status, res.error, res.finished = status, error, now()
            res.steps_done = run.req.nsteps - run.remaining
            try:
                self.backend.close(run.inst)
            finally:
                self.used -= run.nbytes
                del active[run.req.rid]

        while pending or queue or active:
            t = now()
            while pending and pending[0].arrival <= t:
                req = pending.popleft()
                results[req.rid] = SolveResult(req.rid, "queued", req.arrival)
                queue.append(req)
            # cancellation of queued requests
            if self._cancel and queue:
                for req in [r for r in queue if r.rid in self._cancel]:
                    queue.remove(req)
                    results[req.rid].status, results[req.rid].finished = "cancelled", now()
            # admission: first come first served, smaller requests may pass one that does not fit yet
            for req in list(queue):
                if len(active) >= self.max_active:
                    break
                try:
                    nb = nbytes_cache.get(req.rid)
                    if nb is None:
                        nb = nbytes_cache[req.rid] = int(self.backend.device_bytes(req))
                except Exception as exc:  # invalid box: report, never admit
                    queue.remove(req)
                    results[req.rid].status, results[req.rid].error = "rejected", str(exc)
                    results[req.rid].finished = now()
                    continue
                if nb > self.budget:
                    queue.remove(req)
                    results[req.rid].status = "rejected"
                    results[req.rid].error = f"needs {nb} bytes, budget {self.budget}"
                    results[req.rid].finished = now()
                    continue
                if self.used + nb > self.budget:
                    continue
                queue.remove(req)
                self.used += nb
                self.peak_used = max(self.peak_used, self.used)
                try:
                    inst = self.backend.create(req, self._priority(req, nb))
                except Exception as exc:
                    self.used -= nb
                    results[req.rid].status, results[req.rid].error = "failed", str(exc)
                    results[req.rid].finished = now()
                    continue
                results[req.rid].admitted = now()
                active[req.rid] = _Run(req, inst, nb, int(req.nsteps))
            # advance: re-issue to every run whose chunk has finished
            busy = False
            for rid in list(active):
                run = active[rid]
                if run.in_flight:
                    try:
                        if not self.backend.query(run.inst):
                            busy = True
                            continue
                        self.backend.synchronize(run.inst)
                    except Exception as exc:
                        run.in_flight = 0
                        finish(run, "failed", str(exc))
                        continue
                    run.remaining -= run.in_flight
                    run.in_flight = 0
                if rid in self._cancel:
                    finish(run, "cancelled")
                    continue
                if run.remaining == 0:
                    res = results[rid]
                    try:
                        res.ek, res.ek_tot, res.time = self.backend.result(run.inst)
                        finish(run, "done")
                    except Exception as exc:
                        finish(run, "failed", str(exc))
                    continue
                n = min(self.chunk, run.remaining)
                try:
                    self.backend.step_async(run.inst, n)
                except Exception as exc:
                    finish(run, "failed", str(exc))
                    continue
                run.in_flight = n
                busy = True
            if not busy and not queue and pending:
                wait = pending[0].arrival - now()
                if wait > 0:
                    self.sleep(min(wait, 0.05))
            elif busy and self.idle_sleep:
                self.sleep(self.idle_sleep)
        return results


def summarize(results: Dict[int, SolveResult], makespan: float) -> dict:
    done = [r for r in results.values() if r.status == "done"]
    lat = np.array([r.latency for r in done]) if done else np.zeros(0)
    return {
        "requests": len(results), "done": len(done),
        "rejected": sum(r.status == "rejected" for r in results.values()),
        "failed": sum(r.status == "failed" for r in results.values()),
        "cancelled": sum(r.status == "cancelled" for r in results.values()),
        "solves_per_s": len(done) / makespan if makespan > 0 else 0.0,
        "p50_latency_s": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_latency_s": float(np.percentile(lat, 99)) if lat.size else None,
        "makespan_s": makespan,
    }


def synthetic_workload(n: int, rate: float = 20.0, seed: int = 0, sizes=(32, 64, 128, 256),
                       weights=(0.4, 0.3, 0.2, 0.1), steps=(200, 2000), precision: int = 1) -> List[SolveRequest]:
    """Poisson arrivals of LES and DNS runs of seeded spectra (the served workload)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        N = int(rng.choice(sizes, p=np.asarray(weights) / np.sum(weights)))
        les = bool(rng.random() < 0.5)
        cs = float(rng.uniform(0.10, 0.20)) if les else 0.0
        nu = float(rng.uniform(1e-3, 1e-2)) if not les else float(rng.uniform(1e-4, 1e-3))
        out.append(SolveRequest(rid, box_args(N, nu=nu, C_Smag=cs), int(rng.integers(steps[0], steps[1] + 1)),
                                seed=int(rng.integers(0, 2 ** 63)), kp=3.0, precision=precision, arrival=t))
    return out


def box_args(N: int, nu: float, C_Smag: float = 0.0, C_At: float = 0.5, self_adaptive: bool = False) -> HitArgs:
    """A cubic 2 pi box with N retained modes per axis (FFT grid 3N/2)."""
    M = (3 * N) // 2
    return HitArgs(Nx=N, Ny=N, Nz=N, Mx=M, My=M, Mz=M, nu=nu, C_Smag=C_Smag, C_At=C_At, Lx=1, Ly=1, Lz=1,
                   omega_x=0.0, omega_y=0.0, omega_z=0.0, Nx_file=-1, Ny_file=-1, Nz_file=-1, isReLambda=False,
                   isInitialFieldFromBinaryFile=False, isInitialFieldFromASCIIFile=False, isNotCubic=False,
                   isRotating=False, isLES=C_Smag > 0, isComplexConjugateCorrected=False,
                   isSelfAdaptive=self_adaptive)
