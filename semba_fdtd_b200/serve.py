"""Served form: FDTD solves admitted as they arrive and folded into the
batched step (continuous batching).

* Requests arrive on a Poisson clock (seeded).  Each is planned on the host
  (:class:`~semba_fdtd_b200.batch.Plan`, no device memory; a pool of planner
  threads works ahead of admission) and admitted when its device footprint
  -- fields and media, CPML psi, ADE state, sources, time vector and whole
  probe traces, as laid out in the arena -- fits the arena's free memory (the
  HBM budget) and a free instance slot exists.  Admission is first come,
  first served, with a bounded look-ahead (`backfill`) past a head request
  that does not fit yet.
* Admitted solves stay resident (fields, state and probe buffers) and join
  the next chunk of batched steps (one graph replay of 32 steps).
* A finished solve's probe traces are read back at the chunk boundary where
  it completes, its arena memory is freed, and its latency (completion minus
  arrival) recorded.

:func:`run_plain` serves the same stream one solve at a time through the
single-problem path (:class:`~semba_fdtd_b200.Solver`), the baseline the
batched server is compared with.
"""
from __future__ import annotations

import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, Future, ThreadPoolExecutor, wait
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .batch import Batch, Plan
from .case import Problem
from .solver import Solver


@dataclass
class Request:
    rid: int
    arrival: float  # seconds after the start of the run
    problem: Problem
    nsteps: int
    plan: Plan | None = None
    admitted: float | None = None
    finished: float | None = None
    traces: np.ndarray | None = None


def poisson_arrivals(n: int, rate: float, seed: int) -> np.ndarray:
    """Arrival times (s) of n requests at `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))


@dataclass
class ServeStats:
    completed: int = 0
    makespan: float = 0.0
    latencies: list = field(default_factory=list)
    peak_resident: int = 0
    peak_bytes: int = 0
    chunks: int = 0
    refused_admissions: int = 0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies, np.float64)
        return {"completed": self.completed, "makespan_s": self.makespan,
                "solves_per_s": self.completed / self.makespan if self.makespan > 0 else None,
                "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
                "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
                "mean_s": float(lat.mean()) if lat.size else None,
                "peak_resident": self.peak_resident, "peak_arena_bytes": self.peak_bytes, "chunks": self.chunks,
                "refused_admissions": self.refused_admissions}


class Server:
    """Continuous-batching server over one :class:`Batch`.

    `planners` host threads plan arriving requests (the set-up runs in
    libsemba_gpu with the GIL released) at most `plan_ahead` requests ahead
    of admission, overlapping the chunks running on the GPU."""

    def __init__(self, arena_bytes: int, max_instances: int = 512, chunk: int = 32, backfill: int = 16,
                 variant: str = "exact", autotune: bool = False, planners: int = 8, plan_ahead: int = 16):
        self.batch = Batch(arena_bytes, max_instances, variant)
        self.max_instances = max_instances
        self.chunk = chunk
        self.backfill = backfill
        self.variant = variant
        self.autotune = autotune
        self.planners = planners
        self.plan_ahead = plan_ahead

    def close(self) -> None:
        self.batch.close()

    def _fits(self, plan: Plan) -> bool:
        cap, used, largest = self.batch.memory()
        return plan.footprint <= cap - used and plan.largest_buffer <= largest

    def run(self, requests: list[Request], keep_traces: bool = True) -> ServeStats:
        b = self.batch
        st = ServeStats()
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: list[Request] = []
        futures: dict[int, Future] = {}
        active: dict[int, Request] = {}
        pool = ThreadPoolExecutor(max_workers=self.planners)
        t0 = time.perf_counter()
        tuned = not self.autotune

        def now():
            return time.perf_counter() - t0

        def submit_plans():
            for req in waiting[: self.plan_ahead]:
                if req.plan is None and req.rid not in futures:
                    futures[req.rid] = pool.submit(Plan, req.problem, req.nsteps, self.variant)

        def collect_plans():
            for req in waiting:
                f = futures.get(req.rid)
                if f is not None and f.done():
                    req.plan = f.result()
                    del futures[req.rid]

        try:
            while pending or waiting or active:
                t = now()
                while pending and pending[0].arrival <= t:
                    waiting.append(pending.popleft())
                submit_plans()
                collect_plans()
                # the next chunk is queued first: the set-up of the requests
                # admitted below overlaps it on the device's set-up stream
                launched = False
                if active:
                    if not tuned and len(active) >= 4:
                        b.autotune(2)
                        tuned = True
                    b.advance(self.chunk)
                    st.chunks += 1
                    launched = True
                # admission: first come first served with bounded look-ahead
                k = 0
                while k < min(len(waiting), self.backfill) and len(active) < self.max_instances:
                    req = waiting[k]
                    if req.plan is None or not self._fits(req.plan):
                        if req.plan is not None:
                            st.refused_admissions += 1
                        k += 1
                        continue
                    try:
                        slot = b.add(req.plan)
                    except _lib.SembaGpuError:
                        st.refused_admissions += 1
                        k += 1
                        continue
                    req.admitted = now()
                    active[slot] = req
                    waiting.pop(k)
                submit_plans()
                st.peak_resident = max(st.peak_resident, len(active))
                st.peak_bytes = max(st.peak_bytes, b.memory()[1])
                if not launched:
                    if not active:
                        planned = [r for r in waiting[: self.backfill] if r.plan is not None]
                        if waiting and not pending and len(planned) == len(waiting[: self.backfill]):
                            raise _lib.SembaGpuError(f"request {waiting[0].rid} needs {waiting[0].plan.footprint} "
                                                     f"bytes; the arena holds {b.memory()[0]}")
                        # nothing to step: wait for a plan or the next arrival
                        nxt = pending[0].arrival - now() if pending else 0.05
                        wait(list(futures.values()), timeout=max(0.0, min(nxt, 0.05)), return_when=FIRST_COMPLETED)
                    continue
                b.synchronize()
                t = now()
                for slot in [s for s in active if b.done(s)]:
                    req = active.pop(slot)
                    tr = b.probes(slot)
                    req.traces = tr if keep_traces else None
                    req.finished = t
                    b.remove(slot)
                    st.latencies.append(req.finished - req.arrival)
                    st.completed += 1
        finally:
            pool.shutdown(wait=True)
        st.makespan = now() - min((r.arrival for r in requests), default=0.0)
        return st


def run_plain(requests: list[Request], variant: str = "exact", keep_traces: bool = True) -> ServeStats:
    """The same stream, first come first served, one solve at a time through
    the single-problem path (set-up, graph-replayed steps, probe read-back)."""
    st = ServeStats()
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.arrival):
        t = time.perf_counter() - t0
        if t < req.arrival:
            time.sleep(req.arrival - t)
        with Solver(req.problem, variant=variant, max_steps=req.nsteps,
                    probe_capacity=max(1024, req.nsteps + 1)) as s:
            s.step(req.nsteps + 1)
            tr = s.probes()
        req.traces = tr if keep_traces else None
        req.finished = time.perf_counter() - t0
        st.latencies.append(req.finished - req.arrival)
        st.completed += 1
        st.peak_resident = 1
    st.makespan = time.perf_counter() - t0 - min((r.arrival for r in requests), default=0.0)
    return st
