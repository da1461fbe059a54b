"""Continuous-batching request loop over the batched stepper.

Solve requests (a mesh, material, boundary conditions and a cycle count)
arrive over time.  The loop admits each arrived request into the running
batch as soon as an instance slot and enough of the device-memory budget are
free -- the batch itself refuses an instance that would exceed the budget --
keeps its state resident on the device while it runs beside the others,
retires it when its cycles are done (downloading what the caller asked for,
and its energy sums) and frees its memory for the next arrivals.  Admission
is first come, first served, with backfill: a request that does not fit yet
does not block later ones that do.

The GPU advances in quanta of graph-captured cycles; between quanta the host
retires finished instances and admits new ones.  A quantum ends no later
than the earliest finishing instance would (rounded up to ``min_quantum``),
so finished work does not idle for long.

The loop is written against a small backend interface so that the scheduling
logic can be exercised without a GPU (``FakeBackend``); ``BatchBackend``
drives the C ABI.
"""
from __future__ import annotations

import dataclasses
import math
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

ERR_ARG = -1
ERR_OOM = -2


@dataclasses.dataclass
class Outcome:
    """What happened to one request."""

    index: int
    arrival: float
    admitted: float = math.nan
    finished: float = math.nan
    cycles: int = 0
    status: int = 0
    elements: int = 0
    result: Optional[Dict[str, np.ndarray]] = None
    energy: Optional[Dict[str, float]] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class AdmissionError(RuntimeError):
    """The backend has no room for the instance now (slots or memory)."""


class BatchBackend:
    """Backend on the C ABI batch (``capi.Batch``)."""

    def __init__(self, *, budget_bytes: int, max_instances: int = 1024, max_elements: int = 64 << 20,
                 max_nodes: int = 72 << 20, precision: Optional[int] = None, device: int = 0,
                 fields: Sequence[str] = ("u",), assembly: int = 0):
        from . import capi
        self._capi = capi
        self.batch = capi.Batch(max_instances=max_instances, max_elements=max_elements, max_nodes=max_nodes,
                                budget_bytes=budget_bytes, precision=capi.MIXED if precision is None else precision,
                                device=device, assembly=assembly)
        self.fields = tuple(fields)

    def add(self, problem) -> int:
        p = problem
        try:
            slot = self.batch.add(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls)
        except self._capi.EnscError as e:
            if e.code == ERR_OOM:
                raise AdmissionError(str(e)) from None
            raise
        self.batch.set_bcs(slot, p.bc_code, p.bc_value)
        return slot

    def prepare(self, problem):
        p = problem
        return self._capi.Prepared(p.mesh.x0, p.mesh.conn, p.v0, material=p.material, controls=p.controls,
                                   precision=self.batch.precision, assembly=self.batch.assembly)

    def add_prepared(self, token, problem) -> int:
        try:
            slot = self.batch.add_prepared(token)
        except self._capi.EnscError as e:
            if e.code == ERR_OOM:
                raise AdmissionError(str(e)) from None
            raise
        self.batch.set_bcs(slot, problem.bc_code, problem.bc_value)
        return slot

    def release(self, token) -> None:
        token.close()

    def arm(self, slot: int, cycles: int) -> None:
        self.batch.arm(slot, cycles)

    def run(self, cycles: int) -> None:
        self.batch.run(cycles)

    def sync(self) -> int:
        return self.batch.sync()

    def report(self, slot: int) -> Dict[str, float]:
        return self.batch.report(slot)

    def download(self, slot: int) -> Dict[str, np.ndarray]:
        return self.batch.download(slot, self.fields) if self.fields else {}

    def energy(self, slot: int) -> Dict[str, float]:
        return self.batch.energy(slot)

    def remove(self, slot: int) -> None:
        self.batch.remove(slot)

    @property
    def device_bytes(self) -> int:
        return self.batch.device_bytes

    def close(self) -> None:
        self.batch.close()


class FakeBackend:
    """Host-only stand-in with the batch's admission rules (slots, byte
    budget) and cycle accounting, for testing the loop without a GPU."""

    def __init__(self, *, budget_bytes: int, max_instances: int, bytes_per_element: int = 400,
                 seconds_per_element_cycle: float = 1e-9):
        self.t = 0.0                      # simulated seconds
        self.budget = budget_bytes
        self.max_instances = max_instances
        self.bpe = bytes_per_element
        self.spec = seconds_per_element_cycle
        self.slots: Dict[int, dict] = {}
        self.used = 0
        self.peak = 0
        self.peak_instances = 0
        self.cycles_run = 0

    def add(self, problem) -> int:
        need = problem.mesh.n_elements * self.bpe
        if len(self.slots) >= self.max_instances or self.used + need > self.budget:
            raise AdmissionError("no room")
        slot = next(i for i in range(self.max_instances) if i not in self.slots)
        self.slots[slot] = dict(bytes=need, ne=problem.mesh.n_elements, done=0, target=0)
        self.used += need
        self.peak = max(self.peak, self.used)
        self.peak_instances = max(self.peak_instances, len(self.slots))
        return slot

    def prepare(self, problem):
        if problem.mesh.n_elements <= 0:
            raise ValueError("empty mesh")
        return problem

    def add_prepared(self, token, problem) -> int:
        return self.add(token)

    def release(self, token) -> None:
        pass

    def arm(self, slot: int, cycles: int) -> None:
        s = self.slots[slot]
        s["target"] = s["done"] + cycles

    def run(self, cycles: int) -> None:
        work = 0
        for s in self.slots.values():
            n = max(0, min(cycles, s["target"] - s["done"]))
            s["done"] += n
            work += n * s["ne"]
        self.cycles_run += cycles
        self.t += work * self.spec

    def now(self) -> float:
        return self.t

    def sleep(self, dt: float) -> None:
        self.t += max(0.0, dt)

    def sync(self) -> int:
        return sum(1 for s in self.slots.values() if s["done"] < s["target"])

    def report(self, slot: int) -> Dict[str, float]:
        s = self.slots[slot]
        return {"cycles": s["done"], "done": int(s["done"] >= s["target"]), "status": 0}

    def download(self, slot: int) -> Dict[str, np.ndarray]:
        return {}

    def energy(self, slot: int) -> Dict[str, float]:
        return {}

    def remove(self, slot: int) -> None:
        self.used -= self.slots.pop(slot)["bytes"]

    @property
    def device_bytes(self) -> int:
        return self.used

    def close(self) -> None:
        pass


class Server:
    """The request loop.  ``requests`` carry ``index``, ``arrival`` (seconds
    after the start of the stream) and ``problem`` (a workloads.Problem whose
    ``cycles`` is the requested cycle count).

    Admission has a host part (``backend.prepare``: element constants,
    lumped mass, node tables) and a device part (``backend.add_prepared``).
    The host part of the next arrivals runs while the GPU steps the current
    quantum: on ``prepare_workers`` threads, or with ``prepare_workers=0`` on
    the loop's own thread between enqueueing the quantum and waiting for it.
    The device part of requests already prepared also runs during the
    quantum (the batch does it on its own admission stream); they join the
    next quantum.  Between quanta the loop admits again, after retiring the
    finished instances, whatever their memory now lets in.
    At most ``prepare_ahead`` requests are prepared and not yet admitted, which
    bounds the host memory they hold.  ``stats`` accumulates where the loop's
    time went."""

    def __init__(self, backend, *, min_quantum: int = 64, max_quantum: int = 1024,
                 clock: Callable[[], float] = time.perf_counter, sleep: Callable[[float], None] = time.sleep,
                 prepare_workers: int = 0, prepare_ahead: int = 8):
        self.backend = backend
        self.min_quantum = min_quantum
        self.max_quantum = max_quantum
        self.clock = clock
        self.sleep = sleep
        self.prepare_workers = prepare_workers
        self.prepare_ahead = max(1, prepare_ahead)
        self.stats: Dict[str, float] = {}

    def serve(self, requests: Sequence) -> List[Outcome]:
        pending = sorted(requests, key=lambda r: r.arrival)
        out = {r.index: Outcome(r.index, r.arrival, elements=r.problem.mesh.n_elements) for r in pending}
        waiting: List = []          # arrived, not admitted (arrival order)
        prep: Dict[int, object] = {}  # request index -> future / (token, error) of its host part
        running: Dict[int, tuple] = {}   # slot -> (request, cycles left estimate)
        st = dict(prepare_s=0.0, admit_s=0.0, run_s=0.0, wait_s=0.0, retire_s=0.0, idle_s=0.0, quanta=0,
                  cycles=0)
        self.stats = st
        be = self.backend
        pool = None
        if self.prepare_workers > 0:
            from concurrent.futures import ThreadPoolExecutor
            pool = ThreadPoolExecutor(self.prepare_workers)
        t0 = self.clock()
        now = lambda: self.clock() - t0  # noqa: E731

        def host_part(r):
            try:
                return be.prepare(r.problem), None
            except Exception as e:  # noqa: BLE001 - reported as the request's status
                return None, e

        def start_prepares():
            # the host part of the first prepare_ahead waiting requests
            for r in waiting[:self.prepare_ahead]:
                if r.index in prep:
                    continue
                if pool is not None:
                    prep[r.index] = pool.submit(host_part, r)
                else:
                    c = self.clock()
                    prep[r.index] = host_part(r)
                    st["prepare_s"] += self.clock() - c

        def prepared(r, block: bool):
            f = prep.get(r.index)
            if f is None:
                return None
            if pool is None:
                return f
            if not block and not f.done():
                return None
            return f.result()

        def fail(r, code: int):
            o = out[r.index]
            o.status = code
            o.finished = now()

        def intake():
            # arrivals so far join the waiting list
            t = now()
            while state["next"] < len(pending) and pending[state["next"]].arrival <= t:
                waiting.append(pending[state["next"]])
                state["next"] += 1

        def admit(block_first: bool, fresh: Optional[set] = None) -> List:
            # admit the prepared: first come, first served, with backfill;
            # returns the requests the batch refused
            nonlocal waiting
            c = self.clock()
            still, refused = [], []
            for i, r in enumerate(waiting):
                # with nothing on the device, wait for the first request's host part
                res = prepared(r, block=block_first and not running and i == 0)
                if res is None:
                    still.append(r)
                    continue
                token, err = res
                if err is not None:
                    del prep[r.index]
                    fail(r, getattr(err, "code", ERR_ARG))
                    continue
                try:
                    slot = be.add_prepared(token, r.problem)
                except AdmissionError:
                    still.append(r)
                    refused.append(r)
                    continue
                del prep[r.index]
                be.release(token)
                be.arm(slot, r.problem.cycles)
                running[slot] = (r, r.problem.cycles)
                if fresh is not None:
                    fresh.add(slot)
                out[r.index].admitted = now()
            waiting = still
            st["admit_s"] += self.clock() - c
            return refused

        state = {"next": 0}
        try:
            while state["next"] < len(pending) or waiting or running:
                t = now()
                nxt = state["next"]
                if not running and not waiting and nxt < len(pending) and pending[nxt].arrival > t:
                    c = self.clock()
                    self.sleep(pending[nxt].arrival - t)  # idle until the next arrival
                    st["idle_s"] += self.clock() - c
                intake()
                start_prepares()
                refused = admit(block_first=True)
                if not running:
                    # an empty batch that cannot take a request never will: reject it
                    for r in refused:
                        be.release(prepared(r, block=True)[0])
                        del prep[r.index]
                        fail(r, ERR_OOM)
                    waiting = [r for r in waiting if out[r.index].status == 0]
                    continue
                q = min(left for _, left in running.values())
                q = int(min(self.max_quantum, max(self.min_quantum, q)))
                c = self.clock()
                be.run(q)
                st["run_s"] += self.clock() - c
                st["quanta"] += 1
                st["cycles"] += q
                # while the quantum runs: host parts of the next arrivals, and
                # the device part of those already prepared (the backend puts
                # it beside the running cycles); they join the next quantum
                intake()
                start_prepares()
                fresh: set = set()
                admit(block_first=False, fresh=fresh)
                start_prepares()
                c = self.clock()
                be.sync()
                st["wait_s"] += self.clock() - c
                c = self.clock()
                for slot in list(running):
                    r, left = running[slot]
                    if slot in fresh:
                        continue  # added after the quantum was enqueued: it has not run yet
                    rep = be.report(slot)
                    if rep["done"] or rep["status"]:
                        o = out[r.index]
                        o.cycles = int(rep["cycles"])
                        o.status = int(rep["status"])
                        o.result = be.download(slot)
                        o.energy = be.energy(slot)
                        be.remove(slot)
                        o.finished = now()
                        del running[slot]
                    else:
                        running[slot] = (r, max(0, left - q))
                st["retire_s"] += self.clock() - c
        finally:
            for f in prep.values():
                res = f.result() if pool is not None else f
                if res[0] is not None:
                    be.release(res[0])
            if pool is not None:
                pool.shutdown()
        return [out[r.index] for r in pending]


def summarize(outcomes: Sequence[Outcome]) -> Dict[str, float]:
    """Solves/s over the stream (first arrival to last completion), latency
    percentiles and element-cycles/s."""
    lat = np.array([o.latency for o in outcomes])
    start = min(o.arrival for o in outcomes)
    end = max(o.finished for o in outcomes)
    span = end - start
    work = float(sum(o.elements * o.cycles for o in outcomes))
    return {
        "requests": len(outcomes),
        "makespan_s": span,
        "solves_per_s": len(outcomes) / span if span > 0 else math.inf,
        "p50_latency_s": float(np.percentile(lat, 50)),
        "p99_latency_s": float(np.percentile(lat, 99)),
        "mean_latency_s": float(lat.mean()),
        "element_cycles_per_s": work / span if span > 0 else math.inf,
        "failed": int(sum(1 for o in outcomes if o.status != 0)),
    }
