"""Serving floe-indentation scenarios with continuous batching on one GPU.

Requests arrive over time (e.g. a Poisson process); each asks for a scenario
(SimParams + initial HSSOA) to be advanced by a number of sub-steps.  The
server keeps every admitted scenario's state resident on the device as a
member of one Batch, advances all members together in rounds of
`round_steps` sub-steps, and between rounds:
  * takes out the members that have done their steps (their results are
    copied to the host on a side stream while the next round runs),
  * admits waiting requests, first come first served, while their device
    memory fits the budget and a slot is free (their upload and binning run
    on the side stream too, and the next round waits for them).
The host queues round k + 1 while round k runs and waits only for round k - 1,
so the device does not idle between rounds.  Requests that arrive while
others run join the running batch as memory frees up, and their work
overlaps on the device.  Completion latency is measured from arrival to the
moment the host holds the result.

A request can be cancelled (dropped from the queue or the batch) or evicted:
its state, simulation time, step index and force bins are downloaded, its
device memory is freed and it goes back to the head of the queue, to resume
where it stopped when memory allows.

This is host-side scheduling over the icy_batch_* C-ABI; the reference has
no counterpart (it runs one scenario per process).
"""
import collections
import dataclasses
import time

import numpy as np

from .batch import Batch, device_bytes
from .hssoa import HostSideSOA


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float              # seconds after the start of the run
    params: object              # SimParams (None until `make` has built the scenario)
    soa: HostSideSOA            # initial state (released once its upload is done)
    steps: int                  # sub-steps to run (a multiple of the round length)
    make: object = None         # () -> (params, soa): builds the scenario when it reaches the queue head
    slot: int = -1
    admitted: float = None
    done: float = None
    steps_done: int = 0
    bytes: int = 0
    result: HostSideSOA = None
    sim_time: float = None
    bins: np.ndarray = None
    cancelled: bool = False
    evictions: int = 0
    resume_time: float = 0.0     # simulation time / step index to resume from after an eviction
    resume_step: int = 0
    bins_before: np.ndarray = None
    npts: int = 0                # points and HSSOA capacity of the scenario (kept after release)
    capacity: int = 0
    upload_round: int = -1       # the round queued after the upload: the buffer is free once it is done

    def ensure(self):
        """Build the scenario now if it was deferred; returns (params, soa)."""
        if self.soa is None and self.make is not None:
            self.params, self.soa = self.make()
            self.make = None
        if self.soa is not None:
            self.npts, self.capacity = self.soa.size, self.soa.capacity
        return self.params, self.soa

    @property
    def points(self):
        return self.npts


class Server:
    """Continuous batching of requests on one device under a memory budget.

    max_instances bounds the requests resident at once; a batch of at most
    300 slots keeps its members' kernel arguments in the constant bank
    (faster steps)."""

    def __init__(self, budget_bytes=150e9, max_instances=128, round_steps=50, device=0, keep_results=True,
                 keep_inputs=True, reserve_bytes=None):
        self.batch = Batch(max_instances, device=device)
        # device memory for the admitted requests, mapped up front (up to 24 GB by
        # default): an admission then takes its buffers from memory the pool holds
        if reserve_bytes is None:
            reserve_bytes = min(float(budget_bytes), 24e9)
        if reserve_bytes > 0:
            self.batch.reserve(reserve_bytes)
        self.keep_inputs = keep_inputs   # False: release each request's initial state once uploaded
        self.budget = float(budget_bytes)
        self.round_steps = int(round_steps)
        self.max_instances = int(max_instances)
        self.keep_results = keep_results
        self.used = 0.0
        self.running = {}
        self.retired = []        # [(slot, request, buffer)] taken out, results being copied: slots still held
        self.queue = collections.deque()
        self.completed = []
        self.cancelled = []
        self.rounds = 0
        self.peak_live = 0
        self.peak_bytes = 0.0
        self._scratch = {}      # free page-locked download buffers by capacity, when results are not kept
        # uploaded inputs released while rounds are in flight: freeing page-locked
        # memory synchronises the device, so they are freed when it is idle
        self._released = []

    def close(self):
        self.batch.close()

    def _admit(self, now):
        # a retired member's slot stays taken until its results are collected
        while self.queue and len(self.running) + len(self.retired) < self.max_instances:
            r = self.queue[0]
            r.ensure()
            need = device_bytes(r.params, r.capacity)
            if need > self.budget:   # larger than the whole budget: refuse instead of waiting forever
                raise RuntimeError(f"request {r.rid} needs {need} bytes, budget {self.budget}")
            if self.used + need > self.budget:
                break
            self.queue.popleft()
            r.slot = self.batch.add_async(r.params, r.soa)
            r.upload_round = self.rounds + 1
            if r.evictions:
                self.batch.set_clock(r.slot, r.resume_time, r.resume_step)
            r.bytes = need
            if r.admitted is None:
                r.admitted = now
            self.used += need
            self.running[r.slot] = r
        self.peak_live = max(self.peak_live, len(self.running))
        self.peak_bytes = max(self.peak_bytes, self.used)

    def _out_buffer(self, capacity):
        """Result buffer: a new one when results are kept, else a page-locked one
        from the free list (returned by _release)."""
        if self.keep_results:
            return HostSideSOA(capacity)
        cap = 1 << max(int(capacity) - 1, 1).bit_length()
        free = self._scratch.setdefault(cap, [])
        return free.pop() if free else HostSideSOA(cap, pinned=True)

    def _release(self, buf):
        if not self.keep_results:
            self._scratch.setdefault(buf.capacity, []).append(buf)

    def _retire_finished(self):
        """Members whose steps are all queued leave the batch; their results
        are copied after the queued rounds.  Returns [(slot, request, buffer)]."""
        out = []
        for slot, r in list(self.running.items()):
            if r.steps_done >= r.steps:
                buf = self._out_buffer(r.capacity)
                self.batch.retire(slot, buf)
                del self.running[slot]
                out.append((slot, r, buf))
        return out

    def _collect(self, retired, t0):
        for slot, r, buf in retired:
            r.sim_time, _, r.bins = self.batch.collect(slot, wait=True)
            if r.bins_before is not None:
                r.bins = r.bins + r.bins_before
            r.done = time.perf_counter() - t0
            if self.keep_results:
                r.result = buf
            else:
                self._release(buf)
            self.used -= r.bytes
            self.completed.append(r)

    def _running(self, rid):
        for slot, r in self.running.items():
            if r.rid == rid:
                return slot, r
        return None, None

    def cancel(self, rid):
        """Drop request rid, queued or running; returns whether it was found."""
        for r in list(self.queue):
            if r.rid == rid:
                self.queue.remove(r)
                r.cancelled = True
                self.cancelled.append(r)
                return True
        slot, r = self._running(rid)
        if r is None:
            return False
        self.batch.remove(slot)
        self.used -= r.bytes
        del self.running[slot]
        r.cancelled = True
        self.cancelled.append(r)
        return True

    def evict(self, rid):
        """Move running request rid off the device (state kept on the host) and
        put it at the head of the queue; returns whether it was running."""
        slot, r = self._running(rid)
        if r is None:
            return False
        state = HostSideSOA(r.capacity)
        r.resume_time, r.resume_step, bins = self.batch.download(slot, state)
        r.bins_before = bins if r.bins_before is None else r.bins_before + bins
        self.batch.remove(slot)
        self.used -= r.bytes
        del self.running[slot]
        r.soa = state
        r.evictions += 1
        self.queue.appendleft(r)
        return True

    def run(self, requests, on_round=None):
        """Serve `requests` (arrival times relative to now); returns stats.
        on_round(server, round_index) is called after every round is queued."""
        pending = sorted(requests, key=lambda r: r.arrival)
        pi = 0
        work = 0.0
        sat = []                # (time, work) of the rounds queued while requests waited for admission
        t0 = time.perf_counter()
        while pi < len(pending) or self.queue or self.running or self.retired:
            now = time.perf_counter() - t0
            while pi < len(pending) and pending[pi].arrival <= now:
                self.queue.append(pending[pi])
                pi += 1
            self._admit(now)
            stepped = False
            if self.running:
                self.batch.step(self.round_steps)
                stepped = True
                self.rounds += 1
                rw = 0.0
                for r in self.running.values():
                    r.steps_done += self.round_steps
                    rw += r.points * self.round_steps
                work += rw
                if self.queue:
                    sat.append((time.perf_counter() - t0, rw))
            finished = self._retire_finished()
            # at most this round in flight; the previous round's results are copied by now
            self.batch.wait_steps(1)
            self._collect(self.retired, t0)
            # the rounds before this one are done: uploads queued before them no longer
            # read their host buffers
            if not self.keep_inputs:
                for r in self.running.values():
                    if r.soa is not None and 0 <= r.upload_round < self.rounds:
                        self._released.append(r.soa)
                        r.soa = None
            self.retired = finished
            if stepped and on_round is not None:
                on_round(self, self.rounds)
            if not self.running and not self.retired and not self.queue:
                self._released.clear()   # nothing in flight: freeing costs no stall
                if pi < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[pi].arrival - (time.perf_counter() - t0))))
        self.batch.wait_steps(0)
        makespan = time.perf_counter() - t0
        self._released.clear()
        lat = np.array([r.done - r.arrival for r in self.completed]) if self.completed else np.zeros(1)
        # the device's rate while the server was saturated (requests waiting): the
        # rounds queued then, over the time between the first and the last (the host
        # queues a round only when the one before the last has finished)
        sat_s = sat[-1][0] - sat[0][0] if len(sat) > 2 else 0.0
        sat_rate = sum(w for _, w in sat[1:]) / sat_s if sat_s > 0 else None
        return {
            "requests": len(self.completed),
            "budget_bytes": self.budget,
            "peak_budget_fraction": self.peak_bytes / self.budget if self.budget > 0 else None,
            "cancelled": len(self.cancelled),
            "evictions": sum(r.evictions for r in self.completed),
            "makespan_s": makespan,
            "particle_steps": work,
            "particle_steps_per_s": work / makespan if makespan > 0 else 0.0,
            "saturated_particle_steps_per_s": sat_rate,
            "saturated_s": sat_s,
            "latency_p50_s": float(np.percentile(lat, 50)),
            "latency_p99_s": float(np.percentile(lat, 99)),
            "latency_mean_s": float(lat.mean()),
            "rounds": self.rounds,
            "peak_live": self.peak_live,
            "peak_device_bytes": self.peak_bytes,
        }


def poisson_requests(scenes, rate, n, steps_range=(200, 5000), round_steps=50, seed=11):
    """n requests at Poisson arrival `rate` (per second); each takes a scene
    (params, soa) from `scenes` in turn and a step count uniform in
    steps_range, rounded to a multiple of round_steps."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = steps_range
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        p, soa = scenes[k % len(scenes)]
        steps = int(rng.integers(lo // round_steps, hi // round_steps + 1)) * round_steps
        r = Request(rid=k, arrival=t, params=p.copy(), soa=soa, steps=max(steps, round_steps))
        r.ensure()
        out.append(r)
    return out


def seeded_requests(rate, n, points_range=(5_000, 2_000_000), steps_range=(200, 5000), round_steps=50, seed=11,
                    pinned=True):
    """n requests at Poisson arrival `rate` (per second), each its own seeded
    floe-indentation scenario: points log-uniform in points_range, E uniform
    5e8-2e9 Pa, friction angle uniform 45-70 deg, indenter 0.5-3 m/s, a step
    count uniform in steps_range rounded to a multiple of round_steps.  The
    scenario (parameters and initial points) is built when the request
    reaches the head of the queue, so the host holds only the ones waiting
    for admission or being uploaded."""
    from .workloads import floe_scenario, make_workload
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    lo, hi = steps_range
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        npts = int(round(np.exp(rng.uniform(np.log(points_range[0]), np.log(points_range[1])))))
        w = floe_scenario(npts, E=float(rng.uniform(5e8, 2e9)), phi=float(rng.uniform(45, 70)),
                          v_ind=float(rng.uniform(0.5, 3.0)), seed=seed * 100000 + k)
        steps = int(rng.integers(lo // round_steps, hi // round_steps + 1)) * round_steps
        out.append(Request(rid=k, arrival=t, params=None, soa=None, steps=max(steps, round_steps),
                           make=lambda w=w: make_workload(w, pinned=pinned)))
    return out
