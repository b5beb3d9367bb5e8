"""Continuous-batching server of cavity solves on one GPU.

Requests (box cavity, order, final time, Gaussian pulse, 8 probes) arrive on a
stream.  The server admits them into a CavityPool as HBM budget and slots free up,
keeps their fields resident, advances every admitted cavity together (one launch
per N present per LSRK stage, all in one CUDA graph), and as each finishes returns
its probe traces and energy history and frees its memory.  Requests that arrive
while others are on the GPU join the running batch at the next step boundary.
Latency = completion time - arrival time.

Admission policy:
  "fifo"  arrival order, as many as the budget holds (every admitted cavity
          shares the GPU: processor sharing);
  "sjf"   shortest remaining work first among the waiting requests, and new
          admissions only while the resident cavities hold fewer than
          ``saturation_nodes`` nodes -- enough to keep HBM busy, so admitting more
          would only stretch every running request.  A request larger than that
          runs on its own, as in the serial path; small ones batch together.
  "hrrn"  as "sjf", but the waiting requests go in order of highest response ratio
          (waiting time + service time) / service time, the service time taken
          proportional to the request's work: short requests still go first
          while the queue is fresh, and a long one rises as it waits, so it is not
          starved by a stream of short ones (the tail latency "sjf" pays).
  "guard" as "hrrn", but a request that has waited longer than a guard goes first,
          oldest first, and the requests behind it wait until it fits under the
          node limit: a bound on how long a large request can be passed over, so
          that under overload the tail latency is no worse than first come, first
          served, while the short requests still batch ahead.  The guard is
          ``guard_s`` seconds, or by default ``guard_services`` times the mean
          estimated service time of the requests seen so far (their work at a
          rate of EST_BYTES_PER_S of HBM traffic), which scales with the stream.

The serial baseline serves the same stream one request at a time with the
single-mesh FP64 solver (DgSolver), the reference's execution model.
"""
from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np

from .pool import FINISHED, CavityPool, PoolFull
from .workloads import Cavity


@dataclass
class Result:
    request: int
    arrival: float
    admitted: float
    finished: float
    probes: np.ndarray       # [nsteps+1, 8, 6]
    energy: np.ndarray       # [nsteps+1] (NaN where not recorded)
    retired: float = 0.0     # when the server saw it finished and freed its slot
                             # (its results reach the host by `finished`)

    @property
    def latency(self):
        return self.finished - self.arrival


def hrrn_key(req: Cavity, t: float, time_scale: float = 1.0) -> float:
    """Sort key of the "hrrn" policy at time t: the response ratio (wait + service) /
    service, highest first, with the service time proportional to the request's
    DOF-stages (only the order matters, so 1 + wait / work, negated)."""
    wait = max(0.0, t - req.arrival * time_scale)
    return -(wait / max(req.dof_stages, 1.0))


class Server:
    def __init__(self, hbm_budget_bytes: int, max_slots: int = 512, precision: str = "fp32",
                 chunk: int | None = None, energy_every: int = 10, policy: str = "sjf",
                 saturation_nodes: int = 8 << 20, chunk_ms: float = 3.0,
                 guard_s: float | None = None, guard_services: float = 16.0):
        if policy not in ("fifo", "sjf", "hrrn", "guard"):
            raise ValueError("policy must be 'fifo', 'sjf', 'hrrn' or 'guard'")
        self.pool = CavityPool(hbm_budget_bytes, max_slots=max_slots, precision=precision)
        self.chunk = None if chunk is None else int(chunk)
        self.chunk_ms = float(chunk_ms)
        self.energy_every = int(energy_every)
        self.policy = policy
        self.saturation_nodes = int(saturation_nodes)
        self.guard_s = guard_s
        self.guard_services = float(guard_services)

    def close(self):
        self.pool.close()

    # HBM bytes one step moves per resident node (32 B per DOF-stage, 6 DOF, 5 stages)
    # and a conservative rate for them: the estimate only sizes the chunks
    STEP_BYTES_PER_NODE = 32 * 6 * 5
    EST_BYTES_PER_S = 3.5e12
    MIN_STEP_S = 25e-6   # five launches of a nearly empty step graph

    def chunk_steps(self, resident_nodes: int) -> int:
        """Steps queued per round: a fixed chunk when one was given, else enough
        steps for about chunk_ms of GPU work at the resident size (4..64), so that a
        round's host bookkeeping stays well below the GPU time it runs behind."""
        if self.chunk is not None:
            return self.chunk
        step_s = max(self.MIN_STEP_S, resident_nodes * self.STEP_BYTES_PER_NODE / self.EST_BYTES_PER_S)
        return int(min(64, max(4, round(self.chunk_ms * 1e-3 / step_s))))

    @classmethod
    def est_service_s(cls, req: Cavity) -> float:
        """Service time of a request estimated from its work alone."""
        return req.npts * req.nsteps * cls.STEP_BYTES_PER_NODE / cls.EST_BYTES_PER_S

    def order_pending(self, pending, requests, t, time_scale=1.0, mean_service_s=0.0):
        """The waiting requests (indices into requests) in admission order at time t."""
        if self.policy == "sjf":
            return sorted(pending, key=lambda i: requests[i].dof_stages)
        if self.policy in ("hrrn", "guard"):
            out = sorted(pending, key=lambda i: hrrn_key(requests[i], t, time_scale))
            if self.policy == "guard":
                g = self.guard_s if self.guard_s is not None else self.guard_services * mean_service_s
                waited = lambda i: t - requests[i].arrival * time_scale
                old = sorted((i for i in out if waited(i) > g), key=lambda i: requests[i].arrival)
                if old:
                    olds = set(old)
                    out = old + [i for i in out if i not in olds]
            return out
        return list(pending)  # fifo: arrival order

    def admit(self, req: Cavity):
        s = self.pool.add_box(req.N, req.nel, req.lo, req.hi, req.c0, req.dt, req.nsteps,
                              periodic=req.periodic, probes=req.probes,
                              energy_every=self.energy_every)
        self.pool.init_pulse(s, req.pulses)
        return s

    def run(self, requests, time_scale: float = 1.0, log=None):
        """Serve the stream in real time (arrivals replayed at time_scale x the
        request timestamps).  Returns the results in request order and the
        wall time of the whole run.

        The host never waits for the GPU to drain: each round queues the next
        chunk of steps first and only then waits for the status snapshot queued
        after the previous chunk (nwb_pool_query_begin/end), so the GPU works
        on the new chunk while the host retires finished requests (their
        results copied asynchronously, complete by the next snapshot) and
        admits new ones (queued behind the running chunk)."""
        pending = []
        arrivals = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
        nxt = 0
        running = {}            # slot -> (request index, admit time)
        fetching = {}           # request index -> (admit time, result buffers in flight)
        snapshot = False        # a status snapshot is queued
        results = [None] * len(requests)
        seen_s, seen_n = 0.0, 0  # estimated service of the requests arrived so far
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0
        while nxt < len(arrivals) or pending or running or fetching:
            t = now()
            while nxt < len(arrivals) and requests[arrivals[nxt]].arrival * time_scale <= t:
                pending.append(arrivals[nxt])
                seen_s += self.est_service_s(requests[arrivals[nxt]])
                seen_n += 1
                nxt += 1
            if pending:
                pending = self.order_pending(pending, requests, t, time_scale,
                                             seen_s / max(seen_n, 1))
            resident = sum(requests[i].npts for i, _ in running.values())
            while pending:
                i = pending[0]
                if (self.policy != "fifo" and running and
                        resident + requests[i].npts > self.saturation_nodes):
                    break
                try:
                    s = self.admit(requests[i])
                except PoolFull:
                    break
                pending.pop(0)
                running[s] = (i, now())
                resident += requests[i].npts
            if not running and not snapshot:
                if nxt < len(arrivals):          # idle until the next arrival
                    wait = requests[arrivals[nxt]].arrival * time_scale - now()
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            if running:
                self.pool.step(self.chunk_steps(resident))
            if snapshot:
                status, _ = self.pool.query_end()
                # result copies queued before that snapshot have landed
                for i, (ta, tr, r) in fetching.items():
                    results[i] = Result(i, requests[i].arrival * time_scale, ta, now(), r["probes"],
                                        r["energy"], retired=tr)
                    if log:
                        log(results[i])
                fetching = {}
                for s in [s for s in running if status[s] == FINISHED]:
                    i, ta = running.pop(s)
                    fetching[i] = (ta, now(), self.pool.results_async(s))
                    self.pool.remove(s)
            snapshot = bool(running or fetching)
            if snapshot:
                self.pool.query_begin()
        return results, now()


def serve_serial(requests, precision="fp64", time_scale: float = 1.0, energy_every: int = 10):
    """The same stream served one request at a time with the single-mesh solver,
    the reference's execution model (Case::simulate, src/case.cpp:562-655: one
    solve per process, a step at a time, probes recorded after every step and the
    energy every output step).  Box solver built per request, device initial
    state; the probes (ProbeManager::record) and the energy are evaluated on the
    device and only their values are read back, which spares it the reference's
    full per-step download."""
    order = sorted(range(len(requests)), key=lambda i: requests[i].arrival)
    results = [None] * len(requests)
    t0 = time.perf_counter()
    for i in order:
        req = requests[i]
        wait = req.arrival * time_scale - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ta = time.perf_counter() - t0
        probes, energy = solve_one(req, precision, energy_every)
        tf = time.perf_counter() - t0
        results[i] = Result(i, req.arrival * time_scale, ta, tf, probes, energy, retired=tf)
    return results, time.perf_counter() - t0


def solve_one(req: Cavity, precision: str = "fp64", energy_every: int = 10):
    """One request alone on the single-mesh solver, as serve_serial runs it: a
    step at a time, the 8 probes read after every step, the energy every
    energy_every steps and at the end.  Returns (probes, energy)."""
    from . import DgSolver
    from .pool import box_probes
    s = DgSolver(precision)
    s.initializeBox(req.N, req.nel, req.lo, req.hi, req.c0, periodic=req.periodic)
    s.initPulse(req.pulses)
    np_ = len(req.probes)
    if np_:
        off, w = box_probes(req.N, req.nel, req.lo, req.hi, req.probes)
        s.probeSetup(off, w)
    probes = np.zeros((req.nsteps + 1, np_, 6))
    energy = np.full(req.nsteps + 1, np.nan)
    energy[0] = s.energy()
    if np_:
        probes[0] = s.probeRead()
    for n in range(1, req.nsteps + 1):
        s.step(req.dt, 0.0)
        if np_:
            probes[n] = s.probeRead()
        if n % energy_every == 0 or n == req.nsteps:
            energy[n] = s.energy()
    s.finalize()
    return probes, energy


def serial_service_times(requests, precision: str = "fp64", energy_every: int = 10):
    """Service time of every request on the serial path (solve_one), the requests
    run back to back in list order with nothing else on the GPU."""
    out = []
    for req in requests:
        t = time.perf_counter()
        solve_one(req, precision, energy_every)
        out.append(time.perf_counter() - t)
    return np.asarray(out)


def fifo_finish_times(arrivals, service):
    """Finish times of a server that takes one request at a time in arrival order
    (the serial path): finish_i = max(arrival_i, finish_{i-1}) + service_i.  Given
    each request's service time this is the serial server's schedule exactly, for
    any arrival times, since its service does not depend on the queue."""
    arrivals = np.asarray(arrivals, float)
    service = np.asarray(service, float)
    order = np.argsort(arrivals, kind="stable")
    fin = np.empty_like(arrivals)
    t = 0.0
    for i in order:
        t = max(t, arrivals[i]) + service[i]
        fin[i] = t
    return fin


def latency_stats(results):
    lat = np.array([r.latency for r in results if r is not None])
    return latency_summary(lat)


def latency_summary(lat):
    lat = np.asarray(lat, float)
    return dict(n=int(lat.size), p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                mean=float(lat.mean()), max=float(lat.max()))
