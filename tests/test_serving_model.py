"""The serving loop's admission policies on a model of the pool, on the CPU.

The real Server (nekwave_b200/serving.py) runs against a stand-in pool on a virtual
clock: a pool step advances every resident cavity by one step and takes
max(floor, resident nodes / rate) seconds (the per-N stage kernels are HBM-bound and
run one after another, so a step costs the resident nodes' traffic).  The serial
path is a server that takes one request at a time in arrival order, with each
request's service time from the same rate at a lower efficiency plus a per-step
host round trip (its probes are read after every step).  Rates are calibrated on
the B200 measurements of the sweep (the pool's 125 GDOF-stage/s, the serial path's
117).  The model decides nothing at run time; it shows why the "guard" policy is
the recommended one: under overload "hrrn" passes the largest requests over until
the stream ends and its p99 can exceed first come, first served, while "guard"
bounds that wait."""
import numpy as np
import pytest

from nekwave_b200 import serving
from nekwave_b200.pool import FINISHED, FREE, RUNNING
from nekwave_b200.workloads import serving_requests

NODE_STEPS_PER_S = 125e9 / 30   # pool: 125 GDOF-stage/s = 4.17e9 node-steps/s
STEP_FLOOR_S = 1.2e-4           # a nearly empty step graph (every N present, 5 stages)
SERIAL_EFF = 117.0 / 125.0      # serial path's rate relative to the pool's
SERIAL_STEP_S = 5e-5            # per step: launch, probe read and its host round trip
SERIAL_SETUP_S = 0.01           # per request: solver creation and initial state


class Clock:
    def __init__(self):
        self.t = 0.0

    def perf_counter(self):
        return self.t

    def sleep(self, s):
        self.t += max(0.0, s)


class TimedPool:
    """CavityPool stand-in whose steps take model time on the virtual clock."""

    def __init__(self, clock, budget, max_slots=512, precision="fp64"):
        self.clock, self.max_slots = clock, max_slots
        self.slots = {}    # slot -> [npts, nsteps, done]

    def add_box(self, N, nel, lo, hi, c0, dt, nsteps, periodic=(False,) * 3, probes=None,
                energy_every=0):
        free = [s for s in range(self.max_slots) if s not in self.slots]
        if not free:
            raise serving.PoolFull("no slot")
        self.slots[free[0]] = [nel[0] * nel[1] * nel[2] * N ** 3, nsteps, 0]
        return free[0]

    def init_pulse(self, slot, pulses):
        pass

    def step(self, nsteps=1):
        for _ in range(nsteps):
            live = [v for v in self.slots.values() if v[2] < v[1]]
            if not live:
                return
            nodes = sum(v[0] for v in live)
            self.clock.t += max(STEP_FLOOR_S, nodes / NODE_STEPS_PER_S)
            for v in live:
                v[2] += 1

    def query_begin(self):
        status = np.full(self.max_slots, FREE, dtype=np.int32)
        done = np.zeros(self.max_slots, dtype=np.int32)
        for s, (_, nsteps, d) in self.slots.items():
            status[s] = FINISHED if d >= nsteps else RUNNING
            done[s] = d
        self._snap = (status, done)

    def query_end(self):
        return self._snap

    def results_async(self, slot):
        return {"probes": None, "energy": None}

    def remove(self, slot):
        del self.slots[slot]

    def close(self):
        pass


def serial_service(r):
    return (r.npts * r.nsteps / (NODE_STEPS_PER_S * SERIAL_EFF) + r.nsteps * SERIAL_STEP_S
            + SERIAL_SETUP_S)


def run_model(monkeypatch, policy, seed, mult, n=100):
    clock = Clock()
    monkeypatch.setattr(serving.time, "perf_counter", clock.perf_counter)
    monkeypatch.setattr(serving.time, "sleep", clock.sleep)
    monkeypatch.setattr(serving, "CavityPool", lambda *a, **k: TimedPool(clock, *a, **k))
    base = serving_requests(n, 1.0, seed=seed, t_scale=0.125)
    svc = np.array([serial_service(r) for r in base])
    mu = n / svc.sum()
    for r in base:
        r.arrival = r.arrival / (mult * mu)
    arr = np.array([r.arrival for r in base])
    fin = serving.fifo_finish_times(arr, svc)
    serial = serving.latency_summary(fin - arr)
    srv = serving.Server(1 << 50, max_slots=512, precision="fp64", policy=policy)
    res, wall = srv.run(base)
    srv.close()
    pool = serving.latency_stats(res)
    return pool, serial, n / wall, n / fin.max()


@pytest.mark.parametrize("seed", [100, 101, 102, 103, 104])
def test_guard_keeps_p99_under_serial_fifo_at_and_above_capacity(monkeypatch, seed):
    for mult in (1.0, 2.0, 4.0):
        pool, serial, pool_rate, serial_rate = run_model(monkeypatch, "guard", seed, mult)
        assert pool_rate >= serial_rate, (mult, pool_rate, serial_rate)
        assert pool["p99"] < serial["p99"], (mult, pool["p99"], serial["p99"])
        assert pool["p50"] < serial["p50"], (mult, pool["p50"], serial["p50"])


def test_hrrn_tail_exceeds_serial_fifo_under_overload(monkeypatch):
    """The case the guard exists for (seed 100, twice the serial capacity)."""
    pool, serial, _, _ = run_model(monkeypatch, "hrrn", 100, 2.0)
    guard, _, _, _ = run_model(monkeypatch, "guard", 100, 2.0)
    assert pool["p99"] > serial["p99"] > guard["p99"]
    assert pool["p50"] < guard["p50"] < serial["p50"]
