"""Admission logic of the serving loop (nekwave_b200/serving.py) on the CPU: the
server runs against a stand-in for CavityPool that advances each resident cavity by
the requested number of steps and charges each its three state arrays against the
budget, so the policies can be checked without a GPU."""
import numpy as np
import pytest

from nekwave_b200 import serving
from nekwave_b200.pool import FINISHED, FREE, RUNNING
from nekwave_b200.workloads import Cavity

BYTES_PER_NODE = 3 * 6 * 8  # u[2] and k, six FP64 components


class FakePool:
    """The CavityPool calls the server makes, with a log of every admission."""

    def __init__(self, budget, max_slots=512, precision="fp64"):
        self.budget, self.max_slots = budget, max_slots
        self.slots = {}     # slot -> [npts, nsteps, done]
        self.log = []       # (request npts, nsteps, resident nodes after, cavities running before)
        self.max_resident = 0

    def resident(self):
        return sum(v[0] for v in self.slots.values())

    def add_box(self, N, nel, lo, hi, c0, dt, nsteps, periodic=(False,) * 3, probes=None,
                energy_every=0):
        npts = nel[0] * nel[1] * nel[2] * N ** 3
        free = [s for s in range(self.max_slots) if s not in self.slots]
        if not free or (self.resident() + npts) * BYTES_PER_NODE > self.budget:
            raise serving.PoolFull("over budget")
        running_before = len(self.slots)
        self.slots[free[0]] = [npts, nsteps, 0]
        self.log.append((npts, nsteps, self.resident(), running_before))
        self.max_resident = max(self.max_resident, self.resident())
        return free[0]

    def init_pulse(self, slot, pulses):
        assert slot in self.slots

    def step(self, nsteps=1):
        for v in self.slots.values():
            v[2] = min(v[1], v[2] + nsteps)

    def query(self):
        status = np.full(self.max_slots, FREE, dtype=np.int32)
        done = np.zeros(self.max_slots, dtype=np.int32)
        for s, (_, nsteps, d) in self.slots.items():
            status[s] = FINISHED if d >= nsteps else RUNNING
            done[s] = d
        return status, done

    def query_begin(self):
        # the snapshot reflects every step queued so far (the stand-in steps at once)
        self._snap = self.query()

    def query_end(self):
        snap, self._snap = self._snap, None
        assert snap is not None, "query_end without query_begin"
        return snap

    def results(self, slot, state=True, energy=True, probes=True):
        nsteps = self.slots[slot][1]
        return {"probes": np.zeros((nsteps + 1, 8, 6)), "energy": np.zeros(nsteps + 1)}

    def results_async(self, slot):
        assert self.slots[slot][2] >= self.slots[slot][1], "results of an unfinished cavity"
        return self.results(slot)

    def remove(self, slot):
        del self.slots[slot]

    def close(self):
        pass


def requests(sizes):
    """Cavities of (N, elements per direction, steps), arriving in list order."""
    out = []
    for i, (N, n, steps) in enumerate(sizes):
        out.append(Cavity(N, (n, n, n), (0, 0, 0), (1, 1, 1), 1.0, steps, 1e-3,
                          [(0.0, 0, 0, 0, 0.0)] * 6, arrival=1e-6 * i))
    return out


SIZES = [(8, 6, 40), (4, 2, 10), (9, 8, 30), (5, 3, 200), (6, 4, 5), (7, 5, 60), (4, 3, 100),
         (8, 2, 7)]


@pytest.fixture
def fake(monkeypatch):
    made = []

    def make(*a, **k):
        made.append(FakePool(*a, **k))
        return made[-1]

    monkeypatch.setattr(serving, "CavityPool", make)
    return made


def run(policy, reqs, budget=1 << 40, saturation=1 << 40, chunk=4):
    srv = serving.Server(budget, max_slots=16, precision="fp64", chunk=chunk, policy=policy,
                         saturation_nodes=saturation)
    results, _ = srv.run(reqs, time_scale=0.0)
    srv.close()
    return results


@pytest.mark.parametrize("policy", ["fifo", "sjf", "hrrn"])
def test_every_request_completes_with_its_histories(fake, policy):
    reqs = requests(SIZES)
    results = run(policy, reqs)
    for i, r in enumerate(results):
        assert r is not None and r.request == i
        assert r.finished >= r.admitted >= 0.0 and r.latency >= 0.0
        assert r.energy.shape == (reqs[i].nsteps + 1,) and r.probes.shape == (reqs[i].nsteps + 1, 8, 6)
    assert not fake[0].slots  # every finished cavity was removed


def test_fifo_admits_in_arrival_order(fake):
    reqs = requests(SIZES)
    run("fifo", reqs)
    assert [(n, s) for n, s, _, _ in fake[0].log] == [(r.npts, r.nsteps) for r in reqs]


def test_sjf_admits_shortest_work_first(fake):
    reqs = requests(SIZES)
    run("sjf", reqs)
    order = sorted(reqs, key=lambda r: r.dof_stages)
    assert [(n, s) for n, s, _, _ in fake[0].log] == [(r.npts, r.nsteps) for r in order]


def test_sjf_keeps_resident_nodes_under_saturation(fake):
    reqs = requests(SIZES)
    sat = 300_000
    results = run("sjf", reqs, saturation=sat)
    assert all(r is not None for r in results)
    for npts, _, resident, running_before in fake[0].log:
        # over the limit only when it runs alone (a request larger than the limit)
        assert resident <= sat or running_before == 0


def test_full_pool_defers_admission(fake):
    reqs = requests(SIZES)
    largest = max(r.npts for r in reqs)
    budget = (largest + 10_000) * BYTES_PER_NODE  # the largest cavity fits, with little room
    results = run("fifo", reqs, budget=budget)
    assert all(r is not None for r in results)
    assert fake[0].max_resident * BYTES_PER_NODE <= budget


def test_hrrn_orders_by_response_ratio():
    """A long request that has waited rises above short ones that have not; among
    requests that waited alike, shorter work goes first (as in sjf)."""
    big, small, mid = requests([(6, 4, 40), (4, 2, 10), (6, 4, 20)])  # work 110 : 1 : 55
    big.arrival, small.arrival, mid.arrival = 0.0, 9.99, 9.99
    order = sorted([small, big, mid], key=lambda r: serving.hrrn_key(r, 10.0))
    # the long one waited 1000x longer for 110x the work: its ratio is the highest
    assert order == [big, small, mid]
    early = sorted([small, big, mid], key=lambda r: serving.hrrn_key(r, 9.99 + 1e-12))
    assert early[0] is big  # the others have hardly waited
    fresh = sorted([big, mid, small], key=lambda r: serving.hrrn_key(r, 20.0, time_scale=0.0))
    assert fresh == [small, mid, big]  # equal waits: shortest work first


def test_hrrn_keeps_resident_nodes_under_saturation(fake):
    reqs = requests(SIZES)
    sat = 300_000
    results = run("hrrn", reqs, saturation=sat)
    assert all(r is not None for r in results)
    for npts, _, resident, running_before in fake[0].log:
        assert resident <= sat or running_before == 0


def test_fifo_finish_times_match_a_one_at_a_time_simulation():
    """The serial path's schedule from service times equals a step-by-step simulation
    of a server that takes one request at a time in arrival order."""
    r = np.random.Generator(np.random.PCG64(5))
    for rate in (0.25, 1.0, 4.0):
        arr = np.cumsum(r.exponential(1.0 / rate, 200))
        svc = r.exponential(1.0, 200)
        perm = r.permutation(200)             # requests need not be listed in arrival order
        fin = serving.fifo_finish_times(arr[perm], svc[perm])
        clock, want = 0.0, np.empty(200)
        for i in range(200):                  # arr is sorted: serve in index order
            start = arr[i] if arr[i] > clock else clock
            clock = start + svc[i]
            want[i] = clock
        assert np.array_equal(fin, want[perm])
        lat = fin - arr[perm]
        assert (lat >= svc[perm] - 1e-12).all()
    st = serving.latency_summary([1.0, 2.0, 3.0])
    assert st["p50"] == 2.0 and st["max"] == 3.0 and st["n"] == 3


def test_serving_requests_final_time_scale():
    """t_scale shortens the final times only: sizes, orders, pulses, probes and
    arrivals are those of the unscaled stream."""
    from nekwave_b200.workloads import serving_requests
    a = serving_requests(20, 1.0, seed=3)
    b = serving_requests(20, 1.0, seed=3, t_scale=0.125)
    for x, y in zip(a, b):
        assert (x.N, x.nel, x.lo, x.hi, x.arrival) == (y.N, y.nel, y.lo, y.hi, y.arrival)
        assert x.pulses == y.pulses and x.probes == y.probes
        assert abs(y.T - 0.125 * x.T) < 1e-15 * x.T
        assert y.nsteps <= x.nsteps and abs(y.dt * y.nsteps - y.T) < 1e-12


def test_adaptive_chunk_follows_the_resident_size(monkeypatch):
    """Without a fixed chunk the server queues about chunk_ms of GPU work per round:
    many steps while few nodes are resident, four once a step alone takes longer."""
    monkeypatch.setattr(serving, "CavityPool", FakePool)
    srv = serving.Server(1 << 40, max_slots=16, precision="fp64", policy="fifo")
    small, mid, big = srv.chunk_steps(1000), srv.chunk_steps(1 << 20), srv.chunk_steps(64 << 20)
    assert small == 64 and big == 4 and 4 <= mid <= 64 and small >= mid >= big
    fixed = serving.Server(1 << 40, max_slots=16, precision="fp64", chunk=7)
    assert fixed.chunk_steps(1000) == 7 and fixed.chunk_steps(64 << 20) == 7


def test_guard_puts_requests_past_the_guard_first_oldest_first(monkeypatch):
    """The "guard" policy orders as "hrrn" until a request has waited longer than the
    guard; then the requests past it go first in arrival order."""
    monkeypatch.setattr(serving, "CavityPool", FakePool)
    big1, big2, small, mid = requests([(6, 4, 400), (6, 4, 300), (4, 2, 10), (6, 4, 20)])
    big1.arrival, big2.arrival, small.arrival, mid.arrival = 0.0, 1.0, 9.0, 9.5
    reqs = [big1, big2, small, mid]
    srv = serving.Server(1 << 40, max_slots=16, precision="fp64", policy="guard", guard_s=8.5)
    hr = serving.Server(1 << 40, max_slots=16, precision="fp64", policy="hrrn")
    pend = [2, 3, 1, 0]
    # at t = 9.6 both large requests have waited past 8.5 s: oldest first, then hrrn
    assert srv.order_pending(pend, reqs, 9.6) == [0, 1, 2, 3]
    # at t = 9.2 only the first has
    assert srv.order_pending(pend, reqs, 9.2)[0] == 0
    assert srv.order_pending(pend, reqs, 9.2)[1:] == [i for i in hr.order_pending(pend, reqs, 9.2) if i != 0]
    # no request past the guard: the hrrn order itself
    early = serving.Server(1 << 40, max_slots=16, precision="fp64", policy="guard", guard_s=100.0)
    assert early.order_pending(pend, reqs, 9.6) == hr.order_pending(pend, reqs, 9.6)
    # default guard: guard_services x the mean estimated service time given
    auto = serving.Server(1 << 40, max_slots=16, precision="fp64", policy="guard", guard_services=2.0)
    assert auto.order_pending(pend, reqs, 9.6, mean_service_s=4.0)[:2] == [0, 1]   # guard 8 s
    assert auto.order_pending(pend, reqs, 9.6, mean_service_s=4.5)[0] == 0        # guard 9 s
    assert auto.order_pending(pend, reqs, 9.6, mean_service_s=5.0) == hr.order_pending(pend, reqs, 9.6)


def test_guard_completes_every_request_under_the_node_limit(fake):
    reqs = requests(SIZES)
    sat = 300_000
    srv = serving.Server(1 << 40, max_slots=16, precision="fp64", chunk=4, policy="guard",
                         saturation_nodes=sat, guard_s=0.0)
    results, _ = srv.run(reqs, time_scale=0.0)
    srv.close()
    assert all(r is not None for r in results)
    for npts, _, resident, running_before in fake[0].log:
        assert resident <= sat or running_before == 0
    # a zero guard admits in arrival order: first come, first served
    assert [x[0] for x in fake[0].log] == [r.npts for r in reqs]
