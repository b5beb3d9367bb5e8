"""Serving: continuous batching of a request stream.  Each request's probe traces
and energy history must be the same served alone and served in the mix; the box
solver path must equal the mesh path."""
import numpy as np
import pytest

from nekwave_b200 import DgSolver, Mesh
from nekwave_b200.serving import Server, latency_stats, serve_serial
from nekwave_b200.workloads import cavity_state, serving_requests

pytestmark = pytest.mark.gpu


def small_stream(n=8, rate=200.0):
    return serving_requests(n, rate, seed=5, max_nel=5, max_order=5)


@pytest.mark.parametrize("policy,chunk", [("fifo", 3), ("sjf", 3), ("hrrn", 3), ("guard", 3),
                                          ("guard", None)])
def test_each_request_same_alone_and_in_the_mix(gpu, policy, chunk):
    reqs = small_stream()
    srv = Server(4 << 30, max_slots=64, precision="fp64", chunk=chunk, energy_every=1, policy=policy,
                 saturation_nodes=20000, guard_s=0.01)
    mixed, wall = srv.run(reqs)
    srv.close()
    assert all(r is not None for r in mixed)
    st = latency_stats(mixed)
    assert st["n"] == len(reqs) and st["p99"] >= st["p50"] > 0
    for i in (0, 3, len(reqs) - 1):
        solo = Server(2 << 30, max_slots=4, precision="fp64", chunk=5, energy_every=1)
        one = reqs[i]
        one.arrival = 0.0
        res, _ = solo.run([one])
        solo.close()
        np.testing.assert_array_equal(res[0].probes, mixed[i].probes)
        np.testing.assert_array_equal(res[0].energy, mixed[i].energy)


def test_requests_overlap_on_the_device(gpu):
    """Requests admitted while others run: at least two are resident at once."""
    reqs = small_stream(6, rate=1e6)
    srv = Server(4 << 30, max_slots=64, precision="fp32", chunk=2)
    res, _ = srv.run(reqs)
    srv.close()
    spans = sorted((r.admitted, r.finished) for r in res)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))


def test_sjf_admits_the_smallest_waiting_request_first(gpu):
    """All requests waiting at once, residency capped below any two of them: they
    run one at a time in order of work."""
    reqs = small_stream(6, rate=1e9)
    srv = Server(4 << 30, max_slots=64, precision="fp64", chunk=2, policy="sjf", saturation_nodes=1)
    res, _ = srv.run(reqs)
    srv.close()
    order = [r.request for r in sorted(res, key=lambda r: r.admitted)]
    work = [reqs[i].dof_stages for i in order]
    assert work == sorted(work)
    # residency on the GPU (admission to retirement) never overlaps; results reach
    # the host by `finished`, one status round after retirement
    spans = sorted((r.admitted, r.retired) for r in res)
    assert all(spans[k + 1][0] >= spans[k][1] for k in range(len(spans) - 1))
    assert all(r.admitted <= r.retired <= r.finished for r in res)


def test_serving_energy_matches_single_mesh_solver(gpu):
    req = small_stream(1)[0]
    srv = Server(2 << 30, max_slots=2, precision="fp64", chunk=4, energy_every=1)
    res, _ = srv.run([req])
    srv.close()
    s = DgSolver()
    s.initializeBox(req.N, req.nel, req.lo, req.hi, req.c0)
    s.initPulse(req.pulses)
    s.steps(req.dt, req.nsteps)
    e = s.energy()
    s.finalize()
    assert abs(res[0].energy[-1] - e) <= 1e-13 * e
    # the serial baseline records the same histories (probes every step, energy at
    # its output steps and the last one)
    ser, _ = serve_serial([req], energy_every=1)
    assert abs(ser[0].energy[-1] - e) <= 1e-13 * e
    np.testing.assert_allclose(ser[0].energy, res[0].energy, rtol=1e-13, atol=0)
    assert ser[0].probes.shape == res[0].probes.shape == (req.nsteps + 1, len(req.probes), 6)
    scale = np.abs(res[0].probes).max()
    assert scale > 0 and np.abs(ser[0].probes - res[0].probes).max() <= 1e-12 * scale


@pytest.mark.parametrize("N,nel,per", [(5, (4, 3, 2), (False, False, False)),
                                       (8, (3, 3, 3), (True, True, True))])
def test_box_solver_equals_mesh_solver(gpu, N, nel, per):
    lo, hi = (0.0, 0.0, 0.0), (1.0, 0.75, 0.5)
    m = Mesh(N)
    m.createBoxMesh(*nel, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], *per)
    a = DgSolver()
    a.initializeBox(N, nel, lo, hi, 1.0, periodic=per)
    pulses = [(1.0, 0.5, 0.3, 0.2, 0.15)] * 6
    a.initPulse(pulses)
    u0 = a.downloadState()
    req = type("R", (), {"pulses": pulses})()
    host = cavity_state(req, m.getCoordX(), m.getCoordY(), m.getCoordZ())
    assert np.max(np.abs(u0 - host)) < 1e-14
    b = DgSolver()
    b.initialize(m, 1.0)
    b.uploadState(u0)
    dt = 0.5 * m.computeMinNodeDistance()
    a.steps(dt, 5)
    b.steps(dt, 5)
    np.testing.assert_array_equal(a.downloadState(), b.downloadState())
    a.finalize()
    b.finalize()
