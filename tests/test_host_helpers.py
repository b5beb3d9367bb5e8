"""Host-side helpers on the CPU: probe location and Lagrange weights (the data
ProbeManager::init builds, src/probe.cpp:11-96) and the seeded workload generators
the benchmark and the serving loop use."""
import math

import numpy as np
import pytest

from nekwave_b200 import Mesh
from nekwave_b200.pool import lagrange_weights, locate_probes
from nekwave_b200.workloads import batch_instances, box_dxmin, serving_requests


@pytest.mark.parametrize("N", [2, 4, 7, 10])
def test_lagrange_weights_interpolate_polynomials(N):
    m = Mesh(N)
    m.createBoxMesh(1, 1, 1, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, False, False, False)
    z = np.asarray(m.getGllZ())
    rng = np.random.Generator(np.random.PCG64(N))
    for xi in rng.uniform(-1.0, 1.0, 20):
        L = lagrange_weights(z, xi)
        assert abs(L.sum() - 1.0) < 1e-13
        for deg in range(N):  # degree < N is reproduced exactly
            assert abs(L @ z ** deg - xi ** deg) < 1e-12
    # on a node the basis is the unit vector (the reference's exact-node shortcut)
    for i in range(N):
        L = lagrange_weights(z, z[i] + 1e-14)
        assert L[i] == 1.0 and np.count_nonzero(L) == 1


def test_probe_weights_reproduce_coordinates():
    """Tensor weights of a located probe, applied to the element's node coordinates,
    give the probe's position; points outside the box clamp to its surface."""
    N, nel, lo, hi = 5, (3, 2, 4), (0.0, -1.0, 0.5), (1.5, 1.0, 2.5)
    m = Mesh(N)
    m.createBoxMesh(*nel, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], False, False, False)
    x, y, zc = m.getCoordX(), m.getCoordY(), m.getCoordZ()
    rng = np.random.Generator(np.random.PCG64(1))
    pts = [np.asarray(lo) + (np.asarray(hi) - np.asarray(lo)) * rng.uniform(0, 1, 3) for _ in range(12)]
    pts.append(np.array([2.0, 0.0, 1.0]))  # outside in x: clamps to x = 1.5
    elem, w = locate_probes(m, pts)
    w = np.asarray(w).reshape(len(pts), 3, N)
    for p, e, wp in zip(pts, elem, w):
        W = np.einsum("k,j,i->kji", wp[2], wp[1], wp[0]).ravel()
        sl = slice(e * N ** 3, (e + 1) * N ** 3)
        got = np.array([W @ x[sl], W @ y[sl], W @ zc[sl]])
        want = np.clip(p, lo, hi)
        assert np.max(np.abs(got - want)) < 1e-12, (p, got)


def test_batch_instances_are_seeded_and_in_range():
    a, b = batch_instances(64, seed=3), batch_instances(64, seed=3)
    assert [(c.N, c.nel, c.hi) for c in a] == [(c.N, c.nel, c.hi) for c in b]
    assert [(c.N, c.nel) for c in batch_instances(64, seed=4)] != [(c.N, c.nel) for c in a]
    for c in a:
        assert 4 <= c.N <= 9 and all(2 <= n <= 12 for n in c.nel)
        assert c.dt == pytest.approx(0.5 * box_dxmin(c.N, c.nel, c.lo, c.hi), rel=1e-15)


def test_serving_requests_arrive_in_order_and_end_on_their_final_time():
    reqs = serving_requests(40, rate=2.0, seed=5)
    arrivals = [r.arrival for r in reqs]
    assert all(b > a for a, b in zip(arrivals, arrivals[1:]))
    for r in reqs:
        assert len(r.probes) == 8
        assert r.nsteps == max(1, math.ceil(r.T / (0.5 * box_dxmin(r.N, r.nel, r.lo, r.hi))))
        assert abs(r.nsteps * r.dt - r.T) < 1e-12 * r.T  # the last step lands on T
