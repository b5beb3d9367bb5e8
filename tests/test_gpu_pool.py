"""Cavity pool (nwb_pool_*): many independent cavities advanced by one
persistent launch per LSRK stage.  Each cavity must give the single-mesh
solver's result (same fused stage arithmetic), bit for bit, alone or in any mix;
admission respects the HBM budget; energy and probes are recorded per step."""
import numpy as np
import pytest

from nekwave_b200 import DgSolver, Mesh
from nekwave_b200.pool import FINISHED, CavityPool, PoolFull, locate_probes
from tests.gpu_helpers import rel_l2

pytestmark = pytest.mark.gpu

CASES = [  # N, nel, lo, hi, periodic, c0, nsteps
    (4, (3, 2, 2), (0, 0, 0), (1.5, 1, 1), (False,) * 3, 1.0, 3),
    (6, (2, 2, 3), (0, 0, 0), (1, 1, 2), (True, False, True), 0.0, 5),
    (9, (2, 1, 1), (-1, 0, 0), (1, 0.5, 0.5), (False,) * 3, 1.0, 4),
    (2, (4, 3, 2), (0, 0, 0), (1, 1, 1), (False,) * 3, 1.0, 7),
    (5, (3, 3, 3), (0, 0, 0), (1, 1, 1), (False,) * 3, 0.5, 6),
    (8, (2, 2, 2), (0, 0, 0), (1, 1, 1), (True, True, True), 0.0, 2),
]


def make_mesh(N, nel, lo, hi, per):
    m = Mesh(N)
    m.createBoxMesh(*nel, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], *per)
    return m


def pulse_state(m, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    x, y, z = m.getCoordX(), m.getCoordY(), m.getCoordZ()
    lo = np.array([x.min(), y.min(), z.min()])
    hi = np.array([x.max(), y.max(), z.max()])
    u = np.zeros(6 * m.getTotalPoints())
    n = m.getTotalPoints()
    for c in range(6):
        r0 = lo + (hi - lo) * rng.uniform(0.25, 0.75, 3)
        s = 0.2 * float(np.min(hi - lo))
        u[c * n:(c + 1) * n] = np.exp(-((x - r0[0]) ** 2 + (y - r0[1]) ** 2 + (z - r0[2]) ** 2) / s ** 2)
    return u


def probe_points(m, seed, k=3):
    rng = np.random.Generator(np.random.PCG64(seed + 100))
    b = m.box
    lo, hi = np.array(b["lo"]), np.array(b["hi"])
    return [lo + (hi - lo) * rng.uniform(0.05, 0.95, 3) for _ in range(k)]


def single(m, c0, dt, nsteps, u0):
    s = DgSolver()
    s.initialize(m, c0)
    s.uploadState(u0)
    energies = [s.energy()]
    states = [u0.copy()]
    for _ in range(nsteps):
        s.step(dt, 0.0)
        energies.append(s.energy())
        states.append(s.downloadState())
    s.finalize()
    return states, np.array(energies)


def interp_probes(m, states, points):
    elem, w = locate_probes(m, points)
    N = m.getN()
    w = w.reshape(len(points), 3, N)
    n = m.getTotalPoints()
    out = np.zeros((len(states), len(points), 6))
    for t, u in enumerate(states):
        for p in range(len(points)):
            W = np.einsum("k,j,i->kji", w[p, 2], w[p, 1], w[p, 0]).ravel()
            base = elem[p] * N ** 3
            for c in range(6):
                out[t, p, c] = np.dot(W, u[c * n + base:c * n + base + N ** 3])
    return out


@pytest.mark.parametrize("mode", [0, 1])
def test_pool_matches_single_mesh_solver(gpu, mode):
    pool = CavityPool(2 << 30, max_slots=16)
    pool.set_mode(mode)
    meshes, slots, refs = [], [], []
    for i, (N, nel, lo, hi, per, c0, ns) in enumerate(CASES):
        m = make_mesh(N, nel, lo, hi, per)
        dt = 0.5 * m.computeMinNodeDistance()
        u0 = pulse_state(m, i)
        pts = probe_points(m, i)
        s = pool.add(m, c0, dt, ns, probes=pts)
        pool.upload(s, u0)
        meshes.append((m, pts))
        slots.append(s)
        refs.append(single(m, c0, dt, ns, u0))
    pool.step(max(c[-1] for c in CASES) + 2)  # extra steps: finished cavities stay put
    status, done = pool.query()
    for i, s in enumerate(slots):
        assert status[s] == FINISHED and done[s] == CASES[i][-1]
        r = pool.results(s)
        states, energies = refs[i]
        np.testing.assert_array_equal(r["state"], states[-1])
        np.testing.assert_allclose(r["energy"], energies, rtol=1e-13, atol=0)
        m, pts = meshes[i]
        np.testing.assert_allclose(r["probes"], interp_probes(m, states, pts), rtol=0, atol=1e-12)
    pool.close()


def test_each_cavity_same_alone_and_in_the_mix(gpu):
    N, nel, lo, hi, per, c0, ns = CASES[1]
    m = make_mesh(N, nel, lo, hi, per)
    dt = 0.5 * m.computeMinNodeDistance()
    u0 = pulse_state(m, 7)
    alone = CavityPool(1 << 30, max_slots=4)
    s = alone.add(m, c0, dt, ns)
    alone.upload(s, u0)
    alone.step(ns)
    a = alone.results(s)
    alone.close()
    mix = CavityPool(2 << 30, max_slots=32)
    others = []
    for i, (N2, nel2, lo2, hi2, per2, c02, ns2) in enumerate(CASES * 2):
        m2 = make_mesh(N2, nel2, lo2, hi2, per2)
        o = mix.add(m2, c02, 0.5 * m2.computeMinNodeDistance(), ns2 + i)
        mix.upload(o, pulse_state(m2, 50 + i))
        others.append(o)
        if i == 3:
            s2 = mix.add(m, c0, dt, ns)
            mix.upload(s2, u0)
    best, ms = mix.autotune(reps=2)   # timing launches leave every state as it was
    assert best in (0, 1) and all(t > 0 for t in ms)
    mix.step(ns + 20)
    b = mix.results(s2)
    mix.close()
    np.testing.assert_array_equal(a["state"], b["state"])
    np.testing.assert_array_equal(a["energy"], b["energy"])


def test_admission_by_hbm_budget(gpu):
    m = make_mesh(6, (4, 4, 4), (0, 0, 0), (1, 1, 1), (False,) * 3)
    per_cavity = 3 * 6 * m.getTotalPoints() * 8
    pool = CavityPool(int(2.5 * per_cavity) + (1 << 20), max_slots=8)
    a = pool.add(m, 1.0, 1e-3, 2)
    b = pool.add(m, 1.0, 1e-3, 2)
    with pytest.raises(PoolFull):
        pool.add(m, 1.0, 1e-3, 2)
    pool.remove(a)
    c = pool.add(m, 1.0, 1e-3, 2)
    assert c == a
    info = pool.info()
    assert info["slots_used"] == 2 and info["used_bytes"] <= info["budget_bytes"]
    few = CavityPool(1 << 30, max_slots=1)
    few.add(m, 1.0, 1e-3, 2)
    with pytest.raises(PoolFull):
        few.add(m, 1.0, 1e-3, 2)
    few.close()
    pool.close()


def test_box_fast_path_equals_mesh_path(gpu):
    N, nel, lo, hi, per, c0, ns = 7, (3, 2, 2), (0.0, -0.5, 0.0), (1.2, 0.5, 0.8), (False,) * 3, 1.0, 4
    m = make_mesh(N, nel, lo, hi, per)
    dt = 0.5 * m.computeMinNodeDistance()
    pulses = [(1.0, 0.6, 0.0, 0.4, 0.2) if c in (2, 3) else (0.0, 0, 0, 0, 0.0) for c in range(6)]
    pool = CavityPool(1 << 30, max_slots=4)
    a = pool.add_box(N, nel, lo, hi, c0, dt, ns, probes=[(0.3, 0.1, 0.5)])
    pool.init_pulse(a, pulses)
    # the same initial state from the host, on the host mesh
    n = m.getTotalPoints()
    u0 = np.zeros(6 * n)
    from nekwave_b200.pool import CavityPool as _  # noqa: F401
    st0 = pool.results(a, energy=False, probes=False)["state"]
    x, y, z = m.getCoordX(), m.getCoordY(), m.getCoordZ()
    for c in (2, 3):
        u0[c * n:(c + 1) * n] = np.exp(-((x - 0.6) ** 2 + y ** 2 + (z - 0.4) ** 2) / 0.04)
    assert np.max(np.abs(st0 - u0)) < 1e-14
    b = pool.add(m, c0, dt, ns, probes=[(0.3, 0.1, 0.5)])
    pool.upload(b, st0)
    pool.step(ns)
    ra, rb = pool.results(a), pool.results(b)
    np.testing.assert_array_equal(ra["state"], rb["state"])
    np.testing.assert_array_equal(ra["energy"], rb["energy"])
    np.testing.assert_array_equal(ra["probes"], rb["probes"])
    pool.close()


def test_fp32_bulk_pool_error_vs_fp64(gpu):
    N, nel, lo, hi, per, c0, ns = 6, (4, 3, 3), (0, 0, 0), (1, 1, 1), (False,) * 3, 1.0, 40
    m = make_mesh(N, nel, lo, hi, per)
    dt = 0.5 * m.computeMinNodeDistance()
    u0 = pulse_state(m, 3)
    out = {}
    for prec in ("fp64", "fp32"):
        pool = CavityPool(1 << 30, max_slots=2, precision=prec)
        s = pool.add(m, c0, dt, ns)
        pool.upload(s, u0)
        pool.step(ns)
        out[prec] = pool.results(s)
        pool.close()
    err = rel_l2(out["fp32"]["state"], out["fp64"]["state"])
    assert err < 1e-5, err
    assert np.all(np.abs(out["fp32"]["energy"] / out["fp64"]["energy"] - 1) < 1e-5)


def test_fp32_bulk_smooth_pulse_within_1e6_and_pool_equals_single(gpu):
    """The FP32-bulk class on a resolved smooth field (periodic box, 16^3 elements of
    8 points, Gaussian Ez of width 3.2 element sizes, central flux, 500 steps): its
    state stays within 1e-6 relative L2 of the FP64 path, and the pool evolves the
    cavity bit for bit as the single-mesh FP32 solver does."""
    N, nel, lo, hi, per, c0, ns = 8, (16, 16, 16), (0, 0, 0), (0.5, 0.5, 0.5), (True,) * 3, 0.0, 500
    m = make_mesh(N, nel, lo, hi, per)
    dt = 0.5 * m.computeMinNodeDistance()
    x, y, z = m.getCoordX(), m.getCoordY(), m.getCoordZ()
    n = m.getTotalPoints()
    u0 = np.zeros(6 * n)
    u0[2 * n:3 * n] = np.exp(-((x - 0.22) ** 2 + (y - 0.27) ** 2 + (z - 0.25) ** 2) / 0.1 ** 2)
    out = {}
    for prec in ("fp64", "fp32"):
        s = DgSolver(prec)
        s.initialize(m, c0)
        s.uploadState(u0)
        s.steps(dt, ns)
        out[prec] = s.downloadState()
        s.finalize()
    err = rel_l2(out["fp32"], out["fp64"])
    assert err < 1e-6, err
    pool = CavityPool(1 << 30, max_slots=2, precision="fp32")
    s = pool.add(m, c0, dt, ns)
    pool.upload(s, u0)
    pool.step(ns)
    np.testing.assert_array_equal(pool.results(s)["state"], out["fp32"])
    pool.close()


def test_fp32_bulk_meets_1e6_on_the_least_resolved_batch_instances(gpu):
    """The FP32-bulk gate on the batched workload's hardest cavities: of the 256
    seeded instances (400 steps each, upwind, PEC), the 12 whose pulse spans the
    fewest elements, advanced in an FP32-bulk pool and an FP64 pool.  Every
    instance stays within 1e-6 relative L2 of FP64 (elements whose field departs
    from linear across the element run the FP64 arithmetic); the errors are
    recorded (fp32_gate_batch.json)."""
    from nekwave_b200.workloads import batch_instances
    from tests.gpu_helpers import record
    inst = batch_instances(256, seed=0, steps=400)

    def resolution(c):  # pulse width in element sizes, along the coarsest axis
        return c.pulses[2][4] / max((c.hi[a] - c.lo[a]) / c.nel[a] for a in range(3))

    pick = sorted(inst, key=resolution)[:12]
    out = {}
    for prec in ("fp64", "fp32"):
        pool = CavityPool(8 << 30, max_slots=len(pick), precision=prec)
        slots = [pool.add_box(c.N, c.nel, c.lo, c.hi, c.c0, c.dt, c.nsteps) for c in pick]
        for s, c in zip(slots, pick):
            pool.init_pulse(s, c.pulses)
        pool.step(400)
        out[prec] = [pool.results(s, energy=False, probes=False)["state"] for s in slots]
        pool.close()
    errs = [rel_l2(a, b) for a, b in zip(out["fp32"], out["fp64"])]
    record("fp32_gate_batch.json", {"instances": len(pick), "steps": 400,
                                    "resolution_elements": [resolution(c) for c in pick],
                                    "N": [c.N for c in pick], "rel_l2": errs, "max": max(errs)})
    assert max(errs) <= 1e-6, errs
