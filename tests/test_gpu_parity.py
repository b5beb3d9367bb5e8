"""Parity of the CUDA path (libnwb, through its C ABI) with the oracle on the
same seeded inputs, plus the reference's own golden vectors.

FP64 tolerance: the CUDA path contracts a*b+c into FMAs and sums each residual
in a fixed order that differs from the reference's (its lift is an atomicAdd in
arbitrary order), so results agree to rounding, not bitwise.  The bound used is
a relative max error of 1e-12 for one right-hand side and a relative L2 error
of 1e-12 for a few steps, 1e-10 for 200 steps.
"""
import glob
import os

import numpy as np
import pytest

from nekwave_b200 import DgSolver, Mesh
from oracle import oracle as O
from tests.gpu_helpers import random_state, rel_l2, rel_max, smooth_state, solver_for

pytestmark = pytest.mark.gpu

RHS_TOL = 1e-12
STEP_TOL = 1e-12

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.mark.parametrize("N", range(2, 11))
@pytest.mark.parametrize("c0", [0.0, 1.0])
def test_rhs_pec_box_all_orders(gpu, N, c0):
    m = O.box_mesh(N, (3, 2, 2), (0.0, -1.0, 0.0), (1.5, 1.0, 0.75))
    s = solver_for(m, c0)
    assert s.info()["geometry"] == 0
    u = random_state(m, N)
    s.uploadState(u)
    got = s.evalRhs()
    want = O.rhs(m, c0, u)
    assert rel_max(got, want) < RHS_TOL
    np.testing.assert_array_equal(s.downloadState(), u)  # evalRhs leaves the state alone
    s.finalize()


@pytest.mark.parametrize("N,nel,per", [(4, (2, 2, 2), (1, 1, 1)), (5, (3, 1, 2), (1, 0, 1)),
                                       (8, (2, 3, 2), (0, 1, 0)), (7, (1, 1, 1), (1, 1, 1)),
                                       (3, (5, 4, 3), (0, 0, 1))])
@pytest.mark.parametrize("c0", [0.0, 0.5, 1.0])
def test_rhs_periodic_and_mixed(gpu, N, nel, per, c0):
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 2, 1), per)
    s = solver_for(m, c0)
    u = random_state(m, 7)
    s.uploadState(u)
    assert rel_max(s.evalRhs(), O.rhs(m, c0, u)) < RHS_TOL
    s.finalize()


@pytest.mark.parametrize("N", [3, 5, 8])
def test_rhs_affine_parallelepiped(gpu, N):
    A = [[1.0, 0.3, 0.1], [-0.2, 1.1, 0.05], [0.1, 0.2, 0.9]]
    m = O.warped_box_mesh(N, (3, 2, 2), linear=A)
    s = solver_for(m, 1.0)
    assert s.info()["geometry"] == 1
    u = random_state(m, 3)
    s.uploadState(u)
    assert rel_max(s.evalRhs(), O.rhs(m, 1.0, u)) < RHS_TOL
    s.finalize()


@pytest.mark.parametrize("N", [2, 4, 6, 9])
@pytest.mark.parametrize("c0", [0.0, 1.0])
def test_rhs_trilinear_per_node_geometry(gpu, N, c0):
    m = O.warped_box_mesh(N, (3, 3, 2), warp=0.06)
    s = solver_for(m, c0)
    assert s.info()["geometry"] == 2
    u = random_state(m, 5)
    s.uploadState(u)
    assert rel_max(s.evalRhs(), O.rhs(m, c0, u)) < RHS_TOL
    s.finalize()


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_against_reference_golden_vectors(gpu, path):
    g = np.load(path)
    m = O.box_mesh(int(g["N"]), tuple(g["nel"]), tuple(g["lo"]), tuple(g["hi"]),
                   tuple(bool(p) for p in g["periodic"]))
    c0 = float(g["c0"])
    s = solver_for(m, c0)
    s.uploadState(g["u0"])
    assert rel_max(s.evalRhs(), g["rhs"]) < RHS_TOL
    for n in range(int(g["steps"])):
        s.step(float(g["dt"]), 0.0)
        assert abs(s.energy() - g["energies"][n]) <= 1e-12 * abs(g["energies"][n])
    assert rel_l2(s.downloadState(), g["u1"]) < STEP_TOL
    s.finalize()


@pytest.mark.parametrize("N,nel,per,c0", [(4, (2, 2, 2), (0, 0, 0), 1.0), (6, (2, 2, 3), (1, 1, 1), 0.0),
                                          (8, (2, 2, 2), (1, 0, 0), 1.0)])
@pytest.mark.parametrize("graph", [False, True])
def test_steps_match_oracle(gpu, N, nel, per, c0, graph):
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 1, 1), per)
    s = solver_for(m, c0)
    u = smooth_state(m, 11)
    dt = 0.5 * O.dxmin(m)
    s.uploadState(u)
    if graph:
        s.steps(dt, 6)
    else:
        for _ in range(6):
            s.step(dt, 0.0)
    want, _ = O.step(m, c0, dt, 6, u)
    assert rel_l2(s.downloadState(), want) < STEP_TOL
    s.finalize()


def tm110_exact(m, T):
    n, w = m.npts, np.pi * np.sqrt(2.0)
    ex = np.zeros(6 * n)
    ex[2 * n:3 * n] = np.sin(np.pi * m.x) * np.sin(np.pi * m.y) * np.cos(w * T)
    ex[3 * n:4 * n] = -np.sin(np.pi * m.x) * np.cos(np.pi * m.y) * np.sin(w * T) / np.sqrt(2.0)
    ex[4 * n:5 * n] = np.cos(np.pi * m.x) * np.sin(np.pi * m.y) * np.sin(w * T) / np.sqrt(2.0)
    return ex


def test_tm110_cavity_200_steps(gpu):
    """PEC unit cube, 4^3 elements, 5 GLL points, upwind, CFL 0.5, 200 LSRK45 steps,
    Ez = sin(pi x) sin(pi y): the oracle after 200 steps and the analytic TM110 mode."""
    m = O.box_mesh(5, (4, 4, 4), (0, 0, 0), (1, 1, 1))
    dt = 0.5 * O.dxmin(m)
    u0 = tm110_exact(m, 0.0)
    s = solver_for(m, 1.0)
    s.uploadState(u0)
    s.steps(dt, 200)
    got = s.downloadState()
    want, _ = O.step(m, 1.0, dt, 200, u0)
    assert rel_l2(got, want) < 1e-10
    assert rel_l2(got, tm110_exact(m, 200 * dt)) < 5e-5
    e0 = O.energy(m, u0)
    assert s.energy() <= e0  # upwind never gains energy
    s.finalize()


def test_upwind_energy_monotone_stability_case(gpu):
    """MaxwellStabilityTest (tests/nekwave_test.cpp:212-293): N=4, 2x2x2 on
    [-0.5,0.5]^3, upwind, Ez = exp(-50 r^2), dt = 0.005, energy never increases."""
    m = O.box_mesh(4, (2, 2, 2), (-.5, -.5, -.5), (.5, .5, .5))
    u = np.zeros(6 * m.npts)
    u[2 * m.npts:3 * m.npts] = np.exp(-50.0 * (m.x ** 2 + m.y ** 2 + m.zc ** 2))
    s = solver_for(m, 1.0)
    s.uploadState(u)
    prev = s.energy()
    assert abs(prev - O.energy(m, u)) <= 1e-13 * prev
    for _ in range(20):
        s.step(0.005, 0.0)
        e = s.energy()
        assert np.isfinite(e) and e <= prev + 1e-12
        prev = e
    s.finalize()


def test_central_flux_conserves_energy_periodic(gpu):
    """Central flux on a periodic box: the semi-discrete operator conserves the
    discrete energy (u^T M rhs(u) = 0 to rounding), the fully discrete drift is the
    LSRK45 dissipation (it shrinks ~32x when dt halves) and matches the oracle."""
    m = O.box_mesh(6, (4, 4, 4), (0, 0, 0), (1, 1, 1), (True, True, True))
    u = smooth_state(m, 2)
    s = solver_for(m, 0.0)
    s.uploadState(u)
    r = s.evalRhs()
    wts = np.tile(m.jac * np.tile(m.w3, m.nelt), 6)
    assert abs(np.sum(u * wts * r)) / np.sum(u * wts * u) < 1e-14
    e0 = s.energy()
    dt = 0.5 * O.dxmin(m)
    drifts = []
    for f in (1, 2):
        s.uploadState(u)
        s.steps(dt / f, 100 * f)
        e1 = s.energy()
        want, _ = O.step(m, 0.0, dt / f, 100 * f, u)
        assert abs(e1 - O.energy(m, want)) <= 1e-12 * e0
        drifts.append((e0 - e1) / e0)
    assert drifts[0] > 0 and drifts[1] > 0
    assert 20.0 < drifts[0] / drifts[1] < 45.0
    s.finalize()


def test_bitwise_deterministic(gpu):
    m = O.box_mesh(6, (4, 3, 3), (0, 0, 0), (1, 1, 1), (True, False, False))
    u = random_state(m, 1)
    outs = []
    for _ in range(2):
        s = solver_for(m, 1.0)
        s.uploadState(u)
        s.steps(1e-3, 5)
        outs.append(s.downloadState())
        s.finalize()
    np.testing.assert_array_equal(outs[0], outs[1])


def test_rhs_linearity_full_size_c3(gpu):
    """Size-independent property at the PEC cavity size (64x64x32, 6 points):
    RHS(a u + b v) = a RHS(u) + b RHS(v) to rounding."""
    from nekwave_b200 import DgSolver, Mesh
    mesh = Mesh(6)
    mesh.createBoxMesh(64, 64, 32, 0.0, 2.0, 0.0, 2.0, 0.0, 1.0)
    s = DgSolver()
    s.initialize(mesh, 1.0)
    rng = np.random.Generator(np.random.PCG64(0))
    n = 6 * mesh.getTotalPoints()
    u = rng.standard_normal(n)
    v = rng.standard_normal(n)
    s.uploadState(u)
    ru = s.evalRhs()
    s.uploadState(v)
    rv = s.evalRhs()
    s.uploadState(2.0 * u - 0.5 * v)
    rw = s.evalRhs()
    assert rel_l2(rw, 2.0 * ru - 0.5 * rv) < 1e-13
    s.finalize()


@pytest.mark.parametrize("N", range(2, 11))
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_every_launch_shape_matches_oracle(gpu, N, prec):
    """Each launch shape the autotuner may pick computes the same stage."""
    m = O.box_mesh(N, (3, 3, 2), (0, 0, 0), (1, 1, 1), (True, False, True))
    s = solver_for(m, 1.0, prec)
    u = random_state(m, 9)
    s.uploadState(u)
    want = O.rhs(m, 1.0, u)
    dt = 0.5 * O.dxmin(m)
    want_steps, _ = O.step(m, 1.0, dt, 2, u)
    tol = RHS_TOL if prec == "fp64" else 1e-4
    nv = s.info()["variant_count"]
    assert nv >= 3
    for v in range(nv):
        s.setVariant(v)
        s.uploadState(u)
        assert rel_max(s.evalRhs(), want) < tol, v
        s.steps(dt, 2)
        assert rel_l2(s.downloadState(), want_steps) < (STEP_TOL if prec == "fp64" else 1e-5), v
    s.uploadState(u)
    best, ms = s.autotune(reps=3)
    assert 0 <= best < nv and len(ms) == nv and all(t > 0 for t in ms)
    # the default shape is kept unless another beats it by more than 1%
    assert best == 0 or ms[best] * 1.01 < ms[0], (best, ms[best], ms[0])
    assert min(ms) * 1.01 >= ms[best] * (1 - 1e-6)
    np.testing.assert_array_equal(s.downloadState(), u)  # autotuning leaves the state alone
    s.finalize()


@pytest.mark.parametrize("N", [5, 6, 8, 9])
@pytest.mark.parametrize("nel", [(1, 1, 1), (2, 1, 1)])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_every_launch_shape_on_self_neighbour_meshes(gpu, N, nel, prec):
    """Fully periodic meshes of one or two elements: across every face an element
    meets itself or the other element of its tile, so the face phase takes its
    neighbour traces from the resident tile, and tiles of several elements are
    ragged (fewer valid elements than the shape holds)."""
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 1, 1), (True, True, True))
    s = solver_for(m, 1.0, prec)
    u = random_state(m, 5)
    want = O.rhs(m, 1.0, u)
    tol = RHS_TOL if prec == "fp64" else 1e-4
    for v in range(s.info()["variant_count"]):
        s.setVariant(v)
        s.uploadState(u)
        assert rel_max(s.evalRhs(), want) < tol, v
    s.finalize()


@pytest.mark.parametrize("N,nel", [(4, (24, 24, 24)), (5, (20, 16, 16)), (6, (16, 16, 16)),
                                   (7, (12, 12, 12)), (8, (16, 16, 12)), (9, (12, 12, 10))])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_every_launch_shape_on_meshes_of_many_tiles(gpu, N, nel, prec):
    """Meshes of about a million nodes: several tiles per resident block, so the
    persistent double-buffered shapes walk their whole tile loop (buffer swaps,
    ragged last tile, neighbours in tiles that are in flight)."""
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 1.5, 1), (True, False, False))
    s = solver_for(m, 1.0, prec)
    u = random_state(m, 11)
    want = O.rhs(m, 1.0, u)
    dt = 0.5 * O.dxmin(m)
    want_steps, _ = O.step(m, 1.0, dt, 2, u)
    tol = RHS_TOL if prec == "fp64" else 1e-4
    for v in range(s.info()["variant_count"]):
        s.setVariant(v)
        s.uploadState(u)
        assert rel_max(s.evalRhs(), want) < tol, v
        s.steps(dt, 2)
        assert rel_l2(s.downloadState(), want_steps) < (STEP_TOL if prec == "fp64" else 1e-5), v
    s.finalize()


@pytest.mark.parametrize("N", [3, 5, 6, 8])
@pytest.mark.parametrize("rotate", [False, True])
def test_shuffled_and_rotated_elements(gpu, N, rotate):
    """Element numbering without structure, and (rotate) faces that meet with
    turned frames: the connection-table path of the face phase, with
    non-identity orientations, for every launch shape of the geometry class."""
    from tests.gpu_helpers import shuffled_box_mesh
    m = shuffled_box_mesh(N, (3, 4, 2), (0, 0, 0), (1.5, 1, 0.75), 5, rotate)
    s = solver_for(m, 1.0)
    info = s.info()
    assert info["structured"] == (0, 0, 0)
    assert info["geometry"] == (1 if rotate else 0)
    u = random_state(m, 4)
    want = O.rhs(m, 1.0, u)
    dt = 0.5 * O.dxmin(m)
    want_steps, _ = O.step(m, 1.0, dt, 2, u)
    for v in range(info["variant_count"]):
        s.setVariant(v)
        s.uploadState(u)
        assert rel_max(s.evalRhs(), want) < RHS_TOL, v
        s.steps(dt, 2)
        assert rel_l2(s.downloadState(), want_steps) < STEP_TOL, v
    s.finalize()


@pytest.mark.parametrize("per", [(False, False, False), (True, False, True), (True, True, True)])
def test_structured_box_is_recognised(gpu, per):
    m = O.box_mesh(6, (4, 3, 2), (0, 0, 0), (1, 1, 1), per)
    s = solver_for(m, 1.0)
    info = s.info()
    assert info["structured"] == (4, 3, 2)
    assert info["periodic_mask"] == sum(1 << d for d in range(3) if per[d])
    s.finalize()
    b = DgSolver("fp64")
    b.initializeBox(6, (4, 3, 2), (0, 0, 0), (1, 1, 1), 1.0, periodic=per)
    assert b.info()["structured"] == (4, 3, 2)
    b.finalize()


def test_probes_equal_the_reference_record_bit_for_bit(gpu):
    """nwb_probe_read = ProbeManager::record: the same weights and node order, the
    same multiply-then-add roundings, on the state after a few steps."""
    from nekwave_b200.pool import locate_probes
    N, nel = 6, (3, 2, 2)
    mesh = Mesh(N)
    mesh.createBoxMesh(*nel, 0.0, 1.5, 0.0, 1.0, 0.0, 1.0, False, False, False)
    s = DgSolver()
    s.initialize(mesh, 1.0)
    u0 = random_state(O.box_mesh(N, nel, (0, 0, 0), (1.5, 1, 1)), 12)
    s.uploadState(u0)
    s.steps(0.5 * mesh.computeMinNodeDistance(), 3)
    pts = [(0.1, 0.2, 0.3), (1.4, 0.9, 0.95), (0.75, 0.5, 0.5), (0.5, 0.5, 0.0)]
    elems, w1d = locate_probes(mesh, pts)
    w1d = w1d.reshape(len(pts), 3, N)
    # ProbeManager's full weights: w[i + N(j + N k)] = wr[i] ws[j] wt[k]
    wfull = np.einsum("pk,pj,pi->pkji", w1d[:, 2], w1d[:, 1], w1d[:, 0]).reshape(len(pts), -1)
    off = elems.astype(np.int64) * N ** 3
    s.probeSetup(off, wfull)
    got = s.probeRead()
    s.probesAt(mesh, pts)                 # the same set-up from the points alone
    np.testing.assert_array_equal(s.probeRead(), got)
    u = s.downloadState()
    npts = u.size // 6
    want = np.zeros((len(pts), 6))
    for p in range(len(pts)):
        for c in range(6):
            acc = 0.0
            for q in range(N ** 3):
                acc = acc + wfull[p, q] * u[c * npts + off[p] + q]
            want[p, c] = acc
    np.testing.assert_array_equal(got, want)
    s.finalize()


def test_snapshot_while_stepping_equals_a_synchronous_download(gpu):
    m = O.box_mesh(8, (6, 6, 6), (0, 0, 0), (1, 1, 1), (True, True, True))
    u0 = smooth_state(m, 3)
    dt = 0.5 * O.dxmin(m)
    a = solver_for(m, 0.0)
    a.uploadState(u0)
    a.steps(dt, 7)
    want = a.downloadState()
    a.finalize()
    b = solver_for(m, 0.0)
    b.uploadState(u0)
    host = np.empty(6 * m.npts)
    b.steps(dt, 7)
    b.snapshotBegin(host)
    b.steps(dt, 20)            # keeps stepping while the copy is in flight
    b.snapshotWait()
    np.testing.assert_array_equal(host, want)
    b.snapshotBegin(host)      # a second snapshot after the 20 further steps
    b.snapshotWait()
    np.testing.assert_array_equal(host, b.downloadState())
    b.finalize()


@pytest.mark.parametrize("N,nel", [(8, (6, 6, 6)), (5, (3, 5, 4))])
def test_pipelined_upload_step_download_equals_the_blocking_calls(gpu, N, nel):
    """uploadBegin + step + snapshotBegin for a run of different input states (the
    pipelined end-to-end pattern: step i+1's upload in flight while step i runs and
    its result is downloaded) gives, per input, the result of the blocking
    uploadState + step + downloadState, bit for bit; a blocking upload after an
    asynchronous one is ordered behind it."""
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 1, 1), (True, True, True))
    dt = 0.5 * O.dxmin(m)
    ins = [smooth_state(m, s) for s in (3, 4, 5, 6)]
    a = solver_for(m, 0.0)
    want = []
    for u in ins:
        a.uploadState(u)
        a.step(dt)
        want.append(a.downloadState())
    a.finalize()
    b = solver_for(m, 0.0)
    outs = [np.empty(6 * m.npts) for _ in ins]
    for u, o in zip(ins, outs):
        b.uploadBegin(u)
        b.steps(dt, 1, sync=False)
        b.snapshotBegin(o)
    b.snapshotWait()
    b.uploadWait()
    for o, w in zip(outs, want):
        np.testing.assert_array_equal(o, w)
    b.uploadBegin(ins[0])
    b.uploadState(ins[1])      # the blocking upload lands after the asynchronous one
    b.uploadWait()
    np.testing.assert_array_equal(b.downloadState(), ins[1])
    b.finalize()


def test_nonfinite_state_is_reported_not_hidden(gpu):
    """A NaN in the state: nwb_energy returns NWB_ENONFINITE (with the energy), the
    context stays usable and a finite state afterwards is fine again."""
    from nekwave_b200._lib import NwbError
    m = O.box_mesh(4, (2, 2, 2), (0, 0, 0), (1, 1, 1))
    s = solver_for(m, 1.0)
    u = random_state(m, 2)
    bad = u.copy()
    bad[17] = np.nan
    s.uploadState(bad)
    s.steps(0.5 * O.dxmin(m), 2)
    with pytest.raises(NwbError, match="NWB_ENONFINITE"):
        s.energy()
    s.uploadState(u)
    assert abs(s.energy() - O.energy(m, u)) <= 1e-13 * O.energy(m, u)
    with pytest.raises(NwbError, match="NWB_EINVAL"):
        s.uploadState(u[:-6])
    s.finalize()


def _pmc_meshes(N):
    """Unit cube with PMC (bc 2) walls at x = 0, 1: the axis-aligned class (box
    elements) and the per-node class (the same walls on a warped mesh)."""
    from tests.test_pmc_oracle import pmc_x_cube
    box = pmc_x_cube(N, (3, 2, 2))
    warped = O.warped_box_mesh(N, (3, 2, 2), warp=0.05)
    fp = np.arange(warped.nfp)
    face = (fp // (N * N)) % 6
    xw = np.isclose(warped.x[warped.vmin], 0.0) | np.isclose(warped.x[warped.vmin], 1.0)
    warped.bc = warped.bc.copy()
    warped.bc[((face == 1) | (face == 3)) & xw & (warped.vplus < 0)] = 2
    return box, warped


@pytest.mark.parametrize("N", range(2, 11))
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_true_pmc_option_every_launch_shape(gpu, N, prec):
    """NWB_SOLVER_TRUE_PMC against the oracle's PMC option (pinned to the analytic
    PMC cavity mode on the CPU), on every launch shape of the box class and on the
    per-node class; without the flag the same mesh gives the reference's PEC
    mapping of bc 2."""
    box, warped = _pmc_meshes(N)
    tol = RHS_TOL if prec == "fp64" else 1e-4
    stol = STEP_TOL if prec == "fp64" else 1e-5
    for m, geo in ((box, 0), (warped, 2)):
        assert np.count_nonzero(m.bc == 2) > 0
        u = random_state(m, 11)
        dt = 0.5 * O.dxmin(m)
        for true_pmc in (False, True):
            s = solver_for(m, 1.0, prec, true_pmc=true_pmc)
            info = s.info()
            assert info["geometry"] == geo
            if true_pmc:  # the structured-box neighbour rule knows PEC walls only
                assert info["structured"] == (0, 0, 0)
            want = O.rhs(m, 1.0, u, true_pmc=true_pmc)
            want_steps, _ = O.step(m, 1.0, dt, 2, u, true_pmc=true_pmc)
            for v in range(info["variant_count"]):
                s.setVariant(v)
                s.uploadState(u)
                assert rel_max(s.evalRhs(), want) < tol, (geo, true_pmc, v)
                s.steps(dt, 2)
                assert rel_l2(s.downloadState(), want_steps) < stol, (geo, true_pmc, v)
            s.finalize()


@pytest.mark.parametrize("N,nel", [(5, (4, 4, 4)), (8, (6, 5, 4))])
def test_max_norms_equal_the_host_loop_bit_for_bit(gpu, N, nel):
    """nwb_max_norms against Case::getMaxE/getMaxH (src/case.cpp:768-794) restated
    in numpy (elementwise roundings, no contraction): equal bit for bit, also with
    a NaN node, which the host's comparison passes over."""
    m = O.box_mesh(N, nel, (0, 0, 0), (1, 1, 1))
    s = solver_for(m, 1.0)
    u = random_state(m, 21)
    n = m.npts

    def host(u):
        c = u.reshape(6, n)
        e = np.sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2])
        h = np.sqrt((c[3] * c[3] + c[4] * c[4]) + c[5] * c[5])
        return float(np.nanmax(e)), float(np.nanmax(h))

    s.uploadState(u)
    assert s.maxNorms() == host(u)
    u[4 * n + 17] = np.nan
    s.uploadState(u)
    assert s.maxNorms() == host(u)
    s.finalize()
