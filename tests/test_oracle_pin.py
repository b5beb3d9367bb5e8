"""The oracle is pinned to the reference: golden vectors made by the reference
compiled from its own sources (tests/golden/make_golden.py) and, where that
build exists, a live comparison.  CPU only."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.make_golden import CASES, initial_state, mesh_checksum

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _mesh(g):
    return O.box_mesh(int(g["N"]), tuple(g["nel"]), tuple(g["lo"]), tuple(g["hi"]),
                      tuple(bool(p) for p in g["periodic"]))


def test_golden_files_present():
    assert {os.path.basename(p)[:-4] for p in GOLDEN} == set(CASES)


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: os.path.basename(p)[:-4])
def test_oracle_matches_golden_bitwise(path):
    g = np.load(path)
    m = _mesh(g)
    np.testing.assert_array_equal(mesh_checksum(m), g["mesh_checksum"])
    assert O.dxmin(m) == float(g["dxmin"])
    u0 = g["u0"]
    np.testing.assert_array_equal(O.rhs(m, float(g["c0"]), u0), g["rhs"])
    u1, k1 = O.step(m, float(g["c0"]), float(g["dt"]), int(g["steps"]), u0)
    np.testing.assert_array_equal(u1, g["u1"])
    np.testing.assert_array_equal(k1, g["k1"])
    assert O.energy(m, u0) == float(g["energy0"])


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden_inputs_regenerate(name):
    N, nel, lo, hi, per, c0, ic, steps, dt = CASES[name]
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    np.testing.assert_array_equal(initial_state(_mesh(g), ic), g["u0"])


@pytest.mark.skipif(not O.ref_available(), reason="reference host build not present")
@pytest.mark.parametrize("N,nel,per,c0", [(2, (2, 2, 3), (0, 0, 0), 1.0), (6, (2, 2, 2), (1, 0, 0), 0.0),
                                          (7, (1, 2, 2), (0, 1, 1), 1.0), (9, (1, 1, 2), (0, 0, 1), 0.5)])
def test_oracle_matches_reference_build_live(N, nel, per, c0):
    lo, hi = (0.0, -1.0, 0.5), (2.0, 1.0, 1.25)
    m = O.box_mesh(N, nel, lo, hi, per)
    r = O.ref_box_mesh(N, nel, lo, hi, per)
    for k in ("D", "w3", "x", "y", "zc", "jac", "met", "vmin", "vplus", "bc", "nx", "ny", "nz", "dA"):
        np.testing.assert_array_equal(getattr(m, k), getattr(r, k), err_msg=k)
    u = np.random.Generator(np.random.PCG64(N)).standard_normal(6 * m.npts)
    np.testing.assert_array_equal(O.rhs(m, c0, u), O.ref_rhs(r, c0, u))
    a = O.step(m, c0, 1e-3, 2, u)
    b = O.ref_step(r, c0, 1e-3, 2, u)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("N", range(2, 11))
def test_gll_identities(N):
    """MeshQuadratureTest (tests/nekwave_test.cpp:65-129) on the restated operators."""
    z, w, D, w3 = O.gll(N)
    Dm = D.reshape(N, N).T  # Dm[i, j] = D[i + j N]
    assert abs(w.sum() - 2.0) < 1e-12
    np.testing.assert_allclose(z + z[::-1], 0.0, atol=1e-12)
    np.testing.assert_allclose(Dm @ np.ones(N), 0.0, atol=1e-11)
    np.testing.assert_allclose(Dm @ z, 1.0, atol=1e-11)
    m = O.box_mesh(N, (2, 2, 2), (-1, -1, -1), (1, 1, 1))
    vol = sum(float(np.sum(m.jac[e * N ** 3:(e + 1) * N ** 3] * w3)) for e in range(m.nelt))
    assert abs(vol - 8.0) < 1e-10


def test_periodic_pairing_coordinates():
    """PeriodicBCTest (tests/nekwave_test.cpp:353-414): periodic partners coincide up to
    the period; PEC faces have no partner."""
    m = O.box_mesh(4, (3, 2, 2), (0, 0, 0), (2, 1, 1), (True, False, True))
    have = m.vplus >= 0
    dx = np.abs(m.x[m.vmin[have]] - m.x[m.vplus[have]])
    dy = np.abs(m.y[m.vmin[have]] - m.y[m.vplus[have]])
    dz = np.abs(m.zc[m.vmin[have]] - m.zc[m.vplus[have]])
    assert np.all((dx < 1e-12) | (np.abs(dx - 2.0) < 1e-12))
    assert np.all(dy < 1e-12)
    assert np.all((dz < 1e-12) | (np.abs(dz - 1.0) < 1e-12))
    assert np.all(m.bc[~have] == 1)


def test_tm110_oracle_tracks_analytic():
    """The oracle itself follows the TM110 cavity mode on the PEC unit cube."""
    m = O.box_mesh(5, (4, 4, 4), (0, 0, 0), (1, 1, 1))
    dt = 0.5 * O.dxmin(m)
    n = m.npts
    u = np.zeros(6 * n)
    u[2 * n:3 * n] = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    steps = 40
    uu, _ = O.step(m, 1.0, dt, steps, u)
    T, w = steps * dt, np.pi * np.sqrt(2.0)
    ex = np.zeros_like(u)
    ex[2 * n:3 * n] = np.sin(np.pi * m.x) * np.sin(np.pi * m.y) * np.cos(w * T)
    ex[3 * n:4 * n] = -np.sin(np.pi * m.x) * np.cos(np.pi * m.y) * np.sin(w * T) / np.sqrt(2.0)
    ex[4 * n:5 * n] = np.cos(np.pi * m.x) * np.sin(np.pi * m.y) * np.sin(w * T) / np.sqrt(2.0)
    assert np.linalg.norm(uu - ex) / np.linalg.norm(ex) < 1e-4
