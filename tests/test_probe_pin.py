"""Probe location pinned to the reference's own ProbeManager::init
(src/probe.cpp:33-96, compiled from its source into oracle/_ref/libnwref_host.so):
libnwb's box-probe locator (nwb_box_probes, which nwb_pool_add_box uses) and the
Python one (nekwave_b200.pool.locate_probes, used by DgSolver.probesAt) must pick
the same element and give bit-identical tensor Lagrange weights for seeded
points, points outside the box (clamped), points on GLL nodes and points on
element boundaries."""
import ctypes as C

import numpy as np
import pytest

from nekwave_b200 import Mesh, _lib
from nekwave_b200.pool import locate_probes
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="reference host build absent")

CASES = [(5, (4, 3, 2), (0.0, -1.0, 0.5), (1.0, 1.0, 2.0)),
         (8, (3, 3, 3), (0.0, 0.0, 0.0), (1.7, 0.9, 1.3)),
         (4, (6, 2, 5), (-0.5, 0.0, 0.0), (0.5, 2.0, 1.0))]


def points_for(N, nel, lo, hi, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    lo, hi, nel = np.array(lo), np.array(hi), np.array(nel)
    pts = [lo + (hi - lo) * rng.uniform(0, 1, 3) for _ in range(12)]
    pts += [lo - 0.3 * (hi - lo), hi + 0.1, np.array([lo[0] - 1.0, hi[1] + 2.0, 0.5 * (lo[2] + hi[2])])]
    h = (hi - lo) / nel
    z = O.gll(N)[0]
    # on GLL nodes (exact reference coordinates of element (1, 0, last))
    pts.append(lo + h * (np.array([1, 0, nel[2] - 1]) + (z[[1, 0, N - 2]] + 1.0) / 2.0))
    # on element boundaries (ties between neighbours)
    pts.append(lo + h * np.array([1.0, 1.0, 1.0]))
    pts.append(lo + h * np.array([2.0, 0.5, float(nel[2])]))
    return np.array(pts)


def tensor(w1d, N):
    wr, ws, wt = w1d[:N], w1d[N:2 * N], w1d[2 * N:]
    out = np.empty(N ** 3)
    for k in range(N):
        for j in range(N):
            for i in range(N):
                out[i + N * (j + N * k)] = wr[i] * ws[j] * wt[k]  # src/probe.cpp: Lr[i]*Ls[j]*Lt[k]
    return out


@pytest.mark.parametrize("N,nel,lo,hi", CASES)
def test_box_probes_equal_probe_manager(N, nel, lo, hi):
    pts = points_for(N, nel, lo, hi, N)
    off_ref, w_ref = O.ref_probes(N, nel, lo, hi, pts)
    P = len(pts)
    elem = np.zeros(P, np.int32)
    w1d = np.zeros(P * 3 * N)
    xyz = np.ascontiguousarray(pts)
    _lib.check(_lib.lib().nwb_box_probes(N, nel[0], nel[1], nel[2], lo[0], hi[0], lo[1], hi[1],
                                         lo[2], hi[2], P, _lib.dptr(xyz), _lib.iptr(elem),
                                         _lib.dptr(w1d)))
    np.testing.assert_array_equal(elem.astype(np.int64) * N ** 3, off_ref)
    for q in range(P):
        np.testing.assert_array_equal(tensor(w1d[q * 3 * N:(q + 1) * 3 * N], N), w_ref[q])


@pytest.mark.parametrize("N,nel,lo,hi", CASES)
def test_python_locate_probes_equal_probe_manager(N, nel, lo, hi):
    pts = points_for(N, nel, lo, hi, 100 + N)
    off_ref, w_ref = O.ref_probes(N, nel, lo, hi, pts)
    mesh = Mesh(N)
    mesh.createBoxMesh(*nel, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])
    elems, w1d = locate_probes(mesh, [tuple(p) for p in pts])
    np.testing.assert_array_equal(elems.astype(np.int64) * N ** 3, off_ref)
    w1d = w1d.reshape(len(pts), 3 * N)
    for q in range(len(pts)):
        np.testing.assert_array_equal(tensor(w1d[q], N), w_ref[q])
