"""Shared helpers of the GPU parity tests (imported by test modules only)."""
import json
import os

import numpy as np

from nekwave_b200 import DgSolver, Mesh
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def record(name: str, data: dict) -> None:
    """Write a measurement a GPU test takes (timings, parity figures) as JSON into
    the directory NWB_TEST_OUT names (default: test_out/ at the repository root)."""
    out = os.environ.get("NWB_TEST_OUT", os.path.join(ROOT, "test_out"))
    os.makedirs(out, exist_ok=True)
    with open(os.path.join(out, name), "w") as f:
        json.dump(data, f, indent=1)


def solver_for(m: "O.MeshArrays", c0: float, precision: str = "fp64",
               true_pmc: bool = False) -> DgSolver:
    """libnwb solver on exactly the oracle's mesh arrays."""
    mesh = Mesh.from_arrays(m.N, m.nelt, z=m.z, w=m.w, D=m.D, w3=m.w3, jac=m.jac, met=m.met,
                            vmin=m.vmin, vplus=m.vplus, bc=m.bc, nx=m.nx, ny=m.ny, nz=m.nz,
                            dA=m.dA, x=m.x, y=m.y, zc=m.zc)
    s = DgSolver(precision)
    s.initialize(mesh, c0, true_pmc=true_pmc)
    s._keep_mesh = mesh
    return s


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def random_state(m, seed):
    return np.random.Generator(np.random.PCG64(seed)).standard_normal(6 * m.npts)


def smooth_state(m, seed):
    """Band-limited seeded fields (Gaussian pulses in all six components)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lo = np.array([m.x.min(), m.y.min(), m.zc.min()])
    hi = np.array([m.x.max(), m.y.max(), m.zc.max()])
    u = np.zeros(6 * m.npts)
    for c in range(6):
        r0 = lo + (hi - lo) * rng.uniform(0.3, 0.7, 3)
        sig = 0.15 * float(np.min(hi - lo))
        u[c * m.npts:(c + 1) * m.npts] = np.exp(-((m.x - r0[0]) ** 2 + (m.y - r0[1]) ** 2 +
                                                  (m.zc - r0[2]) ** 2) / sig ** 2)
    return u


def shuffled_box_mesh(N, nel, lo, hi, seed, rotate=True):
    """A box mesh (PEC walls) whose elements are numbered in a seeded random order
    and, with rotate, every other element has its local frame turned 90 degrees
    about z (its faces renumbered accordingly): neighbour faces then meet with
    non-identity orientations and the element order carries no structure."""
    corners, fk, fb, ff = O.box_corners(nel, lo, hi, (False, False, False))
    nelt = corners.shape[0]
    rot = (np.arange(nelt) % 2 == 1) if rotate else np.zeros(nelt, bool)
    newface = np.array([3, 0, 1, 2, 4, 5])  # old face -> face of the turned frame
    cr, fk2, fb2, ff2 = corners.copy(), fk.copy(), fb.copy(), ff.copy()
    for e in np.nonzero(rot)[0]:
        cr[e] = corners[e][[1, 2, 3, 0, 5, 6, 7, 4]]
        fk2[e, newface] = fk[e]
        fb2[e, newface] = fb[e]
        ff2[e, newface] = ff[e]
    has = fb2 >= 0
    nbrot = np.zeros_like(has)
    nbrot[has] = rot[fb2[has]]
    ff2[nbrot] = newface[ff2[nbrot]]
    perm = np.random.Generator(np.random.PCG64(seed)).permutation(nelt)
    inv = np.empty(nelt, np.int64)
    inv[perm] = np.arange(nelt)
    fb3 = fb2[perm].copy()
    fb3[fb3 >= 0] = inv[fb3[fb3 >= 0]]
    return O.hex_mesh(N, cr[perm], fk2[perm], fb3, ff2[perm])
