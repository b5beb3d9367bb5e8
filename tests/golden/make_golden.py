"""Generates the golden vectors in tests/golden/ from the reference itself.

The reference is compiled from its own sources by oracle/Makefile into
oracle/_ref/libnwref_host.so (its Mesh and its CUDA kernel bodies run on the
host, single rank, lift summed in face-point order).  Each case stores the
inputs, the reference's right-hand side and its state after a few LSRK45
steps, plus a checksum of its mesh arrays.  Run:

    make -C oracle && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import oracle as O  # noqa: E402

# name: (N, nel, lo, hi, periodic, c0, ic, steps, dt)
CASES = {
    # MaxwellStabilityTest geometry (tests/nekwave_test.cpp:212-293)
    "stability_n4": (4, (2, 2, 2), (-.5, -.5, -.5), (.5, .5, .5), (0, 0, 0), 1.0, "pulse50", 5, 0.005),
    # TM110 cavity on the PEC unit cube, 4^3 elements, 5 points per direction
    "tm110_n5": (5, (4, 4, 4), (0, 0, 0), (1, 1, 1), (0, 0, 0), 1.0, "tm110", 10, None),
    # fully periodic, central flux, 8 points per direction, random state
    "periodic_n8": (8, (3, 2, 2), (0, 0, 0), (1, 1, 1), (1, 1, 1), 0.0, "random", 2, 1e-3),
    # mixed periodic/PEC on a non-cubic box, 3 points per direction
    "mixed_n3": (3, (2, 3, 4), (0, 0, 0), (2, 2, 1), (1, 0, 1), 1.0, "random", 3, 2e-3),
}


def initial_state(m, ic, seed=0):
    n = m.npts
    u = np.zeros(6 * n)
    if ic == "pulse50":
        u[2 * n:3 * n] = np.exp(-50.0 * (m.x ** 2 + m.y ** 2 + m.zc ** 2))
    elif ic == "tm110":
        u[2 * n:3 * n] = np.sin(np.pi * m.x) * np.sin(np.pi * m.y)
    else:
        u[:] = np.random.Generator(np.random.PCG64(seed)).standard_normal(6 * n)
    return u


def mesh_checksum(m):
    parts = [m.D, m.w3, m.jac, m.met.ravel(), m.nx, m.ny, m.nz, m.dA,
             m.vmin.astype(np.float64), m.vplus.astype(np.float64), m.bc.astype(np.float64)]
    return np.array([float(np.sum(p * np.arange(1, p.size + 1) % 7.0)) for p in parts])


def main():
    for name, (N, nel, lo, hi, per, c0, ic, steps, dt) in CASES.items():
        m = O.ref_box_mesh(N, nel, lo, hi, per)
        if dt is None:
            dt = 0.5 * m.dxmin_ref
        u0 = initial_state(m, ic)
        rhs = O.ref_rhs(m, c0, u0)
        u1, k1 = O.ref_step(m, c0, dt, steps, u0)
        energies = []
        uu = u0.copy(); kk = np.zeros_like(u0)
        for _ in range(steps):
            uu, kk = O.ref_step(m, c0, dt, 1, uu, kk)
            energies.append(O.energy(m, uu))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), N=N, nel=nel, lo=lo, hi=hi,
                            periodic=per, c0=c0, dt=dt, steps=steps, u0=u0, rhs=rhs, u1=u1,
                            k1=k1, energy0=O.energy(m, u0), energies=np.array(energies),
                            dxmin=m.dxmin_ref, mesh_checksum=mesh_checksum(m))
        print(name, m.npts, "points")


if __name__ == "__main__":
    main()
