"""Known answers of the reference's own studies and tests, for the oracle (CPU) and
libnwb (GPU).

The plane wave of the reference's convergence study
(examples/numerical_analysis/convergence_test/convergence_test.cpp:68-79, 89-187):
a TEM wave Ez = cos(pi x + pi y - omega t), Hx = Ez / sqrt 2, Hy = -Ez / sqrt 2,
omega = sqrt(2) pi, in a periodic box [-1, 1]^2 x [-0.5, 0.5]; dt from the
reference's automatic CFL (safety 0.2: 0.2 * 1.75 / sqrt 3 * dxmin), rounded down so
that a whole number of steps reaches T; the error is the discrete L2 norm of
(Ez, Hx, Hy) with the quadrature weights J w_i w_j w_k, as the study forms it.  One
period instead of the study's ten, and two elements in z (the wave does not vary
along z) so that no element is its own z-neighbour.  Below it, the cavity modes of the
reference's two regression tests."""
import math

import numpy as np

from oracle import oracle as O

OMEGA = math.sqrt(2.0) * math.pi
PERIOD = math.sqrt(2.0)


def mesh(N, nel):
    return O.box_mesh(N, (nel, nel, 2), (-1.0, -1.0, -0.5), (1.0, 1.0, 0.5), (True, True, True))


def exact(m, t):
    n = m.npts
    ez = np.cos(math.pi * m.x + math.pi * m.y - OMEGA * t)
    u = np.zeros(6 * n)
    u[2 * n:3 * n] = ez
    u[3 * n:4 * n] = ez / math.sqrt(2.0)
    u[4 * n:5 * n] = -ez / math.sqrt(2.0)
    return u


def steps_for(m, periods=1):
    """(dt, nsteps) reaching periods * PERIOD exactly (convergence_test.cpp:131-136)."""
    T = periods * PERIOD
    dt = 0.2 * 1.75 / math.sqrt(3.0) * O.dxmin(m)
    ns = max(1, math.ceil(T / dt))
    return T / ns, ns


def l2_error(m, u, t):
    n = m.npts
    d = u - exact(m, t)
    w = m.w
    w3 = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    dv = m.jac * np.tile(w3, m.nelt)
    sq = d[2 * n:3 * n] ** 2 + d[3 * n:4 * n] ** 2 + d[4 * n:5 * n] ** 2
    return math.sqrt(float(np.sum(sq * dv)))


def eoc(e_coarse, e_fine):
    """Empirical order of convergence for a halved element size."""
    return math.log(e_coarse / e_fine) / math.log(2.0)


# the studies: h-refinement at 5 points per direction (degree 4), p-refinement on 4 x 4 x 2
H_STUDY = [(5, nel) for nel in (2, 4, 8)]
P_STUDY = [(N, 4) for N in range(3, 9)]
EOC_MIN = 4.5  # degree 4: the study's expected order is 5
EOC_MIN_NOTE = "the last h-refinement pair at degree 4 converges at order >= 4.5"


# ---- the reference's two regression cavities (tests/3dboxpec_test, tests/3dboxper_test) ----
# Their NekCEM .rea meshes are not in the reference tree; the same modes run here on box
# meshes of 4 x 4 x 4 elements at 4 points per direction (the cases' order 4), central
# flux, 50 steps at the automatic dt of Case::preprocess (safety 0.4:
# dt = 0.4 * 1.75 / sqrt 3 * dxmin, src/case.cpp:207-210), against the cases' pass
# threshold of 0.05 relative L2.
MODE_THRESHOLD = 0.05
MODE_STEPS = 50


def mode_mesh(name, nel=4):
    if name == "3dboxpec":  # PEC cube [-1, 1]^3
        return O.box_mesh(4, (nel,) * 3, (-1.0,) * 3, (1.0,) * 3, (False,) * 3)
    # periodic cube [0, 2 pi]^3 (the case rescales its mesh to it, src/case.cpp:165-175)
    return O.box_mesh(4, (nel,) * 3, (0.0,) * 3, (2.0 * math.pi,) * 3, (True,) * 3)


def mode_exact(name, m, t):
    """The cases' exact fields (tests/3dboxpec_test/3dboxpec_test.cpp:29-47, 71-92;
    tests/3dboxper_test/3dboxper_test.cpp:25-35, 57-77); their initial conditions are
    these at t = 0."""
    n = m.npts
    x, y, z = m.x, m.y, m.zc
    u = np.zeros(6 * n)
    if name == "3dboxpec":
        pi = math.pi
        th = math.cos(pi * math.sqrt(3.0) * t) / math.sqrt(6.0)
        te = math.sin(pi * math.sqrt(3.0) * t) / math.sqrt(2.0)
        u[0:n] = -np.cos(pi * x) * np.sin(pi * y) * np.sin(pi * z) * te
        u[n:2 * n] = np.sin(pi * x) * np.cos(pi * y) * np.sin(pi * z) * te
        u[3 * n:4 * n] = -np.sin(pi * x) * np.cos(pi * y) * np.cos(pi * z) * th
        u[4 * n:5 * n] = -np.cos(pi * x) * np.sin(pi * y) * np.cos(pi * z) * th
        u[5 * n:6 * n] = 2.0 * np.cos(pi * x) * np.cos(pi * y) * np.sin(pi * z) * th
    else:
        w = math.sqrt(3.0)
        th, te = math.sin(w * t) / w, math.cos(w * t)
        u[n:2 * n] = np.cos(x) * np.sin(y) * np.sin(z) * te
        u[2 * n:3 * n] = np.cos(x) * np.cos(y) * np.cos(z) * te
        u[3 * n:4 * n] = 2.0 * np.cos(x) * np.sin(y) * np.cos(z) * th
        u[4 * n:5 * n] = -np.sin(x) * np.cos(y) * np.cos(z) * th
        u[5 * n:6 * n] = np.sin(x) * np.sin(y) * np.sin(z) * th
    return u


def mode_dt(m):
    return 0.4 * 1.75 / math.sqrt(3.0) * O.dxmin(m)


def mode_rel_l2(m, u, t, name):
    """The cases' relative L2 error: all six components, weights J w3."""
    n = m.npts
    ex = mode_exact(name, m, t)
    w = m.w
    w3 = (w[:, None, None] * w[None, :, None] * w[None, None, :]).ravel()
    dv = m.jac * np.tile(w3, m.nelt)
    d = u - ex
    num = sum(d[c * n:(c + 1) * n] ** 2 for c in range(6))
    den = sum(ex[c * n:(c + 1) * n] ** 2 for c in range(6))
    return math.sqrt(float(np.sum(num * dv)) / float(np.sum(den * dv)))
