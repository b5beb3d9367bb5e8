"""The plane-wave known answer of the reference's convergence study
(examples/numerical_analysis/convergence_test/convergence_test.cpp:68-79, 89-187):
a TEM wave Ez = cos(pi x + pi y - omega t), Hx = Ez / sqrt 2, Hy = -Ez / sqrt 2,
omega = sqrt(2) pi, in a periodic box [-1, 1]^2 x [-0.5, 0.5]; dt from the
reference's automatic CFL (safety 0.2: 0.2 * 1.75 / sqrt 3 * dxmin), rounded down so
that a whole number of steps reaches T; the error is the discrete L2 norm of
(Ez, Hx, Hy) with the quadrature weights J w_i w_j w_k, as the study forms it.  One
period instead of the study's ten, and two elements in z (the wave does not vary
along z) so that no element is its own z-neighbour."""
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
