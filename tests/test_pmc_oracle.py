"""The oracle's true-PMC option (the checker of libnwb's NWB_SOLVER_TRUE_PMC),
pinned to an analytic cavity mode on the CPU.

The reference mirrors PMC faces as PEC walls (src/dg_solver.cpp:92-98,
src/device/dg_kernels.cu:243-251), so no reference output exists for a true PMC
wall.  The unit cube with PMC walls at x = 0, 1 and PEC walls elsewhere carries
the mode (c = 1, omega = pi sqrt 2)
    Ez = cos(pi x) sin(pi y) cos(wt)
    Hx = -(1/sqrt 2) cos(pi x) cos(pi y) sin(wt),  Hy = -(1/sqrt 2) sin(pi x) sin(pi y) sin(wt)
(n x H = 0 on the PMC walls, n x E = 0 on the PEC walls).  The oracle with the
option tracks it as closely as the PEC-cube TM110 mode is tracked; with the
option off (the reference's behaviour) the walls reflect it wrongly."""
import numpy as np

from oracle import oracle as O


def pmc_x_cube(N, nel):
    m = O.box_mesh(N, nel, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    fp = np.arange(m.nfp)
    face = (fp // (N * N)) % 6
    m.bc = m.bc.copy()
    m.bc[(face == 1) | (face == 3)] = 2  # r = +-1: the x walls of a box element ...
    xw = np.isclose(m.x[m.vmin], 0.0) | np.isclose(m.x[m.vmin], 1.0)
    m.bc[(m.bc == 2) & ~xw] = 0  # ... on the boundary only
    m.bc[(m.bc == 0) & (m.vplus < 0)] = 1
    return m


def mode(m, t):
    w = np.pi * np.sqrt(2.0)
    n = m.npts
    u = np.zeros(6 * n)
    u[2 * n:3 * n] = np.cos(np.pi * m.x) * np.sin(np.pi * m.y) * np.cos(w * t)
    u[3 * n:4 * n] = -np.cos(np.pi * m.x) * np.cos(np.pi * m.y) * np.sin(w * t) / np.sqrt(2.0)
    u[4 * n:5 * n] = -np.sin(np.pi * m.x) * np.sin(np.pi * m.y) * np.sin(w * t) / np.sqrt(2.0)
    return u


def test_true_pmc_option_tracks_the_pmc_cavity_mode():
    N, nel, steps = 5, (4, 4, 4), 100
    m = pmc_x_cube(N, nel)
    assert np.count_nonzero(m.bc == 2) == 2 * nel[1] * nel[2] * N * N
    dt = 0.5 * O.dxmin(m)
    u0 = mode(m, 0.0)
    exact = mode(m, steps * dt)
    pmc, _ = O.step(m, 1.0, dt, steps, u0, true_pmc=True)
    pec, _ = O.step(m, 1.0, dt, steps, u0, true_pmc=False)
    err_pmc = np.linalg.norm(pmc - exact) / np.linalg.norm(exact)
    err_pec = np.linalg.norm(pec - exact) / np.linalg.norm(exact)
    assert err_pmc < 1e-4, err_pmc
    assert err_pec > 100 * err_pmc, (err_pec, err_pmc)


def test_option_off_is_the_reference_behaviour():
    """With the option off a bc-2 point is a PEC mirror: the same RHS as bc 1."""
    m = pmc_x_cube(4, (2, 2, 2))
    u = np.random.Generator(np.random.PCG64(3)).standard_normal(6 * m.npts)
    as_pec = O.box_mesh(4, (2, 2, 2), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    np.testing.assert_array_equal(O.rhs(m, 1.0, u), O.rhs(as_pec, 1.0, u))
    assert not np.array_equal(O.rhs(m, 1.0, u, true_pmc=True), O.rhs(m, 1.0, u))
