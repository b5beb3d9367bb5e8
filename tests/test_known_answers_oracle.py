"""CPU: the oracle on the known answers of the reference (tests/known_answers.py): the
plane wave of its convergence study (one period, h- and p-refinement, central and
upwind flux) and the cavity modes of its two regression cases.  The GPU path is held
to the same answers in test_gpu_validation_against_known_answers.py."""
import pytest

from oracle import oracle as O
from tests import known_answers as W


@pytest.mark.parametrize("c0", [0.0, 1.0])
def test_oracle_plane_wave_h_refinement(c0):
    errs = []
    for N, nel in W.H_STUDY:
        m = W.mesh(N, nel)
        dt, ns = W.steps_for(m)
        u, _ = O.step(m, c0, dt, ns, W.exact(m, 0.0))
        errs.append(W.l2_error(m, u, ns * dt))
    assert errs[0] > errs[1] > errs[2]
    assert W.eoc(errs[1], errs[2]) >= W.EOC_MIN, (errs, W.EOC_MIN_NOTE)


@pytest.mark.parametrize("c0", [0.0, 1.0])
def test_oracle_plane_wave_p_refinement(c0):
    errs = []
    for N, nel in W.P_STUDY:
        m = W.mesh(N, nel)
        dt, ns = W.steps_for(m)
        u, _ = O.step(m, c0, dt, ns, W.exact(m, 0.0))
        errs.append(W.l2_error(m, u, ns * dt))
    assert all(a > b for a, b in zip(errs, errs[1:])), errs  # spectral: every order helps
    assert errs[-1] < 1e-6, errs


@pytest.mark.parametrize("name", ["3dboxpec", "3dboxper"])
def test_oracle_regression_cavity_modes(name):
    """The reference's 3dboxpec and 3dboxper regression cases on box meshes: under
    their 0.05 threshold on 4^3 elements, and (a check that the threshold means
    something) above it on 2^3."""
    errs = {}
    for nel in (2, 4):
        m = W.mode_mesh(name, nel)
        dt = W.mode_dt(m)
        u, _ = O.step(m, 0.0, dt, W.MODE_STEPS, W.mode_exact(name, m, 0.0))
        errs[nel] = W.mode_rel_l2(m, u, W.MODE_STEPS * dt, name)
    assert errs[4] <= W.MODE_THRESHOLD < errs[2], errs
