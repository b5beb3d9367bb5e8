"""CPU: the oracle on the plane-wave known answer of the reference's convergence study
(one period, h- and p-refinement, central and upwind flux); the GPU path is held to
the same answer in test_gpu_wave_convergence.py."""
import pytest

from oracle import oracle as O
from tests import plane_wave as W


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
