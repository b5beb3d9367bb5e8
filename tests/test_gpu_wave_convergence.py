"""The plane-wave known answer of the reference's convergence study on libnwb
(examples/numerical_analysis/convergence_test/convergence_test.cpp: a TEM wave in a
periodic box, h-refinement at degree 4 and p-refinement at 3..8 points, central and
upwind flux; one period here): each run equals the oracle's (pinned to the
reference's own build) to the step-parity tolerance, and the errors against the
analytic wave converge as the study expects (tests/plane_wave.py)."""
import pytest

from oracle import oracle as O
from tests import plane_wave as W
from tests.gpu_helpers import record, rel_l2, solver_for

pytestmark = pytest.mark.gpu

STEPS_TOL = 1e-10  # relative L2 to the oracle after up to ~220 steps


def _run(N, nel, c0):
    m = W.mesh(N, nel)
    dt, ns = W.steps_for(m)
    u0 = W.exact(m, 0.0)
    s = solver_for(m, c0)
    s.uploadState(u0)
    s.steps(dt, ns)
    got = s.downloadState()
    s.finalize()
    want, _ = O.step(m, c0, dt, ns, u0)
    return rel_l2(got, want), W.l2_error(m, got, ns * dt), W.l2_error(m, want, ns * dt), ns


@pytest.mark.parametrize("c0", [0.0, 1.0])
def test_plane_wave_convergence_matches_the_oracle_and_the_analytic_wave(gpu, c0):
    rows = {}
    for study, cases in (("h", W.H_STUDY), ("p", W.P_STUDY)):
        errs = []
        for N, nel in cases:
            d, e_gpu, e_ref, ns = _run(N, nel, c0)
            assert d < STEPS_TOL, (study, N, nel, d)
            assert abs(e_gpu - e_ref) <= 1e-6 * e_ref + 1e-13, (study, N, nel, e_gpu, e_ref)
            errs.append(e_gpu)
            rows[f"{study} N={N} nel={nel}"] = dict(steps=ns, rel_l2_vs_oracle=d, l2_error=e_gpu)
        if study == "h":
            assert errs[0] > errs[1] > errs[2]
            assert W.eoc(errs[1], errs[2]) >= W.EOC_MIN, (errs, W.EOC_MIN_NOTE)
        else:
            assert all(a > b for a, b in zip(errs, errs[1:])), errs
            assert errs[-1] < 1e-6, errs
    record(f"plane_wave_c0_{c0:g}.json", rows)
