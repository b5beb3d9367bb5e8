"""Known answers of the reference on libnwb (tests/known_answers.py).

The plane wave of the reference's convergence study
(examples/numerical_analysis/convergence_test/convergence_test.cpp: a TEM wave in a
periodic box, h-refinement at degree 4 and p-refinement at 3..8 points, central and
upwind flux; one period here) and the cavity modes of its regression cases
tests/3dboxpec_test and tests/3dboxper_test (box meshes in place of their missing
NekCEM meshes): each run equals the oracle's (pinned to the reference's own build) to
the step-parity tolerance, and its error against the analytic fields is what the
study and the cases expect.
"""
import pytest

from oracle import oracle as O
from tests import known_answers as W
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


@pytest.mark.parametrize("name", ["3dboxpec", "3dboxper"])
def test_regression_cavity_modes_under_the_reference_threshold(gpu, name):
    m = W.mode_mesh(name, 4)
    dt = W.mode_dt(m)
    u0 = W.mode_exact(name, m, 0.0)
    s = solver_for(m, 0.0)
    s.uploadState(u0)
    s.steps(dt, W.MODE_STEPS)
    got = s.downloadState()
    s.finalize()
    want, _ = O.step(m, 0.0, dt, W.MODE_STEPS, u0)
    d = rel_l2(got, want)
    err = W.mode_rel_l2(m, got, W.MODE_STEPS * dt, name)
    record(f"mode_{name}.json", dict(rel_l2_vs_oracle=d, rel_l2_vs_exact=err, steps=W.MODE_STEPS))
    assert d < STEPS_TOL, d
    assert err <= W.MODE_THRESHOLD, err
