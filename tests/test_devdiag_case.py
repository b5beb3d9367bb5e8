"""CPU: the device-diagnostics front end that nekwave_b200/ref_shim/make_devdiag_case.py
makes from the reference's src/case.cpp (skipped where the reference sources are not
on this machine; REF names their root as in the Makefiles)."""
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASE = os.path.join(os.environ.get("REF", "/root/reference"), "src", "case.cpp")

pytestmark = pytest.mark.skipif(not os.path.exists(CASE), reason="reference sources not present")


def _transform():
    sys.path.insert(0, os.path.join(ROOT, "nekwave_b200", "ref_shim"))
    try:
        import make_devdiag_case as M
    finally:
        sys.path.pop(0)
    src = open(CASE).read()
    return src, M.transform(src)


def _simulate_body(text):
    i = text.index("void Case::simulate()")
    return text[i:text.index("void Case::postprocess()", i)]


def test_the_time_loop_downloads_only_the_probe_elements():
    src, out = _transform()
    a, b = _simulate_body(src), _simulate_body(out)
    # the reference: a full download inside the loop and one after it
    assert a.count("dgSolver_->downloadState(state_.data(), state_.size());") == 2
    # the front end: only the one after the loop, the probe elements per step
    assert b.count("dgSolver_->downloadState(state_.data(), state_.size());") == 1
    assert b.rindex("dgSolver_->downloadState(") > b.rindex("while (true)")
    assert b.count("nwb_dropin::download_probe_elements(") == 1


def test_diagnostics_on_the_device_and_saves_on_the_background_writer():
    src, out = _transform()
    b = _simulate_body(out)
    for host_call in ("getMaxE()", "getMaxH()", "computeTotalEnergy()"):
        assert host_call not in b, host_call
    assert b.count("nwb_dropin::device_diagnostics(*dgSolver_, &maxE, &maxH, &energy);") == 1
    assert b.count("nwb_dropin::SnapshotWriter snapWriter;") == 1
    assert b.count("snapWriter.save(*dgSolver_, step, currentTime_,") == 1
    # the save block's writeStep runs inside the job handed to the writer
    save = b.index("snapWriter.save(")
    write = b.index("hdf5Writer_->writeStep(step, currentTime_, state_.data(), npts, &derived);")
    close = b.index("});", write)
    assert save < write < close
    # nothing else of the reference's file changed
    rest = re.sub(r"void Case::simulate\(\).*?void Case::postprocess\(\)", "", out, flags=re.S)
    rest_src = re.sub(r"void Case::simulate\(\).*?void Case::postprocess\(\)", "", src, flags=re.S)
    assert rest.replace('#include "device_diag.hpp"\n', "") == rest_src


def test_the_generator_refuses_a_changed_reference():
    sys.path.insert(0, os.path.join(ROOT, "nekwave_b200", "ref_shim"))
    try:
        import make_devdiag_case as M
    finally:
        sys.path.pop(0)
    src = open(CASE).read().replace("double maxE = getMaxE();", "double maxE = getMaxNormE();")
    with pytest.raises(SystemExit):
        M.transform(src)
