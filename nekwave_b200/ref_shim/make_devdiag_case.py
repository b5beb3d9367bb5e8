"""Writes a device-diagnostics variant of the reference's Case::simulate.

    python make_devdiag_case.py <reference src/case.cpp> <output .cpp>

Reads the reference's case.cpp where it lies and writes a copy (into the build
directory only) whose time loop no longer downloads the full state every step:

  * the per-step DgSolver::downloadState (src/case.cpp:588) becomes a download of
    the probe elements only (nwb_dropin::download_probe_elements), which is all
    ProbeManager::record reads;
  * the save block (src/case.cpp:604-625) runs in the background: its body
    becomes a job of an nwb_dropin::SnapshotWriter, which copies the state to
    pinned host memory behind the steps queued so far and runs the job (derived
    fields, Hdf5Writer::writeStep) on its own thread with that copy, in step
    order, while the loop goes on; the writer finishes before simulate() returns.
    Inside the job the names the body uses, state_, currentTime_ and step, refer
    to the snapshot and its step and time;
  * the full state is downloaded after the loop, as before;
  * max|E|, max|H| and the energy of the output steps (src/case.cpp:632-634) are
    reduced on the device (nwb_dropin::device_diagnostics).

Each edit is anchored on one statement of the original and must match exactly
once; a reference whose loop has changed makes this script fail instead of
producing a front end that silently reads stale host data.
"""
import sys


def replace_once(text, old, new, after=None):
    start = 0
    if after is not None:
        start = text.index(after)
    i = text.find(old, start)
    if i < 0 or (after is None and text.count(old) != 1):
        raise SystemExit(f"make_devdiag_case: anchor not found exactly once: {old.strip()!r}")
    return text[:i] + new + text[i + len(old):]


def transform(src: str) -> str:
    out = replace_once(src, '#include "case.hpp"\n', '#include "case.hpp"\n#include "device_diag.hpp"\n')
    # the in-loop download (the one inside the "Case::downloadState" range)
    out = replace_once(out, "dgSolver_->downloadState(state_.data(), state_.size());",
                       "nwb_dropin::download_probe_elements(*dgSolver_, probes_, "
                       "mesh_->getNumPointsPerElement(), state_);",
                       after='nvtxRangePushA("Case::downloadState");')
    out = replace_once(out, "const int saveFreq = std::max(1, config_.saveFreq);\n",
                       "const int saveFreq = std::max(1, config_.saveFreq);\n"
                       "    nwb_dropin::SnapshotWriter snapWriter;  // the save block's background writer\n")
    out = replace_once(out, "if (hdf5Writer_ && (step % saveFreq == 0 || isFinal)) {\n",
                       "if (hdf5Writer_ && (step % saveFreq == 0 || isFinal)) {\n"
                       "            snapWriter.save(*dgSolver_, step, currentTime_,\n"
                       "                            [this, npts](int step, double currentTime_, const double* snap) {\n"
                       "            const struct { const double* p; const double* data() const { return p; } } "
                       "state_{snap};\n")
    end = ("hdf5Writer_->writeStep(step, currentTime_, state_.data(), npts, &derived);\n"
           "#ifndef USE_HIP\n            nvtxRangePop();\n#endif\n")
    out = replace_once(out, end, end + "            });\n")
    out = replace_once(out, "double maxE = getMaxE();", "double maxE = 0.0, maxH = 0.0, energy = 0.0;\n"
                       "            nwb_dropin::device_diagnostics(*dgSolver_, &maxE, &maxH, &energy);")
    out = replace_once(out, "double maxH = getMaxH();", "")
    out = replace_once(out, "double energy = computeTotalEnergy();", "")
    return out


def main():
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    with open(sys.argv[1]) as f:
        src = f.read()
    with open(sys.argv[2], "w") as f:
        f.write(transform(src))


if __name__ == "__main__":
    main()
