// device_diag.hpp -- device-resident diagnostics for the reference's front end on
// the drop-in DgSolver (dg_solver.cpp in this directory).
//
// Case::simulate downloads the whole state after every step (src/case.cpp:588)
// for its probes (:596) and, every output step, for max|E|, max|H| and the energy
// (:632-634), all computed on the host.  With these calls a front end downloads
// only what it reads:
//   download_probe_elements  the N^3 nodes of each probe's element (the only
//                            nodes ProbeManager::record reads, src/probe.cpp:192-216)
//                            into their places of the host state, so record()
//                            gives the same values as after a full download;
//   device_diagnostics       max|E| and max|H| (equal to Case::getMaxE/getMaxH
//                            bit for bit) and the energy (Case::computeTotalEnergy
//                            to rounding) reduced on the device.
//   SnapshotWriter           the save steps' output (src/case.cpp:604-625) off the
//                            time loop: the state is copied to pinned host memory
//                            behind the steps already queued while later steps run,
//                            and the writer's work (derived fields, Hdf5Writer::
//                            writeStep) runs on a background thread, in step order.
// The full state then crosses the host link only at save steps, and not inside the
// loop's critical path.
// make_devdiag_case.py turns the reference's case.cpp into such a front end.
#pragma once

#include <functional>
#include <memory>
#include <vector>

class DgSolver;
class ProbeManager;

namespace nwb_dropin {

void download_probe_elements(const DgSolver& solver, const ProbeManager& probes, int nodes_per_elem,
                             std::vector<double>& state);
void device_diagnostics(const DgSolver& solver, double* max_e, double* max_h, double* energy);

// Background writer of state snapshots.  save() queues a copy of the solver's state
// as of the steps run so far and returns; once the copy is complete, job(step, time,
// state) runs on the writer thread with the snapshot ([6][npts], the layout of
// DgSolver::downloadState).  Jobs run one at a time in save() order; two snapshot
// buffers are used in turn, so a save waits only when the job two saves back has
// not finished.  A snapshot's job is queued when its copy is complete, which the
// next save() or finish() checks.  finish() waits for every queued copy and job and
// rethrows the first exception a job threw (the jobs after it are dropped); the
// destructor does the same and reports the exception on stderr.  Only the thread
// that calls save() touches the solver, which must outlive the last finish(); a job
// must not touch it.
class SnapshotWriter {
public:
    using Job = std::function<void(int step, double time, const double* state)>;
    SnapshotWriter();
    ~SnapshotWriter();
    SnapshotWriter(const SnapshotWriter&) = delete;
    SnapshotWriter& operator=(const SnapshotWriter&) = delete;
    void save(const DgSolver& solver, int step, double time, Job job);
    void finish();

private:
    struct State;
    std::unique_ptr<State> st_;
};

}  // namespace nwb_dropin
