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
// The full state then crosses the host link only at save steps.
// make_devdiag_case.py turns the reference's case.cpp into such a front end.
#pragma once

#include <vector>

class DgSolver;
class ProbeManager;

namespace nwb_dropin {

void download_probe_elements(const DgSolver& solver, const ProbeManager& probes, int nodes_per_elem,
                             std::vector<double>& state);
void device_diagnostics(const DgSolver& solver, double* max_e, double* max_h, double* energy);

}  // namespace nwb_dropin
