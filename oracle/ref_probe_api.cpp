// ref_probe_api.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry point around the reference's own ProbeManager::init (src/probe.cpp,
// compiled unchanged into oracle/_ref/libnwref_host.so): locates probe points
// on a reference Mesh and copies out each probe's element offset and its N^3
// tensor Lagrange weights, which the probe-location tests compare with libnwb's
// box-probe locator and the Python one.
#include "mesh.hpp"
#include "probe.hpp"

#include <array>
#include <cstring>
#include <vector>

extern "C" {

// xyz: [nprobes][3]; elem_offset: [nprobes] (element * N^3); weights: [nprobes][N^3].
void nwref_probe_init(void* mesh, int nprobes, const double* xyz, long* elem_offset,
                      double* weights) {
    const Mesh* m = static_cast<Mesh*>(mesh);
    std::vector<std::array<double, 3>> pts(nprobes);
    for (int q = 0; q < nprobes; ++q) pts[q] = {{xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]}};
    ProbeManager pm;
    pm.init(*m, pts, "none");
    const size_t n3 = static_cast<size_t>(m->getN()) * m->getN() * m->getN();
    for (int q = 0; q < nprobes; ++q) {
        const ProbePoint& p = pm.getProbes()[q];
        elem_offset[q] = p.elemOffset;
        std::memcpy(weights + q * n3, p.interpWeights.data(), sizeof(double) * n3);
    }
}

}  // extern "C"
