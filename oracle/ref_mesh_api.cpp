// ref_mesh_api.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points around the reference's own Mesh (src/mesh.cpp, compiled
// unchanged): builds a box mesh with Mesh::createBoxMesh and copies out the
// arrays the hot path consumes.  Linked into both oracle/_ref libraries.
#include "mesh.hpp"

#include <cstring>
#include <vector>

extern "C" {

// ---- reference Mesh (src/mesh.cpp) ------------------------------------------
void* nwref_mesh_box(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                     double ymin, double ymax, double zmin, double zmax, int px, int py,
                     int pz) {
    Mesh* mesh = new Mesh(N, 1);
    if (!mesh->createBoxMesh(nelx, nely, nelz, xmin, xmax, ymin, ymax, zmin, zmax, px != 0,
                             py != 0, pz != 0)) {
        delete mesh;
        return nullptr;
    }
    return mesh;
}

void nwref_mesh_free(void* h) { delete static_cast<Mesh*>(h); }

void nwref_mesh_sizes(void* h, long* nelt, long* npts, long* nfp) {
    const Mesh* m = static_cast<Mesh*>(h);
    *nelt = m->getNumElements();
    *npts = m->getTotalPoints();
    long n = 0;
    for (const auto& fd : m->getFaceData()) n += static_cast<long>(fd.points.size());
    *nfp = n;
}

// Node coordinates only (Mesh::getCoordX/Y/Z), for initial states of large meshes.
void nwref_mesh_coords(void* h, double* x, double* y, double* zc) {
    const Mesh* m = static_cast<Mesh*>(h);
    const long npts = m->getTotalPoints();
    std::memcpy(x, m->getCoordX().data(), sizeof(double) * npts);
    std::memcpy(y, m->getCoordY().data(), sizeof(double) * npts);
    std::memcpy(zc, m->getCoordZ().data(), sizeof(double) * npts);
}

double nwref_mesh_dxmin(void* h) { return static_cast<Mesh*>(h)->computeMinNodeDistance(); }

// Copies the mesh arrays out, face data flattened exactly as
// DgSolver::Impl::initialize does (src/dg_solver.cpp:76-112).
void nwref_mesh_export(void* h, double* z, double* w, double* D, double* w3, double* x,
                       double* y, double* zc, double* jac, double* met, int* vmin,
                       int* vplus, int* bc, double* nx, double* ny, double* nz, double* dA) {
    const Mesh* m = static_cast<Mesh*>(h);
    const int N = m->getN();
    const long npts = m->getTotalPoints();
    std::memcpy(z, m->getGllZ().data(), sizeof(double) * N);
    std::memcpy(w, m->getGllW().data(), sizeof(double) * N);
    std::memcpy(D, m->getD().data(), sizeof(double) * N * N);
    std::memcpy(w3, m->getW3().data(), sizeof(double) * N * N * N);
    std::memcpy(x, m->getCoordX().data(), sizeof(double) * npts);
    std::memcpy(y, m->getCoordY().data(), sizeof(double) * npts);
    std::memcpy(zc, m->getCoordZ().data(), sizeof(double) * npts);
    std::memcpy(jac, m->getJac().data(), sizeof(double) * npts);
    const std::vector<double>* mets[9] = {&m->getRx(), &m->getSx(), &m->getTx(),
                                          &m->getRy(), &m->getSy(), &m->getTy(),
                                          &m->getRz(), &m->getSz(), &m->getTz()};
    for (int c = 0; c < 9; ++c) std::memcpy(met + c * npts, mets[c]->data(), sizeof(double) * npts);
    long p = 0;
    for (const auto& fd : m->getFaceData()) {
        int code = 0;
        if (fd.bcType == "PEC" || fd.bcType == "W" || fd.bcType == "V" || fd.bcType == "v")
            code = 1;
        else if (fd.bcType == "PMC" || fd.bcType == "SYM" || fd.bcType == "S" ||
                 fd.bcType == "s")
            code = 2;
        for (const auto& pt : fd.points) {
            vmin[p] = pt.volIdxMinus;
            vplus[p] = pt.volIdxPlus;
            int c = code;
            if (pt.volIdxPlus < 0 && c == 0) c = 1;
            bc[p] = c;
            nx[p] = pt.nx;
            ny[p] = pt.ny;
            nz[p] = pt.nz;
            dA[p] = pt.dA;
            ++p;
        }
    }
}

}  // extern "C"
