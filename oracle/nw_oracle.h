/*
 * nw_oracle.h -- CPU restatement of NekWave's DG-SEM Maxwell right-hand side and
 * LSRK45 step, used ONLY as test infrastructure (the checker for the CUDA path and
 * the timed CPU baseline).  Nothing in the product links this library.
 *
 * Parity pin: every function here is checked against the reference compiled from its
 * own sources (oracle/Makefile -> oracle/_ref/) and against the committed golden
 * vectors in tests/golden/ that were generated from that build.
 *
 * Conventions follow the reference exactly:
 *   - N = GLL points per direction (reference Mesh::getN, src/mesh.cpp:56-61).
 *   - node index  e*N^3 + i + N*(j + N*k)          (src/mesh.cpp:216)
 *   - element index ex + nelx*(ey + nely*ez)       (src/mesh.cpp:705-707)
 *   - D column-major, D[i + j*N] = d l_j / dxi (xi_i) (src/mesh.cpp:113-131)
 *   - state SoA [Ex,Ey,Ez,Hx,Hy,Hz][npts]           (src/dg_solver.hpp:8-14)
 *   - face points flattened element-major, face 0..5, q, p (src/mesh.cpp:1003-1004,
 *     flattening in src/dg_solver.cpp:76-112)
 *   - metrics packed as met[9][npts] in the order rx,sx,tx,ry,sy,ty,rz,sz,tz.
 */
#ifndef NW_ORACLE_H
#define NW_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* GLL nodes z[N], weights w[N], derivative matrix D[N*N] (column-major), w3[N^3].
 * Restates Mesh::setupGLL (src/mesh.cpp:64-145). */
void nwo_gll(int N, double* z, double* w, double* D, double* w3);

/* Structured box mesh: restates Mesh::createBoxMesh (src/mesh.cpp:683-843),
 * Mesh::computeMetricsFromCorners (src/mesh.cpp:188-314), Mesh::setupFaceData
 * (src/mesh.cpp:985-1080) and the face flattening of DgSolver::Impl::initialize
 * (src/dg_solver.cpp:76-112).  Output arrays are caller-allocated:
 *   x,y,z,jac: npts; met: 9*npts; face arrays: nfp = 6*N*N*nelt.
 * bc[p] is the reference's per-point code: 1 = PEC mirror, 0 = neighbour trace.
 * Returns 0 on success, -1 on bad arguments. */
int nwo_box_mesh(int N, int nelx, int nely, int nelz,
                 double xmin, double xmax, double ymin, double ymax,
                 double zmin, double zmax, int px, int py, int pz,
                 double* x, double* y, double* z, double* jac, double* met,
                 int* vmin, int* vplus, int* bc,
                 double* nx, double* ny, double* nz, double* dA);

/* General hexahedral mesh from element corners (corners[nelt][8][3], the
 * reference's corner order, src/mesh.cpp:718-727) and a face table per
 * (element, face): kind 0 = interior (neighbour node found by coordinate match),
 * 1 = periodic (direct (p,q) map), 2 = PEC; fnb/fnf = neighbour element/face.
 * Restates computeMetricsFromCorners + setupFaceData + the flattening. */
int nwo_hex_mesh(int N, int nelt, const double* corners, const int* fkind,
                 const int* fnb, const int* fnf,
                 double* x, double* y, double* z, double* jac, double* met,
                 int* vmin, int* vplus, int* bc,
                 double* nx, double* ny, double* nz, double* dA);

/* Corners and face table of createBoxMesh (src/mesh.cpp:700-830). */
int nwo_box_corners(int nelx, int nely, int nelz,
                    double xmin, double xmax, double ymin, double ymax,
                    double zmin, double zmax, int px, int py, int pz,
                    double* corners, int* fkind, int* fnb, int* fnf);

/* Smallest distance between adjacent GLL nodes (src/mesh.cpp:883-930). */
double nwo_dxmin(int N, int nelt, const double* x, const double* y, const double* z);

/* Semi-discrete right-hand side rhs = M^{-1}(K u + F*): the reference's six
 * single-rank kernels in the order of DgSolver::Impl::step (src/dg_solver.cpp:393-487):
 * volume curl (src/device/dg_kernels.cu:41-155) twice, restrict (:170-190),
 * flux (:220-304), lift (:316-338, summed in face-point order), inverse mass
 * (:353-382).  u, rhs: 6*npts. */
void nwo_rhs(int N, int nelt, const double* D, const double* w3,
             const double* jac, const double* met,
             int nfp, const int* vmin, const int* vplus, const int* bc,
             const double* nx, const double* ny, const double* nz, const double* dA,
             double c0, const double* u, double* rhs);

/* Off (default): bc != 0 points are PEC mirrors, as in the reference
 * (src/device/dg_kernels.cu:243-251).  On: bc 2 points are PMC mirrors
 * ([[E]] = 0, [[H]] = -2 H^-), the checker of libnwb's NWB_SOLVER_TRUE_PMC. */
void nwo_set_true_pmc(int on);

/* nsteps LSRK45 steps of size dt (src/dg_solver.cpp:306-527, coefficients :58-69,
 * update kernel src/device/dg_kernels.cu:393-408).  u and k (6*npts) are updated
 * in place; k must be zero before the first step (src/dg_solver.cpp:125). */
void nwo_step(int N, int nelt, const double* D, const double* w3,
              const double* jac, const double* met,
              int nfp, const int* vmin, const int* vplus, const int* bc,
              const double* nx, const double* ny, const double* nz, const double* dA,
              double c0, double dt, int nsteps, double* u, double* k);

/* Discrete energy 1/2 sum J w_i w_j w_k (|E|^2+|H|^2) (src/case.cpp:733-766). */
double nwo_energy(int N, int nelt, const double* wgll, const double* jac, const double* u);

/* LSRK45 coefficient tables (src/dg_solver.cpp:58-69). */
void nwo_lsrk45(double* a5, double* b5);

/* Number of OpenMP threads the oracle uses (1 when built without OpenMP). */
int nwo_threads(void);

#ifdef __cplusplus
}
#endif
#endif
