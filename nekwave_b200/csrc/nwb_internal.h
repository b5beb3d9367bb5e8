// nwb_internal.h -- types shared by the host side (nwb_api.cpp) and the CUDA
// kernels (stage_kernels.cu, diag_kernels.cu).
#pragma once

#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

namespace nwb {

// One-time kernel set-up per device.  cudaFuncSetAttribute (and the occupancy a
// launcher derives from it) applies to the current device's context only, so a
// launcher keeps one flag per device index: a process that creates solvers on
// several GPUs sets each kernel up on each of them.
constexpr int kMaxDeviceSlots = 64;
inline cudaError_t current_device_slot(int* dev) {
    cudaError_t e = cudaGetDevice(dev);
    if (e != cudaSuccess) return e;
    if (*dev < 0 || *dev >= kMaxDeviceSlots) return cudaErrorInvalidDevice;
    return cudaSuccess;
}
// Raises kern's dynamic shared-memory limit to smem on the current device, once
// per device (flags: one zero-initialised static array per kernel).
template <typename K>
cudaError_t set_smem_once(K kern, int smem, std::atomic<int>* flags) {
    int dev = 0;
    cudaError_t e = current_device_slot(&dev);
    if (e != cudaSuccess) return e;
    if (flags[dev].load(std::memory_order_acquire)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    flags[dev].store(1, std::memory_order_release);
    return cudaSuccess;
}

// Geometry classes the mesh analysis sorts a mesh into (nwb_api.cpp).
enum GeoKind : int {
    GEO_BOX = 0,     // affine, axis-aligned: metrics diag(rx, sy, tz) per element
    GEO_AFFINE = 1,  // affine: full constant J^{-T} per element
    GEO_NODAL = 2    // per-node metrics and per-face-point normals/lift/neighbours
};

// Per-element geometry for the affine classes.  The reference weights the volume
// curl by w3*J (src/device/dg_kernels.cu:127) and divides by J*w3 again in the
// inverse-mass kernel (:369-370); the two cancel, so only J^{-T} remains.  The
// lift of face f is dA/(J w3) at its nodes, which for an affine element is the
// constant |J J^{-T} n_ref| / (J w_end) (src/mesh.cpp:1011-1038).
struct alignas(16) ElemGeo {
    double met[9];      // rx sx tx ry sy ty rz sz tz
    double nrm[6][3];   // outward unit normal of face f
    double lift[6];     // dA/(J w3) at the nodes of face f
    double jdet;        // J (energy weight); 34 doubles = 272 bytes
};
static_assert(sizeof(ElemGeo) == 272, "ElemGeo layout");

// Face connection code of (element, face):
//   -1                          PEC mirror ([[E]] = -2E^-, [[H]] = 0); the reference
//                               applies it to PMC faces too (src/device/dg_kernels.cu:243-251)
//   -2                          true PMC mirror ([[E]] = 0, [[H]] = -2H^-), only for
//                               solvers created with NWB_SOLVER_TRUE_PMC
//   (eB << 6) | (fB << 3) | o   neighbour element eB, its face fB, orientation o
// Orientation o maps (p,q) on this face to (p',q') on the neighbour face:
//   (a,b) = (o & 4) ? (q,p) : (p,q);  p' = (o & 1) ? N-1-a : a;  q' = (o & 2) ? N-1-b : b.
constexpr int kConnPEC = -1;
constexpr int kConnPMC = -2;

struct StageParams {
    const double* u_in;     // [6][stride]
    double* u_out;          // [6][stride]
    double* k;              // [6][stride], updated in place
    long long stride;       // component stride (doubles)
    int nelt;
    int _pad0;
    const double* D;        // [N*N] column-major
    const ElemGeo* geo;     // [nelt]       (GEO_BOX, GEO_AFFINE)
    const int* conn;        // [nelt*6]     (GEO_BOX, GEO_AFFINE)
    const double* met_n;    // [9][stride]  (GEO_NODAL)
    const double* fnrm;     // [3][nfp]     (GEO_NODAL)
    const double* flift;    // [nfp]        (GEO_NODAL)
    const int* fplus;       // [nfp] neighbour node, -1 mirror (GEO_NODAL)
    long long nfp;
    int* err;               // device status word: a kernel whose bounded wait expires
                            // records a nonzero code here (null: none kept)
    double c0;              // flux penalty: 0 central, 1 upwind
    double a, b, dt;        // LSRK45 stage coefficients and step
    int snel[3];            // structured box mesh: elements per axis (x fastest), or 0
    int spmask;             // structured box mesh: periodic axes (bit 0 x, 1 y, 2 z)
    double Dc[100];         // D again, by value: kernels that index it with constants
                            // read it as an operand from the parameter bank
    double zl[10];          // line coordinates: D zl = 1, zl[0] = -1 (the GLL nodes for
                            // a GLL D); FP32-bulk fits a linear function with them
};

// Launch configuration of one fused-stage-kernel variant.
struct StageConfig {
    int ks;       // threads per (i,j) node column
    int epb;      // elements per block
    int threads;  // threads per block
    int smem;     // dynamic shared memory bytes
    int ksmem;    // 1: k staged in shared memory, 0: prefetched to L2 and read directly
    int minb;     // minimum resident blocks requested from the register allocator
};

}  // namespace nwb

#include <vector>
#include "nwb.h"

namespace nwb {

// Host-side result of the mesh analysis (nwb_api.cpp): geometry class and, for
// the affine classes, the compressed per-element geometry and connections.
struct Analysis {
    int geo = GEO_NODAL;
    std::vector<ElemGeo> egeo;
    std::vector<int> conn;
    std::vector<double> jac_e;
};
// true_pmc: bc_type 2 faces become kConnPMC (per-node class: neighbour -2) instead
// of the reference's PEC mirror.
nwb_status analyse_mesh(const nwb_mesh_desc* m, Analysis* A, bool true_pmc = false);

// Box meshes without per-node arrays (box_mesh.cpp).
void gll(int N, std::vector<double>& z, std::vector<double>& w, std::vector<double>& D);
// Line coordinates from the differentiation matrix alone: the z with D z = 1 and
// z[0] = -1 (unique, as D maps exactly the constants to zero).  For a GLL D these
// are the GLL nodes; the reference's DgSolver::initialize reads no nodes, so the
// solver derives them.
void line_coords(int N, const double* D, double* z);
void trilinear_point(const double c[8][3], double r, double s, double t, double* X, double* J,
                     double met[9]);
void box_geometry(int N, int nelx, int nely, int nelz, const double lo[3], const double hi[3],
                  int pmask, const std::vector<double>& z, const std::vector<double>& w,
                  std::vector<ElemGeo>& geo, std::vector<int>& conn);
void box_probes(int N, int nelx, int nely, int nelz, const double lo[3], const double hi[3],
                const std::vector<double>& z, int nprobes, const double* xyz, std::vector<int>& elem,
                std::vector<double>& wts);
nwb_status set_error(nwb_status s, const char* fmt, ...);

// Fused stage kernel (stage_inst.cu, one object per N).  Variant 0 exists for
// every (N, geometry, precision); the axis-aligned class has more variants,
// which the autotuner times.  Returns cudaErrorInvalidValue for an unknown
// combination.  p == nullptr only reports the configuration (and performs the
// one-time kernel attribute set-up).
cudaError_t launch_stage(int N, int geo, int f32, int variant, const StageParams* p,
                         cudaStream_t st, StageConfig* cfg_out);
int stage_variant_count(int N, int geo, int f32);
template <int N>
cudaError_t launch_stage_n(int geo, int f32, int variant, const StageParams* p, cudaStream_t st,
                           StageConfig* cfg);
template <int N>
int stage_variant_count_n(int geo, int f32);

// FP64 energy of the state u (diag_kernels.cu): nblocks partial sums, then one
// fixed-order final sum into *out (device).  J comes from jac_e (per element,
// affine meshes) or jac_n (per node).
cudaError_t launch_energy(const double* u, long long stride, int N, int nelt,
                          const double* jac_e, const double* jac_n, const double* w3,
                          double* partial, int nblocks, double* out, cudaStream_t st);
int energy_blocks(int nelt);
// Largest |E| and |H| over the nodes of u (diag_kernels.cu), out[0], out[1] on the
// device; partial holds 2*nblocks doubles.
cudaError_t launch_max_norms(const double* u, long long stride, long long npts, double* partial,
                             int nblocks, double* out, cudaStream_t st);

// Large buffer write that evicts L2 (benchmark hygiene).
cudaError_t launch_l2_flush(void* buf, size_t bytes, cudaStream_t st);
// Probe values [nprobes][Ex..Hz] of state u (diag_kernels.cu).
cudaError_t launch_probes(const double* u, long long stride, int N3, const long long* offset,
                          const double* w, int nprobes, double* out, cudaStream_t st);

}  // namespace nwb
