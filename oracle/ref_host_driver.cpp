// ref_host_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Drives the reference's own code on the host: its Mesh (src/mesh.cpp, compiled
// unchanged) and its CUDA kernel bodies (src/device/dg_kernels.cu:1-453, compiled
// as C++ through the shim in ref_shim/).  The stage order is the one of
// DgSolver::Impl::step (src/dg_solver.cpp:330-505) on a single rank.  Built by
// oracle/Makefile into oracle/_ref/libnwref_host.so; used to pin the C
// restatement (nw_oracle.c), to generate the golden vectors and as the timed
// CPU baseline.  Never linked by the product.
#include "mesh.hpp"

#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

struct nw_host_dim3 { unsigned x, y, z; };
thread_local nw_host_dim3 blockIdx, threadIdx, blockDim;
thread_local int nw_cpu_phase;
// Dynamic shared memory of the volume kernel: (N^2 + 3 N^3) doubles, N <= 16.
thread_local double s_mem[16 * 16 + 3 * 16 * 16 * 16];

// Kernel bodies of src/device/dg_kernels.cu, compiled for the host.
void gpu_volume_curl_kernel(const double*, const double*, const double*, double*, double*,
                            double*, const double*, const double*, const double*,
                            const double*, const double*, const double*, const double*,
                            const double*, const double*, const double*, const double*,
                            const double*, double, int, int);
void gpu_restrict_faces_kernel(const double*, double*, double*, const int*, int, int);
void gpu_compute_flux_kernel(const double*, const double*, const double*, const int*,
                             const int*, const double*, const double*, const double*,
                             double*, double, int, int);
void gpu_add_flux_kernel(const double*, const int*, const double*, double*, int, int);
void gpu_inv_mass_kernel(double*, const double*, const double*, int, int, int);
void gpu_lsrk45_update_kernel(double*, double*, const double*, double, double, double,
                              int, int);

namespace {

// Runs a 1-D grid on the host.  Blocks are distributed over OpenMP threads;
// kernels with a barrier run every block in two phases (see ref_shim/gpu_runtime.hpp).
template <class F>
void run_grid(long nblocks, int bdim, bool has_barrier, bool parallel, F&& f) {
#pragma omp parallel for schedule(static) if (parallel)
    for (long b = 0; b < nblocks; ++b) {
        blockIdx = {static_cast<unsigned>(b), 0u, 0u};
        blockDim = {static_cast<unsigned>(bdim), 1u, 1u};
        for (int ph = has_barrier ? 0 : 1; ph < 2; ++ph) {
            nw_cpu_phase = ph;
            for (int t = 0; t < bdim; ++t) {
                threadIdx = {static_cast<unsigned>(t), 0u, 0u};
                f();
            }
        }
    }
}

struct Geo {
    int N, nelt, nfp;
    const double *D, *w3, *jac, *met;
    const int *vmin, *vplus, *bc;
    const double *nx, *ny, *nz, *dA;
};

// One right-hand-side evaluation in the order of src/dg_solver.cpp:393-487.
// deterministic != 0 runs the atomic lift kernel on one thread in face-point order.
void ref_rhs(const Geo& g, double c0, const double* u, double* rhs, double* fEN,
             double* fHN, double* flux, int deterministic) {
    const int N = g.N, nelt = g.nelt, nfp = g.nfp;
    const int nxyz = N * N * N;
    const int npts = nelt * nxyz;
    const double* m = g.met;
    const double *rx = m, *sx = m + npts, *tx = m + 2L * npts, *ry = m + 3L * npts,
                 *sy = m + 4L * npts, *ty = m + 5L * npts, *rz = m + 6L * npts,
                 *sz = m + 7L * npts, *tz = m + 8L * npts;
    const double *Ex = u, *Ey = u + npts, *Ez = u + 2L * npts;
    const double *Hx = u + 3L * npts, *Hy = u + 4L * npts, *Hz = u + 5L * npts;
    double *rEx = rhs, *rEy = rhs + npts, *rEz = rhs + 2L * npts;
    double *rHx = rhs + 3L * npts, *rHy = rhs + 4L * npts, *rHz = rhs + 5L * npts;

    run_grid(nelt, nxyz, true, true, [&] {
        gpu_volume_curl_kernel(Hx, Hy, Hz, rEx, rEy, rEz, g.D, g.w3, g.jac, rx, sx, tx, ry,
                               sy, ty, rz, sz, tz, 1.0, N, nelt);
    });
    run_grid(nelt, nxyz, true, true, [&] {
        gpu_volume_curl_kernel(Ex, Ey, Ez, rHx, rHy, rHz, g.D, g.w3, g.jac, rx, sx, tx, ry,
                               sy, ty, rz, sz, tz, -1.0, N, nelt);
    });
    const int bs = 256;
    const long nb = (nfp + bs - 1) / bs;
    run_grid(nb, bs, false, true, [&] {
        gpu_restrict_faces_kernel(u, fEN, fHN, g.vmin, nfp, npts);
    });
    run_grid(nb, bs, false, true, [&] {
        gpu_compute_flux_kernel(u, fEN, fHN, g.vplus, g.bc, g.nx, g.ny, g.nz, flux, c0, nfp,
                                npts);
    });
    run_grid(nb, bs, false, deterministic == 0, [&] {
        gpu_add_flux_kernel(flux, g.vmin, g.dA, rhs, nfp, npts);
    });
    const long nbm = (static_cast<long>(nelt) * nxyz + bs - 1) / bs;
    run_grid(nbm, bs, false, true, [&] {
        gpu_inv_mass_kernel(rhs, g.jac, g.w3, nelt, nxyz, npts);
    });
}

}  // namespace

extern "C" {

// ---- reference kernels on the host --------------------------------------------
void nwref_rhs(int N, int nelt, const double* D, const double* w3, const double* jac,
               const double* met, int nfp, const int* vmin, const int* vplus, const int* bc,
               const double* nx, const double* ny, const double* nz, const double* dA,
               double c0, const double* u, double* rhs, int deterministic) {
    Geo g{N, nelt, nfp, D, w3, jac, met, vmin, vplus, bc, nx, ny, nz, dA};
    std::vector<double> fEN(3L * nfp), fHN(3L * nfp), flux(6L * nfp);
    ref_rhs(g, c0, u, rhs, fEN.data(), fHN.data(), flux.data(), deterministic);
}

// nsteps LSRK45 steps (src/dg_solver.cpp:306-527); u and k updated in place.
void nwref_step(int N, int nelt, const double* D, const double* w3, const double* jac,
                const double* met, int nfp, const int* vmin, const int* vplus,
                const int* bc, const double* nx, const double* ny, const double* nz,
                const double* dA, double c0, double dt, int nsteps, double* u, double* k,
                int deterministic) {
    // Carpenter-Kennedy coefficients as written in src/dg_solver.cpp:58-69.
    const double rk4a[5] = {0.0, -567301805773.0 / 1357537059087.0,
                            -2404267990393.0 / 2016746695238.0,
                            -3550918686646.0 / 2091501179385.0,
                            -1275806237668.0 / 842570457699.0};
    const double rk4b[5] = {1432997174477.0 / 9575080441755.0,
                            5161836677717.0 / 13612068292357.0,
                            1720146321549.0 / 2090206949498.0,
                            3134564353537.0 / 4481467310338.0,
                            2277821191437.0 / 14882151754819.0};
    Geo g{N, nelt, nfp, D, w3, jac, met, vmin, vplus, bc, nx, ny, nz, dA};
    const int npts = nelt * N * N * N;
    std::vector<double> fEN(3L * nfp), fHN(3L * nfp), flux(6L * nfp), rhs(6L * npts);
    const long nb = (6L * npts + 255) / 256;
    for (int s = 0; s < nsteps; ++s) {
        for (int st = 0; st < 5; ++st) {
            ref_rhs(g, c0, u, rhs.data(), fEN.data(), fHN.data(), flux.data(), deterministic);
            run_grid(nb, 256, false, true, [&] {
                gpu_lsrk45_update_kernel(u, k, rhs.data(), rk4a[st], rk4b[st], dt, npts, npts);
            });
        }
    }
}

int nwref_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Host threads for the next runs (n >= 1); returns the previous count.
int nwref_set_threads(int n) {
#ifdef _OPENMP
    const int old = omp_get_max_threads();
    if (n >= 1) omp_set_num_threads(n);
    return old;
#else
    (void)n;
    return 1;
#endif
}

}  // extern "C"
