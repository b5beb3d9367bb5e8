// ref_gpu_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points around the reference's own GPU solver: its DgSolver
// (src/dg_solver.cpp) and kernels (src/device/dg_kernels.cu), compiled unchanged
// for sm_100a by oracle/Makefile into oracle/_ref/libnwref_cuda.so.  The GPU
// tests use it as the reference CUDA build on the same B200 (parity and the
// reference's own step time, driven like
// examples/numerical_analysis/convergence_test/convergence_test.cpp:108-148).
#include "dg_solver.hpp"
#include "mesh.hpp"

#include <cuda_runtime.h>

extern "C" {

void* nwref_mesh_box(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                     double ymin, double ymax, double zmin, double zmax, int px, int py,
                     int pz);

void* nwref_gpu_create(void* mesh, double c0) {
    DgSolver* s = new DgSolver();
    s->initialize(*static_cast<Mesh*>(mesh), c0);
    return s;
}

void nwref_gpu_upload(void* h, const double* state, size_t n) {
    static_cast<DgSolver*>(h)->uploadState(state, n);
}

void nwref_gpu_download(void* h, double* state, size_t n) {
    static_cast<DgSolver*>(h)->downloadState(state, n);
}

// Runs nsteps reference steps and returns their device time in milliseconds
// (CUDA events on the default stream around the loop; each reference step ends
// with a stream synchronize, src/dg_solver.cpp:519).
double nwref_gpu_steps(void* h, double dt, int nsteps) {
    DgSolver* s = static_cast<DgSolver*>(h);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    double t = 0.0;
    for (int i = 0; i < nsteps; ++i) {
        s->step(dt, t);
        t += dt;
    }
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

void nwref_gpu_destroy(void* h) {
    DgSolver* s = static_cast<DgSolver*>(h);
    s->finalize();
    delete s;
}

}  // extern "C"
