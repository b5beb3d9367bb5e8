// Host shim for compiling the reference's CUDA kernel bodies as plain C++.
// TEST INFRASTRUCTURE ONLY (oracle/_ref build).  It stands in for the
// reference's src/device/gpu_runtime.hpp when its kernels (extracted at build
// time from src/device/dg_kernels.cu:1-453) are compiled for the host:
//   * blockIdx / threadIdx / blockDim become thread-local variables set by the
//     host grid runner in ref_host_driver.cpp;
//   * __shared__ storage is thread-local, one copy per OpenMP thread;
//   * __syncthreads() ends phase 0 of a two-phase block run: phase 0 performs
//     the (idempotent) shared-memory loads of every thread, phase 1 reloads and
//     computes, which is what a barrier guarantees on the device;
//   * atomicAdd is an OpenMP atomic capture.
#ifndef NW_DEVICE_GPU_RUNTIME_HPP
#define NW_DEVICE_GPU_RUNTIME_HPP
#include <cstdio>
#include <cstdlib>

struct nw_host_dim3 { unsigned x, y, z; };
extern thread_local nw_host_dim3 blockIdx, threadIdx, blockDim;
extern thread_local int nw_cpu_phase;

#define __global__
#define __shared__ thread_local
#define __syncthreads() do { if (nw_cpu_phase == 0) return; } while (0)

inline double atomicAdd(double* addr, double v) {
    double old;
#pragma omp atomic capture
    { old = *addr; *addr += v; }
    return old;
}

typedef void* cudaStream_t;
#define NW_GPU_CHECK(call) ((void)0)
#endif
