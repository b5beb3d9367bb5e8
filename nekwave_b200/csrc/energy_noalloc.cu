// energy_noalloc.cu -- the discrete energy of a device-resident state, computed
// without allocating any device memory.
//
// nwb_energy needs per-block partial sums in global memory, which the solver
// allocates with cudaMalloc when it is created.  Some callers cannot allocate:
// a server that admits work against a fixed HBM budget and must not grow its
// footprint behind the admission check, a host framework whose own caching
// allocator owns all device memory, or a loop on a latency-critical path where
// cudaMalloc's implicit device synchronisation is not acceptable.  For them,
// nwb_energy_noalloc takes the state, the Jacobians and the weights as device
// pointers, writes the energy to a device pointer, and keeps its per-element
// partial sums in a fixed array in the library's own device memory
// (NWB_ENERGY_NOALLOC_MAX_ELEMENTS doubles, 1 MiB, held on every GPU that loads
// the library until the process exits).
//
// All calls share that array: calls whose kernels overlap on the GPU (different
// streams, different host threads) race on it and must be ordered by the
// caller.  Every call writes all the partials it reads, so nothing left from an
// earlier call is ever summed.
#include "nwb.h"

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

extern "C" void nwb_set_error_(const char* msg);

namespace {

// Per-element partial sums.  In host code this name is only a host-side handle
// of the symbol, never a device address; the address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) double g_energy_partials[NWB_ENERGY_NOALLOC_MAX_ELEMENTS];

constexpr int kWarpsPerBlock = 8;
constexpr int kMaxDevices = 64;

// One warp per element: lane-strided sum over the element's nodes in a fixed
// order, then a fixed shuffle tree.
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
energy_element_kernel(const double* __restrict__ u, long long stride, int N3, int nelt,
                      const double* __restrict__ jac, int jac_per_node,
                      const double* __restrict__ w3, double* __restrict__ partials) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.x * kWarpsPerBlock + warp;
    if (e >= nelt) return;
    const long long base = static_cast<long long>(e) * N3;
    double acc = 0.0;
    for (int m = lane; m < N3; m += 32) {
        const long long p = base + m;
        const double J = jac_per_node ? jac[p] : jac[e];
        const double ex = u[p], ey = u[stride + p], ez = u[2 * stride + p];
        const double hx = u[3 * stride + p], hy = u[4 * stride + p], hz = u[5 * stride + p];
        acc += 0.5 * ((ex * ex + ey * ey + ez * ez) + (hx * hx + hy * hy + hz * hz)) * (J * w3[m]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) partials[e] = acc;
}

// One block: fixed-order strided sums, then a fixed tree.
__global__ void __launch_bounds__(256)
energy_sum_kernel(const double* __restrict__ partials, int n, double* __restrict__ out) {
    __shared__ double s[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += 256) acc += partials[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = s[0];
}

std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

// Device address of g_energy_partials on the current device, looked up once per
// device (with that device current) and cached.
nwb_status scratch_address(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        nwb_set_error_("nwb_energy_noalloc: no usable current CUDA device");
        return NWB_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_energy_partials);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            nwb_set_error_("nwb_energy_noalloc: cudaGetSymbolAddress of the scratch array failed");
            return NWB_ECUDA;
        }
        g_addr[dev] = static_cast<double*>(p);
    }
    *out = g_addr[dev];
    return NWB_OK;
}

}  // namespace

extern "C" nwb_status nwb_energy_noalloc(const double* d_state, long long stride, int N, int nelt,
                                         const double* d_jac, int jac_per_node, const double* d_w3,
                                         double* d_energy, void* stream) {
    if (!d_state || !d_jac || !d_w3 || !d_energy) {
        nwb_set_error_("nwb_energy_noalloc: null device pointer");
        return NWB_EINVAL;
    }
    if (N < 2 || N > 10 || nelt < 1) {
        nwb_set_error_("nwb_energy_noalloc: need 2 <= N <= 10 and nelt >= 1");
        return NWB_EINVAL;
    }
    if (nelt > NWB_ENERGY_NOALLOC_MAX_ELEMENTS) {
        nwb_set_error_("nwb_energy_noalloc: nelt exceeds NWB_ENERGY_NOALLOC_MAX_ELEMENTS (131072), "
                       "the size of its fixed scratch array; use nwb_energy for larger meshes");
        return NWB_EINVAL;
    }
    const long long N3 = static_cast<long long>(N) * N * N;
    if (stride < static_cast<long long>(nelt) * N3) {
        nwb_set_error_("nwb_energy_noalloc: stride smaller than nelt*N^3");
        return NWB_EINVAL;
    }
    double* partials = nullptr;
    nwb_status st = scratch_address(&partials);
    if (st != NWB_OK) return st;
    // every pointer must be device memory of the current device: the kernels run
    // there, and the scratch address above is that device's
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        nwb_set_error_("nwb_energy_noalloc: no usable current CUDA device");
        return NWB_ECUDA;
    }
    const void* ptrs[4] = {d_state, d_jac, d_w3, d_energy};
    for (const void* q : ptrs) {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, q) != cudaSuccess) {
            cudaGetLastError();
            nwb_set_error_("nwb_energy_noalloc: a pointer argument is not a CUDA pointer");
            return NWB_EINVAL;
        }
        const bool on_dev = a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
        if (!on_dev || a.device != dev) {
            nwb_set_error_("nwb_energy_noalloc: every pointer must be device memory of the "
                           "current device (nwb_set_device)");
            return NWB_EINVAL;
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (nelt + kWarpsPerBlock - 1) / kWarpsPerBlock;
    energy_element_kernel<<<blocks, 32 * kWarpsPerBlock, 0, s>>>(
        d_state, stride, static_cast<int>(N3), nelt, d_jac, jac_per_node, d_w3, partials);
    energy_sum_kernel<<<1, 256, 0, s>>>(partials, nelt, d_energy);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        nwb_set_error_(cudaGetErrorString(e));
        return NWB_ECUDA;
    }
    return NWB_OK;
}
