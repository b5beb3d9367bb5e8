// diag_kernels.cu -- device diagnostics: the FP64 discrete energy of
// Case::computeTotalEnergy (src/case.cpp:733-766) as a deterministic two-pass
// reduction, and an L2-evicting buffer write used between timed iterations.
#include "nwb_internal.h"

namespace nwb {
namespace {

constexpr int kEnergyThreads = 256;

// Block b sums 1/2 (|E|^2 + |H|^2) J w3 over a contiguous range of nodes with a
// fixed per-thread order and a fixed shuffle tree, so repeated calls agree bit
// for bit.  jac_e (per element) or jac_n (per node) supplies J.
__global__ void __launch_bounds__(kEnergyThreads)
energy_partials_kernel(const double* __restrict__ u, long long stride, int N3,
                       long long npts, const double* __restrict__ jac_e,
                       const double* __restrict__ jac_n, const double* __restrict__ w3,
                       double* __restrict__ partial) {
    const long long per = (npts + gridDim.x - 1) / gridDim.x;
    const long long lo = per * blockIdx.x;
    const long long hi = min(npts, lo + per);
    double acc = 0.0;
    for (long long p = lo + threadIdx.x; p < hi; p += blockDim.x) {
        const long long e = p / N3;
        const int m = static_cast<int>(p - e * N3);
        const double J = jac_n ? jac_n[p] : jac_e[e];
        const double dV = J * w3[m];
        const double ex = u[p], ey = u[stride + p], ez = u[2 * stride + p];
        const double hx = u[3 * stride + p], hy = u[4 * stride + p], hz = u[5 * stride + p];
        const double eSq = ex * ex + ey * ey + ez * ez;
        const double hSq = hx * hx + hy * hy + hz * hz;
        acc += 0.5 * (eSq + hSq) * dV;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    __shared__ double warp_sums[kEnergyThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kEnergyThreads / 32; ++w) s += warp_sums[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void energy_final_kernel(const double* __restrict__ partial, int n,
                                    double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < n; ++b) s += partial[b];
        *out = s;
    }
}

// Largest |E| and |H| over the nodes of a contiguous range per block, as
// Case::getMaxE / getMaxH (src/case.cpp:768-794) form them on the host:
// sqrt((x*x + y*y) + z*z) with separate multiply, add and square-root roundings
// (no contraction), kept when larger than the running maximum (a NaN node never
// is).  The maximum does not depend on the order, so the result equals the
// host's bit for bit.  partial[2b] = max|E|, partial[2b+1] = max|H| of block b.
__device__ __forceinline__ double norm3_rn(double x, double y, double z) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}

__global__ void __launch_bounds__(kEnergyThreads)
maxnorm_partials_kernel(const double* __restrict__ u, long long stride, long long npts,
                        double* __restrict__ partial) {
    const long long per = (npts + gridDim.x - 1) / gridDim.x;
    const long long lo = per * blockIdx.x;
    const long long hi = min(npts, lo + per);
    double me = 0.0, mh = 0.0;
    for (long long p = lo + threadIdx.x; p < hi; p += blockDim.x) {
        const double e = norm3_rn(u[p], u[stride + p], u[2 * stride + p]);
        const double h = norm3_rn(u[3 * stride + p], u[4 * stride + p], u[5 * stride + p]);
        if (e > me) me = e;
        if (h > mh) mh = h;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const double oe = __shfl_down_sync(0xffffffffu, me, off);
        const double oh = __shfl_down_sync(0xffffffffu, mh, off);
        if (oe > me) me = oe;
        if (oh > mh) mh = oh;
    }
    __shared__ double warp_max[2][kEnergyThreads / 32];
    if ((threadIdx.x & 31) == 0) {
        warp_max[0][threadIdx.x >> 5] = me;
        warp_max[1][threadIdx.x >> 5] = mh;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double m = 0.0;
        for (int w = 0; w < kEnergyThreads / 32; ++w)
            if (warp_max[threadIdx.x][w] > m) m = warp_max[threadIdx.x][w];
        partial[2 * blockIdx.x + threadIdx.x] = m;
    }
}

__global__ void maxnorm_final_kernel(const double* __restrict__ partial, int n,
                                     double* __restrict__ out) {
    if (blockIdx.x == 0 && threadIdx.x < 2) {
        double m = 0.0;
        for (int b = 0; b < n; ++b)
            if (partial[2 * b + threadIdx.x] > m) m = partial[2 * b + threadIdx.x];
        out[threadIdx.x] = m;
    }
}

// ProbeManager::record (src/probe.cpp:192-216): thread (probe, component) sums
// w[p] * u[offset + p] over the probe element's N^3 nodes in node order, with
// separate multiply and add roundings as on the host, so the values equal the
// reference's bit for bit on the same state and weights.
__global__ void probe_kernel(const double* __restrict__ u, long long stride, int N3,
                             const long long* __restrict__ offset, const double* __restrict__ w,
                             int nprobes, double* __restrict__ out) {
    const int pr = blockIdx.x;
    const int c = threadIdx.x;
    if (pr >= nprobes || c >= 6) return;
    const double* wp = w + static_cast<long long>(pr) * N3;
    const double* up = u + c * stride + offset[pr];
    double acc = 0.0;
    for (int p = 0; p < N3; ++p) acc = __dadd_rn(acc, __dmul_rn(wp[p], up[p]));
    out[pr * 6 + c] = acc;
}

__global__ void l2_flush_kernel(int4* __restrict__ buf, size_t n16) {
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t x = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; x < n16; x += stride)
        buf[x] = make_int4(static_cast<int>(x), 0, 0, 0);
}

}  // namespace

int energy_blocks(int nelt) {
    const int b = (nelt + 3) / 4;
    return b < 1 ? 1 : (b > 1184 ? 1184 : b);
}

cudaError_t launch_energy(const double* u, long long stride, int N, int nelt,
                          const double* jac_e, const double* jac_n, const double* w3,
                          double* partial, int nblocks, double* out, cudaStream_t st) {
    const int N3 = N * N * N;
    const long long npts = static_cast<long long>(nelt) * N3;
    energy_partials_kernel<<<nblocks, kEnergyThreads, 0, st>>>(u, stride, N3, npts, jac_e, jac_n,
                                                               w3, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    energy_final_kernel<<<1, 32, 0, st>>>(partial, nblocks, out);
    return cudaGetLastError();
}

cudaError_t launch_max_norms(const double* u, long long stride, long long npts, double* partial,
                             int nblocks, double* out, cudaStream_t st) {
    maxnorm_partials_kernel<<<nblocks, kEnergyThreads, 0, st>>>(u, stride, npts, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    maxnorm_final_kernel<<<1, 32, 0, st>>>(partial, nblocks, out);
    return cudaGetLastError();
}

cudaError_t launch_probes(const double* u, long long stride, int N3, const long long* offset,
                          const double* w, int nprobes, double* out, cudaStream_t st) {
    if (nprobes <= 0) return cudaSuccess;
    probe_kernel<<<nprobes, 32, 0, st>>>(u, stride, N3, offset, w, nprobes, out);
    return cudaGetLastError();
}

cudaError_t launch_l2_flush(void* buf, size_t bytes, cudaStream_t st) {
    const size_t n16 = bytes / 16;
    l2_flush_kernel<<<148 * 4, 256, 0, st>>>(static_cast<int4*>(buf), n16);
    return cudaGetLastError();
}

}  // namespace nwb
