// stage_dmma.cuh -- fused LSRK45 stage for 8 points per direction, axis-aligned
// elements, FP64, with the r and s contractions on the FP64 tensor cores
// (mma.sync m8n8k4 f64) and the residual split by field between two warps.
//
// Why: in the SIMT forms every lane reads, for each r and s derivative it forms,
// the N values of a row or column from shared memory, and a 64-bit warp load costs
// two wavefronts however many lanes share an address; ncu shows those loads
// keeping the L1/shared pipe at 80-90 % at N = 8.  As an 8x8x8 product per plane
// and component, a warp reads each node value once per direction (one 64-bit
// fragment load per lane per k-step) and keeps D in two registers.  tcgen05 has no
// FP64 kind; mma.sync .f64 is sm_100a's FP64 tensor-core instruction.
//
// Block = one element, 64 threads = 2 warps (or 128 threads, two warps per field
// taking four planes each):
//   1. cp.async of u_in (16-byte copies), D, geometry, connections; k lines of the
//      element into L2;
//   2. face phase (face_phase2, one thread per face point, six per thread);
//   3. warp 0 forms the E residual from V = H (+curl H), warp 1 the H residual from
//      V = E (-curl E).  Lane 4g + t owns nodes (i = 2t, 2t+1; j = g) of every
//      plane k.  Per plane: the r derivatives of Vz, Vy in the original form
//      (A = rows of the plane, B = D^T) and the s derivatives of Vz, Vx in the
//      swapped form (A = D, B = columns of the plane) land on the same two nodes;
//      the t derivatives of Vy, Vx are SIMT sums over the lane's two node columns,
//      read once into registers, with D(k,l) from the kernel's parameter bank.
//      Then the lifted face terms in face order 0..5 and the LSRK update in FP64,
//      two adjacent nodes per 16-byte access.
// Fragment layout (m8n8k4, A row-major 8x4, B column-major 4x8, C 8x8): lane
// L = 4g + t holds A[g][t], B[t][g], C[g][2t] and C[g][2t+1].
#pragma once

#include "stage_mma.cuh"
#include "stage_pipe.cuh"

namespace nwb {
namespace stage {

struct DmmaLayout8 {
    static constexpr int u = 0;                                   // [6][512] doubles
    static constexpr int geo = u + 6 * 512 * 8;
    static constexpr int conn = geo + static_cast<int>(sizeof(ElemGeo));
    static constexpr int D = conn + 32;
    static constexpr int flux = D + 64 * 8;                       // [6 faces][6 comps][64]
    static constexpr int total = flux + 36 * 64 * 8;
};

// Planes K0 .. K0+NK-1 of the column phase of one warp (field src -> dst).
template <int K0, int NK>
__device__ __forceinline__ void dmma8_planes(const StageParams& P, const double* su, const double* V,
                                             const double* Fl, int g, int t, int dst, double sgn,
                                             double d0, double d1, const double (&cx)[8][2],
                                             const double (&cy)[8][2], double rx, double sy, double tz,
                                             long long ebase, const double* __restrict__ Dc) {
    constexpr int N = 8, N3 = 512;
    const double A = P.a, B = P.b, DT = P.dt;
    const long long S = P.stride;
#pragma unroll
    for (int k = K0; k < K0 + NK; ++k) {
        const int ms = 64 * k + 8 * g + 2 * t;  // first of the lane's two nodes
        double2 kold[3];
#pragma unroll
        for (int c = 0; c < 3; ++c)
            kold[c] = __ldcg(reinterpret_cast<const double2*>(P.k + (dst + c) * S + ebase + ms));
        // r (original form): A[g][t] = V(l = t, j = g, k)
        double zr0 = 0.0, zr1 = 0.0, yr0 = 0.0, yr1 = 0.0;
        dmma_f64(zr0, zr1, V[2 * N3 + 64 * k + 8 * g + t], d0);
        dmma_f64(zr0, zr1, V[2 * N3 + 64 * k + 8 * g + 4 + t], d1);
        dmma_f64(yr0, yr1, V[1 * N3 + 64 * k + 8 * g + t], d0);
        dmma_f64(yr0, yr1, V[1 * N3 + 64 * k + 8 * g + 4 + t], d1);
        // s (swapped form): B[t][g] = V(i = g, l = t, k)
        double zs0 = 0.0, zs1 = 0.0, xs0 = 0.0, xs1 = 0.0;
        dmma_f64(zs0, zs1, d0, V[2 * N3 + 64 * k + 8 * t + g]);
        dmma_f64(zs0, zs1, d1, V[2 * N3 + 64 * k + 8 * (4 + t) + g]);
        dmma_f64(xs0, xs1, d0, V[0 * N3 + 64 * k + 8 * t + g]);
        dmma_f64(xs0, xs1, d1, V[0 * N3 + 64 * k + 8 * (4 + t) + g]);
        // t: sums over the cached columns, D(k, l) from Dc (the parameter bank when the
        // caller has it there, else shared memory: the same values either way)
        double yt0 = 0.0, yt1 = 0.0, xt0 = 0.0, xt1 = 0.0;
#pragma unroll
        for (int l = 0; l < 8; ++l) {
            const double dk = Dc[k + 8 * l];
            yt0 += dk * cy[l][0]; yt1 += dk * cy[l][1];
            xt0 += dk * cx[l][0]; xt1 += dk * cx[l][1];
        }
        double rhs0[3], rhs1[3];
        rhs0[0] = sgn * (sy * zs0 - tz * yt0);
        rhs0[1] = sgn * (tz * xt0 - rx * zr0);
        rhs0[2] = sgn * (rx * yr0 - sy * xs0);
        rhs1[0] = sgn * (sy * zs1 - tz * yt1);
        rhs1[1] = sgn * (tz * xt1 - rx * zr1);
        rhs1[2] = sgn * (rx * yr1 - sy * xs1);
        add_lifts<N, 3>(Fl, dst, 2 * t, g, k, rhs0);
        add_lifts<N, 3>(Fl, dst, 2 * t + 1, g, k, rhs1);
        // LSRK45 (src/device/dg_kernels.cu:404-406), FP64
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double kn0 = A * kold[c].x + DT * rhs0[c];
            const double kn1 = A * kold[c].y + DT * rhs1[c];
            const double2 uo = *reinterpret_cast<const double2*>(su + (dst + c) * N3 + ms);
            __stcs(reinterpret_cast<double2*>(P.k + (dst + c) * S + ebase + ms), make_double2(kn0, kn1));
            __stcs(reinterpret_cast<double2*>(P.u_out + (dst + c) * S + ebase + ms),
                   make_double2(uo.x + B * kn0, uo.y + B * kn1));
        }
    }
}

// One element: WPF warps per field, 1 (64 threads, each warp all 8 planes of its
// field) or 2 (128 threads, each warp 4 planes; the face phase then has 3 points
// per thread).  Dc: D (column-major) where the t contraction reads it -- the
// kernel's parameter copy when the caller has one (constant-bank operands), else
// the tile's shared copy at smem + DmmaLayout8::D (the same values either way).
// All threads of the block call it; threads beyond 64*WPF take part in the
// barriers only.  e_ahead >= 0: thread 0 also pulls the u_in and k of that element
// into L2, for the block that loads it later.
template <int WPF>
__device__ __forceinline__ void dmma8_tile(const StageParams& P, const int e, unsigned char* smem,
                                           const int tid, const double* Dc, const int e_ahead = -1) {
    constexpr int N = 8, N3 = 512, NT = 64 * WPF;
    static_assert(WPF == 1 || WPF == 2, "one or two warps per field");
    using L = DmmaLayout8;
    double* su = reinterpret_cast<double*>(smem + L::u);
    ElemGeo* sg = reinterpret_cast<ElemGeo*>(smem + L::geo);
    int* sc = reinterpret_cast<int*>(smem + L::conn);
    double* sD = reinterpret_cast<double*>(smem + L::D);
    double* sflux = reinterpret_cast<double*>(smem + L::flux);

    if (tid < NT) {
        issue2<N, GEO_BOX, 1, NT, false>(P, e, su, sg, sc, tid);
        if (tid < 64) cp_async8(sD + tid, P.D + tid);
        if (tid == 0 && e_ahead >= 0) prefetch_tile_l2<N3>(P, e_ahead, 1);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();

    FaceGather<face_points_per_thread<N, WPF>()> G;
    face_phase2<N, GEO_BOX, false, WPF, 1, false, false>(P, e, su, sg, sc, sflux, tid, G);
    __syncthreads();
    if (tid >= NT) return;

    const int warp = tid >> 5, lane = tid & 31;
    const int field = warp / WPF, part = warp % WPF;
    const int g = lane >> 2, t = lane & 3;
    const int src = field == 0 ? 3 : 0;  // differentiated field
    const int dst = 3 - src;             // residual components formed
    const double sgn = field == 0 ? 1.0 : -1.0;
    const double* V = su + src * N3;
    const double d0 = sD[g + 8 * t];        // D(q = g, l = t)
    const double d1 = sD[g + 8 * (4 + t)];  // D(q = g, l = 4 + t)
    // the lane's two node columns of Vx and Vy (t derivatives)
    double cx[8][2], cy[8][2];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const double2 a = *reinterpret_cast<const double2*>(V + 0 * N3 + 64 * l + 8 * g + 2 * t);
        const double2 b = *reinterpret_cast<const double2*>(V + 1 * N3 + 64 * l + 8 * g + 2 * t);
        cx[l][0] = a.x; cx[l][1] = a.y;
        cy[l][0] = b.x; cy[l][1] = b.y;
    }
    const double rx = sg->met[0], sy = sg->met[4], tz = sg->met[8];
    const long long ebase = static_cast<long long>(e) * N3;
    if constexpr (WPF == 1) {
        dmma8_planes<0, 8>(P, su, V, sflux, g, t, dst, sgn, d0, d1, cx, cy, rx, sy, tz, ebase, Dc);
    } else {
        if (part == 0) dmma8_planes<0, 4>(P, su, V, sflux, g, t, dst, sgn, d0, d1, cx, cy, rx, sy, tz, ebase, Dc);
        else dmma8_planes<4, 4>(P, su, V, sflux, g, t, dst, sgn, d0, d1, cx, cy, rx, sy, tz, ebase, Dc);
    }
}

// AHEAD (0, 1, 2): block e also pulls into L2 the element of the block that starts
// about AHEAD/2 waves of resident blocks later (tile_ahead); 0: no prefetch.
template <int MINB, int WPF, int AHEAD>
__global__ void __launch_bounds__(64 * WPF, MINB) stage_dmma8_kernel(const __grid_constant__ StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int e_ahead = AHEAD > 0 ? tile_ahead<(AHEAD > 0 ? AHEAD : 1), MINB>(blockIdx.x) : -1;
    dmma8_tile<WPF>(P, blockIdx.x, smem, threadIdx.x, P.Dc, e_ahead);
}

template <int MINB, int WPF = 1, int AHEAD = 0>
cudaError_t launch_dmma8(const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    constexpr int smem = DmmaLayout8::total;
    auto kern = stage_dmma8_kernel<MINB, WPF, AHEAD>;
    if (cfg) *cfg = StageConfig{WPF, 1, 64 * WPF, smem, 0, MINB};
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (!p) return cudaSuccess;
    kern<<<p->nelt, 64 * WPF, smem, st>>>(*p);
    return cudaGetLastError();
}

}  // namespace stage
}  // namespace nwb
