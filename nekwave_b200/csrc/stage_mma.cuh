// stage_mma.cuh -- the fused LSRK45 stage with the GLL contractions on the FP64
// tensor cores (mma.sync m8n8k4 f64), for 8 points per direction, axis-aligned
// affine elements, FP64.
//
// Why: the SIMT tile (stage_kernel.cuh) has each thread compute whole node
// derivatives, so every node value is read from shared memory N times per
// direction; ncu shows that kernel bound by the L1/shared-memory pipe (90 %),
// not by DRAM.  As an 8x8 MMA the same contraction reads each value once per
// direction and keeps D in a register fragment.  tcgen05 has no FP64 kind, so
// this is the FP64 tensor-core path of sm_100a.
//
// Fragment layout (m8n8k4, A row-major 8x4, B column-major 4x8, C 8x8): lane
// L = 4g + t holds A[g][t], B[t][g], C[g][2t] and C[g][2t+1].
// Two forms of the same contraction d(q, line) = sum_l D(q, l) u(line, l):
//   original  A = u (rows = lines), B = D^T  ->  C[line][q]
//   swapped   A = D,  B = u (cols = lines)   ->  C[q][line]
// Both take D(q = g, l = t) and D(g, 4 + t) as the lane's D registers.  With the
// r contraction in the original form and the s contraction in the swapped form,
// lane 4g + t receives both derivatives at the same nodes (i = 2t, 2t+1; j = g),
// so six residual components leave the registers already combined; only the
// t contraction (swapped form: nodes k = g, i = 2t, 2t+1) is added through
// shared memory.
//
// Shared-memory pitches (rows j, planes k, in doubles): the tile u uses
// (12, 100), so every half-warp fragment load of r, s and t touches 16
// distinct bank pairs; the residual tile uses (8, 72), so the 16-byte
// residual stores of both phases are conflict-free.
//
// One element per block of 128 threads (4 warps):
//   1. cp.async the element's u_in and geometry; each thread also loads the
//      neighbour traces of its three face points (one per direction) and the
//      LSRK register of its four update nodes into registers now, so that
//      latency overlaps the contractions;
//   2. r and s contractions, combined in registers, written to the residual tile;
//   3. t contractions, added to the residual tile;
//   4. faces one direction at a time (opposite faces share no node): numerical
//      flux in FP64, times the lift dA/(J w3), added to the residual tile;
//   5. LSRK update per node with coalesced loads and streaming stores.
// The residual's terms are summed in a fixed order: bitwise deterministic.
#pragma once

#include "stage_kernel.cuh"

namespace nwb {
namespace stage {

__device__ __forceinline__ void dmma_f64(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

struct MmaLayout8 {
    static constexpr int UJ = 12, UK = 100, UE = 8 * UK;  // u tile pitches (doubles)
    static constexpr int RJ = 8, RK = 72, RE = 8 * RK;    // residual tile pitches
    static constexpr int u = 0;
    static constexpr int r = u + 6 * UE * 8;
    static constexpr int D = r + 6 * RE * 8;
    static constexpr int geo = D + 64 * 8;
    static constexpr int total = geo + static_cast<int>(sizeof(ElemGeo));
};

__device__ __forceinline__ void st2(double* p, double a, double b) {
    *reinterpret_cast<double2*>(p) = make_double2(a, b);
}

template <bool KSMEM_UNUSED = false>
__device__ __forceinline__ void stage_tile_mma8(const StageParams& P, const int e,
                                                unsigned char* smem, const int tid) {
    constexpr int N = 8, N3 = 512;
    using L = MmaLayout8;
    constexpr int UJ = L::UJ, UK = L::UK, UE = L::UE, RJ = L::RJ, RK = L::RK, RE = L::RE;
    double* s_u = reinterpret_cast<double*>(smem + L::u);
    double* s_r = reinterpret_cast<double*>(smem + L::r);
    double* s_D = reinterpret_cast<double*>(smem + L::D);
    ElemGeo* s_geo = reinterpret_cast<ElemGeo*>(smem + L::geo);
    const int lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t4 = lane & 3;
    const long long S = P.stride;
    const long long gbase = static_cast<long long>(e) * N3;

    // ---- 1. loads --------------------------------------------------------------
    // each warp copies 4 rows of 8 nodes per pass; the rows of one half-warp are
    // two apart, which puts them on disjoint bank pairs
    {
        const int i = lane & 7, rsel = lane >> 3;
        const int roff = (rsel == 1) ? 2 : ((rsel == 2) ? 1 : rsel);  // 0, 2, 1, 3
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double* src = P.u_in + c * S + gbase;
#pragma unroll
            for (int n = 0; n < 4; ++n) {
                const int row = 4 * (warp + 4 * n) + roff;  // row = j + 8 k, 0..63
                const int j = row & 7, k = row >> 3;
                cp_async8(s_u + c * UE + i + UJ * j + UK * k, src + 8 * row + i);
            }
        }
    }
    if (tid < 64) cp_async8(s_D + tid, P.D + tid);
    if (tid < 34) cp_async8(reinterpret_cast<double*>(s_geo) + tid,
                            reinterpret_cast<const double*>(P.geo + e) + tid);
    cp_async_commit();
    // this thread's face points: one per direction (r: faces 3,1; s: 0,2; t: 4,5)
    const int side = tid >> 6;
    const int pq = tid & 63, p = pq & 7, q = pq >> 3;
    double nb[3][6];
    bool mirror[3];
    int wall[3];  // wall code of a mirror face (kConnPEC or kConnPMC)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int f = d == 0 ? (side ? 1 : 3) : (d == 1 ? (side ? 2 : 0) : (side ? 5 : 4));
        const int cd = __ldg(P.conn + e * 6 + f);
        mirror[d] = cd < 0;
        wall[d] = cd;
        if (!mirror[d]) {
            const int eB = cd >> 6, fB = (cd >> 3) & 7, o = cd & 7;
            int a = (o & 4) ? q : p;
            int b = (o & 4) ? p : q;
            if (o & 1) a = N - 1 - a;
            if (o & 2) b = N - 1 - b;
            const long long vB = static_cast<long long>(eB) * N3 + face_local<N>(fB, a, b);
#pragma unroll
            for (int c = 0; c < 6; ++c) nb[d][c] = __ldg(P.u_in + c * S + vB);
        } else {
#pragma unroll
            for (int c = 0; c < 6; ++c) nb[d][c] = 0.0;
        }
    }
    // the LSRK register of this thread's four epilogue nodes, loaded now (shared
    // memory, not registers, limits the resident blocks, so they are free)
    double kold[4][6];
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
        for (int c = 0; c < 6; ++c) kold[n][c] = __ldcg(P.k + c * S + gbase + tid + 128 * n);
    cp_async_wait<0>();
    __syncthreads();

    const double d0 = s_D[g + 8 * t4];        // D(q = g, l = t)
    const double d1 = s_D[g + 8 * (4 + t4)];  // D(q = g, l = 4 + t)
    const double rx = s_geo->met[0], sy = s_geo->met[4], tz = s_geo->met[8];

    // ---- 2. r and s contractions, combined in registers --------------------------
    // residual components: 0 Ex, 1 Ey, 2 Ez, 3 Hx, 4 Hy, 5 Hz (E: +curl H, H: -curl E)
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        const int k = warp + 4 * n;
        // r (original form): A[line j = g][l = t] = u(i = 4h + t, j = g, k)
        auto rder = [&](int c, double& c0, double& c1) {
            const double* U = s_u + c * UE + UK * k + UJ * g + t4;
            c0 = 0.0;
            c1 = 0.0;
            dmma_f64(c0, c1, U[0], d0);
            dmma_f64(c0, c1, U[4], d1);
        };
        // s (swapped form): B[l = t][line i = g] = u(i = g, j = 4h + t, k)
        auto sder = [&](int c, double& c0, double& c1) {
            const double* U = s_u + c * UE + UK * k + g + UJ * t4;
            c0 = 0.0;
            c1 = 0.0;
            dmma_f64(c0, c1, d0, U[0]);
            dmma_f64(c0, c1, d1, U[4 * UJ]);
        };
        double hzr0, hzr1, hyr0, hyr1, ezr0, ezr1, eyr0, eyr1;
        double hzs0, hzs1, hxs0, hxs1, ezs0, ezs1, exs0, exs1;
        rder(5, hzr0, hzr1); rder(4, hyr0, hyr1); rder(2, ezr0, ezr1); rder(1, eyr0, eyr1);
        sder(5, hzs0, hzs1); sder(3, hxs0, hxs1); sder(2, ezs0, ezs1); sder(0, exs0, exs1);
        // nodes (i = 2t, 2t+1; j = g; k)
        double* R = s_r + RK * k + RJ * g + 2 * t4;
        st2(R + 0 * RE, sy * hzs0, sy * hzs1);                               // Ex (+ t term)
        st2(R + 1 * RE, -rx * hzr0, -rx * hzr1);                             // Ey (+ t term)
        st2(R + 2 * RE, rx * hyr0 - sy * hxs0, rx * hyr1 - sy * hxs1);       // Ez
        st2(R + 3 * RE, -sy * ezs0, -sy * ezs1);                             // Hx (+ t term)
        st2(R + 4 * RE, rx * ezr0, rx * ezr1);                               // Hy (+ t term)
        st2(R + 5 * RE, sy * exs0 - rx * eyr0, sy * exs1 - rx * eyr1);       // Hz
    }
    __syncthreads();

    // ---- 3. t contractions (swapped form), added to the residual ------------------
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const int job = warp + 4 * n;        // 32 jobs: 4 fields x 8 tiles j
        const int fi = job >> 3, j = job & 7;
        const int src = fi == 0 ? 4 : (fi == 1 ? 3 : (fi == 2 ? 1 : 0));   // Hy, Hx, Ey, Ex
        const int dst = fi == 0 ? 0 : (fi == 1 ? 1 : (fi == 2 ? 3 : 4));   // Ex, Ey, Hx, Hy
        const double sc = (fi == 0 || fi == 3) ? -tz : tz;
        // B[l = t][line i = g] = u(i = g, j, k = 4h + t)
        const double* U = s_u + src * UE + UJ * j + g + UK * t4;
        double c0 = 0.0, c1 = 0.0;
        dmma_f64(c0, c1, d0, U[0]);
        dmma_f64(c0, c1, d1, U[4 * UK]);
        // nodes (k = g; i = 2t, 2t+1; j)
        double* R = s_r + dst * RE + RK * g + RJ * j + 2 * t4;
        const double2 v = *reinterpret_cast<const double2*>(R);
        st2(R, v.x + sc * c0, v.y + sc * c1);
    }
    __syncthreads();

    // ---- 4. surface terms, one direction at a time --------------------------------
    const double hc0 = 0.5 * P.c0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int f = d == 0 ? (side ? 1 : 3) : (d == 1 ? (side ? 2 : 0) : (side ? 5 : 4));
        const int m = face_local<N>(f, p, q);
        const int mi = m & 7, mj = (m >> 3) & 7, mk = m >> 6;
        const int mu = mi + UJ * mj + UK * mk, mr = mi + RJ * mj + RK * mk;
        double own[6], jmp[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) own[c] = s_u[c * UE + mu];
        if (mirror[d]) {
            wall_jumps(wall[d], own[0], own[1], own[2], own[3], own[4], own[5], jmp);
        } else {
#pragma unroll
            for (int c = 0; c < 6; ++c) jmp[c] = nb[d][c] - own[c];
        }
        double fl[6];
        numerical_flux<double>(s_geo->nrm[f][0], s_geo->nrm[f][1], s_geo->nrm[f][2], hc0, jmp[0],
                               jmp[1], jmp[2], jmp[3], jmp[4], jmp[5], fl);
        const double lift = s_geo->lift[f];
#pragma unroll
        for (int c = 0; c < 6; ++c) s_r[c * RE + mr] += lift * fl[c];
        __syncthreads();
    }

    // ---- 5. LSRK45 update (src/device/dg_kernels.cu:404-406), FP64 -------------
    const double A = P.a, B = P.b, DT = P.dt;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const int x = tid + 128 * n;
        const int i = x & 7, j = (x >> 3) & 7, k = x >> 6;
        const int au = i + UJ * j + UK * k, ar = i + RJ * j + RK * k;
        const long long gi = gbase + x;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double kn = A * kold[n][c] + DT * s_r[c * RE + ar];
            __stcs(P.k + c * S + gi, kn);
            __stcs(P.u_out + c * S + gi, s_u[c * UE + au] + B * kn);
        }
    }
}

template <int MINB>
__global__ void __launch_bounds__(128, MINB) stage_kernel_mma8(const StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    stage_tile_mma8(P, blockIdx.x, smem, threadIdx.x);
}

template <int MINB>
cudaError_t launch_mma8(const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    constexpr int smem = MmaLayout8::total;
    auto kern = stage_kernel_mma8<MINB>;
    if (cfg) *cfg = StageConfig{2, 1, 128, smem, 0, MINB};
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (!p) return cudaSuccess;
    kern<<<p->nelt, 128, smem, st>>>(*p);
    return cudaGetLastError();
}

}  // namespace stage
}  // namespace nwb
