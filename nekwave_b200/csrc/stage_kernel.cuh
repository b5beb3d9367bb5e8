// stage_kernel.cuh -- the fused LSRK45 stage kernel for sm_100a.
//
// One launch performs, for every element, everything the reference does in
// seven launches per stage (src/dg_solver.cpp:393-505):
//   volume curl of H and E        (src/device/dg_kernels.cu:41-155, twice)
//   face traces, numerical flux   (:170-304; PEC mirror and neighbour traces)
//   surface lift and inverse mass (:316-382, without atomics)
//   LSRK45 update                 (:393-408)
// The state is ping-ponged (u_in -> u_out) because neighbour traces of u_in are
// read while other blocks write their updated elements; k is updated in place.
//
// Block = EPB elements; each element is handled by a team of KS*N*N threads,
// thread (i,j,h) owning node column (i,j) for the planes k of its share h.
// Per block:
//   1. cp.async stages u_in of the EPB elements in shared memory; k is either
//      staged too (second commit group, it arrives while the flux and volume
//      work runs) or prefetched into L2 and read directly by its owner thread;
//   2. face phase: one thread per face point computes the numerical flux from
//      its own trace (shared memory) and the neighbour trace (shared memory if
//      the neighbour is in the same block, else global/L2), multiplies it by the
//      FP64 lift dA/(J w3) and stores it in shared memory;
//   3. column phase: GLL sum-factorised derivatives from shared memory, the
//      physical curl, the lifted face terms of the faces the node lies on, the
//      LSRK update in FP64, and coalesced stores of k and u_out.
// Each residual entry is formed once by one thread in a fixed order: the
// kernel is deterministic (the reference's atomic lift is not).
#pragma once
#include "nwb_internal.h"

#include <atomic>
#include <type_traits>

namespace nwb {
namespace stage {

__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int n>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(n) : "memory");
}

// Local node of face point (p,q) on face f: Mesh::getFaceNodeVolIndex without
// the element offset (src/mesh.cpp:955-981).
template <int N>
__device__ __forceinline__ int face_local(int f, int p, int q) {
    switch (f) {
        case 0: return p + N * N * q;                      // s = -1: i=p, j=0,   k=q
        case 1: return (N - 1) + N * p + N * N * q;        // r = +1: i=N-1, j=p, k=q
        case 2: return p + N * (N - 1) + N * N * q;        // s = +1: i=p, j=N-1, k=q
        case 3: return N * p + N * N * q;                  // r = -1: i=0,   j=p, k=q
        case 4: return p + N * q;                          // t = -1: i=p, j=q,   k=0
        default: return p + N * q + N * N * (N - 1);       // t = +1: i=p, j=q,   k=N-1
    }
}

constexpr int align16(int b) { return (b + 15) & ~15; }

template <int N, bool F32, int EPB, bool KSMEM>
struct SmemLayout {
    static constexpr int N2 = N * N, N3 = N2 * N;
    static constexpr int u = 0;
    static constexpr int k = u + EPB * 6 * N3 * 8;
    static constexpr int D = k + (KSMEM ? EPB * 6 * N3 * 8 : 0);
    static constexpr int geo = D + align16(N2 * 8);
    static constexpr int conn = geo + EPB * static_cast<int>(sizeof(ElemGeo));
    static constexpr int flux = conn + align16(EPB * 6 * 4);
    static constexpr int uc = flux + EPB * 36 * N2 * 8;
    static constexpr int total = uc + (F32 ? EPB * 6 * N3 * 4 : 0);
};

// Numerical flux of src/device/dg_kernels.cu:264-294 for jumps dE = E+ - E-,
// dH = H+ - H-: fH = -1/2 n x[[E]] - c0/2 n x(n x[[H]]), fE = +1/2 n x[[H]] - c0/2 n x(n x[[E]]).
template <typename T>
__device__ __forceinline__ void numerical_flux(T nx, T ny, T nz, T hc0, T dEx, T dEy, T dEz,
                                               T dHx, T dHy, T dHz, T f[6]) {
    const T nxE_x = ny * dEz - nz * dEy;
    const T nxE_y = nz * dEx - nx * dEz;
    const T nxE_z = nx * dEy - ny * dEx;
    const T nxH_x = ny * dHz - nz * dHy;
    const T nxH_y = nz * dHx - nx * dHz;
    const T nxH_z = nx * dHy - ny * dHx;
    const T nnE_x = ny * nxE_z - nz * nxE_y;
    const T nnE_y = nz * nxE_x - nx * nxE_z;
    const T nnE_z = nx * nxE_y - ny * nxE_x;
    const T nnH_x = ny * nxH_z - nz * nxH_y;
    const T nnH_y = nz * nxH_x - nx * nxH_z;
    const T nnH_z = nx * nxH_y - ny * nxH_x;
    const T half = T(0.5);
    // residual order: E components first, then H (the reference lifts flux[3..5]
    // into resE and flux[0..2] into resH, src/device/dg_kernels.cu:329-336)
    f[0] = half * nxH_x - hc0 * nnE_x;
    f[1] = half * nxH_y - hc0 * nnE_y;
    f[2] = half * nxH_z - hc0 * nnE_z;
    f[3] = -half * nxE_x - hc0 * nnH_x;
    f[4] = -half * nxE_y - hc0 * nnH_y;
    f[5] = -half * nxE_z - hc0 * nnH_z;
}

// Jumps at a wall face point (neighbour code < 0) from the own traces (E-, H-).
// kConnPEC: the PEC mirror [[E]] = -2E-, [[H]] = 0 of src/device/dg_kernels.cu:243-251,
// which the reference also applies to PMC faces.  kConnPMC (solvers created with
// NWB_SOLVER_TRUE_PMC only): the PMC mirror [[E]] = 0, [[H]] = -2H-.
__device__ __forceinline__ void wall_jumps(long long code, double Ex, double Ey, double Ez,
                                           double Hx, double Hy, double Hz, double jmp[6]) {
    if (code == kConnPMC) {
        jmp[0] = 0.0; jmp[1] = 0.0; jmp[2] = 0.0;
        jmp[3] = -2.0 * Hx; jmp[4] = -2.0 * Hy; jmp[5] = -2.0 * Hz;
    } else {
        jmp[0] = -2.0 * Ex; jmp[1] = -2.0 * Ey; jmp[2] = -2.0 * Ez;
        jmp[3] = 0.0; jmp[4] = 0.0; jmp[5] = 0.0;
    }
}

// One tile (EPB consecutive elements starting at e0) of one stage.  Called by
// all threads of a block; threads tid >= EPB*KS*N*N take part in the barriers
// only (the batched kernel runs every N in blocks of one fixed size).
template <int N, int GEO, bool F32, int KS, int EPB, bool KSMEM, bool UNROLL_K = true>
__device__ __forceinline__ void stage_tile(const StageParams& P, const int e0,
                                           unsigned char* smem, const int tid) {
    using TC = typename std::conditional<F32, float, double>::type;
    constexpr int N2 = N * N, N3 = N2 * N;
    constexpr int TPE = KS * N2;          // threads per element
    constexpr int NT = EPB * TPE;         // threads per block
    constexpr int KPT = (N + KS - 1) / KS;
    constexpr int CS = EPB * N3;          // component stride in shared memory
    using L = SmemLayout<N, F32, EPB, KSMEM>;

    double* s_u = reinterpret_cast<double*>(smem + L::u);
    double* s_k = reinterpret_cast<double*>(smem + L::k);
    double* s_D = reinterpret_cast<double*>(smem + L::D);
    ElemGeo* s_geo = reinterpret_cast<ElemGeo*>(smem + L::geo);
    int* s_conn = reinterpret_cast<int*>(smem + L::conn);
    double* s_flux = reinterpret_cast<double*>(smem + L::flux);
    TC* s_uc;
    if constexpr (F32) s_uc = reinterpret_cast<TC*>(smem + L::uc);
    else s_uc = reinterpret_cast<TC*>(s_u);

    const int team = tid / TPE;
    const int lt = tid - team * TPE;
    const int loc = lt % N2;
    const int h = lt / N2;
    const int i = loc % N;
    const int j = loc / N;
    const int nvalid = min(EPB, P.nelt - e0);
    const bool loader = tid < NT;
    const int e = e0 + team;
    const bool active = team < nvalid;
    const long long S = P.stride;

    // ---- 1. stage u_in (+ D, geometry) then k in shared memory ---------------
    if (loader) {
        const long long gbase = static_cast<long long>(e0) * N3;
        const int cnt = nvalid * N3;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double* src = P.u_in + c * S + gbase;
            for (int x = tid; x < cnt; x += NT) cp_async8(s_u + c * CS + x, src + x);
        }
        for (int x = tid; x < N2; x += NT) cp_async8(s_D + x, P.D + x);
        if constexpr (GEO != GEO_NODAL) {
            const double* gsrc = reinterpret_cast<const double*>(P.geo + e0);
            double* gdst = reinterpret_cast<double*>(s_geo);
            const int gcnt = nvalid * static_cast<int>(sizeof(ElemGeo) / 8);
            for (int x = tid; x < gcnt; x += NT) cp_async8(gdst + x, gsrc + x);
            for (int x = tid; x < nvalid * 6; x += NT) s_conn[x] = P.conn[e0 * 6 + x];
        }
        cp_async_commit();
        if constexpr (KSMEM) {
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const double* src = P.k + c * S + gbase;
                for (int x = tid; x < cnt; x += NT) cp_async8(s_k + c * CS + x, src + x);
            }
        } else {
            // pull this block's k lines into L2 now; the owner threads read them
            // in the column phase
            const int lines = (cnt * 8 + 127) / 128;
            for (int x = tid; x < 6 * lines; x += NT) {
                const int c = x / lines, ln = x - c * lines;
                const double* a = P.k + c * S + gbase + ln * 16;
                asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a));
            }
        }
    }
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if constexpr (F32) {
        // FP32 copy of the tile as deviations from the element's centre node:
        // the derivatives are unchanged (rows of D sum to zero) and the rounding
        // error scales with the variation across the element instead of |u|
        constexpr int centre = (N / 2) * (1 + N + N2);
        const int cnt = loader ? nvalid * N3 : 0;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            for (int x = tid; x < cnt; x += NT) {
                const double ref = s_u[c * CS + (x / N3) * N3 + centre];
                s_uc[c * CS + x] = static_cast<float>(s_u[c * CS + x] - ref);
            }
        __syncthreads();
    }

    // ---- 2. face phase: lifted numerical flux per face point -----------------
    if (active) {
        // traces and jumps in FP64 in both precision classes: a jump is a small
        // difference of two nearly equal traces and is rounded only afterwards
        const double* U = s_u + team * N3;
        for (int fp = lt; fp < 6 * N2; fp += TPE) {
            const int f = fp / N2;
            const int pq = fp - f * N2;
            const int p = pq % N, q = pq / N;
            const int m = face_local<N>(f, p, q);
            const double Exm = U[0 * CS + m], Eym = U[1 * CS + m], Ezm = U[2 * CS + m];
            const double Hxm = U[3 * CS + m], Hym = U[4 * CS + m], Hzm = U[5 * CS + m];
            long long vB = kConnPEC;  // neighbour node (global index), < 0: a wall code
            double nxd, nyd, nzd, lift;
            if constexpr (GEO == GEO_NODAL) {
                const long long g = (static_cast<long long>(e) * 6 + f) * N2 + pq;
                vB = P.fplus[g];
                nxd = P.fnrm[g];
                nyd = P.fnrm[P.nfp + g];
                nzd = P.fnrm[2 * P.nfp + g];
                lift = P.flift[g];
            } else {
                const int cd = s_conn[team * 6 + f];
                vB = cd;
                if (cd >= 0) {
                    const int eB = cd >> 6, fB = (cd >> 3) & 7, o = cd & 7;
                    int a = (o & 4) ? q : p;
                    int b = (o & 4) ? p : q;
                    if (o & 1) a = N - 1 - a;
                    if (o & 2) b = N - 1 - b;
                    vB = static_cast<long long>(eB) * N3 + face_local<N>(fB, a, b);
                }
                const ElemGeo& G = s_geo[team];
                nxd = G.nrm[f][0];
                nyd = G.nrm[f][1];
                nzd = G.nrm[f][2];
                lift = G.lift[f];
            }
            double jmp[6];
            if (vB < 0) {
                wall_jumps(vB, Exm, Eym, Ezm, Hxm, Hym, Hzm, jmp);
            } else {
                const long long eB = vB / N3;
                double vals[6];
                if (eB >= e0 && eB < e0 + nvalid) {
                    const int sidx = static_cast<int>(vB - static_cast<long long>(e0) * N3);
#pragma unroll
                    for (int c = 0; c < 6; ++c) vals[c] = s_u[c * CS + sidx];
                } else {
#pragma unroll
                    for (int c = 0; c < 6; ++c) vals[c] = __ldg(P.u_in + c * S + vB);
                }
                jmp[0] = vals[0] - Exm; jmp[1] = vals[1] - Eym; jmp[2] = vals[2] - Ezm;
                jmp[3] = vals[3] - Hxm; jmp[4] = vals[4] - Hym; jmp[5] = vals[5] - Hzm;
            }
            TC fl[6];
            numerical_flux<TC>(static_cast<TC>(nxd), static_cast<TC>(nyd), static_cast<TC>(nzd),
                               static_cast<TC>(0.5 * P.c0), static_cast<TC>(jmp[0]),
                               static_cast<TC>(jmp[1]), static_cast<TC>(jmp[2]),
                               static_cast<TC>(jmp[3]), static_cast<TC>(jmp[4]),
                               static_cast<TC>(jmp[5]), fl);
            double* F = s_flux + (team * 6 + f) * 6 * N2 + pq;
#pragma unroll
            for (int c = 0; c < 6; ++c) F[c * N2] = lift * static_cast<double>(fl[c]);
        }
    }
    cp_async_wait<0>();
    __syncthreads();

    // ---- 3. column phase: volume curl + face terms + LSRK update --------------
    if (!active) return;
    const TC* U = s_uc + team * N3;
    const double* Fl = s_flux + team * 36 * N2;
    TC Dr[N], Ds[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        Dr[l] = static_cast<TC>(s_D[i + l * N]);
        Ds[l] = static_cast<TC>(s_D[j + l * N]);
    }
    TC m_[9];
    if constexpr (GEO != GEO_NODAL) {
#pragma unroll
        for (int c = 0; c < 9; ++c) m_[c] = static_cast<TC>(s_geo[team].met[c]);
    }
    const double A = P.a, B = P.b, DT = P.dt;
    const long long ebase = static_cast<long long>(e) * N3;

    // the k-planes of a thread: unrolled (more independent work in flight) unless
    // the caller must stay within a tight register budget
#pragma unroll (UNROLL_K ? KPT : 1)
    for (int kk = 0; kk < KPT; ++kk) {
        const int k = h * KPT + kk;
        if (KS > 1 && k >= N) break;
        const int mloc = i + N * j + N2 * k;
        double rhs[6];
        if constexpr (GEO == GEO_BOX) {
            // only the six derivatives a curl needs when J^{-T} = diag(rx, sy, tz)
            TC Hz_r = 0, Hy_r = 0, Ez_r = 0, Ey_r = 0;
            TC Hz_s = 0, Hx_s = 0, Ez_s = 0, Ex_s = 0;
            TC Hy_t = 0, Hx_t = 0, Ey_t = 0, Ex_t = 0;
#pragma unroll
            for (int l = 0; l < N; ++l) {
                const TC dr = Dr[l], ds = Ds[l];
                const TC dt = static_cast<TC>(s_D[k + l * N]);
                const int ir = N2 * k + N * j + l;
                const int is = N2 * k + N * l + i;
                const int it = N2 * l + N * j + i;
                Hz_r += dr * U[5 * CS + ir]; Hy_r += dr * U[4 * CS + ir];
                Ez_r += dr * U[2 * CS + ir]; Ey_r += dr * U[1 * CS + ir];
                Hz_s += ds * U[5 * CS + is]; Hx_s += ds * U[3 * CS + is];
                Ez_s += ds * U[2 * CS + is]; Ex_s += ds * U[0 * CS + is];
                Hy_t += dt * U[4 * CS + it]; Hx_t += dt * U[3 * CS + it];
                Ey_t += dt * U[1 * CS + it]; Ex_t += dt * U[0 * CS + it];
            }
            const TC rx = m_[0], sy = m_[4], tz = m_[8];
            rhs[0] = static_cast<double>(sy * Hz_s - tz * Hy_t);
            rhs[1] = static_cast<double>(tz * Hx_t - rx * Hz_r);
            rhs[2] = static_cast<double>(rx * Hy_r - sy * Hx_s);
            rhs[3] = static_cast<double>(tz * Ey_t - sy * Ez_s);
            rhs[4] = static_cast<double>(rx * Ez_r - tz * Ex_t);
            rhs[5] = static_cast<double>(sy * Ex_s - rx * Ey_r);
        } else {
            TC dr_[6] = {0, 0, 0, 0, 0, 0}, ds_[6] = {0, 0, 0, 0, 0, 0}, dt_[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int l = 0; l < N; ++l) {
                const TC dr = Dr[l], ds = Ds[l];
                const TC dt = static_cast<TC>(s_D[k + l * N]);
                const int ir = N2 * k + N * j + l;
                const int is = N2 * k + N * l + i;
                const int it = N2 * l + N * j + i;
#pragma unroll
                for (int c = 0; c < 6; ++c) {
                    dr_[c] += dr * U[c * CS + ir];
                    ds_[c] += ds * U[c * CS + is];
                    dt_[c] += dt * U[c * CS + it];
                }
            }
            TC rx, sx, tx, ry, sy, ty, rz, sz, tz;
            if constexpr (GEO == GEO_NODAL) {
                const long long g = ebase + mloc;
                rx = static_cast<TC>(P.met_n[0 * S + g]); sx = static_cast<TC>(P.met_n[1 * S + g]);
                tx = static_cast<TC>(P.met_n[2 * S + g]); ry = static_cast<TC>(P.met_n[3 * S + g]);
                sy = static_cast<TC>(P.met_n[4 * S + g]); ty = static_cast<TC>(P.met_n[5 * S + g]);
                rz = static_cast<TC>(P.met_n[6 * S + g]); sz = static_cast<TC>(P.met_n[7 * S + g]);
                tz = static_cast<TC>(P.met_n[8 * S + g]);
            } else {
                rx = m_[0]; sx = m_[1]; tx = m_[2]; ry = m_[3]; sy = m_[4];
                ty = m_[5]; rz = m_[6]; sz = m_[7]; tz = m_[8];
            }
            // physical curl, src/device/dg_kernels.cu:140-149; E residual = +curl H,
            // H residual = -curl E
#pragma unroll
            for (int fld = 0; fld < 2; ++fld) {
                const int o = fld == 0 ? 3 : 0;
                const TC u1r = dr_[o], u1s = ds_[o], u1t = dt_[o];
                const TC u2r = dr_[o + 1], u2s = ds_[o + 1], u2t = dt_[o + 1];
                const TC u3r = dr_[o + 2], u3s = ds_[o + 2], u3t = dt_[o + 2];
                const TC c1 = (u3r * ry + u3s * sy + u3t * ty) - (u2r * rz + u2s * sz + u2t * tz);
                const TC c2 = (u1r * rz + u1s * sz + u1t * tz) - (u3r * rx + u3s * sx + u3t * tx);
                const TC c3 = (u2r * rx + u2s * sx + u2t * tx) - (u1r * ry + u1s * sy + u1t * ty);
                const double sg = fld == 0 ? 1.0 : -1.0;
                rhs[3 * fld + 0] = sg * static_cast<double>(c1);
                rhs[3 * fld + 1] = sg * static_cast<double>(c2);
                rhs[3 * fld + 2] = sg * static_cast<double>(c3);
            }
        }
        // lifted face terms, faces in the reference's order 0..5
        if (j == 0) {
            const double* F = Fl + 0 * 6 * N2 + (i + N * k);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        if (i == N - 1) {
            const double* F = Fl + 1 * 6 * N2 + (j + N * k);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        if (j == N - 1) {
            const double* F = Fl + 2 * 6 * N2 + (i + N * k);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        if (i == 0) {
            const double* F = Fl + 3 * 6 * N2 + (j + N * k);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        if (k == 0) {
            const double* F = Fl + 4 * 6 * N2 + (i + N * j);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        if (k == N - 1) {
            const double* F = Fl + 5 * 6 * N2 + (i + N * j);
#pragma unroll
            for (int c = 0; c < 6; ++c) rhs[c] += F[c * N2];
        }
        // LSRK45 (src/device/dg_kernels.cu:404-406), FP64
        const int sl = team * N3 + mloc;
        const long long g = ebase + mloc;
        double kold[6];
#pragma unroll
        for (int c = 0; c < 6; ++c) kold[c] = KSMEM ? s_k[c * CS + sl] : __ldcg(P.k + c * S + g);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double kn = A * kold[c] + DT * rhs[c];
            __stcs(P.k + c * S + g, kn);
            __stcs(P.u_out + c * S + g, s_u[c * CS + sl] + B * kn);
        }
    }
}

template <int N, int GEO, bool F32, int KS, int EPB, bool KSMEM, int MINB>
__global__ void __launch_bounds__(EPB * KS * N * N, MINB)
    stage_kernel(const StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    stage_tile<N, GEO, F32, KS, EPB, KSMEM>(P, blockIdx.x * EPB, smem, threadIdx.x);
}

// Launch of one variant.  The opt-in shared-memory size is set on the first
// call, which the solver makes at creation (outside any stream capture).
template <int N, int GEO, bool F32, int KS, int EPB, bool KSMEM, int MINB>
cudaError_t launch_cfg(const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    constexpr int threads = EPB * KS * N * N;
    constexpr int smem = SmemLayout<N, F32, EPB, KSMEM>::total;
    auto kern = stage_kernel<N, GEO, F32, KS, EPB, KSMEM, MINB>;
    if (cfg) *cfg = StageConfig{KS, EPB, threads, smem, KSMEM ? 1 : 0, MINB};
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (!p) return cudaSuccess;
    const int blocks = (p->nelt + EPB - 1) / EPB;
    kern<<<blocks, threads, smem, st>>>(*p);
    return cudaGetLastError();
}

}  // namespace stage
}  // namespace nwb
