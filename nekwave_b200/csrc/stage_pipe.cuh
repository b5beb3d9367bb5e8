// stage_pipe.cuh -- second family of fused stage kernels.
//
// Same arithmetic as stage_tile (stage_kernel.cuh): per element the volume curl,
// the numerical flux with its lift, and the LSRK45 update, each residual entry
// formed once in a fixed order.  Independent options change the schedule
// and the shared-memory traffic:
//
//   PIPE   the block stays resident and walks the tiles t = blockIdx.x,
//          blockIdx.x + gridDim.x, ...; while it computes tile t, the asynchronous
//          copies of its next tile (u_in, per-element geometry and connections) are
//          in flight into a second buffer and that tile's k lines are being pulled
//          into L2.  Without PIPE a block computes one tile, as stage_tile does.
//   SPLIT  (KS = 2) the two threads of a node column split the residual by field
//          instead of by planes: thread h = 0 forms the E residual (curl H) and
//          h = 1 the H residual (-curl E), each for all N planes (KS = 1: one thread
//          forms both, one after the other, with the same arithmetic).  The components
//          a thread differentiates along t are read once per column into
//          registers, so shared memory serves only the r and s derivatives, and
//          each thread lifts, updates and stores three components.
//   PAD    rows of the shared-memory tile are N+1 doubles apart (node (i,j,k) of
//          an element at i + (N+1)(j + N k)), which spreads the traces of the
//          r-faces (i = 0, N-1) and the rows of the r-derivative over the banks.
//   CONSTD (with SPLIT, FP64) the plane loop is unrolled, so the t-derivative's
//          D(k,l) are compile-time indices into a kernel-parameter copy of D (Dc,
//          StageParams::Dc or the pool's per-N parameter) and enter the FMAs as
//          constant-bank operands instead of shared loads.
//   FACEFIRST (without PIPE) the whole face phase runs from global memory (own and
//          neighbour traces, connections, normals and lifts through the read-only
//          path) while the tile's copies are in flight; the column phase follows
//          the wait.  The face phase's latency then overlaps the tile's.
//   DSMEM  (with SPLIT) the D rows a thread contracts with are read from shared
//          memory at each use instead of being held in 2N registers, which buys
//          resident blocks for the latency-bound orders at the price of more
//          shared loads.
//   EARLY  (without PIPE) the neighbour traces of the tile's face points are
//          requested from global memory right after the tile's copies are issued,
//          before the block waits for them, so both latencies overlap.  On a
//          structured box mesh (StageParams::snel) the neighbour element follows
//          from the element index, so no connection-table read precedes them.
//
// In every form the face phase requests the neighbour values of all of a thread's
// face points before it forms any flux, and each node's k is read before the
// derivative sums that hide its latency.
#pragma once
#include "stage_kernel.cuh"

#include <cstdint>

namespace nwb {
namespace stage {

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
    unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}

// Number of SM identifiers of the GPU (%nsmid: at least the number of SMs).
__device__ __forceinline__ int sm_ids() {
    unsigned n;
    asm("mov.u32 %0, %%nsmid;\n" : "=r"(n));
    return static_cast<int>(n);
}

// Tile of the block that starts about AHEAD/2 waves of resident blocks after block
// b (a wave = the SMs times the MINB resident blocks per SM), or -1 past the grid.
// Blocks are handed out in about index order, so that block starts about half a
// (AHEAD = 1) or one (AHEAD = 2) block lifetime later; the order is not guaranteed,
// and a pull that misses only costs L2 traffic.
template <int AHEAD, int MINB>
__device__ __forceinline__ int tile_ahead(int b) {
    const long long a = static_cast<long long>(b) + static_cast<long long>(sm_ids()) * MINB * AHEAD / 2;
    return a < static_cast<long long>(gridDim.x) ? static_cast<int>(a) : -1;
}

// Nodes [g0, g0 + cnt) of the six components of u and of k (component stride S)
// pulled into L2 by twelve bulk prefetches (one thread; nothing waits on them), for
// the block that will load them later: its own copies then read L2 instead of DRAM.
// The ranges are rounded out to 16-byte boundaries, which stay inside the state
// arrays (components are 512-byte aligned and padded to 64 doubles).
__device__ __forceinline__ void prefetch_nodes_l2(const double* u, const double* k, long long S,
                                                  long long g0, long long cnt) {
    const long long a0 = g0 & ~1ll, a1 = (g0 + cnt + 1) & ~1ll;
    const unsigned bytes = static_cast<unsigned>((a1 - a0) * 8);
#pragma unroll
    for (int c = 0; c < 6; ++c)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(u + c * S + a0), "r"(bytes)
                     : "memory");
#pragma unroll
    for (int c = 0; c < 6; ++c)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(k + c * S + a0), "r"(bytes)
                     : "memory");
}

// The u_in and k of the tile of elements [e0, e0 + n) pulled into L2.
template <int N3>
__device__ __forceinline__ void prefetch_tile_l2(const StageParams& P, int e0, int n) {
    prefetch_nodes_l2(P.u_in, P.k, P.stride, static_cast<long long>(e0) * N3, static_cast<long long>(n) * N3);
}

// The no-op L2 pull of a tile function (see bulk_tile).
struct NoPull {
    __device__ __forceinline__ void operator()() const {}
};

// FP32-bulk, affine classes: an element runs the FP64 column arithmetic when the
// largest deviation of its tile from the per-element linear fit exceeds this
// fraction of the largest deviation from its centre value (in any component).
constexpr float kFp64Fallback = 0.125f;

// Shared-memory index of local node n = i + N j + N^2 k of a tile (element-major).
template <int N, bool PAD>
__device__ __forceinline__ int pidx(int n) {
    if constexpr (PAD) return n + n / N;
    else return n;
}

template <int N, bool F32, int EPB, bool PIPE, bool PAD>
struct Layout2 {
    static constexpr int N2 = N * N, N3 = N2 * N;
    static constexpr int EN3 = PAD ? N2 * (N + 1) : N3;                  // element stride
    static constexpr int CS = EPB * EN3;                                  // component stride
    static constexpr int NB = PIPE ? 2 : 1;                               // buffers
    static constexpr int tile = 6 * CS * 8;
    static constexpr int geo_b = EPB * static_cast<int>(sizeof(ElemGeo));
    static constexpr int conn_b = align16(EPB * 6 * 4);
    static constexpr int u0 = 0;
    static constexpr int geo0 = u0 + NB * tile;
    static constexpr int conn0 = geo0 + NB * geo_b;
    static constexpr int D = conn0 + NB * conn_b;
    static constexpr int flux = D + align16(N2 * 8);
    static constexpr int uc = flux + EPB * 36 * N2 * 8;
    // FP32-bulk: the tile's deviations [6][CS] floats, then per element the linear
    // fit ([6][4]: centre value, slopes along r, s, t) and its curl ([6]), then zl,
    // then per element the largest deviation and variation (FP64 fallback test)
    static constexpr int LIN = 30;
    static constexpr int total = uc + (F32 ? align16(6 * CS * 4) + align16((EPB * LIN + 10) * 8) +
                                                 align16(EPB * 2 * 4)
                                           : 0);
    static_assert(tile % 16 == 0 && geo_b % 16 == 0, "16-byte aligned buffers");
};

// Asynchronous copies of the tile that starts at element e0 into one buffer set.
// Unpadded even N: the tile and every component start on a 16-byte boundary
// (e0*N^3*8 and stride*8 are multiples of 16), so the copies move 16 bytes each.
template <int N, int GEO, int EPB, int NT, bool PAD>
__device__ __forceinline__ void issue2(const StageParams& P, const int e0, double* su, ElemGeo* sg,
                                       int* sc, const int tid) {
    constexpr int N3 = N * N * N;
    constexpr int CS = EPB * (PAD ? N * N * (N + 1) : N3);
    const int nvalid = min(EPB, P.nelt - e0);
    const long long gbase = static_cast<long long>(e0) * N3;
    const long long S = P.stride;
    const int cnt = nvalid * N3;
    if constexpr (N % 2 == 0 && !PAD) {
        const int c2 = cnt / 2;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double* src = P.u_in + c * S + gbase;
            double* dst = su + c * CS;
            for (int x = tid; x < c2; x += NT) cp_async16(dst + 2 * x, src + 2 * x);
        }
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double* src = P.u_in + c * S + gbase;
            double* dst = su + c * CS;
            for (int x = tid; x < cnt; x += NT) cp_async8(dst + pidx<N, PAD>(x), src + x);
        }
    }
    if constexpr (GEO != GEO_NODAL) {
        constexpr int chunks = static_cast<int>(sizeof(ElemGeo) / 16);
        const char* gsrc = reinterpret_cast<const char*>(P.geo + e0);
        char* gdst = reinterpret_cast<char*>(sg);
        for (int x = tid; x < nvalid * chunks; x += NT) cp_async16(gdst + 16 * x, gsrc + 16 * x);
        for (int x = tid; x < nvalid * 6; x += NT) cp_async4(sc + x, P.conn + e0 * 6 + x);
    }
    // the tile's k lines into L2; the owner threads read them in the column phase
    const int lines = (cnt * 8 + 127) / 128;
    for (int x = tid; x < 6 * lines; x += NT) {
        const int c = x / lines, ln = x - c * lines;
        const double* a = P.k + c * S + gbase + ln * 16;
        asm volatile("prefetch.global.L2 [%0];\n" ::"l"(a));
    }
}

// Lifted face terms of node (i,j,k) for the NC components starting at c0, added
// in the reference's face order 0..5.
template <int N, int NC>
__device__ __forceinline__ void add_lifts(const double* Fl, int c0, int i, int j, int k, double* rhs) {
    constexpr int N2 = N * N;
    if (j == 0) {
        const double* F = Fl + 0 * 6 * N2 + (i + N * k) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
    if (i == N - 1) {
        const double* F = Fl + 1 * 6 * N2 + (j + N * k) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
    if (j == N - 1) {
        const double* F = Fl + 2 * 6 * N2 + (i + N * k) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
    if (i == 0) {
        const double* F = Fl + 3 * 6 * N2 + (j + N * k) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
    if (k == 0) {
        const double* F = Fl + 4 * 6 * N2 + (i + N * j) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
    if (k == N - 1) {
        const double* F = Fl + 5 * 6 * N2 + (i + N * j) + c0 * N2;
#pragma unroll
        for (int c = 0; c < NC; ++c) rhs[c] += F[c * N2];
    }
}

// Numerical flux of one face point.  On an axis-aligned element (GEO_BOX) the
// normal of face f lies along the axis of its reference direction (x for faces 1
// and 3, y for 0 and 2, z for 4 and 5).  When its other two components are exactly
// zero, n = s e_d, n x v = s (e_d x v) and n x (n x v) = -(v without its d
// component), so the flux of src/device/dg_kernels.cu:264-294 reduces to eight
// products (the normal components of both fields are zero); otherwise, and for
// the other classes, the general form.  Used where a warp's face points never
// span two faces (N^2 a multiple of 32): elsewhere the three branches diverge
// within a warp and cost more than they save.
template <typename TC, int GEO, int N>
__device__ __forceinline__ void face_flux(int f, double nxd, double nyd, double nzd, double c0,
                                          const double* jmp, TC* fl) {
    if constexpr (GEO == GEO_BOX && (N * N) % 32 == 0) {
        const TC dEx = static_cast<TC>(jmp[0]), dEy = static_cast<TC>(jmp[1]), dEz = static_cast<TC>(jmp[2]);
        const TC dHx = static_cast<TC>(jmp[3]), dHy = static_cast<TC>(jmp[4]), dHz = static_cast<TC>(jmp[5]);
        const TC hc0 = static_cast<TC>(0.5 * c0);
        if ((f == 1 || f == 3) && nyd == 0.0 && nzd == 0.0) {
            const TC hs = static_cast<TC>(0.5 * nxd);
            fl[0] = TC(0); fl[3] = TC(0);
            fl[1] = hc0 * dEy - hs * dHz; fl[2] = hs * dHy + hc0 * dEz;
            fl[4] = hs * dEz + hc0 * dHy; fl[5] = hc0 * dHz - hs * dEy;
            return;
        }
        if ((f == 0 || f == 2) && nxd == 0.0 && nzd == 0.0) {
            const TC hs = static_cast<TC>(0.5 * nyd);
            fl[1] = TC(0); fl[4] = TC(0);
            fl[0] = hs * dHz + hc0 * dEx; fl[2] = hc0 * dEz - hs * dHx;
            fl[3] = hc0 * dHx - hs * dEz; fl[5] = hs * dEx + hc0 * dHz;
            return;
        }
        if ((f == 4 || f == 5) && nxd == 0.0 && nyd == 0.0) {
            const TC hs = static_cast<TC>(0.5 * nzd);
            fl[2] = TC(0); fl[5] = TC(0);
            fl[0] = hc0 * dEx - hs * dHy; fl[1] = hs * dHx + hc0 * dEy;
            fl[3] = hs * dEy + hc0 * dHx; fl[4] = hc0 * dHy - hs * dEx;
            return;
        }
    }
    numerical_flux<TC>(static_cast<TC>(nxd), static_cast<TC>(nyd), static_cast<TC>(nzd),
                       static_cast<TC>(0.5 * c0), static_cast<TC>(jmp[0]), static_cast<TC>(jmp[1]),
                       static_cast<TC>(jmp[2]), static_cast<TC>(jmp[3]), static_cast<TC>(jmp[4]),
                       static_cast<TC>(jmp[5]), fl);
}

// Neighbour element across face f of element e of a structured box mesh
// (x-fastest element order, faces 0..5 = y-, x+, y+, x-, z-, z+), -1 where the
// face lies on a non-periodic wall; the matching face is the opposite one with
// the identity orientation.
__device__ __forceinline__ int struct_neighbour(const StageParams& P, int ex, int ey, int ez, int e,
                                                int f) {
    const int nx = P.snel[0], ny = P.snel[1], nz = P.snel[2], pm = P.spmask;
    const int sx = 1, sy = nx, sz = nx * ny;
    switch (f) {
        case 0: return ey > 0 ? e - sy : ((pm & 2) ? e + sy * (ny - 1) : -1);
        case 1: return ex < nx - 1 ? e + sx : ((pm & 1) ? e - sx * (nx - 1) : -1);
        case 2: return ey < ny - 1 ? e + sy : ((pm & 2) ? e - sy * (ny - 1) : -1);
        case 3: return ex > 0 ? e - sx : ((pm & 1) ? e + sx * (nx - 1) : -1);
        case 4: return ez > 0 ? e - sz : ((pm & 4) ? e + sz * (nz - 1) : -1);
        default: return ez < nz - 1 ? e + sz : ((pm & 4) ? e - sz * (nz - 1) : -1);
    }
}

// Neighbour values of the face points of one thread (FPT of them): the global
// node vB across each point (< 0: the wall code kConnPEC or kConnPMC) and its six
// field values.
template <int FPT>
struct FaceGather {
    double nb[FPT][6];
    long long vB[FPT];
};

// Fill a FaceGather.  FROM_SMEM: the tile is resident (connections from sc,
// neighbours inside the tile from su); otherwise only global memory is read, so
// it may run while the tile's copies are still in flight.
template <int N, int GEO, int KS, int EPB, bool PAD, bool FROM_SMEM, int FPT, int CSX = 0>
__device__ __forceinline__ void gather2(const StageParams& P, const int e0, const double* su,
                                        const int* sc, const int tid, FaceGather<FPT>& G) {
    constexpr int N2 = N * N, N3 = N2 * N;
    constexpr int TPE = KS * N2;
    // component stride of the shared tile (CSX: a tile with slack between components)
    constexpr int CS = CSX ? CSX : EPB * (PAD ? N2 * (N + 1) : N3);
    const int team = tid / TPE;
    const int lt = tid - team * TPE;
    const int nvalid = min(EPB, P.nelt - e0);
    const int e = e0 + team;
    const long long S = P.stride;
    // the tile-resident form reads the connection table from shared memory; the
    // early form uses the structure when there is one
    const bool structured = !FROM_SMEM && P.snel[0] > 0;
    int ex = 0, ey = 0, ez = 0;
    if (structured) {
        ex = e % P.snel[0];
        const int r = e / P.snel[0];
        ey = r % P.snel[1];
        ez = r / P.snel[1];
    }
#pragma unroll
    for (int q = 0; q < FPT; ++q) {
        const int fp = lt + q * TPE;
        long long vB = kConnPEC;  // < 0: a wall code
        if (team < nvalid && fp < 6 * N2) {
            const int f = fp / N2;
            const int pq = fp - f * N2;
            const int p = pq % N, qq = pq / N;
            int eB = -1;
            if constexpr (GEO == GEO_NODAL) {
                vB = P.fplus[(static_cast<long long>(e) * 6 + f) * N2 + pq];
                if (vB >= 0) eB = static_cast<int>(vB / N3);
            } else if (structured) {
                eB = struct_neighbour(P, ex, ey, ez, e, f);
                if (eB >= 0) {
                    constexpr int opp[6] = {2, 3, 0, 1, 5, 4};
                    vB = static_cast<long long>(eB) * N3 + face_local<N>(opp[f], p, qq);
                }
            } else {
                int cd;
                if constexpr (FROM_SMEM) cd = sc[team * 6 + f];
                else cd = __ldg(P.conn + e * 6 + f);
                vB = cd;
                if (cd >= 0) {
                    const int fB = (cd >> 3) & 7, o = cd & 7;
                    eB = cd >> 6;
                    int a = (o & 4) ? qq : p;
                    int b = (o & 4) ? p : qq;
                    if (o & 1) a = N - 1 - a;
                    if (o & 2) b = N - 1 - b;
                    vB = static_cast<long long>(eB) * N3 + face_local<N>(fB, a, b);
                }
            }
            if (vB >= 0) {
                bool in_tile = false;
                if constexpr (FROM_SMEM) in_tile = eB >= e0 && eB < e0 + nvalid;
                if (in_tile) {
                    const int el = eB - e0;
                    constexpr int EN3 = PAD ? N2 * (N + 1) : N3;  // element stride in the tile
                    const int sidx = el * EN3 + pidx<N, PAD>(static_cast<int>(vB - static_cast<long long>(eB) * N3));
#pragma unroll
                    for (int c = 0; c < 6; ++c) G.nb[q][c] = su[c * CS + sidx];
                } else {
#pragma unroll
                    for (int c = 0; c < 6; ++c) G.nb[q][c] = __ldg(P.u_in + c * S + vB);
                }
            }
        }
        G.vB[q] = vB;
    }
}

// Face phase and column phase of one tile whose u_in, geometry and connections
// are resident in (su, sg, sc).  All threads of the block call it; threads
// tid >= EPB*KS*N*N take part in the barrier only.
template <int N, int KS>
__host__ __device__ constexpr int face_points_per_thread() {
    return (6 * N * N + KS * N * N - 1) / (KS * N * N);
}

// Face phase of one tile: one thread per face point (FPT per thread), neighbour
// values of all of a thread's points requested first (unless EARLY already did),
// then the numerical flux of each point times its lift, stored in sflux
// [team][face][component][point].  The caller synchronises afterwards.
template <int N, int GEO, bool F32, int KS, int EPB, bool PAD, bool EARLY, int CSX = 0>
__device__ __forceinline__ void face_phase2(const StageParams& P, const int e0, const double* su,
                                            const ElemGeo* sg, const int* sc, double* sflux,
                                            const int tid,
                                            FaceGather<face_points_per_thread<N, KS>()>& G) {
    using TC = typename std::conditional<F32, float, double>::type;
    constexpr int N2 = N * N;
    constexpr int RP = PAD ? N + 1 : N;
    constexpr int EN3 = RP * N * N;
    constexpr int TPE = KS * N2;
    constexpr int CS = CSX ? CSX : EPB * EN3;
    constexpr int FPT = face_points_per_thread<N, KS>();
    const int team = tid / TPE;
    const int lt = tid - team * TPE;
    const int nvalid = min(EPB, P.nelt - e0);
    const int e = e0 + team;
    const bool active = team < nvalid;
    if constexpr (!EARLY) gather2<N, GEO, KS, EPB, PAD, true, FPT, CSX>(P, e0, su, sc, tid, G);
    if (active) {
        const double* U = su + team * EN3;
#pragma unroll
        for (int q = 0; q < FPT; ++q) {
            const int fp = lt + q * TPE;
            if (fp >= 6 * N2) break;
            const int f = fp / N2;
            const int pq = fp - f * N2;
            const int p = pq % N, qq = pq / N;
            const int m = pidx<N, PAD>(face_local<N>(f, p, qq));
            const double Exm = U[0 * CS + m], Eym = U[1 * CS + m], Ezm = U[2 * CS + m];
            const double Hxm = U[3 * CS + m], Hym = U[4 * CS + m], Hzm = U[5 * CS + m];
            double nxd, nyd, nzd, lift;
            if constexpr (GEO == GEO_NODAL) {
                const long long g = (static_cast<long long>(e) * 6 + f) * N2 + pq;
                nxd = P.fnrm[g];
                nyd = P.fnrm[P.nfp + g];
                nzd = P.fnrm[2 * P.nfp + g];
                lift = P.flift[g];
            } else {
                const ElemGeo& G = sg[team];
                nxd = G.nrm[f][0];
                nyd = G.nrm[f][1];
                nzd = G.nrm[f][2];
                lift = G.lift[f];
            }
            double jmp[6];
            if (G.vB[q] < 0) {
                wall_jumps(G.vB[q], Exm, Eym, Ezm, Hxm, Hym, Hzm, jmp);
            } else {
                jmp[0] = G.nb[q][0] - Exm; jmp[1] = G.nb[q][1] - Eym; jmp[2] = G.nb[q][2] - Ezm;
                jmp[3] = G.nb[q][3] - Hxm; jmp[4] = G.nb[q][4] - Hym; jmp[5] = G.nb[q][5] - Hzm;
            }
            TC fl[6];
            face_flux<TC, GEO, N>(f, nxd, nyd, nzd, P.c0, jmp, fl);
            double* F = sflux + (team * 6 + f) * 6 * N2 + pq;
#pragma unroll
            for (int c = 0; c < 6; ++c) F[c * N2] = lift * static_cast<double>(fl[c]);
        }
    }
}

// Face phase from global memory only: own and neighbour traces, connections (or
// the box structure), normals and lifts, so that it runs while the tile's copies
// are in flight.  Writes the lifted fluxes into sflux like face_phase2; the caller
// synchronises after waiting for the tile.
template <int N, int GEO, bool F32, int KS, int EPB>
__device__ __forceinline__ void face_phase_global(const StageParams& P, const int e0, double* sflux,
                                                  const int tid) {
    using TC = typename std::conditional<F32, float, double>::type;
    constexpr int N2 = N * N, N3 = N2 * N;
    constexpr int TPE = KS * N2;
    constexpr int FPT = face_points_per_thread<N, KS>();
    const int team = tid / TPE;
    const int lt = tid - team * TPE;
    const int e = e0 + team;
    if (team >= min(EPB, P.nelt - e0)) return;
    const long long S = P.stride;
    FaceGather<FPT> G;
    gather2<N, GEO, KS, EPB, false, false>(P, e0, nullptr, nullptr, tid, G);
    double own[FPT][6];
#pragma unroll
    for (int q = 0; q < FPT; ++q) {
        const int fp = lt + q * TPE;
        if (fp < 6 * N2) {
            const int f = fp / N2;
            const int pq = fp - f * N2;
            const long long g = static_cast<long long>(e) * N3 + face_local<N>(f, pq % N, pq / N);
#pragma unroll
            for (int c = 0; c < 6; ++c) own[q][c] = __ldg(P.u_in + c * S + g);
        }
    }
#pragma unroll
    for (int q = 0; q < FPT; ++q) {
        const int fp = lt + q * TPE;
        if (fp >= 6 * N2) break;
        const int f = fp / N2;
        const int pq = fp - f * N2;
        double nxd, nyd, nzd, lift;
        if constexpr (GEO == GEO_NODAL) {
            const long long gf = (static_cast<long long>(e) * 6 + f) * N2 + pq;
            nxd = __ldg(P.fnrm + gf);
            nyd = __ldg(P.fnrm + P.nfp + gf);
            nzd = __ldg(P.fnrm + 2 * P.nfp + gf);
            lift = __ldg(P.flift + gf);
        } else {
            const ElemGeo* Gp = P.geo + e;
            nxd = __ldg(&Gp->nrm[f][0]);
            nyd = __ldg(&Gp->nrm[f][1]);
            nzd = __ldg(&Gp->nrm[f][2]);
            lift = __ldg(&Gp->lift[f]);
        }
        double jmp[6];
        if (G.vB[q] < 0) {
            wall_jumps(G.vB[q], own[q][0], own[q][1], own[q][2], own[q][3], own[q][4], own[q][5], jmp);
        } else {
#pragma unroll
            for (int c = 0; c < 6; ++c) jmp[c] = G.nb[q][c] - own[q][c];
        }
        TC fl[6];
        face_flux<TC, GEO, N>(f, nxd, nyd, nzd, P.c0, jmp, fl);
        double* F = sflux + (team * 6 + f) * 6 * N2 + pq;
#pragma unroll
        for (int c = 0; c < 6; ++c) F[c * N2] = lift * static_cast<double>(fl[c]);
    }
}

// Barrier of the threads that share one tile (the whole block in every form here).
struct CtaBar {
    __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// The N values of a node row p[0..N-1] in shared memory with 16-byte loads.  Even N:
// p must be 16-byte aligned.  Odd N: the loads start at the 16-byte boundary at or
// below p, so they also read one neighbouring value (p[-1] or p[N]), which must lie
// inside the tile's shared memory and is discarded.
template <int N>
__device__ __forceinline__ void row_pairs(const double* p, double (&r)[N]) {
    if constexpr (N % 2 == 0) {
        const double2* b = reinterpret_cast<const double2*>(p);
#pragma unroll
        for (int q = 0; q < N / 2; ++q) {
            const double2 v = b[q];
            r[2 * q] = v.x;
            r[2 * q + 1] = v.y;
        }
    } else {
        const int a = static_cast<int>((reinterpret_cast<uintptr_t>(p) >> 3) & 1);
        const double2* b = reinterpret_cast<const double2*>(p - a);
        double w[N + 1];
#pragma unroll
        for (int q = 0; q < (N + 1) / 2; ++q) {
            const double2 v = b[q];
            w[2 * q] = v.x;
            w[2 * q + 1] = v.y;
        }
#pragma unroll
        for (int l = 0; l < N; ++l) r[l] = a ? w[l + 1] : w[l];
    }
}

// VROW (FP64 field split on unpadded tiles whose components and elements start on
// 16-byte boundaries for even N: the bulk-copy tile): the r-derivative's node rows
// are read with 16-byte loads (row_pairs), half the shared loads of that sum.  The
// arithmetic and its order are unchanged.  ILP2 (axis-aligned field split): each
// derivative sum is formed as two partial sums (even and odd l) added at the end,
// two independent FMA chains per sum instead of one (a different rounding order).
template <int N, int GEO, bool F32, int KS, int EPB, bool SPLIT, bool PAD, bool CONSTD = false,
          bool EARLY = false, bool FACEDONE = false, bool DSMEM = false, class Bar = CtaBar,
          int CSX = 0, bool KSM = false, bool VROW = false, bool ILP2 = false>
__device__ __forceinline__ void compute2(const StageParams& P, const int e0, const double* su,
                                         const ElemGeo* sg, const int* sc, const double* sD,
                                         double* sflux, unsigned char* smem_uc, const int tid,
                                         FaceGather<face_points_per_thread<N, KS>()>& G,
                                         const double* __restrict__ Dc = nullptr, Bar bar = Bar(),
                                         const double* sk = nullptr) {
    using TC = typename std::conditional<F32, float, double>::type;
    constexpr int N2 = N * N, N3 = N2 * N;
    constexpr int RP = PAD ? N + 1 : N;              // row pitch in shared memory
    constexpr int PP = RP * N;                       // plane pitch
    constexpr int EN3 = PP * N;                      // element stride
    constexpr int TPE = KS * N2;
    constexpr int NT = EPB * TPE;
    constexpr int KPT = (N + KS - 1) / KS;
    constexpr int CS = CSX ? CSX : EPB * EN3;
    static_assert(CSX == 0 || !F32, "tiles with slack: FP64 only");
    static_assert(!KSM || (!PAD && !F32), "k in shared memory: unpadded FP64 tiles");
    static_assert(!SPLIT || KS == 1 || KS == 2, "the field split: one or two threads per column");
    static_assert(!CONSTD || (SPLIT && !F32), "constant-bank D: FP64 field split only");
    static_assert(!VROW || (SPLIT && !F32 && !PAD && CSX % 2 == 0), "row pairs: FP64 split, unpadded");

    const int team = tid / TPE;
    const int lt = tid - team * TPE;
    const int loc = lt % N2;
    const int h = lt / N2;
    const int i = loc % N;
    const int j = loc / N;
    const int nvalid = min(EPB, P.nelt - e0);
    const int e = e0 + team;
    const bool active = team < nvalid;
    const long long S = P.stride;

    const TC* s_uc;
    // FP32-bulk, affine classes: per element the linear fit's curl, added in FP64
    constexpr int LIN = 30;
    const double* s_lin = nullptr;
    unsigned* s_fb = nullptr;  // per element: bits of the largest |w| and |u - centre|
    if constexpr (F32 && GEO == GEO_NODAL) {
        // FP32 copy of the tile as deviations from the element's centre node: the
        // derivatives are unchanged (rows of D sum to zero) and the rounding error
        // scales with the variation across the element instead of |u|
        TC* w = reinterpret_cast<TC*>(smem_uc);
        constexpr int centre = (N / 2) * (1 + RP + PP);
        const int cnt = tid < NT ? nvalid * EN3 : 0;
#pragma unroll
        for (int c = 0; c < 6; ++c)
            for (int x = tid; x < cnt; x += NT) {
                const double ref = su[c * CS + (x / EN3) * EN3 + centre];
                w[c * CS + x] = static_cast<float>(su[c * CS + x] - ref);
            }
        s_uc = w;
    } else if constexpr (F32) {
        // FP32 copy of the tile as deviations w = u - L from a linear function L of
        // the line coordinates zl, one per element and component (centre value and
        // the slopes between opposite faces through the centre lines).  D zl = 1, so
        // grad u = grad_FP32(w) + grad L, and on an affine element curl L is one
        // constant per residual component, formed here in FP64 and added to the
        // residual.  The FP32 rounding then scales with the departure from linear
        // across the element instead of with the variation.
        TC* w = reinterpret_cast<TC*>(smem_uc);
        constexpr int lin_off = (6 * CS * 4 + 15) & ~15;  // after the deviations (Layout2::uc)
        double* lin = reinterpret_cast<double*>(smem_uc + lin_off);
        double* szl = lin + EPB * LIN;
        s_fb = reinterpret_cast<unsigned*>(szl + 10);
        if (tid < 2 * EPB) s_fb[tid] = 0u;  // formed in (c), after the face phase's barrier
        constexpr int ic = N / 2;
        const double inv = 1.0 / (P.zl[N - 1] - P.zl[0]);
        const int nlin = tid < NT ? nvalid * 6 : 0;
        if (tid == 0) {
            // constant indices: a runtime index would move a caller's local P into
            // local memory
#pragma unroll
            for (int x = 0; x < N; ++x) szl[x] = P.zl[x];
        }
        // (a) centre value and slopes of each component
        for (int x = tid; x < nlin; x += NT) {
            const int el = x / 6, c = x - 6 * el;
            const double* U = su + c * CS + el * EN3;
            double* Lc = lin + el * LIN + 4 * c;
            Lc[0] = U[ic + RP * ic + PP * ic];
            Lc[1] = (U[(N - 1) + RP * ic + PP * ic] - U[RP * ic + PP * ic]) * inv;
            Lc[2] = (U[ic + RP * (N - 1) + PP * ic] - U[ic + PP * ic]) * inv;
            Lc[3] = (U[ic + RP * ic + PP * (N - 1)] - U[ic + RP * ic]) * inv;
        }
        // (b) curl of L with the residual's sign: +curl H_L for E, -curl E_L for H
        // (physical gradient = J^-T applied to the slopes; met = rx,sx,tx,ry,...,tz)
        for (int x = tid; x < nlin; x += NT) {
            const int el = x / 6, rc = x - 6 * el;
            const int fld = rc / 3, q = rc - 3 * fld;
            const int o = fld == 0 ? 3 : 0;  // the differentiated field
            const double* m = sg[el].met;
            double gr[3][3];                 // gr[comp][axis]
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double* U = su + (o + c) * CS + el * EN3;
                const double ar = (U[(N - 1) + RP * ic + PP * ic] - U[RP * ic + PP * ic]) * inv;
                const double as = (U[ic + RP * (N - 1) + PP * ic] - U[ic + PP * ic]) * inv;
                const double at = (U[ic + RP * ic + PP * (N - 1)] - U[ic + RP * ic]) * inv;
#pragma unroll
                for (int d = 0; d < 3; ++d) gr[c][d] = m[3 * d] * ar + m[3 * d + 1] * as + m[3 * d + 2] * at;
            }
            const double cx = gr[2][1] - gr[1][2], cy = gr[0][2] - gr[2][0], cz = gr[1][0] - gr[0][1];
            const double cq = q == 0 ? cx : (q == 1 ? cy : cz);
            lin[el * LIN + 24 + rc] = fld == 0 ? cq : -cq;
        }
        // (c), the deviations, follows the face phase's barrier
        s_uc = w;
        s_lin = lin;
    } else {
        s_uc = reinterpret_cast<const TC*>(su);
    }

    // ---- face phase (unless the caller ran it from global memory) -------------------
    if constexpr (!FACEDONE)
        face_phase2<N, GEO, F32, KS, EPB, PAD, EARLY, CSX>(P, e0, su, sg, sc, sflux, tid, G);
    bar.sync();

    if constexpr (F32 && GEO != GEO_NODAL) {
        // (c) FP32-bulk deviations w = u - L: each thread takes its own node column
        // (i, j) of its element, planes h, h + KS, ... (the fit is complete: it was
        // formed before the face phase's barrier)
        if (active) {
            TC* w = reinterpret_cast<TC*>(smem_uc);
            const double* szl = s_lin + EPB * LIN;
            constexpr int ic = N / 2;
            const double zi = szl[i] - szl[ic], zj = szl[j] - szl[ic];
            float wmax = 0.f, vmax = 0.f;
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const double* Lc = s_lin + team * LIN + 4 * c;
                const double base = Lc[0] + Lc[1] * zi + Lc[2] * zj;
                const double at = Lc[3];
                const int col = c * CS + team * EN3 + i + RP * j;
                for (int k = h; k < N; k += KS) {
                    const double Lv = base + at * (szl[k] - szl[ic]);
                    const float wv = static_cast<float>(su[col + PP * k] - Lv);
                    w[col + PP * k] = wv;
                    wmax = fmaxf(wmax, fabsf(wv));
                    vmax = fmaxf(vmax, fabsf(static_cast<float>(su[col + PP * k] - Lc[0])));
                }
            }
            // non-negative floats order as their bit patterns
            atomicMax(s_fb + 2 * team, __float_as_uint(wmax));
            atomicMax(s_fb + 2 * team + 1, __float_as_uint(vmax));
        }
        bar.sync();
    }

    // ---- column phase: volume curl + face terms + LSRK update ------------------
    if (!active) return;
    const TC* U = s_uc + team * EN3;
    const double* Uf = su + team * EN3;
    const double* Fl = sflux + team * 36 * N2;
    TC Dr[N], Ds[N];
#pragma unroll
    for (int l = 0; l < N; ++l) {
        Dr[l] = static_cast<TC>(sD[i + l * N]);
        Ds[l] = static_cast<TC>(sD[j + l * N]);
    }
    TC m_[9];
    if constexpr (GEO != GEO_NODAL) {
#pragma unroll
        for (int c = 0; c < 9; ++c) m_[c] = static_cast<TC>(sg[team].met[c]);
    }
    const double A = P.a, B = P.b, DT = P.dt;
    const long long ebase = static_cast<long long>(e) * N3;

    if constexpr (SPLIT) {
        // FP32-bulk: an element whose deviations from its linear fit are not small
        // against its variation (a field resolved within one or two elements, where
        // the fit removes little) runs the FP64 arithmetic on u itself: its FP32
        // rounding would not shrink with the deviations there.
        bool fb64 = false;
        if constexpr (F32 && GEO != GEO_NODAL)
            fb64 = __uint_as_float(s_fb[2 * team]) > kFp64Fallback * __uint_as_float(s_fb[2 * team + 1]);
        // the column work in arithmetic type TX (TC, or FP64 for a fallback element)
        auto columns = [&](auto zero) {
        using TX = decltype(zero);
        constexpr bool SAME = std::is_same<TX, TC>::value;
        const TX* ubase;
        if constexpr (SAME) ubase = U;
        else ubase = Uf;
        auto met = [&](int c) -> TX {
            if constexpr (SAME) return m_[c];
            else return static_cast<TX>(sg[team].met[c]);
        };
        // field hf = 0: E residual from V = H (+curl H); hf = 1: H residual from V = E
        // (-curl E).  KS = 2: thread h takes field h; KS = 1: one thread takes both,
        // one after the other, with the same arithmetic per node.
#pragma unroll 1
        for (int hf = (KS == 2 ? h : 0); hf < (KS == 2 ? h + 1 : 2); ++hf) {
        const int src = hf == 0 ? 3 : 0;
        const int dst = 3 - src;
        const double sgn = hf == 0 ? 1.0 : -1.0;
        const TX* V = ubase + src * CS;
        constexpr int NC = GEO == GEO_BOX ? 2 : 3;  // components differentiated along t
        TX col[NC][N];
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int l = 0; l < N; ++l) col[c][l] = V[c * CS + i + RP * j + PP * l];
        // CONSTD (plane loop unrolled): k of the next plane is requested before this
        // plane's stores, which the compiler may not move a later load above, so its
        // latency overlaps the sums (B200: 3-5% faster at N = 7, 9; the rolled loop
        // is faster without it)
        double knext[3];
        // KSM: k staged in shared memory with the tile's layout (unpadded)
        const double* Kf = KSM ? sk + team * EN3 : nullptr;
        if constexpr (CONSTD) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
                knext[c] = KSM ? Kf[(dst + c) * CS + i + RP * j] : __ldcg(P.k + (dst + c) * S + ebase + i + N * j);
        }
#pragma unroll (CONSTD ? N : 1)
        for (int k = 0; k < N; ++k) {
            const int mn = i + N * j + N2 * k;           // node in natural numbering
            const int ms = i + RP * j + PP * k;          // node in shared memory
            const long long g = ebase + mn;
            double kold[3];
            if constexpr (CONSTD) {
#pragma unroll
                for (int c = 0; c < 3; ++c) kold[c] = knext[c];
                if (k + 1 < N) {
#pragma unroll
                    for (int c = 0; c < 3; ++c)
                        knext[c] = KSM ? Kf[(dst + c) * CS + ms + PP] : __ldcg(P.k + (dst + c) * S + g + N2);
                }
            } else {
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    kold[c] = KSM ? Kf[(dst + c) * CS + ms] : __ldcg(P.k + (dst + c) * S + g);
            }
            double rhs[3];
            if constexpr (GEO == GEO_BOX) {
                TX Vz_r = 0, Vy_r = 0, Vz_s = 0, Vx_s = 0, Vy_t = 0, Vx_t = 0;
                TX rowz[N], rowy[N];
                if constexpr (VROW) {
                    row_pairs<N>(V + 2 * CS + PP * k + RP * j, rowz);
                    row_pairs<N>(V + 1 * CS + PP * k + RP * j, rowy);
                }
                // ILP2: odd l into a second set of partial sums, added at the end
                TX Wz_r = 0, Wy_r = 0, Wz_s = 0, Wx_s = 0, Wy_t = 0, Wx_t = 0;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    const TX dr = (DSMEM || !SAME) ? static_cast<TX>(sD[i + l * N]) : static_cast<TX>(Dr[l]);
                    const TX ds = (DSMEM || !SAME) ? static_cast<TX>(sD[j + l * N]) : static_cast<TX>(Ds[l]);
                    const TX dt = CONSTD ? static_cast<TX>(Dc[k + l * N]) : static_cast<TX>(sD[k + l * N]);
                    const int is = PP * k + RP * l + i;
                    const bool odd = ILP2 && (l & 1);
                    TX& az_r = odd ? Wz_r : Vz_r; TX& ay_r = odd ? Wy_r : Vy_r;
                    TX& az_s = odd ? Wz_s : Vz_s; TX& ax_s = odd ? Wx_s : Vx_s;
                    TX& ay_t = odd ? Wy_t : Vy_t; TX& ax_t = odd ? Wx_t : Vx_t;
                    if constexpr (VROW) {
                        az_r += dr * rowz[l]; ay_r += dr * rowy[l];
                    } else {
                        const int ir = PP * k + RP * j + l;
                        az_r += dr * V[2 * CS + ir]; ay_r += dr * V[1 * CS + ir];
                    }
                    az_s += ds * V[2 * CS + is]; ax_s += ds * V[0 * CS + is];
                    ay_t += dt * col[1][l]; ax_t += dt * col[0][l];
                }
                if constexpr (ILP2) {
                    Vz_r += Wz_r; Vy_r += Wy_r; Vz_s += Wz_s; Vx_s += Wx_s; Vy_t += Wy_t; Vx_t += Wx_t;
                }
                const TX rx = met(0), sy = met(4), tz = met(8);
                rhs[0] = sgn * static_cast<double>(sy * Vz_s - tz * Vy_t);
                rhs[1] = sgn * static_cast<double>(tz * Vx_t - rx * Vz_r);
                rhs[2] = sgn * static_cast<double>(rx * Vy_r - sy * Vx_s);
            } else {
                TX dr_[3] = {0, 0, 0}, ds_[3] = {0, 0, 0}, dt_[3] = {0, 0, 0};
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    const TX dr = (DSMEM || !SAME) ? static_cast<TX>(sD[i + l * N]) : static_cast<TX>(Dr[l]);
                    const TX ds = (DSMEM || !SAME) ? static_cast<TX>(sD[j + l * N]) : static_cast<TX>(Ds[l]);
                    const TX dt = CONSTD ? static_cast<TX>(Dc[k + l * N]) : static_cast<TX>(sD[k + l * N]);
                    const int ir = PP * k + RP * j + l;
                    const int is = PP * k + RP * l + i;
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        dr_[c] += dr * V[c * CS + ir];
                        ds_[c] += ds * V[c * CS + is];
                        dt_[c] += dt * col[c][l];
                    }
                }
                TX rx, sx, tx, ry, sy, ty, rz, sz, tz;
                if constexpr (GEO == GEO_NODAL) {
                    rx = static_cast<TX>(P.met_n[0 * S + g]); sx = static_cast<TX>(P.met_n[1 * S + g]);
                    tx = static_cast<TX>(P.met_n[2 * S + g]); ry = static_cast<TX>(P.met_n[3 * S + g]);
                    sy = static_cast<TX>(P.met_n[4 * S + g]); ty = static_cast<TX>(P.met_n[5 * S + g]);
                    rz = static_cast<TX>(P.met_n[6 * S + g]); sz = static_cast<TX>(P.met_n[7 * S + g]);
                    tz = static_cast<TX>(P.met_n[8 * S + g]);
                } else {
                    rx = met(0); sx = met(1); tx = met(2); ry = met(3); sy = met(4);
                    ty = met(5); rz = met(6); sz = met(7); tz = met(8);
                }
                // physical curl, src/device/dg_kernels.cu:140-149
                const TX c1 = (dr_[2] * ry + ds_[2] * sy + dt_[2] * ty) - (dr_[1] * rz + ds_[1] * sz + dt_[1] * tz);
                const TX c2 = (dr_[0] * rz + ds_[0] * sz + dt_[0] * tz) - (dr_[2] * rx + ds_[2] * sx + dt_[2] * tx);
                const TX c3 = (dr_[1] * rx + ds_[1] * sx + dt_[1] * tx) - (dr_[0] * ry + ds_[0] * sy + dt_[0] * ty);
                rhs[0] = sgn * static_cast<double>(c1);
                rhs[1] = sgn * static_cast<double>(c2);
                rhs[2] = sgn * static_cast<double>(c3);
            }
            if constexpr (F32 && GEO != GEO_NODAL && SAME) {
#pragma unroll
                for (int c = 0; c < 3; ++c) rhs[c] += s_lin[team * LIN + 24 + dst + c];
            }
            add_lifts<N, 3>(Fl, dst, i, j, k, rhs);
            // LSRK45 (src/device/dg_kernels.cu:404-406), FP64
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double kn = A * kold[c] + DT * rhs[c];
                __stcs(P.k + (dst + c) * S + g, kn);
                __stcs(P.u_out + (dst + c) * S + g, Uf[(dst + c) * CS + ms] + B * kn);
            }
        }
        }
        };
        if constexpr (F32 && GEO != GEO_NODAL) {
            if (fb64) columns(0.0);
            else columns(0.0f);
        } else {
            columns(TC(0));
        }
    } else {
        // one plane at a time: the register budget goes to the batched loads
#pragma unroll 1
        for (int kk = 0; kk < KPT; ++kk) {
            const int k = h * KPT + kk;
            if (KS > 1 && k >= N) break;
            const int mn = i + N * j + N2 * k;
            const int ms = i + RP * j + PP * k;
            const long long g = ebase + mn;
            double kold[6];
#pragma unroll
            for (int c = 0; c < 6; ++c)
                kold[c] = KSM ? sk[c * CS + team * EN3 + ms] : __ldcg(P.k + c * S + g);
            double rhs[6];
            if constexpr (GEO == GEO_BOX) {
                TC Hz_r = 0, Hy_r = 0, Ez_r = 0, Ey_r = 0;
                TC Hz_s = 0, Hx_s = 0, Ez_s = 0, Ex_s = 0;
                TC Hy_t = 0, Hx_t = 0, Ey_t = 0, Ex_t = 0;
#pragma unroll
                for (int l = 0; l < N; ++l) {
                    const TC dr = Dr[l], ds = Ds[l];
                    const TC dt = static_cast<TC>(sD[k + l * N]);
                    const int ir = PP * k + RP * j + l;
                    const int is = PP * k + RP * l + i;
                    const int it = PP * l + RP * j + i;
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
                    const TC dt = static_cast<TC>(sD[k + l * N]);
                    const int ir = PP * k + RP * j + l;
                    const int is = PP * k + RP * l + i;
                    const int it = PP * l + RP * j + i;
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        dr_[c] += dr * U[c * CS + ir];
                        ds_[c] += ds * U[c * CS + is];
                        dt_[c] += dt * U[c * CS + it];
                    }
                }
                TC rx, sx, tx, ry, sy, ty, rz, sz, tz;
                if constexpr (GEO == GEO_NODAL) {
                    rx = static_cast<TC>(P.met_n[0 * S + g]); sx = static_cast<TC>(P.met_n[1 * S + g]);
                    tx = static_cast<TC>(P.met_n[2 * S + g]); ry = static_cast<TC>(P.met_n[3 * S + g]);
                    sy = static_cast<TC>(P.met_n[4 * S + g]); ty = static_cast<TC>(P.met_n[5 * S + g]);
                    rz = static_cast<TC>(P.met_n[6 * S + g]); sz = static_cast<TC>(P.met_n[7 * S + g]);
                    tz = static_cast<TC>(P.met_n[8 * S + g]);
                } else {
                    rx = m_[0]; sx = m_[1]; tx = m_[2]; ry = m_[3]; sy = m_[4];
                    ty = m_[5]; rz = m_[6]; sz = m_[7]; tz = m_[8];
                }
                // physical curl, src/device/dg_kernels.cu:140-149
#pragma unroll
                for (int fld = 0; fld < 2; ++fld) {
                    const int o = fld == 0 ? 3 : 0;
                    const TC u1r = dr_[o], u1s = ds_[o], u1t = dt_[o];
                    const TC u2r = dr_[o + 1], u2s = ds_[o + 1], u2t = dt_[o + 1];
                    const TC u3r = dr_[o + 2], u3s = ds_[o + 2], u3t = dt_[o + 2];
                    const TC c1 = (u3r * ry + u3s * sy + u3t * ty) - (u2r * rz + u2s * sz + u2t * tz);
                    const TC c2 = (u1r * rz + u1s * sz + u1t * tz) - (u3r * rx + u3s * sx + u3t * tx);
                    const TC c3 = (u2r * rx + u2s * sx + u2t * tx) - (u1r * ry + u1s * sy + u1t * ty);
                    const double sg_ = fld == 0 ? 1.0 : -1.0;
                    rhs[3 * fld + 0] = sg_ * static_cast<double>(c1);
                    rhs[3 * fld + 1] = sg_ * static_cast<double>(c2);
                    rhs[3 * fld + 2] = sg_ * static_cast<double>(c3);
                }
            }
            if constexpr (F32 && GEO != GEO_NODAL) {
#pragma unroll
                for (int c = 0; c < 6; ++c) rhs[c] += s_lin[team * LIN + 24 + c];
            }
            add_lifts<N, 6>(Fl, 0, i, j, k, rhs);
            // LSRK45 (src/device/dg_kernels.cu:404-406), FP64
#pragma unroll
            for (int c = 0; c < 6; ++c) {
                const double kn = A * kold[c] + DT * rhs[c];
                __stcs(P.k + c * S + g, kn);
                __stcs(P.u_out + c * S + g, Uf[c * CS + ms] + B * kn);
            }
        }
    }
}

template <int N, int GEO, bool F32, int KS, int EPB, int MINB, bool PIPE, bool SPLIT, bool PAD,
          bool CONSTD, bool EARLY, bool FACEFIRST, bool DSMEM>
__global__ void __launch_bounds__(EPB * KS * N * N, MINB)
    stage2_kernel(const __grid_constant__ StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    using L = Layout2<N, F32, EPB, PIPE, PAD>;
    constexpr int NT = EPB * KS * N * N;
    const int tid = threadIdx.x;
    const int ntiles = (P.nelt + EPB - 1) / EPB;
    int t = blockIdx.x;
    if (t >= ntiles) return;
    double* sD = reinterpret_cast<double*>(smem + L::D);
    double* sflux = reinterpret_cast<double*>(smem + L::flux);
    for (int x = tid; x < N * N; x += NT) cp_async8(sD + x, P.D + x);
    auto su = [&](int b) { return reinterpret_cast<double*>(smem + L::u0 + b * L::tile); };
    auto sg = [&](int b) { return reinterpret_cast<ElemGeo*>(smem + L::geo0 + b * L::geo_b); };
    auto sc = [&](int b) { return reinterpret_cast<int*>(smem + L::conn0 + b * L::conn_b); };
    static_assert(!((EARLY || FACEFIRST) && PIPE), "early forms belong to the one-tile form");
    FaceGather<face_points_per_thread<N, KS>()> G;
    issue2<N, GEO, EPB, NT, PAD>(P, t * EPB, su(0), sg(0), sc(0), tid);
    cp_async_commit();
    if constexpr (!PIPE) {
        if constexpr (FACEFIRST) face_phase_global<N, GEO, F32, KS, EPB>(P, t * EPB, sflux, tid);
        else if constexpr (EARLY) gather2<N, GEO, KS, EPB, PAD, false>(P, t * EPB, nullptr, nullptr, tid, G);
        cp_async_wait<0>();
        __syncthreads();
        compute2<N, GEO, F32, KS, EPB, SPLIT, PAD, CONSTD, EARLY, FACEFIRST, DSMEM>(
            P, t * EPB, su(0), sg(0), sc(0), sD, sflux, smem + L::uc, tid, G, P.Dc);
    } else {
        for (int n = 0; t < ntiles; ++n, t += gridDim.x) {
            const int b = n & 1;
            cp_async_wait<0>();
            __syncthreads();  // tile t resident; every thread is done with the other buffer
            const int tn = t + gridDim.x;
            if (tn < ntiles) issue2<N, GEO, EPB, NT, PAD>(P, tn * EPB, su(b ^ 1), sg(b ^ 1), sc(b ^ 1), tid);
            cp_async_commit();
            compute2<N, GEO, F32, KS, EPB, SPLIT, PAD, CONSTD, false, false, DSMEM>(
                P, t * EPB, su(b), sg(b), sc(b), sD, sflux, smem + L::uc, tid, G, P.Dc);
        }
        cp_async_wait<0>();
    }
}

// Launch of one variant of the family.  PIPE: as many blocks as fit on the device
// at once (queried with the occupancy calculator on the first call, which the
// solver makes at creation, outside any stream capture), never more than tiles.
template <int N, int GEO, bool F32, int KS, int EPB, int MINB, bool PIPE, bool SPLIT, bool PAD,
          bool CONSTD, bool EARLY, bool FACEFIRST, bool DSMEM>
cudaError_t launch2(const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    constexpr int threads = EPB * KS * N * N;
    constexpr int smem = Layout2<N, F32, EPB, PIPE, PAD>::total;
    auto kern = stage2_kernel<N, GEO, F32, KS, EPB, MINB, PIPE, SPLIT, PAD, CONSTD, EARLY, FACEFIRST, DSMEM>;
    if (cfg) *cfg = StageConfig{KS, EPB, threads, smem, 0, MINB};
    // resident blocks on the device, per kernel and device (0: not yet set up)
    static std::atomic<int> resident[kMaxDeviceSlots];
    int dev = 0;
    if (cudaError_t e = current_device_slot(&dev); e != cudaSuccess) return e;
    if (resident[dev].load(std::memory_order_acquire) == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        int sms = 0, occ = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem);
        if (e != cudaSuccess) return e;
        if (occ < 1) return cudaErrorInvalidConfiguration;
        resident[dev].store(occ * sms, std::memory_order_release);
    }
    const int res = resident[dev].load(std::memory_order_acquire);
    if (!p) return cudaSuccess;
    const int tiles = (p->nelt + EPB - 1) / EPB;
    const int blocks = PIPE ? (tiles < res ? tiles : res) : tiles;
    kern<<<blocks, threads, smem, st>>>(*p);
    return cudaGetLastError();
}

}  // namespace stage
}  // namespace nwb
