// stage_bulk.cuh -- the second-family stage kernel with its tile loaded by the
// bulk-copy engine (FP64; axis-aligned and affine classes).
//
// One block per tile.  Thread 0 issues the tile's u_in, its LSRK register k,
// the per-element geometry and the connections as a dozen cp.async.bulk copies
// (plain copies from this GPU's own memory, no multicast) that complete on one
// mbarrier by byte count; every thread waits for them, then compute2 runs the
// face and column phases as in the other one-tile forms, with k read from
// shared memory.  Against the per-thread cp.async loads of those forms this
// takes a few hundred load instructions per block off the issue slots, and the
// column phase no longer waits on L2 for each plane's k: on B200 the stage runs
// 4-10% faster at 5, 6, 7 and 9 points (the defaults there).
//
// Bulk copies start and end on 16-byte boundaries.  A tile whose first node or
// length is odd (odd N) is copied from the boundary at or below its first value
// to the one at or above its last (at most one double more at either end, inside
// the state arrays: components are 512-byte aligned and rounded up to 64
// doubles) into a component slot with two doubles of slack, and read from
// offset (first node & 1).  Connections are copied the same way (the solver pads
// its connection table to a multiple of four entries; a pool cavity's table
// lies in a 256-byte-rounded range of its arena).
//
// The wait is bounded (kWaitNs of the global timer, about a thousand times a
// normal stage).  When it expires the block records a code in *P.err (when the
// caller keeps one), waits once more, bounded, for its copies, and returns.
#pragma once
#include "stage_pipe.cuh"

#include <cstdint>

namespace nwb {
namespace stage {

constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s
constexpr int kErrTileWait = 1;  // a block's wait for its tile expired

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase of the given parity to complete; false when kWaitNs pass first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (;;) {
        for (int k = 0; k < 32; ++k)
            if (mbar_test(bar, parity)) return true;
        if (global_ns() - t0 > kWaitNs) return false;
    }
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void report(const StageParams& P, int code) {
    if (P.err) atomicCAS(P.err, 0, code);
}

// Shared-memory layout of one tile: u_in (and with KSM k) [6][CSR] doubles with
// slack, geometry, connections, D, the lifted fluxes, the mbarrier and a flag.
template <int N, int EPB, bool KSM>
struct BulkLayout {
    static constexpr int N2 = N * N, N3 = N2 * N;
    static constexpr int CSR = (EPB * N3 + 2 + 1) / 2 * 2;
    static constexpr int tile_u = 6 * CSR * 8;
    static constexpr int u0 = 0;
    static constexpr int k0 = u0 + tile_u;
    static constexpr int geo0 = k0 + (KSM ? tile_u : 0);
    static constexpr int geo_b = EPB * static_cast<int>(sizeof(ElemGeo));
    static constexpr int conn0 = geo0 + geo_b;
    static constexpr int conn_b = align16((EPB * 6 + 6) * 4);
    static constexpr int D = conn0 + conn_b;
    static constexpr int flux0 = D + align16(N2 * 8);
    static constexpr int bar = flux0 + EPB * 36 * N2 * 8;
    static constexpr int flag = bar + 8;
    static constexpr int total = flag + 16;
};

// Thread 0's part of a tile load: the tile's u_in (and with KSM its k; otherwise k's
// lines are prefetched into L2), geometry and connections as bulk copies that
// complete on the mbarrier at smem + L::bar, which must be initialised.
template <int N, int EPB, bool KSM>
__device__ __forceinline__ void bulk_issue(const StageParams& P, const int e0, unsigned char* smem) {
    using L = BulkLayout<N, EPB, KSM>;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::bar);
    const long long S = P.stride;
    const long long g0 = static_cast<long long>(e0) * L::N3;
    const int nvalid = min(EPB, P.nelt - e0);
    const long long a0 = g0 & ~1ll, a1 = (g0 + static_cast<long long>(nvalid) * L::N3 + 1) & ~1ll;
    const unsigned ub = static_cast<unsigned>((a1 - a0) * 8);
    const long long c0 = static_cast<long long>(e0) * 6, c1 = c0 + 6 * nvalid;
    const long long ca0 = c0 & ~3ll, ca1 = (c1 + 3) & ~3ll;
    const unsigned cb = static_cast<unsigned>((ca1 - ca0) * 4);
    const unsigned gb = static_cast<unsigned>(nvalid * sizeof(ElemGeo));
    mbar_arrive_expect_tx(bar, (KSM ? 12 : 6) * ub + gb + cb);
    double* su = reinterpret_cast<double*>(smem + L::u0);
#pragma unroll
    for (int c = 0; c < 6; ++c) bulk_g2s(su + c * L::CSR, P.u_in + c * S + a0, ub, bar);
    if constexpr (KSM) {
        double* sk = reinterpret_cast<double*>(smem + L::k0);
#pragma unroll
        for (int c = 0; c < 6; ++c) bulk_g2s(sk + c * L::CSR, P.k + c * S + a0, ub, bar);
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) bulk_prefetch_l2(P.k + c * S + a0, ub);
    }
    bulk_g2s(smem + L::geo0, P.geo + e0, gb, bar);
    bulk_g2s(smem + L::conn0, P.conn + ca0, cb, bar);
}

// Every thread's wait for the tile issued by bulk_issue: true when it is resident.
// On expiry thread 0 records the code, waits once more (bounded) for the copies so
// that none lands in a finished block, and every thread gets false.
template <int N, int EPB, bool KSM>
__device__ __forceinline__ bool bulk_wait_tile(const StageParams& P, unsigned char* smem, const int tid) {
    using L = BulkLayout<N, EPB, KSM>;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::bar);
    int* flag = reinterpret_cast<int*>(smem + L::flag);
    if (tid == 0) *flag = mbar_wait(bar, 0) ? 1 : 0;
    __syncthreads();
    if (!*flag) {
        if (tid == 0) {
            report(P, kErrTileWait);
            mbar_wait(bar, 0);
        }
        return false;
    }
    mbar_test(bar, 0);  // the phase is complete: acquire the tile for this thread
    return true;
}

// One tile of the bulk-copy one-tile form, for the single-mesh kernel below and
// the pool's per-N kernels.  All NT = EPB*KS*N*N threads of the block call it.
// EARLY: the neighbour traces of the face phase are requested from global memory
// (through the box structure when there is one) while the tile's copies are in
// flight.  VROW: the r-derivative's node rows read with 16-byte loads.  Dc: D where
// the t contraction of CONSTD reads it (a parameter copy).  pull: called by thread 0
// right after it has issued the tile's copies (NoPull, or a functor that pulls a
// later block's tile into L2).
template <int N, int GEO, int KS, int EPB, bool CONSTD, bool DSMEM, bool KSM, bool EARLY,
          bool VROW = false, bool ILP2 = false, class Pull = NoPull>
__device__ __forceinline__ void bulk_tile(const StageParams& P, const int e0, unsigned char* smem,
                                          const int tid, const double* Dc, const Pull& pull = Pull()) {
    static_assert(GEO != GEO_NODAL, "per-element geometry and connections");
    using L = BulkLayout<N, EPB, KSM>;
    constexpr int NT = EPB * KS * N * N;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::bar);
    double* sD = reinterpret_cast<double*>(smem + L::D);
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_fence_init();
    }
    for (int x = tid; x < L::N2; x += NT) sD[x] = P.D[x];
    __syncthreads();
    const long long g0 = static_cast<long long>(e0) * L::N3;
    FaceGather<face_points_per_thread<N, KS>()> G;
    if (tid == 0) {
        bulk_issue<N, EPB, KSM>(P, e0, smem);
        pull();
    }
    if constexpr (EARLY) gather2<N, GEO, KS, EPB, false, false>(P, e0, nullptr, nullptr, tid, G);
    if (!bulk_wait_tile<N, EPB, KSM>(P, smem, tid)) return;
    const int off = static_cast<int>(g0 & 1);
    const double* su = reinterpret_cast<const double*>(smem + L::u0) + off;
    const double* sk = KSM ? reinterpret_cast<const double*>(smem + L::k0) + off : nullptr;
    const ElemGeo* sg = reinterpret_cast<const ElemGeo*>(smem + L::geo0);
    const int* sc = reinterpret_cast<const int*>(smem + L::conn0) + ((e0 * 6) & 3);
    double* sflux = reinterpret_cast<double*>(smem + L::flux0);
    compute2<N, GEO, false, KS, EPB, true, false, CONSTD, EARLY, false, DSMEM, CtaBar, L::CSR, KSM, VROW,
             ILP2>(
        P, e0, su, sg, sc, sD, sflux, nullptr, tid, G, Dc, CtaBar(), sk);
}

// Tile taken by block b.  ZCOL on a structured box whose rows hold whole tiles:
// blocks walk the tiles of one (x-tile, y) column through every z before the next
// column, so an element's z-neighbours (nx*ny elements away in memory) are
// loaded by blocks that run at about the same time and their shared face planes
// come from L2 instead of a second DRAM read.  Otherwise tiles in memory order.
template <int EPB, bool ZCOL>
__device__ __forceinline__ int bulk_tile_index(const StageParams& P, int b) {
    if constexpr (ZCOL) {
        const int nx = P.snel[0], ny = P.snel[1], nz = P.snel[2];
        if (nx > 0 && nx % EPB == 0) {
            const int col = b / nz, ez = b - col * nz;
            const int ntx = nx / EPB;
            const int ey = col / ntx, xt = col - ey * ntx;
            return xt + ntx * (ey + ny * ez);
        }
    }
    return b;
}

// Thread 0's L2 pull of the single-mesh kernel: the tile of the block that starts
// about AHEAD/2 waves of resident blocks after this one (tile_ahead), in the same
// tile order.
template <int N3, int EPB, int MINB, int AHEAD, bool ZCOL>
struct MeshPull {
    const StageParams& P;
    __device__ __forceinline__ void operator()() const {
        const int b = tile_ahead<AHEAD, MINB>(blockIdx.x);
        if (b < 0) return;
        const int e = bulk_tile_index<EPB, ZCOL>(P, b) * EPB;
        prefetch_tile_l2<N3>(P, e, min(EPB, P.nelt - e));
    }
};

// AHEAD (0, 1, 2): block b also pulls into L2 the tile of the block that starts
// about AHEAD/2 waves of resident blocks later, so that block's bulk copies read L2
// instead of DRAM; 0: no pull.  On B200 this pays where few blocks are resident
// (6 and 9 points: 3 and 2 per SM), whose tile waits the other blocks hide least.
template <int N, int GEO, int KS, int EPB, int MINB, bool CONSTD, bool DSMEM, bool KSM, bool EARLY,
          bool ZCOL, bool VROW, bool ILP2, int AHEAD>
__global__ void __launch_bounds__(EPB * KS * N * N, MINB)
    stage_bulk_kernel(const __grid_constant__ StageParams P) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int t = bulk_tile_index<EPB, ZCOL>(P, blockIdx.x);
    if constexpr (AHEAD > 0)
        bulk_tile<N, GEO, KS, EPB, CONSTD, DSMEM, KSM, EARLY, VROW, ILP2>(
            P, t * EPB, smem, threadIdx.x, P.Dc, MeshPull<N * N * N, EPB, MINB, AHEAD, ZCOL>{P});
    else
        bulk_tile<N, GEO, KS, EPB, CONSTD, DSMEM, KSM, EARLY, VROW, ILP2>(P, t * EPB, smem, threadIdx.x, P.Dc);
}

template <int N, int GEO, int KS, int EPB, int MINB, bool CONSTD, bool DSMEM, bool KSM, bool EARLY,
          bool ZCOL, bool VROW, bool ILP2, int AHEAD = 0>
cudaError_t launch_bulk(const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    using L = BulkLayout<N, EPB, KSM>;
    constexpr int threads = EPB * KS * N * N;
    auto kern = stage_bulk_kernel<N, GEO, KS, EPB, MINB, CONSTD, DSMEM, KSM, EARLY, ZCOL, VROW, ILP2, AHEAD>;
    if (cfg) *cfg = StageConfig{KS, EPB, threads, L::total, KSM ? 1 : 0, MINB};
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, L::total, attr_set); e != cudaSuccess) return e;
    if (!p) return cudaSuccess;
    kern<<<(p->nelt + EPB - 1) / EPB, threads, L::total, st>>>(*p);
    return cudaGetLastError();
}

}  // namespace stage
}  // namespace nwb
