// batch.cu -- kernels of the multi-cavity pool: one persistent launch per LSRK
// stage advances every resident cavity, whatever its N and element count.
//
// Blocks of kBatchThreads threads take tiles (EPB consecutive elements of one
// cavity) from a work list through a per-stage atomic counter, largest tiles
// first, and run the same fused stage tile as the single-mesh kernel
// (stage_tile in stage_kernel.cuh) with the N-specialised shape of that tile.
// A cavity's arithmetic does not depend on which other cavities share the
// launch, so each result is bit-identical alone and in any mix.
#include "batch.cuh"
#include "stage_kernel.cuh"
#include "stage_pipe.cuh"
#include "stage_dmma.cuh"
#include "stage_bulk.cuh"

namespace nwb {
namespace {

using stage::SmemLayout;
using stage::stage_tile;

// Shape per N for the batch kernel's blocks (kBatchThreads = 128): KS threads
// per column, EPB elements, ALG the kernel family -- the single-mesh default's
// family and arithmetic for each N (stage_variants.h entry 0), in a shape that
// fits, so a cavity in the pool evolves bit for bit as it does alone.  N = 8 in
// FP64 runs the field-split tensor-core tile (stage_dmma.cuh, 128 threads) as the
// single-mesh default does; ALG below is its FP32-bulk shape.
template <int N> struct BShape;
template <> struct BShape<2> { static constexpr int KS = 2, EPB = 16, ALG = 0; };
template <> struct BShape<3> { static constexpr int KS = 1, EPB = 14, ALG = 0; };
template <> struct BShape<4> { static constexpr int KS = 2, EPB = 4, ALG = 4; };
template <> struct BShape<5> { static constexpr int KS = 2, EPB = 2, ALG = 4; };
template <> struct BShape<6> { static constexpr int KS = 2, EPB = 1, ALG = 4; };
template <> struct BShape<7> { static constexpr int KS = 2, EPB = 1, ALG = 4; };
template <> struct BShape<8> { static constexpr int KS = 2, EPB = 1, ALG = 8; };
template <> struct BShape<9> { static constexpr int KS = 1, EPB = 1, ALG = 4; };
template <> struct BShape<10> { static constexpr int KS = 1, EPB = 1, ALG = 0; };

// N = 8 in FP64: the single-mesh default is the field-split tensor-core tile
template <int N, bool F32>
__host__ __device__ constexpr bool dmma_tile() { return N == 8 && !F32; }

template <int N, bool F32>
constexpr int bsmem() {
    using B = BShape<N>;
    if constexpr (dmma_tile<N, F32>()) return stage::DmmaLayout8::total;
    else if constexpr (B::ALG == 0) return SmemLayout<N, F32, B::EPB, false>::total;
    else return stage::Layout2<N, F32, B::EPB, false, (((B::ALG - 2) & 4) != 0)>::total;
}

// One tile of the second family without the persistent loop: stage u_in (and D,
// geometry, connections), wait, compute.  Threads beyond the shape's count take
// part in the barriers only.
template <int N, bool F32, int KS, int EPB, int ALG>
__device__ __forceinline__ void tile2(const StageParams& P, int e0, unsigned char* smem, int tid,
                                      const double* Dc = nullptr) {
    constexpr bool SPLIT = ((ALG - 2) & 2) != 0, PAD = ((ALG - 2) & 4) != 0;
    constexpr bool CONSTD = ((ALG - 2) & 8) != 0;
    static_assert(((ALG - 2) & 1) == 0 && ((ALG - 2) & 16) == 0, "one tile per call, tile resident");
    using L2 = stage::Layout2<N, F32, EPB, false, PAD>;
    constexpr int NT = EPB * KS * N * N;
    double* sD = reinterpret_cast<double*>(smem + L2::D);
    double* su = reinterpret_cast<double*>(smem + L2::u0);
    ElemGeo* sg = reinterpret_cast<ElemGeo*>(smem + L2::geo0);
    int* sc = reinterpret_cast<int*>(smem + L2::conn0);
    if (tid < NT) {
        for (int x = tid; x < N * N; x += NT) stage::cp_async8(sD + x, P.D + x);
        stage::issue2<N, GEO_BOX, EPB, NT, PAD>(P, e0, su, sg, sc, tid);
    }
    stage::cp_async_commit();
    stage::cp_async_wait<0>();
    __syncthreads();
    stage::FaceGather<stage::face_points_per_thread<N, KS>()> G;
    stage::compute2<N, GEO_BOX, F32, KS, EPB, SPLIT, PAD, CONSTD>(P, e0, su, sg, sc, sD,
                                                                  reinterpret_cast<double*>(smem + L2::flux),
                                                                  smem + L2::uc, tid, G, Dc);
}

template <int N, bool F32>
__device__ __forceinline__ void run_tile(const StageParams& P, int e0, unsigned char* smem, int tid) {
    using B = BShape<N>;
    static_assert(B::KS * B::EPB * N * N <= kBatchThreads, "shape too large");
    if constexpr (dmma_tile<N, F32>())
        stage::dmma8_tile<2>(P, e0, smem, tid,
                             reinterpret_cast<const double*>(smem + stage::DmmaLayout8::D));
    else if constexpr (B::ALG == 0)
        stage_tile<N, GEO_BOX, F32, B::KS, B::EPB, false, false>(P, e0, smem, tid);
    else
        tile2<N, F32, B::KS, B::EPB, B::ALG>(P, e0, smem, tid);
}

// Carpenter-Kennedy LSRK45 (src/dg_solver.cpp:58-69).
__constant__ double c_rk4a[5] = {0.0, -567301805773.0 / 1357537059087.0,
                                 -2404267990393.0 / 2016746695238.0,
                                 -3550918686646.0 / 2091501179385.0,
                                 -1275806237668.0 / 842570457699.0};
__constant__ double c_rk4b[5] = {1432997174477.0 / 9575080441755.0,
                                 5161836677717.0 / 13612068292357.0,
                                 1720146321549.0 / 2090206949498.0,
                                 3134564353537.0 / 4481467310338.0,
                                 2277821191437.0 / 14882151754819.0};

template <bool F32>
__global__ void __launch_bounds__(kBatchThreads, 3)
batch_stage_kernel(const SlotDev* __restrict__ slots, const WorkItem* __restrict__ work,
                   const int* __restrict__ ntiles_p, int* __restrict__ counters, int stage, int dry) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_tile;
    const int tid = threadIdx.x;
    const int ntiles = *ntiles_p;
    for (;;) {
        __syncthreads();  // the previous tile is done with shared memory
        if (tid == 0) s_tile = atomicAdd(&counters[stage], 1);
        __syncthreads();
        const int t = s_tile;
        if (t >= ntiles) break;
        const WorkItem w = work[t];
        const SlotDev& S = slots[w.slot];
        if (!S.active) continue;
        const int par = S.par ^ (stage & 1);
        StageParams P;
        P.u_in = S.u[par];
        P.u_out = S.u[par ^ 1];
        P.k = S.k;
        P.stride = S.stride;
        P.nelt = S.nelt;
        P._pad0 = 0;
        P.D = S.D;
        P.geo = S.geo;
        P.conn = S.conn;
        P.met_n = nullptr;
        P.fnrm = nullptr;
        P.flift = nullptr;
        P.fplus = nullptr;
        P.nfp = 0;
        P.err = nullptr;
        P.snel[0] = P.snel[1] = P.snel[2] = 0;  // connections from the slot's table
        P.spmask = 0;
        for (int x = 0; x < 10; ++x) P.zl[x] = S.zl[x];
        P.c0 = S.c0;
        P.a = dry ? 0.0 : c_rk4a[stage];
        P.b = dry ? 0.0 : c_rk4b[stage];
        P.dt = dry ? 0.0 : S.dt;
        switch (w.N) {
            case 2: run_tile<2, F32>(P, w.e0, smem, tid); break;
            case 3: run_tile<3, F32>(P, w.e0, smem, tid); break;
            case 4: run_tile<4, F32>(P, w.e0, smem, tid); break;
            case 5: run_tile<5, F32>(P, w.e0, smem, tid); break;
            case 6: run_tile<6, F32>(P, w.e0, smem, tid); break;
            case 7: run_tile<7, F32>(P, w.e0, smem, tid); break;
            case 8: run_tile<8, F32>(P, w.e0, smem, tid); break;
            case 9: run_tile<9, F32>(P, w.e0, smem, tid); break;
            case 10: run_tile<10, F32>(P, w.e0, smem, tid); break;
            default: break;
        }
    }
}

// Stage parameters of one tile's slot.
__device__ __forceinline__ StageParams slot_params(const SlotDev& S, int stage, int dry) {
    const int par = S.par ^ (stage & 1);
    StageParams P;
    P.u_in = S.u[par];
    P.u_out = S.u[par ^ 1];
    P.k = S.k;
    P.stride = S.stride;
    P.nelt = S.nelt;
    P._pad0 = 0;
    P.D = S.D;
    P.geo = S.geo;
    P.conn = S.conn;
    P.met_n = nullptr;
    P.fnrm = nullptr;
    P.flift = nullptr;
    P.fplus = nullptr;
    P.nfp = 0;
    P.err = nullptr;
    P.snel[0] = P.snel[1] = P.snel[2] = 0;  // connections from the slot's table
    P.spmask = 0;
    for (int x = 0; x < 10; ++x) P.zl[x] = S.zl[x];
    P.c0 = S.c0;
    P.a = dry ? 0.0 : c_rk4a[stage];
    P.b = dry ? 0.0 : c_rk4b[stage];
    P.dt = dry ? 0.0 : S.dt;
    return P;
}

// D of one N by value, for the constant-bank form of the per-N kernels.
struct DParam {
    double d[100];
};

// One block per tile of one N: the single-mesh kernel's tuned shape for that N,
// fully unrolled, reading its slot from the work item (per-N mode).  ALG 0 is the
// first-family tile (stage_kernel.cuh); ALG 2 + flags (SPLIT = 2, PAD = 4,
// CONSTD = 8 with D from dp; no PIPE: the work list is walked one tile per block)
// the second (stage_pipe.cuh).
template <int N, bool F32, int KS, int EPB, bool KSMEM, int MINB, int ALG>
__global__ void __launch_bounds__(EPB * KS * N * N, MINB)
batch_stage_n_kernel(const SlotDev* __restrict__ slots, const WorkItem* __restrict__ work,
                     int stage, int dry, const __grid_constant__ DParam dp) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WorkItem w = work[blockIdx.x];
    const SlotDev& S = slots[w.slot];
    if (!S.active) return;
    const StageParams P = slot_params(S, stage, dry);
    if constexpr (ALG == 0)
        stage_tile<N, GEO_BOX, F32, KS, EPB, KSMEM, true>(P, w.e0, smem, threadIdx.x);
    else
        tile2<N, F32, KS, EPB, ALG>(P, w.e0, smem, threadIdx.x, dp.d);
}

// N = 8 in FP64, per-N mode: the single-mesh default's field-split tensor-core tile
// (128 threads, one element per block), D from dp (CD) or from shared memory.
template <int MINB, bool CD>
__global__ void __launch_bounds__(128, MINB)
batch_dmma8_kernel(const SlotDev* __restrict__ slots, const WorkItem* __restrict__ work, int stage,
                   int dry, const __grid_constant__ DParam dp) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WorkItem w = work[blockIdx.x];
    const SlotDev& S = slots[w.slot];
    if (!S.active) return;
    const StageParams P = slot_params(S, stage, dry);
    stage::dmma8_tile<2>(P, w.e0, smem, threadIdx.x,
                         CD ? dp.d : reinterpret_cast<const double*>(smem + stage::DmmaLayout8::D));
}

template <bool CD>
cudaError_t launch_dmma8_n(int stage, const SlotDev* slots, const WorkItem* work, int ntiles, int dry,
                           const DParam& dp, cudaStream_t st) {
    constexpr int smem = stage::DmmaLayout8::total;
    auto kern = batch_dmma8_kernel<4, CD>;
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    kern<<<ntiles, 128, smem, st>>>(slots, work, stage, dry, dp);
    return cudaGetLastError();
}

// Per-N shapes of the per-N mode: the single-mesh defaults (stage_variants.h entry
// 0), with the persistent form of N = 4 replaced by its one-tile-per-block form.
// N = 8 in FP64 runs batch_dmma8_kernel instead (NShape<8> is its FP32-bulk shape).
// An ALG with CONSTD runs without it for an N whose cavities do not all share the
// pool's D for that N (same arithmetic, D from shared memory).
template <int N> struct NShape;
template <> struct NShape<2> { static constexpr int KS = 2, EPB = 16, KSM = 1, MINB = 1, ALG = 0; };
template <> struct NShape<3> { static constexpr int KS = 1, EPB = 16, KSM = 0, MINB = 4, ALG = 0; };
template <> struct NShape<4> { static constexpr int KS = 2, EPB = 4, KSM = 0, MINB = 4, ALG = 12; };
template <> struct NShape<5> { static constexpr int KS = 2, EPB = 2, KSM = 0, MINB = 4, ALG = 4; };
template <> struct NShape<6> { static constexpr int KS = 2, EPB = 2, KSM = 0, MINB = 3, ALG = 4; };
template <> struct NShape<7> { static constexpr int KS = 2, EPB = 1, KSM = 0, MINB = 4, ALG = 12; };
template <> struct NShape<8> { static constexpr int KS = 2, EPB = 1, KSM = 0, MINB = 4, ALG = 12; };
template <> struct NShape<9> { static constexpr int KS = 2, EPB = 1, KSM = 0, MINB = 2, ALG = 12; };
template <> struct NShape<10> { static constexpr int KS = 2, EPB = 1, KSM = 0, MINB = 2, ALG = 0; };

// FP64 per-N shapes that run the bulk-copy one-tile form (the single-mesh default
// at these N): k staged in shared memory, CD = t-derivative D from the parameters.
// EARLY = neighbour traces requested while the tile's copies fly.  VROW = the
// r-derivative's node rows read with 16-byte loads.  AHEAD = 1: each block pulls
// into L2 the tile of the block half a wave of resident blocks after it (PoolPull).
template <int N> struct NBulk { static constexpr bool on = false, VROW = false, CD = false, EARLY = false; static constexpr int EPB = 1, MINB = 1, AHEAD = 0; };
template <> struct NBulk<5> { static constexpr bool on = true, VROW = false, CD = true, EARLY = true; static constexpr int EPB = 1, MINB = 8, AHEAD = 0; };
template <> struct NBulk<6> { static constexpr bool on = true, VROW = false, CD = true, EARLY = true; static constexpr int EPB = 2, MINB = 3, AHEAD = 1; };
template <> struct NBulk<7> { static constexpr bool on = true, VROW = false, CD = true, EARLY = true; static constexpr int EPB = 1, MINB = 4, AHEAD = 0; };
template <> struct NBulk<9> { static constexpr bool on = true, VROW = false, CD = true, EARLY = true; static constexpr int EPB = 1, MINB = 2, AHEAD = 1; };

// Thread 0's L2 pull in a per-N bulk kernel: the tile of the work item about AHEAD/2
// waves of resident blocks after this block's (that N's tiles are the grid, one per
// block, in work-list order), in whichever cavity it lies.
template <int N>
struct PoolPull {
    const SlotDev* slots;
    const WorkItem* work;
    int stage;
    __device__ __forceinline__ void operator()() const {
        const int b = stage::tile_ahead<NBulk<N>::AHEAD, NBulk<N>::MINB>(blockIdx.x);
        if (b < 0) return;
        const WorkItem w = work[b];
        const SlotDev& S = slots[w.slot];
        if (!S.active) return;
        constexpr long long N3 = N * N * N;
        stage::prefetch_nodes_l2(S.u[S.par ^ (stage & 1)], S.k, S.stride, w.e0 * N3,
                                 min(NBulk<N>::EPB, S.nelt - w.e0) * N3);
    }
};

template <int N, bool CD>
__global__ void __launch_bounds__(NBulk<N>::EPB * 2 * N * N, NBulk<N>::MINB)
batch_bulk_n_kernel(const SlotDev* __restrict__ slots, const WorkItem* __restrict__ work, int stage,
                    int dry, const __grid_constant__ DParam dp) {
    extern __shared__ __align__(16) unsigned char smem[];
    const WorkItem w = work[blockIdx.x];
    const SlotDev& S = slots[w.slot];
    if (!S.active) return;
    const StageParams P = slot_params(S, stage, dry);
    if constexpr (NBulk<N>::AHEAD > 0)
        stage::bulk_tile<N, GEO_BOX, 2, NBulk<N>::EPB, CD, false, true, NBulk<N>::EARLY, NBulk<N>::VROW>(
            P, w.e0, smem, threadIdx.x, dp.d, PoolPull<N>{slots, work, stage});
    else
        stage::bulk_tile<N, GEO_BOX, 2, NBulk<N>::EPB, CD, false, true, NBulk<N>::EARLY, NBulk<N>::VROW>(
            P, w.e0, smem, threadIdx.x, dp.d);
}

template <int N, bool CD>
cudaError_t launch_bulk_n(int stage, const SlotDev* slots, const WorkItem* work, int ntiles, int dry,
                          const DParam& dp, cudaStream_t st) {
    constexpr int smem = stage::BulkLayout<N, NBulk<N>::EPB, true>::total;
    constexpr int threads = NBulk<N>::EPB * 2 * N * N;
    auto kern = batch_bulk_n_kernel<N, CD>;
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    kern<<<ntiles, threads, smem, st>>>(slots, work, stage, dry, dp);
    return cudaGetLastError();
}

template <int N, bool F32, int ALG>
cudaError_t launch_n_alg(int stage, const SlotDev* slots, const WorkItem* work, int ntiles, int dry,
                         const DParam& dp, cudaStream_t st) {
    using Sh = NShape<N>;
    constexpr int threads = Sh::EPB * Sh::KS * N * N;
    constexpr int smem = ALG == 0
        ? SmemLayout<N, F32, Sh::EPB, (Sh::KSM != 0)>::total
        : stage::Layout2<N, F32, Sh::EPB, false, (((ALG - 2) & 4) != 0)>::total;
    auto kern = batch_stage_n_kernel<N, F32, Sh::KS, Sh::EPB, (Sh::KSM != 0), Sh::MINB, ALG>;
    static std::atomic<int> attr_set[kMaxDeviceSlots];  // per kernel and device
    if (cudaError_t e = set_smem_once(kern, smem, attr_set); e != cudaSuccess) return e;
    if (ntiles <= 0) return cudaSuccess;
    kern<<<ntiles, threads, smem, st>>>(slots, work, stage, dry, dp);
    return cudaGetLastError();
}

// Dh: this N's D on the host when every resident cavity of this N uses it (the
// constant-bank form then applies), else null.
template <int N, bool F32>
cudaError_t launch_n(int stage, const SlotDev* slots, const WorkItem* work, int ntiles, int dry,
                     const double* Dh, cudaStream_t st, int* epb_out) {
    using Sh = NShape<N>;
    if (epb_out) *epb_out = (NBulk<N>::on && !F32) ? NBulk<N>::EPB : Sh::EPB;
    if constexpr (NBulk<N>::on && !F32) {
        DParam dp{};
        if constexpr (NBulk<N>::CD) {
            if (Dh) {
                for (int x = 0; x < N * N; ++x) dp.d[x] = Dh[x];
                return launch_bulk_n<N, true>(stage, slots, work, ntiles, dry, dp, st);
            }
            if (ntiles <= 0) {  // set-up call: prepare both forms
                cudaError_t e = launch_bulk_n<N, true>(stage, slots, work, 0, dry, dp, st);
                if (e != cudaSuccess) return e;
            }
        }
        return launch_bulk_n<N, false>(stage, slots, work, ntiles, dry, dp, st);
    }
    if constexpr (dmma_tile<N, F32>()) {
        DParam dp{};
        if (Dh) {
            for (int x = 0; x < N * N; ++x) dp.d[x] = Dh[x];
            return launch_dmma8_n<true>(stage, slots, work, ntiles, dry, dp, st);
        }
        if (ntiles <= 0) {  // set-up call: prepare both forms
            cudaError_t e = launch_dmma8_n<true>(stage, slots, work, 0, dry, dp, st);
            if (e != cudaSuccess) return e;
        }
        return launch_dmma8_n<false>(stage, slots, work, ntiles, dry, dp, st);
    }
    constexpr bool cd_bit = Sh::ALG >= 2 && ((Sh::ALG - 2) & 8) != 0;
    constexpr bool has_cd = cd_bit && !F32;  // the constant-bank D is an FP64 form
    constexpr int ALG_PLAIN = cd_bit ? Sh::ALG - 8 : Sh::ALG;
    DParam dp{};
    if constexpr (has_cd) {
        if (Dh) {
            for (int x = 0; x < N * N; ++x) dp.d[x] = Dh[x];
            return launch_n_alg<N, F32, Sh::ALG>(stage, slots, work, ntiles, dry, dp, st);
        }
        if (ntiles <= 0) {  // set-up call: prepare both forms
            cudaError_t e = launch_n_alg<N, F32, Sh::ALG>(stage, slots, work, 0, dry, dp, st);
            if (e != cudaSuccess) return e;
        }
    }
    return launch_n_alg<N, F32, ALG_PLAIN>(stage, slots, work, ntiles, dry, dp, st);
}

// Does this slot record energy after the step it is taking now (post = 1), or
// is this the initial-state record (post = 0)?
__device__ __forceinline__ bool wants_energy(const SlotDev& S, int post) {
    if (!post) return true;
    const int next = S.done + 1;
    return (next % S.energy_every) == 0 || next == S.nsteps;
}

// Energy partial of each tile, fixed order within the tile.
__global__ void __launch_bounds__(256)
batch_diag_kernel(const SlotDev* __restrict__ slots, const WorkItem* __restrict__ work,
                  const int* __restrict__ ntiles_p, int post, int only_slot) {
    const int ntiles = *ntiles_p;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = blockIdx.x * 8 + warp; t < ntiles; t += gridDim.x * 8) {
        const WorkItem w = work[t];
        if (only_slot >= 0 && w.slot != only_slot) continue;
        const SlotDev& S = slots[w.slot];
        if (!(S.active || !post) || !wants_energy(S, post)) continue;
        const double* u = S.u[post ? (S.par ^ 1) : S.par];
        const int N3 = S.N * S.N * S.N;
        const int e1 = min(S.nelt, w.e0 + S.epb);
        double acc = 0.0;
        for (int e = w.e0; e < e1; ++e) {
            const double J = S.geo[e].jdet;
            const long long base = static_cast<long long>(e) * N3;
            for (int m = lane; m < N3; m += 32) {
                const long long p = base + m;
                const long long st = S.stride;
                const double ex = u[p], ey = u[st + p], ez = u[2 * st + p];
                const double hx = u[3 * st + p], hy = u[4 * st + p], hz = u[5 * st + p];
                acc += 0.5 * ((ex * ex + ey * ey + ez * ez) + (hx * hx + hy * hy + hz * hz)) *
                       (J * S.w3[m]);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (lane == 0) S.partial[w.tile] = acc;
    }
}

// One block per slot: warp 0 sums the energy partials in a fixed order, warps
// 1..kMaxProbes evaluate the probes (tensor-product Lagrange interpolation of
// the element's nodes, as ProbeManager::record does on the host,
// src/probe.cpp:192-216), then thread 0 advances the slot's step bookkeeping.
__global__ void __launch_bounds__(32 * (kMaxProbes + 1))
batch_epilogue_kernel(SlotDev* __restrict__ slots, int nslots, int post, int only_slot,
                      int* __restrict__ counters) {
    if (blockIdx.x == 0 && threadIdx.x < 8 && post) counters[threadIdx.x] = 0;
    const int s = blockIdx.x;
    if (s >= nslots || (only_slot >= 0 && s != only_slot)) return;
    SlotDev& S = slots[s];
    if (post && !S.active) return;
    if (!post && !S.u[0]) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int idx = post ? S.done + 1 : 0;  // history index written by this call
    const double* u = S.u[post ? (S.par ^ 1) : S.par];
    if (warp == 0 && wants_energy(S, post)) {
        double acc = 0.0;
        for (int t = lane; t < S.ntiles; t += 32) acc += S.partial[t];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (lane == 0) S.energy[idx] = acc;
    } else if (warp == 0 && lane == 0) {
        S.energy[idx] = __longlong_as_double(0x7ff8000000000000LL);  // not recorded this step
    }
    if (warp >= 1 && warp - 1 < S.nprobes) {
        const int pr = warp - 1;
        const int N = S.N, N2 = N * N, N3 = N2 * N;
        const double* wr = S.probe_w + pr * 3 * N;
        const double* ws = wr + N;
        const double* wt = ws + N;
        const long long base = static_cast<long long>(S.probe_elem[pr]) * N3;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int m = lane; m < N3; m += 32) {
            const int i = m % N, j = (m / N) % N, k = m / N2;
            const double wgt = wr[i] * ws[j] * wt[k];
#pragma unroll
            for (int c = 0; c < 6; ++c) acc[c] += wgt * u[c * S.stride + base + m];
        }
#pragma unroll
        for (int c = 0; c < 6; ++c) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], off);
        }
        if (lane == 0) {
            double* out = S.probes + (static_cast<long long>(idx) * S.nprobes + pr) * 6;
#pragma unroll
            for (int c = 0; c < 6; ++c) out[c] = acc[c];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && post) {
        S.par ^= 1;
        S.done += 1;
        if (S.done >= S.nsteps) S.active = 0;
    }
}

__global__ void box_pulse_kernel(const BoxPulse b, double* __restrict__ u, long long stride) {
    const int N = b.N, N3 = N * N * N;
    const long long npts = static_cast<long long>(b.nel[0]) * b.nel[1] * b.nel[2] * N3;
    for (long long p = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; p < npts;
         p += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long e = p / N3;
        const int m = static_cast<int>(p - e * N3);
        const int i = m % N, j = (m / N) % N, k = m / (N * N);
        const int ex = static_cast<int>(e % b.nel[0]);
        const int ey = static_cast<int>((e / b.nel[0]) % b.nel[1]);
        const int ez = static_cast<int>(e / (static_cast<long long>(b.nel[0]) * b.nel[1]));
        const double x = b.lo[0] + (ex + 0.5 * (b.z[i] + 1.0)) * b.h[0];
        const double y = b.lo[1] + (ey + 0.5 * (b.z[j] + 1.0)) * b.h[1];
        const double z = b.lo[2] + (ez + 0.5 * (b.z[k] + 1.0)) * b.h[2];
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const double* q = b.pulse + 5 * c;
            double v = 0.0;
            if (q[4] > 0.0) {
                const double dx = x - q[1], dy = y - q[2], dz = z - q[3];
                v = q[0] * exp(-(dx * dx + dy * dy + dz * dz) / (q[4] * q[4]));
            }
            u[c * stride + p] = v;
        }
    }
}

template <bool F32>
int max_batch_smem() {
    int m = 0;
    m = max(m, bsmem<2, F32>()); m = max(m, bsmem<3, F32>()); m = max(m, bsmem<4, F32>());
    m = max(m, bsmem<5, F32>()); m = max(m, bsmem<6, F32>()); m = max(m, bsmem<7, F32>());
    m = max(m, bsmem<8, F32>()); m = max(m, bsmem<9, F32>()); m = max(m, bsmem<10, F32>());
    return m;
}

}  // namespace

cudaError_t launch_batch_stage_n(int N, int f32, int stage, const SlotDev* slots,
                                 const WorkItem* work, int ntiles, int dry, const double* Dh,
                                 cudaStream_t st) {
    switch (N) {
#define NWB_CASE(n) \
        case n: return f32 ? launch_n<n, true>(stage, slots, work, ntiles, dry, Dh, st, nullptr) \
                           : launch_n<n, false>(stage, slots, work, ntiles, dry, Dh, st, nullptr);
        NWB_CASE(2) NWB_CASE(3) NWB_CASE(4) NWB_CASE(5) NWB_CASE(6) NWB_CASE(7) NWB_CASE(8)
        NWB_CASE(9) NWB_CASE(10)
#undef NWB_CASE
        default: return cudaErrorInvalidValue;
    }
}

namespace {
template <int N>
int epb_n(int f32) {
    return (NBulk<N>::on && !f32) ? NBulk<N>::EPB : NShape<N>::EPB;
}
}  // namespace

int batch_epb_n(int N, int f32) {
    switch (N) {
        case 2: return epb_n<2>(f32); case 3: return epb_n<3>(f32); case 4: return epb_n<4>(f32);
        case 5: return epb_n<5>(f32); case 6: return epb_n<6>(f32); case 7: return epb_n<7>(f32);
        case 8: return epb_n<8>(f32); case 9: return epb_n<9>(f32); case 10: return epb_n<10>(f32);
        default: return 1;
    }
}

BatchShape batch_shape(int N, int f32) {
    (void)f32;
    switch (N) {
        case 2: return {BShape<2>::KS, BShape<2>::EPB};
        case 3: return {BShape<3>::KS, BShape<3>::EPB};
        case 4: return {BShape<4>::KS, BShape<4>::EPB};
        case 5: return {BShape<5>::KS, BShape<5>::EPB};
        case 6: return {BShape<6>::KS, BShape<6>::EPB};
        case 7: return {BShape<7>::KS, BShape<7>::EPB};
        case 8: return {BShape<8>::KS, BShape<8>::EPB};
        case 9: return {BShape<9>::KS, BShape<9>::EPB};
        case 10: return {BShape<10>::KS, BShape<10>::EPB};
        default: return {0, 0};
    }
}

int batch_smem(int N, int f32) {
    switch (N) {
        case 2: return f32 ? bsmem<2, true>() : bsmem<2, false>();
        case 3: return f32 ? bsmem<3, true>() : bsmem<3, false>();
        case 4: return f32 ? bsmem<4, true>() : bsmem<4, false>();
        case 5: return f32 ? bsmem<5, true>() : bsmem<5, false>();
        case 6: return f32 ? bsmem<6, true>() : bsmem<6, false>();
        case 7: return f32 ? bsmem<7, true>() : bsmem<7, false>();
        case 8: return f32 ? bsmem<8, true>() : bsmem<8, false>();
        case 9: return f32 ? bsmem<9, true>() : bsmem<9, false>();
        case 10: return f32 ? bsmem<10, true>() : bsmem<10, false>();
        default: return 0;
    }
}

cudaError_t batch_prepare(int f32, int smem) {
    const int cap = f32 ? max_batch_smem<true>() : max_batch_smem<false>();
    if (smem > cap) smem = cap;
    return f32 ? cudaFuncSetAttribute(batch_stage_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, cap)
               : cudaFuncSetAttribute(batch_stage_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
}

cudaError_t launch_batch_stage(int f32, int stage, const SlotDev* slots, const WorkItem* work,
                               const int* ntiles, int* counters, int grid, int smem, int dry,
                               cudaStream_t st) {
    if (f32)
        batch_stage_kernel<true><<<grid, kBatchThreads, smem, st>>>(slots, work, ntiles, counters, stage, dry);
    else
        batch_stage_kernel<false><<<grid, kBatchThreads, smem, st>>>(slots, work, ntiles, counters, stage, dry);
    return cudaGetLastError();
}

cudaError_t launch_box_pulse(const BoxPulse& b, double* u, long long stride, cudaStream_t st) {
    box_pulse_kernel<<<148 * 8, 256, 0, st>>>(b, u, stride);
    return cudaGetLastError();
}

cudaError_t launch_batch_diag(SlotDev* slots, const WorkItem* work, const int* ntiles, int post,
                              int only_slot, int grid, cudaStream_t st) {
    batch_diag_kernel<<<grid, 256, 0, st>>>(slots, work, ntiles, post, only_slot);
    return cudaGetLastError();
}

cudaError_t launch_batch_epilogue(SlotDev* slots, int nslots, int post, int only_slot,
                                  int* counters, cudaStream_t st) {
    if (nslots < 1) return cudaSuccess;
    batch_epilogue_kernel<<<nslots, 32 * (kMaxProbes + 1), 0, st>>>(slots, nslots, post, only_slot,
                                                                  counters);
    return cudaGetLastError();
}

}  // namespace nwb
