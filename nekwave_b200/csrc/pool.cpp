// pool.cpp -- many independent cavities resident on one GPU, advanced together.
//
// The reference solves one mesh per process (Case::simulate, src/case.cpp:529-660).
// A pool keeps many cavities ("slots") resident in HBM at once and advances all
// active ones with one persistent launch per LSRK stage (batch.cu):
//   * admission by a fixed HBM budget: the pool owns one arena allocated at
//     creation and sub-allocates every slot's buffers from it, so admitting a
//     cavity never calls cudaMalloc and fails with NWB_EBUSY when it does not fit
//     (the slot table and the work lists, sized at creation for any admissible
//     set of cavities, live outside the arena);
//   * no host waits on the admission path: host data goes through pinned
//     staging and every copy is queued in stream order behind the steps in
//     flight; status and results can be read back the same way
//     (nwb_pool_query_begin/end, nwb_pool_results_async);
//   * a step of all slots is one CUDA graph (5 stage launches, diagnostics,
//     step epilogue) replayed as often as needed; slots that have taken their
//     steps fall idle on the device, and slots can be added or removed between
//     replays (the graph reads the slot table and the work list from device
//     memory, so it stays valid);
//   * per-slot energy history and probe traces are recorded on the device.
#include "batch.cuh"
#include "nwb.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <new>
#include <vector>


namespace {

using nwb::set_error;

#define NWB_PCU(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return set_error(NWB_ECUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                             __LINE__);                                                       \
    } while (0)

constexpr size_t kAlign = 256;

struct Range {
    size_t off, size;
};

// First-fit sub-allocator over the arena; frees coalesce with their neighbours.
class Arena {
public:
    void reset(size_t bytes) {
        free_.clear();
        free_[0] = bytes;
        total_ = bytes;
        used_ = 0;
    }
    bool alloc(size_t bytes, Range* r) {
        bytes = (std::max<size_t>(bytes, 1) + kAlign - 1) / kAlign * kAlign;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                r->off = it->first;
                r->size = bytes;
                const size_t rest = it->second - bytes;
                const size_t noff = it->first + bytes;
                free_.erase(it);
                if (rest) free_[noff] = rest;
                used_ += bytes;
                return true;
            }
        }
        return false;
    }
    void release(const Range& r) {
        used_ -= r.size;
        auto it = free_.emplace(r.off, r.size).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t used() const { return used_; }
    size_t total() const { return total_; }

private:
    std::map<size_t, size_t> free_;
    size_t total_ = 0, used_ = 0;
};

// Pinned host staging for the pool's host-to-device copies.  A copy from pageable
// memory makes the CUDA runtime wait for everything already queued on the stream
// (the steps of the resident cavities), so admissions, uploads of slot records
// and work lists first copy their data here and then queue a truly asynchronous
// copy.  Two chunks are used in turn; before a chunk is reused, the copies queued
// from it are waited for (an event recorded after them), which in steady state
// have long finished.
class Staging {
public:
    static constexpr size_t kChunk = 48u << 20;  // a 48^3-element box cavity's geometry fits
    cudaError_t init() {
        for (int c = 0; c < 2; ++c) {
            cudaError_t e = cudaHostAlloc(reinterpret_cast<void**>(&buf_[c]), kChunk, cudaHostAllocDefault);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_[c], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    void destroy() {
        for (int c = 0; c < 2; ++c) {
            if (buf_[c]) cudaFreeHost(buf_[c]);
            if (ev_[c]) cudaEventDestroy(ev_[c]);
            buf_[c] = nullptr;
            ev_[c] = nullptr;
        }
    }
    // Pinned space for bytes; nullptr when they exceed a chunk (the caller then
    // copies from its own memory and synchronises).  Copies from the space must be
    // queued on st before the next call.
    void* get(size_t bytes, cudaStream_t st) {
        bytes = (bytes + 15) & ~static_cast<size_t>(15);
        if (bytes > kChunk) return nullptr;
        if (used_ + bytes > kChunk) {
            if (cudaEventRecord(ev_[cur_], st) != cudaSuccess) return nullptr;
            live_[cur_] = true;
            cur_ ^= 1;
            if (live_[cur_] && cudaEventSynchronize(ev_[cur_]) != cudaSuccess) return nullptr;
            used_ = 0;
        }
        void* p = buf_[cur_] + used_;
        used_ += bytes;
        return p;
    }
    // Marks the copies queued so far from the current chunk.
    cudaError_t mark(cudaStream_t st) {
        live_[cur_] = true;
        return cudaEventRecord(ev_[cur_], st);
    }

private:
    char* buf_[2] = {nullptr, nullptr};
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    bool live_[2] = {false, false};
    int cur_ = 0;
    size_t used_ = 0;
};

struct SlotHost {
    bool used = false;
    unsigned gen = 0;     // admission generation: status snapshots of an older one are ignored
    bool dcanon = false;  // its D equals the pool's D for its N (the GLL operator)
    bool uploaded = false;
    bool is_box = false;
    nwb::BoxPulse box{};
    int N = 0, nelt = 0, nsteps = 0, nprobes = 0, energy_every = 1, ntiles = 0, epb = 1;
    long long npts = 0, stride = 0;
    std::vector<Range> ranges;
    nwb::SlotDev dev{};
};

}  // namespace

struct nwb_pool {
    int device = 0;
    cudaStream_t st = nullptr;
    int f32 = 0;
    char* base = nullptr;
    Arena arena;
    int max_slots = 0;
    std::vector<SlotHost> slots;
    nwb::SlotDev* d_slots = nullptr;
    nwb::WorkItem* d_work = nullptr;
    int work_cap = 0;
    int* d_ntiles = nullptr;
    int* d_counters = nullptr;
    bool work_dirty = true;
    int ntiles = 0;
    int smem_needed = 0;
    // per-N mode: tiles cut with each N's own elements-per-block, grouped by N
    nwb::WorkItem* d_work_n = nullptr;
    int work_n_cap = 0;
    int n_off[11] = {}, n_cnt[11] = {};
    int mode = 1;  // 0: one persistent launch for every N, 1: one launch per N (default)
    // the GLL differentiation matrix of each N, for kernels that take D by value
    double canonD[11][100] = {};
    bool canon_set[11] = {};
    cudaStream_t side[11] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[11] = {};
    cudaGraphExec_t graph = nullptr;
    int graph_smem = -1;
    int grid = 0, diag_grid = 0;
    int sms = 148;
    long long launches = 0;
    Staging stage;
    // asynchronous status snapshots (nwb_pool_query_begin/end): the device slot
    // table copied into pinned memory, and each slot's generation when it was taken
    nwb::SlotDev* h_snap = nullptr;
    cudaEvent_t snap_ev = nullptr;
    bool snap_pending = false;
    std::vector<unsigned> snap_gen;
    unsigned next_gen = 1;

    template <class T>
    T* ptr(const Range& r) const {
        return reinterpret_cast<T*>(base + r.off);
    }

    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_smem = -1;
    }

    // Host-to-device copy of bytes through the pinned staging area (asynchronous);
    // data larger than a staging chunk is copied directly, with a synchronisation.
    nwb_status h2d(void* dst, const void* src, size_t bytes) {
        if (!bytes) return NWB_OK;
        void* pin = stage.get(bytes, st);
        if (!pin) {
            NWB_PCU(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
            NWB_PCU(cudaStreamSynchronize(st));
            return NWB_OK;
        }
        std::memcpy(pin, src, bytes);
        NWB_PCU(cudaMemcpyAsync(dst, pin, bytes, cudaMemcpyHostToDevice, st));
        NWB_PCU(stage.mark(st));
        return NWB_OK;
    }

    // The device copy of slot s's record, queued in stream order (no host wait).
    nwb_status write_slot(int s) { return h2d(d_slots + s, &slots[s].dev, sizeof(nwb::SlotDev)); }

    // Work list: every tile of every used slot, largest tiles first, so the
    // dynamic tile counter hands out the long tiles early.
    nwb_status rebuild_work() {
        if (!work_dirty) return NWB_OK;
        std::vector<nwb::WorkItem> w;
        smem_needed = 0;
        for (int s = 0; s < max_slots; ++s) {
            const SlotHost& h = slots[s];
            if (!h.used) continue;
            smem_needed = std::max(smem_needed, nwb::batch_smem(h.N, f32));
            for (int t = 0; t < h.ntiles; ++t) w.push_back(nwb::WorkItem{s, t * h.epb, h.N, t});
        }
        std::stable_sort(w.begin(), w.end(), [&](const nwb::WorkItem& a, const nwb::WorkItem& b) {
            const long long ca = static_cast<long long>(slots[a.slot].epb) * a.N * a.N * a.N;
            const long long cb = static_cast<long long>(slots[b.slot].epb) * b.N * b.N * b.N;
            return ca > cb;
        });
        ntiles = static_cast<int>(w.size());
        std::vector<nwb::WorkItem> wn;
        for (int N = 2; N <= 10; ++N) {
            n_off[N] = static_cast<int>(wn.size());
            const int epb = nwb::batch_epb_n(N, f32);
            for (int s = 0; s < max_slots; ++s) {
                const SlotHost& h = slots[s];
                if (!h.used || h.N != N) continue;
                for (int e0 = 0; e0 < h.nelt; e0 += epb) wn.push_back(nwb::WorkItem{s, e0, N, 0});
            }
            n_cnt[N] = static_cast<int>(wn.size()) - n_off[N];
        }
        // both lists were sized at creation for every admissible cavity set
        if (static_cast<int>(wn.size()) > work_n_cap || ntiles > work_cap)
            return set_error(NWB_EINVAL, "pool work list: %d tiles over its capacity %d", ntiles,
                             work_cap);
        nwb_status r = h2d(d_work_n, wn.data(), sizeof(nwb::WorkItem) * wn.size());
        if (r == NWB_OK) r = h2d(d_work, w.data(), sizeof(nwb::WorkItem) * ntiles);
        if (r == NWB_OK) r = h2d(d_ntiles, &ntiles, sizeof(int));
        if (r != NWB_OK) return r;
        if (mode == 1) drop_graph();  // per-N grids follow the tile counts
        work_dirty = false;
        return NWB_OK;
    }

    nwb_status launch_stages(int dry) {
        for (int s = 0; s < 5; ++s) {
            if (mode == 0) {
                cudaError_t e = nwb::launch_batch_stage(f32, s, d_slots, d_work, d_ntiles, d_counters,
                                                        grid, graph_smem, dry, st);
                if (e != cudaSuccess) return set_error(NWB_ECUDA, "batch stage: %s", cudaGetErrorString(e));
                continue;
            }
            // one launch per N on its own stream: independent branches of the graph
            NWB_PCU(cudaEventRecord(fork_ev, st));
            for (int N = 2; N <= 10; ++N) {
                if (!n_cnt[N]) continue;
                NWB_PCU(cudaStreamWaitEvent(side[N], fork_ev, 0));
                bool all_canon = true;
                for (int q = 0; q < max_slots; ++q)
                    if (slots[q].used && slots[q].N == N && !slots[q].dcanon) all_canon = false;
                cudaError_t e = nwb::launch_batch_stage_n(N, f32, s, d_slots, d_work_n + n_off[N], n_cnt[N],
                                                          dry, all_canon ? canonD[N] : nullptr, side[N]);
                if (e != cudaSuccess) return set_error(NWB_ECUDA, "batch stage N=%d: %s", N, cudaGetErrorString(e));
                NWB_PCU(cudaEventRecord(join_ev[N], side[N]));
                NWB_PCU(cudaStreamWaitEvent(st, join_ev[N], 0));
            }
        }
        return NWB_OK;
    }

    nwb_status launch_step() {
        nwb_status r = launch_stages(0);
        if (r != NWB_OK) return r;
        cudaError_t e = nwb::launch_batch_diag(d_slots, d_work, d_ntiles, 1, -1, diag_grid, st);
        if (e != cudaSuccess) return set_error(NWB_ECUDA, "batch diag: %s", cudaGetErrorString(e));
        e = nwb::launch_batch_epilogue(d_slots, max_slots, 1, -1, d_counters, st);
        if (e != cudaSuccess) return set_error(NWB_ECUDA, "batch epilogue: %s", cudaGetErrorString(e));
        return NWB_OK;
    }

    // Captures the five stages (dry = 1: timing only) or a whole step (dry = 0).
    nwb_status capture(int dry, cudaGraphExec_t* out) {
        cudaGraph_t g = nullptr;
        NWB_PCU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        // a timing graph has no epilogue to reset the tile counters: reset them first
        if (dry) NWB_PCU(cudaMemsetAsync(d_counters, 0, sizeof(int) * 8, st));
        nwb_status r = dry ? launch_stages(1) : launch_step();
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (r != NWB_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (ce != cudaSuccess) return set_error(NWB_ECUDA, "capture: %s", cudaGetErrorString(ce));
        ce = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return set_error(NWB_ECUDA, "instantiate: %s", cudaGetErrorString(ce));
        return NWB_OK;
    }

    nwb_status ensure_graph() {
        nwb_status r = rebuild_work();
        if (r != NWB_OK) return r;
        const int want = std::max(smem_needed, 1024);
        if (graph && graph_smem >= want) return NWB_OK;
        drop_graph();
        graph_smem = want;
        NWB_PCU(nwb::batch_prepare(f32, graph_smem));
        // persistent grid: as many resident blocks as the shared memory allows
        const int by_smem = std::max(1, (227 * 1024) / (graph_smem + 1024));
        grid = sms * std::min(3, by_smem);  // the kernel is built for 3 resident blocks
        diag_grid = sms * 4;
        for (int N = 2; N <= 10; ++N) {  // one-time kernel attribute set-up, outside capture
            cudaError_t e = nwb::launch_batch_stage_n(N, f32, 0, nullptr, nullptr, 0, 0, nullptr, st);
            if (e != cudaSuccess) return set_error(NWB_ECUDA, "per-N set-up: %s", cudaGetErrorString(e));
        }
        return capture(0, &graph);
    }

    void release_slot(int s) {
        for (const Range& r : slots[s].ranges) arena.release(r);
        slots[s] = SlotHost{};
    }
};

extern "C" {

nwb_status nwb_pool_create(size_t hbm_budget_bytes, int max_slots, nwb_precision prec,
                           nwb_pool** out) {
    if (!out) return set_error(NWB_EINVAL, "nwb_pool_create: out is null");
    *out = nullptr;
    if (max_slots < 1 || max_slots > 65536 || hbm_budget_bytes < (1u << 20))
        return set_error(NWB_EINVAL, "nwb_pool_create: need 1..65536 slots and >= 1 MiB budget");
    if (prec != NWB_FP64 && prec != NWB_FP32_BULK)
        return set_error(NWB_EINVAL, "nwb_pool_create: unknown precision");
    nwb_pool* p = new (std::nothrow) nwb_pool();
    if (!p) return set_error(NWB_ENOMEM, "nwb_pool_create: out of host memory");
    p->f32 = prec == NWB_FP32_BULK;
    p->max_slots = max_slots;
    p->slots.resize(max_slots);
    auto bail = [&](nwb_status r) {
        nwb_pool_destroy(p);
        return r;
    };
    cudaError_t e = cudaGetDevice(&p->device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, p->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(set_error(NWB_ECUDA, "nwb_pool_create: %s", cudaGetErrorString(e)));
    e = cudaMalloc(&p->base, hbm_budget_bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return bail(set_error(NWB_ENOMEM, "nwb_pool_create: arena of %zu bytes: %s", hbm_budget_bytes,
                              cudaGetErrorString(e)));
    }
    p->arena.reset(hbm_budget_bytes);
    e = cudaMalloc(&p->d_slots, sizeof(nwb::SlotDev) * max_slots);
    if (e == cudaSuccess) e = cudaMemset(p->d_slots, 0, sizeof(nwb::SlotDev) * max_slots);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_ntiles, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(p->d_ntiles, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&p->d_counters, sizeof(int) * 8);
    if (e == cudaSuccess) e = cudaMemset(p->d_counters, 0, sizeof(int) * 8);
    for (int N = 2; N <= 10 && e == cudaSuccess; ++N) {
        e = cudaStreamCreateWithFlags(&p->side[N], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->join_ev[N], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->fork_ev, cudaEventDisableTiming);
    // Work lists sized once for any set of cavities the budget admits: each element
    // takes at least 3 x 6 x N^3 doubles of the arena (u twice, k), each full tile
    // holds epb elements, and each slot adds at most one partial tile.  With 2-point
    // cavities in 16-element tiles that is one 16-byte entry per 18 KB of budget.
    if (e == cudaSuccess) {
        double min_tile = 1e300;
        for (int N = 2; N <= 10; ++N) {
            const int epb = std::min(nwb::batch_shape(N, p->f32).epb, nwb::batch_epb_n(N, p->f32));
            min_tile = std::min(min_tile, 144.0 * N * N * N * epb);
        }
        const double cap = static_cast<double>(max_slots) + static_cast<double>(hbm_budget_bytes) / min_tile + 1;
        if (cap > 0x7fffffff) e = cudaErrorInvalidValue;
        p->work_cap = p->work_n_cap = static_cast<int>(cap);
    }
    if (e == cudaSuccess) e = cudaMalloc(&p->d_work, sizeof(nwb::WorkItem) * p->work_cap);
    if (e == cudaSuccess) e = cudaMalloc(&p->d_work_n, sizeof(nwb::WorkItem) * p->work_n_cap);
    if (e == cudaSuccess) e = p->stage.init();
    if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void**>(&p->h_snap), sizeof(nwb::SlotDev) * max_slots,
                          cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->snap_ev, cudaEventDisableTiming);
    p->snap_gen.assign(max_slots, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return bail(set_error(NWB_ECUDA, "nwb_pool_create: %s", cudaGetErrorString(e)));
    *out = p;
    return NWB_OK;
}

}  // extern "C"

namespace {

// Admits one cavity given its compressed axis-aligned geometry.
nwb_status admit(nwb_pool* p, int N, int nelt, const double* D, const double* w3,
                 const nwb::ElemGeo* egeo, const int* conn, double c0, double dt, int nsteps,
                 int nprobes, const int* probe_elem, const double* probe_w, int energy_every,
                 int* slot_out, SlotHost** host_out) {
    int s = -1;
    for (int i = 0; i < p->max_slots; ++i)
        if (!p->slots[i].used) {
            s = i;
            break;
        }
    if (s < 0) return set_error(NWB_EBUSY, "nwb_pool_add: all %d slots busy", p->max_slots);
    const int N2 = N * N, N3 = N2 * N;
    const nwb::BatchShape sh = nwb::batch_shape(N, p->f32);
    if (!p->canon_set[N]) {
        std::vector<double> z, w, Dg;
        nwb::gll(N, z, w, Dg);
        for (int x = 0; x < N2; ++x) p->canonD[N][x] = Dg[x];
        p->canon_set[N] = true;
    }
    SlotHost h;
    h.used = true;
    h.dcanon = std::memcmp(p->canonD[N], D, sizeof(double) * N2) == 0;
    h.N = N;
    h.nelt = nelt;
    h.nsteps = nsteps;
    h.nprobes = nprobes;
    h.energy_every = energy_every;
    h.epb = sh.epb;
    h.ntiles = (nelt + sh.epb - 1) / sh.epb;
    h.npts = static_cast<long long>(nelt) * N3;
    h.stride = (h.npts + 63) / 64 * 64;
    // buffers, in one list so a failed admission releases what it took
    const size_t sizes[] = {
        sizeof(double) * 6 * static_cast<size_t>(h.stride),                 // 0 u0
        sizeof(double) * 6 * static_cast<size_t>(h.stride),                 // 1 u1
        sizeof(double) * 6 * static_cast<size_t>(h.stride),                 // 2 k
        sizeof(double) * N2,                                                // 3 D
        sizeof(double) * N3,                                                // 4 w3
        sizeof(nwb::ElemGeo) * nelt,                                        // 5 geo
        sizeof(int) * 6 * static_cast<size_t>(nelt),                        // 6 conn
        sizeof(double) * h.ntiles,                                          // 7 partial
        sizeof(double) * (nsteps + 1),                                      // 8 energy
        sizeof(double) * 6 * static_cast<size_t>(nprobes) * (nsteps + 1),   // 9 probes
        sizeof(int) * std::max(nprobes, 1),                                 // 10 probe elements
        sizeof(double) * 3 * N * std::max(nprobes, 1)};                     // 11 probe weights
    for (size_t b : sizes) {
        Range r;
        if (!p->arena.alloc(b, &r)) {
            for (const Range& q : h.ranges) p->arena.release(q);
            return set_error(NWB_EBUSY, "nwb_pool_add: over the HBM budget (%zu of %zu bytes in use)",
                             p->arena.used(), p->arena.total());
        }
        h.ranges.push_back(r);
    }
    nwb::SlotDev& d = h.dev;
    d.u[0] = p->ptr<double>(h.ranges[0]);
    d.u[1] = p->ptr<double>(h.ranges[1]);
    d.k = p->ptr<double>(h.ranges[2]);
    d.D = p->ptr<double>(h.ranges[3]);
    d.w3 = p->ptr<double>(h.ranges[4]);
    nwb::line_coords(N, D, d.zl);
    d.geo = p->ptr<nwb::ElemGeo>(h.ranges[5]);
    d.conn = p->ptr<int>(h.ranges[6]);
    d.partial = p->ptr<double>(h.ranges[7]);
    d.energy = p->ptr<double>(h.ranges[8]);
    d.probes = p->ptr<double>(h.ranges[9]);
    d.probe_elem = p->ptr<int>(h.ranges[10]);
    d.probe_w = p->ptr<double>(h.ranges[11]);
    d.stride = h.stride;
    d.c0 = c0;
    d.dt = dt;
    d.N = N;
    d.nelt = nelt;
    d.ntiles = h.ntiles;
    d.epb = h.epb;
    d.nprobes = nprobes;
    d.energy_every = energy_every;
    d.nsteps = nsteps;
    d.done = 0;
    d.par = 0;
    d.active = 0;  // set when the initial state arrives
    // queued in stream order after the steps already in flight (the ranges may be
    // a removed cavity's, which those steps may still read); no host wait
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 3 && e == cudaSuccess; ++b)
        e = cudaMemsetAsync(p->base + h.ranges[b].off, 0, sizes[b], p->st);
    nwb_status r = e == cudaSuccess ? NWB_OK : set_error(NWB_ECUDA, "nwb_pool_add: %s", cudaGetErrorString(e));
    auto cp = [&](int idx, const void* src, size_t bytes) {
        if (r == NWB_OK) r = p->h2d(p->base + h.ranges[idx].off, src, bytes);
    };
    cp(3, D, sizes[3]);
    cp(4, w3, sizes[4]);
    cp(5, egeo, sizes[5]);
    cp(6, conn, sizes[6]);
    if (nprobes) {
        cp(10, probe_elem, sizeof(int) * nprobes);
        cp(11, probe_w, sizeof(double) * 3 * N * nprobes);
    }
    if (r != NWB_OK) {
        for (const Range& q : h.ranges) p->arena.release(q);
        return r;
    }
    h.gen = p->next_gen++;
    p->slots[s] = h;
    r = p->write_slot(s);
    if (r != NWB_OK) {
        p->release_slot(s);
        return r;
    }
    p->work_dirty = true;
    *slot_out = s;
    if (host_out) *host_out = &p->slots[s];
    return NWB_OK;
}

}  // namespace

extern "C" {

nwb_status nwb_pool_add(nwb_pool* p, const nwb_mesh_desc* m, double c0, double dt, int nsteps,
                        int nprobes, const int* probe_elem, const double* probe_w,
                        int energy_every, int* slot_out) {
    if (!p || !m || !slot_out) return set_error(NWB_EINVAL, "nwb_pool_add: null argument");
    if (m->N < 2 || m->N > 10 || m->nelt < 1 || nsteps < 1 || !std::isfinite(dt) || dt <= 0 ||
        nprobes < 0 || nprobes > nwb::kMaxProbes || energy_every < 1 ||
        (nprobes > 0 && (!probe_elem || !probe_w)))
        return set_error(NWB_EINVAL, "nwb_pool_add: bad arguments (N 2..10, nsteps >= 1, dt > 0, "
                                     "0..8 probes, energy_every >= 1)");
    nwb::Analysis A;
    try {
        nwb_status r = nwb::analyse_mesh(m, &A);
        if (r != NWB_OK) return r;
    } catch (const std::bad_alloc&) {
        return set_error(NWB_ENOMEM, "nwb_pool_add: out of host memory");
    }
    if (A.geo != nwb::GEO_BOX)
        return set_error(NWB_EINVAL, "nwb_pool_add: the pool takes axis-aligned affine (box) meshes");
    for (int i = 0; i < nprobes; ++i)
        if (probe_elem[i] < 0 || probe_elem[i] >= m->nelt)
            return set_error(NWB_EINVAL, "nwb_pool_add: probe element out of range");
    return admit(p, m->N, m->nelt, m->D, m->w3, A.egeo.data(), A.conn.data(), c0, dt, nsteps, nprobes,
                 probe_elem, probe_w, energy_every, slot_out, nullptr);
}

nwb_status nwb_pool_add_box(nwb_pool* p, int N, int nelx, int nely, int nelz, double xmin,
                            double xmax, double ymin, double ymax, double zmin, double zmax,
                            int periodic_mask, double c0, double dt, int nsteps, int nprobes,
                            const double* probe_xyz, int energy_every, int* slot_out) {
    if (!p || !slot_out) return set_error(NWB_EINVAL, "nwb_pool_add_box: null argument");
    const long long nelt = static_cast<long long>(nelx) * nely * nelz;
    if (N < 2 || N > 10 || nelx < 1 || nely < 1 || nelz < 1 || nelt > (1 << 25) ||
        nelt * N * N * N > 0x7fffffffLL || !(xmax > xmin) || !(ymax > ymin) || !(zmax > zmin) ||
        nsteps < 1 || !std::isfinite(dt) || dt <= 0 || nprobes < 0 || nprobes > nwb::kMaxProbes ||
        energy_every < 1 || (nprobes > 0 && !probe_xyz))
        return set_error(NWB_EINVAL, "nwb_pool_add_box: bad arguments");
    std::vector<double> z, w, D;
    std::vector<nwb::ElemGeo> geo;
    std::vector<int> conn, pe;
    std::vector<double> pw;
    const double lo[3] = {xmin, ymin, zmin}, hi[3] = {xmax, ymax, zmax};
    try {
        nwb::gll(N, z, w, D);
        nwb::box_geometry(N, nelx, nely, nelz, lo, hi, periodic_mask, z, w, geo, conn);
        nwb::box_probes(N, nelx, nely, nelz, lo, hi, z, nprobes, probe_xyz, pe, pw);
    } catch (const std::bad_alloc&) {
        return set_error(NWB_ENOMEM, "nwb_pool_add_box: out of host memory");
    }
    std::vector<double> w3(static_cast<size_t>(N) * N * N);
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) w3[i + N * (j + N * k)] = w[i] * w[j] * w[k];
    SlotHost* h = nullptr;
    nwb_status r = admit(p, N, static_cast<int>(nelt), D.data(), w3.data(), geo.data(), conn.data(), c0,
                         dt, nsteps, nprobes, pe.data(), pw.data(), energy_every, slot_out, &h);
    if (r != NWB_OK) return r;
    h->is_box = true;
    nwb::BoxPulse& b = h->box;
    b = nwb::BoxPulse{};
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = lo[a];
        b.h[a] = (hi[a] - lo[a]) / (a == 0 ? nelx : a == 1 ? nely : nelz);
    }
    b.nel[0] = nelx;
    b.nel[1] = nely;
    b.nel[2] = nelz;
    b.N = N;
    for (int i = 0; i < N; ++i) b.z[i] = z[i];
    return NWB_OK;
}

nwb_status nwb_pool_upload(nwb_pool* p, int s, const double* h, size_t n) {
    if (!p || !h || s < 0 || s >= (p ? p->max_slots : 0))
        return set_error(NWB_EINVAL, "nwb_pool_upload: bad argument");
    SlotHost& sh = p->slots[s];
    if (!sh.used) return set_error(NWB_ENOTFOUND, "nwb_pool_upload: slot %d is free", s);
    if (n != 6 * static_cast<size_t>(sh.npts))
        return set_error(NWB_EINVAL, "nwb_pool_upload: size %zu, expected 6*npts", n);
    nwb_status r = p->rebuild_work();
    if (r != NWB_OK) return r;
    const size_t bytes = sizeof(double) * 6 * static_cast<size_t>(sh.npts);
    void* pin = p->stage.get(bytes, p->st);
    if (pin) std::memcpy(pin, h, bytes);  // queued without waiting for the steps in flight
    NWB_PCU(cudaMemcpy2DAsync(sh.dev.u[0], sizeof(double) * sh.stride, pin ? pin : h,
                              sizeof(double) * sh.npts, sizeof(double) * sh.npts, 6,
                              cudaMemcpyHostToDevice, p->st));
    if (pin) NWB_PCU(p->stage.mark(p->st));
    else NWB_PCU(cudaStreamSynchronize(p->st));
    NWB_PCU(cudaMemsetAsync(sh.dev.k, 0, sizeof(double) * 6 * sh.stride, p->st));
    sh.dev.par = 0;
    sh.dev.done = 0;
    sh.dev.active = 0;
    r = p->write_slot(s);
    if (r != NWB_OK) return r;
    // initial-state energy and probes (history index 0)
    cudaError_t e = nwb::launch_batch_diag(p->d_slots, p->d_work, p->d_ntiles, 0, s, p->sms * 4, p->st);
    if (e == cudaSuccess) e = nwb::launch_batch_epilogue(p->d_slots, p->max_slots, 0, s, p->d_counters, p->st);
    if (e != cudaSuccess) return set_error(NWB_ECUDA, "nwb_pool_upload: %s", cudaGetErrorString(e));
    p->launches += 2;
    sh.dev.active = 1;
    sh.uploaded = true;
    return p->write_slot(s);
}

nwb_status nwb_pool_init_pulse(nwb_pool* p, int s, const double* pulse) {
    if (!p || !pulse || s < 0 || s >= (p ? p->max_slots : 0))
        return set_error(NWB_EINVAL, "nwb_pool_init_pulse: bad argument");
    SlotHost& sh = p->slots[s];
    if (!sh.used || !sh.is_box)
        return set_error(NWB_ENOTFOUND, "nwb_pool_init_pulse: slot %d is not a box cavity", s);
    nwb_status r = p->rebuild_work();
    if (r != NWB_OK) return r;
    nwb::BoxPulse b = sh.box;
    for (int i = 0; i < 30; ++i) b.pulse[i] = pulse[i];
    cudaError_t e = nwb::launch_box_pulse(b, sh.dev.u[0], sh.stride, p->st);
    if (e != cudaSuccess) return set_error(NWB_ECUDA, "nwb_pool_init_pulse: %s", cudaGetErrorString(e));
    NWB_PCU(cudaMemsetAsync(sh.dev.k, 0, sizeof(double) * 6 * sh.stride, p->st));
    sh.dev.par = 0;
    sh.dev.done = 0;
    sh.dev.active = 0;
    r = p->write_slot(s);
    if (r != NWB_OK) return r;
    e = nwb::launch_batch_diag(p->d_slots, p->d_work, p->d_ntiles, 0, s, p->sms * 4, p->st);
    if (e == cudaSuccess) e = nwb::launch_batch_epilogue(p->d_slots, p->max_slots, 0, s, p->d_counters, p->st);
    if (e != cudaSuccess) return set_error(NWB_ECUDA, "nwb_pool_init_pulse: %s", cudaGetErrorString(e));
    p->launches += 3;
    sh.dev.active = 1;
    sh.uploaded = true;
    return p->write_slot(s);
}

nwb_status nwb_pool_step(nwb_pool* p, int nsteps) {
    if (!p || nsteps < 0) return set_error(NWB_EINVAL, "nwb_pool_step: bad argument");
    nwb_status r = p->ensure_graph();
    if (r != NWB_OK) return r;
    for (int i = 0; i < nsteps; ++i) {
        NWB_PCU(cudaGraphLaunch(p->graph, p->st));
        p->launches += 7;
    }
    return NWB_OK;
}

nwb_status nwb_pool_sync(nwb_pool* p) {
    if (!p) return set_error(NWB_EINVAL, "nwb_pool_sync: null pool");
    NWB_PCU(cudaStreamSynchronize(p->st));
    return NWB_OK;
}

nwb_status nwb_pool_query(nwb_pool* p, int* status, int* done, int cap) {
    if (!p || (!status && !done)) return set_error(NWB_EINVAL, "nwb_pool_query: bad argument");
    std::vector<nwb::SlotDev> tmp(p->max_slots);
    NWB_PCU(cudaMemcpyAsync(tmp.data(), p->d_slots, sizeof(nwb::SlotDev) * p->max_slots,
                            cudaMemcpyDeviceToHost, p->st));
    NWB_PCU(cudaStreamSynchronize(p->st));
    for (int s = 0; s < p->max_slots && s < cap; ++s) {
        const SlotHost& h = p->slots[s];
        int st = -1;
        if (h.used) st = !h.uploaded ? 0 : (tmp[s].done >= tmp[s].nsteps ? 2 : 1);
        if (h.used) {
            p->slots[s].dev.done = tmp[s].done;
            p->slots[s].dev.par = tmp[s].par;
            p->slots[s].dev.active = tmp[s].active;
        }
        if (status) status[s] = st;
        if (done) done[s] = h.used ? tmp[s].done : 0;
    }
    return NWB_OK;
}

nwb_status nwb_pool_query_begin(nwb_pool* p) {
    if (!p) return set_error(NWB_EINVAL, "nwb_pool_query_begin: null pool");
    if (p->snap_pending) NWB_PCU(cudaEventSynchronize(p->snap_ev));  // one snapshot in flight
    for (int s = 0; s < p->max_slots; ++s) p->snap_gen[s] = p->slots[s].used ? p->slots[s].gen : 0;
    NWB_PCU(cudaMemcpyAsync(p->h_snap, p->d_slots, sizeof(nwb::SlotDev) * p->max_slots,
                            cudaMemcpyDeviceToHost, p->st));
    NWB_PCU(cudaEventRecord(p->snap_ev, p->st));
    p->snap_pending = true;
    return NWB_OK;
}

nwb_status nwb_pool_query_end(nwb_pool* p, int* status, int* done, int cap) {
    if (!p || (!status && !done)) return set_error(NWB_EINVAL, "nwb_pool_query_end: bad argument");
    if (!p->snap_pending) return set_error(NWB_EINVAL, "nwb_pool_query_end: no nwb_pool_query_begin");
    NWB_PCU(cudaEventSynchronize(p->snap_ev));
    p->snap_pending = false;
    for (int s = 0; s < p->max_slots && s < cap; ++s) {
        SlotHost& h = p->slots[s];
        const nwb::SlotDev& d = p->h_snap[s];
        // a slot admitted or removed since the snapshot was taken: not yet in it
        const bool current = h.used && p->snap_gen[s] == h.gen;
        int st = -1;
        if (h.used) st = (!h.uploaded || !current) ? (h.uploaded ? 1 : 0) : (d.done >= d.nsteps ? 2 : 1);
        if (current) {
            h.dev.done = d.done;
            h.dev.par = d.par;
            h.dev.active = d.active;
        }
        if (status) status[s] = st;
        if (done) done[s] = current ? d.done : 0;
    }
    return NWB_OK;
}

nwb_status nwb_pool_results_async(nwb_pool* p, int s, double* state, double* energy, double* probes) {
    if (!p || s < 0 || s >= p->max_slots) return set_error(NWB_EINVAL, "nwb_pool_results_async: bad argument");
    SlotHost& h = p->slots[s];
    if (!h.used) return set_error(NWB_ENOTFOUND, "nwb_pool_results_async: slot %d is free", s);
    if (h.dev.done < h.nsteps)
        return set_error(NWB_EINVAL, "nwb_pool_results_async: slot %d has not been reported finished "
                                     "by nwb_pool_query_end", s);
    if (state)
        NWB_PCU(cudaMemcpy2DAsync(state, sizeof(double) * h.npts, h.dev.u[h.dev.par], sizeof(double) * h.stride,
                                  sizeof(double) * h.npts, 6, cudaMemcpyDeviceToHost, p->st));
    if (energy)
        NWB_PCU(cudaMemcpyAsync(energy, h.dev.energy, sizeof(double) * (h.nsteps + 1), cudaMemcpyDeviceToHost,
                                p->st));
    if (probes && h.nprobes)
        NWB_PCU(cudaMemcpyAsync(probes, h.dev.probes, sizeof(double) * 6 * h.nprobes * (h.nsteps + 1),
                                cudaMemcpyDeviceToHost, p->st));
    return NWB_OK;
}

nwb_status nwb_pool_results(nwb_pool* p, int s, double* state, double* energy, double* probes) {
    if (!p || s < 0 || s >= p->max_slots) return set_error(NWB_EINVAL, "nwb_pool_results: bad argument");
    SlotHost& h = p->slots[s];
    if (!h.used) return set_error(NWB_ENOTFOUND, "nwb_pool_results: slot %d is free", s);
    nwb::SlotDev d;
    NWB_PCU(cudaMemcpyAsync(&d, p->d_slots + s, sizeof(d), cudaMemcpyDeviceToHost, p->st));
    NWB_PCU(cudaStreamSynchronize(p->st));
    if (state)
        NWB_PCU(cudaMemcpy2DAsync(state, sizeof(double) * h.npts, d.u[d.par], sizeof(double) * h.stride,
                                  sizeof(double) * h.npts, 6, cudaMemcpyDeviceToHost, p->st));
    if (energy)
        NWB_PCU(cudaMemcpyAsync(energy, d.energy, sizeof(double) * (h.nsteps + 1), cudaMemcpyDeviceToHost,
                                p->st));
    if (probes && h.nprobes)
        NWB_PCU(cudaMemcpyAsync(probes, d.probes, sizeof(double) * 6 * h.nprobes * (h.nsteps + 1),
                                cudaMemcpyDeviceToHost, p->st));
    NWB_PCU(cudaStreamSynchronize(p->st));
    return NWB_OK;
}

nwb_status nwb_pool_remove(nwb_pool* p, int s) {
    if (!p || s < 0 || s >= p->max_slots) return set_error(NWB_EINVAL, "nwb_pool_remove: bad argument");
    if (!p->slots[s].used) return set_error(NWB_ENOTFOUND, "nwb_pool_remove: slot %d is free", s);
    // no host wait: the zeroed record and any later admission into the freed ranges
    // are queued after the steps (and result copies) already in flight
    p->release_slot(s);
    nwb_status r = p->write_slot(s);  // zeroed descriptor: inactive, no buffers
    p->work_dirty = true;
    return r;
}

nwb_status nwb_pool_info(const nwb_pool* p, size_t* used_bytes, size_t* budget_bytes, int* slots_used,
                         long long* launches) {
    if (!p) return set_error(NWB_EINVAL, "nwb_pool_info: null pool");
    if (used_bytes) *used_bytes = p->arena.used();
    if (budget_bytes) *budget_bytes = p->arena.total();
    if (slots_used) {
        int n = 0;
        for (const SlotHost& h : p->slots) n += h.used;
        *slots_used = n;
    }
    if (launches) *launches = p->launches;
    return NWB_OK;
}

nwb_status nwb_pool_time_steps(nwb_pool* p, int nsteps, float* ms) {
    if (!p || !ms || nsteps < 1) return set_error(NWB_EINVAL, "nwb_pool_time_steps: bad argument");
    nwb_status r = p->ensure_graph();
    if (r != NWB_OK) return r;
    cudaEvent_t a, b;
    NWB_PCU(cudaEventCreate(&a));
    NWB_PCU(cudaEventCreate(&b));
    NWB_PCU(cudaStreamSynchronize(p->st));
    NWB_PCU(cudaEventRecord(a, p->st));
    r = nwb_pool_step(p, nsteps);
    NWB_PCU(cudaEventRecord(b, p->st));
    NWB_PCU(cudaEventSynchronize(b));
    NWB_PCU(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return r;
}

nwb_status nwb_pool_set_mode(nwb_pool* p, int mode) {
    if (!p || (mode != 0 && mode != 1)) return set_error(NWB_EINVAL, "nwb_pool_set_mode: mode must be 0 or 1");
    NWB_PCU(cudaStreamSynchronize(p->st));
    if (p->mode != mode) {
        p->mode = mode;
        p->drop_graph();
    }
    return NWB_OK;
}

// Times the five stage launches of both modes on the resident cavities (dry
// stages: a = b = dt = 0, which leaves every state as it is and zeroes the LSRK
// registers, which the first stage of the next step multiplies by a = 0) and
// keeps the faster mode.
nwb_status nwb_pool_autotune(nwb_pool* p, int reps, int* best_mode, float* ms_out /* [2] */) {
    if (!p || reps < 1) return set_error(NWB_EINVAL, "nwb_pool_autotune: bad argument");
    float t[2] = {0.f, 0.f};
    for (int m = 0; m < 2; ++m) {
        nwb_status r = nwb_pool_set_mode(p, m);
        if (r == NWB_OK) r = p->ensure_graph();
        if (r != NWB_OK) return r;
        cudaGraphExec_t dry = nullptr;
        r = p->capture(1, &dry);
        if (r != NWB_OK) return r;
        cudaEvent_t a, b;
        NWB_PCU(cudaEventCreate(&a));
        NWB_PCU(cudaEventCreate(&b));
        NWB_PCU(cudaGraphLaunch(dry, p->st));  // warm-up
        NWB_PCU(cudaEventRecord(a, p->st));
        for (int i = 0; i < reps; ++i) NWB_PCU(cudaGraphLaunch(dry, p->st));
        NWB_PCU(cudaEventRecord(b, p->st));
        NWB_PCU(cudaEventSynchronize(b));
        NWB_PCU(cudaEventElapsedTime(&t[m], a, b));
        t[m] /= reps;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        cudaGraphExecDestroy(dry);
        // the dry launches advanced the stage counters of mode 0: reset them
        NWB_PCU(cudaMemsetAsync(p->d_counters, 0, sizeof(int) * 8, p->st));
        NWB_PCU(cudaStreamSynchronize(p->st));
    }
    const int m = t[1] < t[0] ? 1 : 0;
    if (best_mode) *best_mode = m;
    if (ms_out) {
        ms_out[0] = t[0];
        ms_out[1] = t[1];
    }
    return nwb_pool_set_mode(p, m);
}

nwb_status nwb_pool_destroy(nwb_pool* p) {
    if (!p) return NWB_OK;
    if (p->st) cudaStreamSynchronize(p->st);
    p->drop_graph();
    void* ptrs[] = {p->base, p->d_slots, p->d_work, p->d_work_n, p->d_ntiles, p->d_counters};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    for (int N = 2; N <= 10; ++N) {
        if (p->side[N]) cudaStreamDestroy(p->side[N]);
        if (p->join_ev[N]) cudaEventDestroy(p->join_ev[N]);
    }
    if (p->fork_ev) cudaEventDestroy(p->fork_ev);
    if (p->snap_ev) cudaEventDestroy(p->snap_ev);
    if (p->h_snap) cudaFreeHost(p->h_snap);
    p->stage.destroy();
    if (p->st) cudaStreamDestroy(p->st);
    delete p;
    return NWB_OK;
}

}  // extern "C"
