// dg_solver.cpp -- drop-in implementation of NekWave's DgSolver on libnwb.
//
// Implements the reference's own header src/dg_solver.hpp (class DgSolver,
// src/dg_solver.hpp:35-102) on the C ABI of include/nwb.h, so that the
// reference's Case, examples and tests link against the B200 path unchanged:
// build the reference's sources with this file in place of src/dg_solver.cpp and
// without src/device/, and link libnwb.so (recipe: Makefile next to this file).
//
//   DgSolver::initialize    -> nwb_solver_create     (src/dg_solver.cpp:40-241)
//   DgSolver::uploadState   -> nwb_upload_state      (src/dg_solver.cpp:243-262)
//   DgSolver::downloadState -> nwb_download_state    (src/dg_solver.cpp:264-283)
//   DgSolver::step          -> nwb_step + nwb_sync   (src/dg_solver.cpp:306-527)
//   DgSolver::finalize      -> nwb_solver_destroy    (src/dg_solver.cpp:529-582)
//
// It also implements device_diag.hpp, the device diagnostics a front end calls
// in place of its per-step full download and host reductions.
//
// The face points are handed over in the canonical (element, face, q, p) order
// nwb_mesh_desc requires; Mesh::getFaceData lists them per (element, face) in
// the order of Mesh::m_faces, so they are re-ordered by (elementId, faceId).
// Like the reference, any failure prints a message and aborts
// (src/device/gpu_runtime.hpp:146-153).  Environment knobs (no counterpart in
// the reference): NWB_PRECISION=fp32 selects the FP32-bulk class,
// NWB_AUTOTUNE=1 times the stage kernel's launch shapes at initialize.
#include "dg_solver.hpp"
#include "device_diag.hpp"
#include "mesh.hpp"
#include "nwb.h"
#include "probe.hpp"

#include <cuda_runtime.h>

#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <exception>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

void nwb_or_abort(nwb_status s, const char* what) {
    if (s != NWB_OK) {
        std::fprintf(stderr, "[NekWave nwb ERROR] %s: %s (%s)\n", what, nwb_status_string(s),
                     nwb_last_error());
        std::abort();
    }
}

int bc_code(const std::string& t) {
    // src/dg_solver.cpp:92-98
    if (t == "PEC" || t == "W" || t == "V" || t == "v") return 1;
    if (t == "PMC" || t == "SYM" || t == "S" || t == "s") return 2;
    return 0;
}

}  // namespace

class DgSolver::Impl {
public:
    ~Impl() { freeBuffers(); }

    bool initialize(const Mesh& mesh, double c0) {
        freeBuffers();
        if (mesh.isPartitioned() && mesh.getNumHaloPoints() > 0) {
            std::fprintf(stderr, "[NekWave nwb ERROR] partitioned (MPI) meshes are not supported: "
                                 "the B200 path is single-GPU\n");
            std::abort();
        }
        const int N = mesh.getN();
        const int nelt = mesh.getNumElements();
        const size_t nn = static_cast<size_t>(N) * N;
        const size_t nfp = 6 * nn * nelt;
        npts_ = static_cast<size_t>(mesh.getTotalPoints());
        std::vector<int> vmin(nfp), vplus(nfp), bc(nfp);
        std::vector<double> nx(nfp), ny(nfp), nz(nfp), dA(nfp);
        std::vector<char> seen(6 * static_cast<size_t>(nelt), 0);
        for (const auto& fd : mesh.getFaceData()) {
            if (fd.elementId < 0 || fd.elementId >= nelt || fd.faceId < 0 || fd.faceId > 5 ||
                fd.points.size() != nn) {
                std::fprintf(stderr, "[NekWave nwb ERROR] unexpected face data layout\n");
                std::abort();
            }
            const size_t slot = 6 * static_cast<size_t>(fd.elementId) + fd.faceId;
            seen[slot] = 1;
            const int code = bc_code(fd.bcType);
            for (size_t pq = 0; pq < nn; ++pq) {
                const FacePointData& pt = fd.points[pq];
                const size_t fp = slot * nn + pq;
                vmin[fp] = pt.volIdxMinus;
                vplus[fp] = pt.volIdxPlus;
                int c = code;
                if (pt.volIdxPlus < 0 && c == 0) c = 1;  // src/dg_solver.cpp:101-103
                bc[fp] = c;
                nx[fp] = pt.nx;
                ny[fp] = pt.ny;
                nz[fp] = pt.nz;
                dA[fp] = pt.dA;
            }
        }
        for (char s : seen)
            if (!s) {
                std::fprintf(stderr, "[NekWave nwb ERROR] mesh has an element face without face data\n");
                std::abort();
            }
        nwb_mesh_desc d{};
        d.N = N;
        d.nelt = nelt;
        d.D = mesh.getD().data();
        d.w3 = mesh.getW3().data();
        d.jac = mesh.getJac().data();
        const std::vector<double>* m[9] = {&mesh.getRx(), &mesh.getSx(), &mesh.getTx(),
                                           &mesh.getRy(), &mesh.getSy(), &mesh.getTy(),
                                           &mesh.getRz(), &mesh.getSz(), &mesh.getTz()};
        for (int c = 0; c < 9; ++c) d.met[c] = m[c]->data();
        d.vol_idx_minus = vmin.data();
        d.vol_idx_plus = vplus.data();
        d.bc_type = bc.data();
        d.nx = nx.data();
        d.ny = ny.data();
        d.nz = nz.data();
        d.dA = dA.data();
        // libnwb carries its own CUDA runtime: hand it the device the application
        // selected (Comm::init binds rank % numGPUs, src/comm.cpp:35-47)
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) nwb_or_abort(nwb_set_device(dev), "DgSolver::initialize");
        const char* prec = std::getenv("NWB_PRECISION");
        const nwb_precision p = (prec && std::strcmp(prec, "fp32") == 0) ? NWB_FP32_BULK : NWB_FP64;
        nwb_or_abort(nwb_solver_create(&d, c0, p, &s_), "DgSolver::initialize");
        const char* tune = std::getenv("NWB_AUTOTUNE");
        if (tune && std::strcmp(tune, "1") == 0)
            nwb_or_abort(nwb_solver_autotune(s_, 5, nullptr, nullptr, 0), "DgSolver::initialize (autotune)");
        return true;
    }

    void uploadState(const double* h, size_t size) {
        nwb_or_abort(nwb_upload_state(need(), h, size), "DgSolver::uploadState");
    }

    void downloadState(double* h, size_t size) const {
        nwb_or_abort(nwb_download_state(need(), h, size), "DgSolver::downloadState");
    }

    void step(double dt, double /*time: unused, as in src/dg_solver.cpp:307*/) {
        nwb_or_abort(nwb_step(need(), dt, 1), "DgSolver::step");
        nwb_or_abort(nwb_sync(need()), "DgSolver::step");  // the reference's step blocks
    }

    void freeBuffers() {
        if (s_) {
            nwb_solver_destroy(s_);
            s_ = nullptr;
        }
    }

    nwb_solver* handle() const { return s_; }

private:
    nwb_solver* need() const {
        if (!s_) {
            std::fprintf(stderr, "[NekWave nwb ERROR] DgSolver used before initialize\n");
            std::abort();
        }
        return s_;
    }
    nwb_solver* s_ = nullptr;
    size_t npts_ = 0;
};

// libnwb handle of each live DgSolver, for the device diagnostics below (the
// reference's header gives free functions no access to the pimpl).
namespace {
std::mutex g_reg_mu;
std::map<const DgSolver*, nwb_solver*> g_reg;
void reg_set(const DgSolver* d, nwb_solver* s) {
    std::lock_guard<std::mutex> lock(g_reg_mu);
    if (s) g_reg[d] = s;
    else g_reg.erase(d);
}
nwb_solver* reg_get(const DgSolver& d, const char* what) {
    std::lock_guard<std::mutex> lock(g_reg_mu);
    auto it = g_reg.find(&d);
    if (it == g_reg.end()) {
        std::fprintf(stderr, "[NekWave nwb ERROR] %s: DgSolver not initialized\n", what);
        std::abort();
    }
    return it->second;
}
}  // namespace

DgSolver::DgSolver() : impl_(new Impl()) {}
DgSolver::~DgSolver() { reg_set(this, nullptr); }
bool DgSolver::initialize(const Mesh& mesh, double c0) {
    const bool ok = impl_->initialize(mesh, c0);
    reg_set(this, impl_->handle());
    return ok;
}
void DgSolver::uploadState(const double* s, size_t n) { impl_->uploadState(s, n); }
void DgSolver::downloadState(double* s, size_t n) const { impl_->downloadState(s, n); }
void DgSolver::step(double dt, double t) { impl_->step(dt, t); }
void DgSolver::finalize() {
    reg_set(this, nullptr);
    impl_->freeBuffers();
}

namespace nwb_dropin {

void download_probe_elements(const DgSolver& solver, const ProbeManager& probes, int nodes_per_elem,
                             std::vector<double>& state) {
    nwb_solver* s = reg_get(solver, "download_probe_elements");
    for (const ProbePoint& p : probes.getProbes())
        nwb_or_abort(nwb_download_nodes(s, p.elemOffset, nodes_per_elem, state.data(), state.size()),
                     "download_probe_elements");
}

void device_diagnostics(const DgSolver& solver, double* max_e, double* max_h, double* energy) {
    nwb_solver* s = reg_get(solver, "device_diagnostics");
    nwb_or_abort(nwb_max_norms(s, max_e, max_h), "device_diagnostics (max norms)");
    nwb_or_abort(nwb_energy(s, energy), "device_diagnostics (energy)");
}

// ---- SnapshotWriter -------------------------------------------------------------
// The thread that calls save() owns the solver side: it starts a snapshot into a free
// pinned buffer (nwb_snapshot_begin: device copy in stream order, host copy on a side
// stream) and, at the next save() or at finish(), waits for that copy and queues the
// job.  The worker thread only runs jobs on completed buffers.
struct SnapshotWriter::State {
    struct Item {
        int step;
        double time;
        Job job;
        int buf;
    };
    nwb_solver* s = nullptr;
    size_t n = 0;
    double* buf[2] = {nullptr, nullptr};
    int next = 0;
    // the snapshot in flight (the saving thread only)
    bool pending = false;
    Item pend{0, 0.0, Job(), 0};
    // shared with the worker, under mu
    std::mutex mu;
    std::condition_variable cv;
    bool in_use[2] = {false, false};  // from the snapshot's start to its job's end
    std::deque<Item> queue;
    bool busy = false, stop = false;
    std::exception_ptr err;
    std::thread worker;

    void run() {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || !queue.empty(); });
            if (queue.empty()) return;
            Item it = std::move(queue.front());
            queue.pop_front();
            busy = true;
            const bool skip = err != nullptr;  // after a failed job, drop the rest
            lk.unlock();
            std::exception_ptr e;
            if (!skip) {
                try {
                    it.job(it.step, it.time, buf[it.buf]);
                } catch (...) {
                    e = std::current_exception();
                }
            }
            lk.lock();
            if (e && !err) err = e;
            in_use[it.buf] = false;
            busy = false;
            cv.notify_all();
        }
    }
    void hand_over() {
        nwb_or_abort(nwb_snapshot_wait(s), "SnapshotWriter (snapshot copy)");
        std::lock_guard<std::mutex> lk(mu);
        queue.push_back(std::move(pend));
        pending = false;
        cv.notify_all();
    }
};

SnapshotWriter::SnapshotWriter() : st_(new State()) {}

void SnapshotWriter::save(const DgSolver& solver, int step, double time, Job job) {
    State& S = *st_;
    nwb_solver* s = reg_get(solver, "SnapshotWriter::save");
    if (!S.s) {
        nwb_solver_info info;
        nwb_or_abort(nwb_solver_get_info(s, &info), "SnapshotWriter (solver info)");
        S.n = 6 * static_cast<size_t>(info.npts);
        for (double*& b : S.buf) {
            if (cudaHostAlloc(reinterpret_cast<void**>(&b), S.n * sizeof(double), cudaHostAllocDefault) !=
                cudaSuccess) {
                std::fprintf(stderr, "[NekWave nwb ERROR] SnapshotWriter: pinned host allocation failed\n");
                std::abort();
            }
        }
        S.s = s;
        S.worker = std::thread([&S] { S.run(); });
    } else if (s != S.s) {
        std::fprintf(stderr, "[NekWave nwb ERROR] SnapshotWriter: one solver per writer\n");
        std::abort();
    }
    if (S.pending) S.hand_over();
    const int b = S.next;
    {
        std::unique_lock<std::mutex> lk(S.mu);
        S.cv.wait(lk, [&] { return !S.in_use[b]; });
        S.in_use[b] = true;
    }
    nwb_or_abort(nwb_snapshot_begin(s, S.buf[b], S.n), "SnapshotWriter (snapshot)");
    S.pending = true;
    S.pend = State::Item{step, time, std::move(job), b};
    S.next = b ^ 1;
}

void SnapshotWriter::finish() {
    State& S = *st_;
    if (S.pending) S.hand_over();
    std::unique_lock<std::mutex> lk(S.mu);
    S.cv.wait(lk, [&] { return S.queue.empty() && !S.busy; });
    if (S.err) {
        std::exception_ptr e = S.err;
        S.err = nullptr;
        std::rethrow_exception(e);
    }
}

SnapshotWriter::~SnapshotWriter() {
    State& S = *st_;
    try {
        finish();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[NekWave nwb ERROR] SnapshotWriter: a snapshot job failed: %s\n", e.what());
    } catch (...) {
        std::fprintf(stderr, "[NekWave nwb ERROR] SnapshotWriter: a snapshot job failed\n");
    }
    {
        std::lock_guard<std::mutex> lk(S.mu);
        S.stop = true;
        S.cv.notify_all();
    }
    if (S.worker.joinable()) S.worker.join();
    for (double* b : S.buf)
        if (b) cudaFreeHost(b);
}

}  // namespace nwb_dropin
