// nwb_api.cpp -- host side of libnwb: the C ABI of include/nwb.h.
//
// nwb_solver replaces DgSolver::Impl (src/dg_solver.cpp:22-640).  At create time
// the mesh arrays the reference uploads as-is are analysed once on the host and
// compressed into the form the fused stage kernel streams:
//   * affine elements (constant J^{-T} over the element, the case of every box
//     mesh): one ElemGeo record per element (metrics, per-face normal and lift)
//     plus one connection code per face -- O(nelt) geometry instead of the
//     reference's 10 per-node and 7 per-face-point arrays;
//   * anything else: per-node metrics and per-face-point normal/lift/neighbour
//     arrays (the general path).
// One stage is one kernel launch; a time step is five launches, optionally
// replayed from a CUDA graph.
#include "batch.cuh"
#include "nwb.h"
#include "nwb_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

nwb_status fail(nwb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

#define NWB_CU(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            return fail(e_ == cudaErrorMemoryAllocation ? NWB_ENOMEM : NWB_ECUDA,         \
                        "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
        }                                                                                 \
    } while (0)

// Carpenter-Kennedy LSRK45 (src/dg_solver.cpp:58-69).
const double kRK4A[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                         -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double kRK4B[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                         1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                         2277821191437.0 / 14882151754819.0};

inline int face_local(int N, int f, int p, int q) {
    switch (f) {
        case 0: return p + N * N * q;
        case 1: return (N - 1) + N * p + N * N * q;
        case 2: return p + N * (N - 1) + N * N * q;
        case 3: return N * p + N * N * q;
        case 4: return p + N * q;
        default: return p + N * q + N * N * (N - 1);
    }
}

inline void orient(int N, int o, int p, int q, int* pp, int* qq) {
    int a = (o & 4) ? q : p;
    int b = (o & 4) ? p : q;
    if (o & 1) a = N - 1 - a;
    if (o & 2) b = N - 1 - b;
    *pp = a;
    *qq = b;
}

}  // namespace

namespace nwb {

nwb_status set_error(nwb_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

// Wall code of face point fp: 0 (a neighbour), kConnPEC or kConnPMC.  The
// reference mirrors PEC/W/V (bc 1), PMC/SYM/S (bc 2) and neighbourless points as
// PEC alike (src/dg_solver.cpp:92-104, src/device/dg_kernels.cu:243-251); with
// true_pmc, bc 2 points are PMC mirrors instead.
int wall_code(const nwb_mesh_desc* m, long long fp, bool true_pmc) {
    if (true_pmc && m->bc_type[fp] == 2) return nwb::kConnPMC;
    if (m->bc_type[fp] != 0 || m->vol_idx_plus[fp] < 0) return nwb::kConnPEC;
    return 0;
}

nwb_status analyse_mesh(const nwb_mesh_desc* m, Analysis* A, bool true_pmc) {
    const int N = m->N, nelt = m->nelt, N2 = N * N, N3 = N2 * N;
    const long long npts = static_cast<long long>(nelt) * N3;
    // canonical face-point order (src/mesh.cpp:1003-1004) is part of the contract
    for (int e = 0; e < nelt; ++e)
        for (int f = 0; f < 6; ++f)
            for (int pq = 0; pq < N2; ++pq) {
                const long long fp = (static_cast<long long>(e) * 6 + f) * N2 + pq;
                const int want = e * N3 + face_local(N, f, pq % N, pq / N);
                if (m->vol_idx_minus[fp] != want)
                    return fail(NWB_EINVAL,
                                "face point %lld: vol_idx_minus %d, expected %d (face points must be "
                                "element-major, faces 0..5, q, p)",
                                fp, m->vol_idx_minus[fp], want);
                const int vp = m->vol_idx_plus[fp];
                if (vp >= npts)
                    return fail(NWB_EINVAL, "face point %lld: vol_idx_plus %d out of range", fp, vp);
            }
    bool affine = true, box = true;
    A->egeo.assign(nelt, nwb::ElemGeo{});
    A->conn.assign(6 * static_cast<size_t>(nelt), nwb::kConnPEC);
    A->jac_e.assign(nelt, 0.0);
    for (int e = 0; e < nelt && affine; ++e) {
        const long long base = static_cast<long long>(e) * N3;
        nwb::ElemGeo& G = A->egeo[e];
        double scale = 0.0;
        for (int c = 0; c < 9; ++c) {
            G.met[c] = m->met[c][base];
            scale = std::max(scale, std::abs(G.met[c]));
        }
        const double J0 = m->jac[base];
        G.jdet = J0;
        A->jac_e[e] = J0;
        for (int n = 0; n < N3 && affine; ++n) {
            if (std::abs(m->jac[base + n] - J0) > 1e-12 * std::abs(J0)) affine = false;
            for (int c = 0; c < 9; ++c)
                if (std::abs(m->met[c][base + n] - G.met[c]) > 1e-12 * scale) affine = false;
        }
        for (int c : {1, 2, 3, 5, 6, 7})
            if (std::abs(G.met[c]) > 1e-13 * scale) box = false;
        for (int f = 0; f < 6 && affine; ++f) {
            const long long fp0 = (static_cast<long long>(e) * 6 + f) * N2;
            const int pec0 = wall_code(m, fp0, true_pmc);
            const double n0[3] = {m->nx[fp0], m->ny[fp0], m->nz[fp0]};
            const int vm0 = m->vol_idx_minus[fp0];
            const double lift0 = m->dA[fp0] / (m->jac[vm0] * m->w3[vm0 - base]);
            for (int pq = 0; pq < N2; ++pq) {
                const long long fp = fp0 + pq;
                const int pec = wall_code(m, fp, true_pmc);
                const int vm = m->vol_idx_minus[fp];
                const double lift = m->dA[fp] / (m->jac[vm] * m->w3[vm - base]);
                if (pec != pec0 || std::abs(m->nx[fp] - n0[0]) > 1e-12 ||
                    std::abs(m->ny[fp] - n0[1]) > 1e-12 || std::abs(m->nz[fp] - n0[2]) > 1e-12 ||
                    std::abs(lift - lift0) > 1e-12 * std::abs(lift0)) {
                    affine = false;
                    break;
                }
            }
            if (!affine) break;
            for (int c = 0; c < 3; ++c) G.nrm[f][c] = n0[c];
            G.lift[f] = lift0;
            if (pec0) {
                A->conn[6 * static_cast<size_t>(e) + f] = pec0;
                continue;
            }
            const int eB = m->vol_idx_plus[fp0] / N3;
            int found = -1;
            for (int fB = 0; fB < 6 && found < 0; ++fB)
                for (int o = 0; o < 8 && found < 0; ++o) {
                    bool ok = true;
                    for (int pq = 0; pq < N2 && ok; ++pq) {
                        int a, b;
                        orient(N, o, pq % N, pq / N, &a, &b);
                        ok = m->vol_idx_plus[fp0 + pq] == eB * N3 + face_local(N, fB, a, b);
                    }
                    if (ok) found = (fB << 3) | o;
                }
            if (found < 0) { affine = false; break; }
            A->conn[6 * static_cast<size_t>(e) + f] = (eB << 6) | found;
        }
    }
    A->geo = !affine ? nwb::GEO_NODAL : (box ? nwb::GEO_BOX : nwb::GEO_AFFINE);
    if (!affine) {
        A->egeo.clear();
        A->conn.clear();
        A->jac_e.clear();
    }
    return NWB_OK;
}

}  // namespace nwb

namespace {
using nwb::Analysis;

template <class T>
nwb_status dalloc(T** p, size_t count, size_t* total) {
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(NWB_ENOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    *total += bytes;
    return NWB_OK;
}

}  // namespace

extern "C" void nwb_set_error_(const char* msg) { g_err = msg ? msg : ""; }

struct nwb_solver {
    int device = 0;
    cudaStream_t st = nullptr;
    int N = 0, nelt = 0, geo = 0, f32 = 0;
    long long npts = 0, stride = 0, nfp = 0;
    double c0 = 1.0;
    double* u[2] = {nullptr, nullptr};
    double* k = nullptr;
    int cur = 0;
    double* dD = nullptr;
    double hD[100] = {};
    double hzl[10] = {};  // line coordinates of hD (nwb::line_coords)
    int snel[3] = {0, 0, 0};  // structured box mesh (x-fastest elements), 0 = not
    int spmask = 0;
    // probes (nwb_probe_setup): node offset and N^3 weights per probe, device values
    int nprobes = 0;
    long long* dprobe_off = nullptr;
    double* dprobe_w = nullptr;
    double* dprobe_out = nullptr;
    // asynchronous snapshots (nwb_snapshot_begin/wait)
    double* dsnap = nullptr;
    cudaStream_t snap_st = nullptr;
    cudaEvent_t snap_ev = nullptr;
    bool snap_pending = false;
    // asynchronous uploads (nwb_upload_begin/wait): a staging copy of the state
    double* dstage = nullptr;
    cudaStream_t up_st = nullptr;
    cudaEvent_t up_done = nullptr;  // the host copy into dstage has landed
    cudaEvent_t up_free = nullptr;  // the solver stream has copied dstage into the state
    bool up_pending = false;
    nwb::ElemGeo* dgeo = nullptr;
    int* dconn = nullptr;
    double* djac_e = nullptr;
    double* dmet_n = nullptr;
    double* dfnrm = nullptr;
    double* dflift = nullptr;
    int* dfplus = nullptr;
    double* djac_n = nullptr;
    double* dw3 = nullptr;
    double* dpartial = nullptr;
    double* denergy = nullptr;
    int* derr = nullptr;  // kernels record an expired bounded wait here
    int eblocks = 1;
    void* dflush = nullptr;
    size_t flush_bytes = 0;
    nwb::StageConfig cfg{};
    int variant = 0;
    long long launches = 0;
    size_t device_bytes = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    double gdt = 0.0;
    bool is_box = false;
    nwb::BoxPulse box{};

    nwb::StageParams params(int stage, double dt) const {
        nwb::StageParams P{};
        P.u_in = u[cur];
        P.u_out = u[cur ^ 1];
        P.k = k;
        P.stride = stride;
        P.nelt = nelt;
        P.D = dD;
        P.geo = dgeo;
        P.conn = dconn;
        P.met_n = dmet_n;
        P.fnrm = dfnrm;
        P.flift = dflift;
        P.fplus = dfplus;
        P.nfp = nfp;
        P.err = derr;
        P.c0 = c0;
        P.a = kRK4A[stage];
        P.b = kRK4B[stage];
        P.dt = dt;
        for (int x = 0; x < N * N; ++x) P.Dc[x] = hD[x];
        for (int x = 0; x < N; ++x) P.zl[x] = hzl[x];
        for (int d = 0; d < 3; ++d) P.snel[d] = snel[d];
        P.spmask = spmask;
        return P;
    }

    nwb_status launch_stage(int stage, double dt) {
        nwb::StageParams P = params(stage, dt);
        cudaError_t e = nwb::launch_stage(N, geo, f32, variant, &P, st, nullptr);
        if (e != cudaSuccess) return fail(NWB_ECUDA, "stage kernel launch: %s", cudaGetErrorString(e));
        cur ^= 1;
        ++launches;
        return NWB_OK;
    }

    nwb_status launch_step(double dt) {
        for (int s = 0; s < 5; ++s) {
            nwb_status r = launch_stage(s, dt);
            if (r != NWB_OK) return r;
        }
        return NWB_OK;
    }

    void drop_graphs() {
        for (auto& g : gexec)
            if (g) {
                cudaGraphExecDestroy(g);
                g = nullptr;
            }
    }

    // One-step graphs for both ping-pong parities, captured for this dt.
    nwb_status ensure_graphs(double dt) {
        if (gexec[0] && gexec[1] && gdt == dt) return NWB_OK;
        drop_graphs();
        const int cur0 = cur;
        const long long l0 = launches;
        for (int par = 0; par < 2; ++par) {
            cur = par;
            cudaGraph_t g = nullptr;
            NWB_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            nwb_status r = launch_step(dt);
            cudaError_t ce = cudaStreamEndCapture(st, &g);
            if (r != NWB_OK) {
                if (g) cudaGraphDestroy(g);
                cur = cur0;
                return r;
            }
            if (ce != cudaSuccess) {
                cur = cur0;
                return fail(NWB_ECUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(ce));
            }
            ce = cudaGraphInstantiate(&gexec[par], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) {
                cur = cur0;
                return fail(NWB_ECUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ce));
            }
        }
        cur = cur0;
        launches = l0;
        gdt = dt;
        return NWB_OK;
    }

    nwb_status run_steps(double dt, int nsteps, bool graph) {
        if (graph) {
            nwb_status r = ensure_graphs(dt);
            if (r != NWB_OK) return r;
            for (int s = 0; s < nsteps; ++s) {
                NWB_CU(cudaGraphLaunch(gexec[cur], st));
                cur ^= 1;  // five stages: odd number of swaps
                launches += 5;
            }
            return NWB_OK;
        }
        for (int s = 0; s < nsteps; ++s) {
            nwb_status r = launch_step(dt);
            if (r != NWB_OK) return r;
        }
        return NWB_OK;
    }

    void release() {
        drop_graphs();
        void* ptrs[] = {u[0], u[1], k, dD, dgeo, dconn, djac_e, dmet_n, dfnrm, dflift,
                        dfplus, djac_n, dw3, dpartial, denergy, dflush, dprobe_off, dprobe_w, dprobe_out, dsnap,
                        derr, dstage};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        if (st) cudaStreamDestroy(st);
        st = nullptr;
        if (snap_st) cudaStreamDestroy(snap_st);
        snap_st = nullptr;
        if (snap_ev) cudaEventDestroy(snap_ev);
        snap_ev = nullptr;
        if (up_st) cudaStreamDestroy(up_st);
        up_st = nullptr;
        for (cudaEvent_t* ev : {&up_done, &up_free}) {
            if (*ev) cudaEventDestroy(*ev);
            *ev = nullptr;
        }
    }
};

namespace {
nwb_status create_solver(const nwb_mesh_desc* m, int N, int nelt, const double* D, const double* w3,
                         Analysis& A, double c0, nwb_precision prec, nwb_solver** out,
                         bool true_pmc);
}  // namespace

extern "C" {

const char* nwb_last_error(void) { return g_err.c_str(); }

const char* nwb_status_string(nwb_status s) {
    switch (s) {
        case NWB_OK: return "NWB_OK";
        case NWB_EINVAL: return "NWB_EINVAL";
        case NWB_ENOMEM: return "NWB_ENOMEM";
        case NWB_ECUDA: return "NWB_ECUDA";
        case NWB_ETIMEOUT: return "NWB_ETIMEOUT";
        case NWB_ENONFINITE: return "NWB_ENONFINITE";
        case NWB_EBUSY: return "NWB_EBUSY";
        case NWB_ENOTFOUND: return "NWB_ENOTFOUND";
    }
    return "NWB_UNKNOWN";
}

int nwb_version(void) { return NWB_VERSION; }

nwb_status nwb_set_device(int device) {
    NWB_CU(cudaSetDevice(device));
    return NWB_OK;
}

nwb_status nwb_solver_create(const nwb_mesh_desc* m, double c0, nwb_precision prec, nwb_solver** out) {
    return nwb_solver_create_ex(m, c0, prec, 0u, out);
}

nwb_status nwb_solver_create_ex(const nwb_mesh_desc* m, double c0, nwb_precision prec, unsigned flags,
                                nwb_solver** out) {
    if (!out) return fail(NWB_EINVAL, "nwb_solver_create: out is null");
    *out = nullptr;
    if (!m) return fail(NWB_EINVAL, "nwb_solver_create: mesh is null");
    if (m->N < 2 || m->N > 10) return fail(NWB_EINVAL, "nwb_solver_create: N=%d outside 2..10", m->N);
    if (m->nelt < 1) return fail(NWB_EINVAL, "nwb_solver_create: nelt=%d", m->nelt);
    if (prec != NWB_FP64 && prec != NWB_FP32_BULK)
        return fail(NWB_EINVAL, "nwb_solver_create: unknown precision %d", static_cast<int>(prec));
    if (!m->D || !m->w3 || !m->jac || !m->vol_idx_minus || !m->vol_idx_plus || !m->bc_type || !m->nx ||
        !m->ny || !m->nz || !m->dA)
        return fail(NWB_EINVAL, "nwb_solver_create: null mesh array");
    for (int c = 0; c < 9; ++c)
        if (!m->met[c]) return fail(NWB_EINVAL, "nwb_solver_create: null metric array %d", c);
    if (!std::isfinite(c0)) return fail(NWB_EINVAL, "nwb_solver_create: c0 not finite");
    const int N = m->N, N2 = N * N, N3 = N2 * N;
    const long long npts = static_cast<long long>(m->nelt) * N3;
    if (m->nelt > (1 << 25) || npts > 0x7fffffffLL)
        return fail(NWB_EINVAL, "nwb_solver_create: mesh too large for 32-bit node indices");
    if (flags & ~static_cast<unsigned>(NWB_SOLVER_TRUE_PMC))
        return fail(NWB_EINVAL, "nwb_solver_create_ex: unknown flags 0x%x", flags);
    const bool true_pmc = (flags & NWB_SOLVER_TRUE_PMC) != 0;

    Analysis A;
    try {
        nwb_status r = nwb::analyse_mesh(m, &A, true_pmc);
        if (r != NWB_OK) return r;
    } catch (const std::bad_alloc&) {
        return fail(NWB_ENOMEM, "nwb_solver_create: out of host memory");
    }
    return create_solver(m, N, m->nelt, m->D, m->w3, A, c0, prec, out, true_pmc);
}

}  // extern "C"

namespace {

// Connection code of face f of element (ex,ey,ez) of a structured box mesh with
// x-fastest element order (the order of the reference's createBoxMesh).
int box_conn(int ex, int ey, int ez, int f, const int nel[3], int pm) {
    const int nx = nel[0], ny = nel[1], nz = nel[2];
    auto id = [&](int a, int b, int c) { return a + nx * (b + ny * c); };
    int nb = -1;
    switch (f) {
        case 0: nb = ey > 0 ? id(ex, ey - 1, ez) : ((pm & 2) ? id(ex, ny - 1, ez) : -1); break;
        case 1: nb = ex < nx - 1 ? id(ex + 1, ey, ez) : ((pm & 1) ? id(0, ey, ez) : -1); break;
        case 2: nb = ey < ny - 1 ? id(ex, ey + 1, ez) : ((pm & 2) ? id(ex, 0, ez) : -1); break;
        case 3: nb = ex > 0 ? id(ex - 1, ey, ez) : ((pm & 1) ? id(nx - 1, ey, ez) : -1); break;
        case 4: nb = ez > 0 ? id(ex, ey, ez - 1) : ((pm & 4) ? id(ex, ey, nz - 1) : -1); break;
        default: nb = ez < nz - 1 ? id(ex, ey, ez + 1) : ((pm & 4) ? id(ex, ey, 0) : -1); break;
    }
    static const int opp[6] = {2, 3, 0, 1, 5, 4};
    return nb < 0 ? nwb::kConnPEC : ((nb << 6) | (opp[f] << 3));
}

// Recognises the connection table of a structured box mesh (elements x-fastest,
// identity face orientations): the stage kernels can then find neighbours from
// the element index.  Returns false and leaves nel at 0 for any other table.
bool detect_structure(const std::vector<int>& conn, int nelt, int nel[3], int* pm) {
    nel[0] = nel[1] = nel[2] = 0;
    *pm = 0;
    auto step = [&](int e, int f) { const int cd = conn[6 * static_cast<size_t>(e) + f];
                                    return cd == nwb::kConnPEC ? -1 : (cd >> 6); };
    int n[2] = {1, 1}, mask = 0;
    const int face[2] = {1, 2};
    for (int d = 0; d < 2; ++d) {
        const int stride = d == 0 ? 1 : n[0];
        int e = 0;
        for (;;) {
            const int nb = step(e, face[d]);
            if (nb < 0) break;
            if (nb == 0) { mask |= 1 << d; break; }
            if (nb != e + stride || n[d] >= nelt) return false;
            e = nb;
            ++n[d];
        }
    }
    if (nelt % (n[0] * n[1]) != 0) return false;
    const int nz = nelt / (n[0] * n[1]);
    const int zb = step(0, 4);
    if (zb >= 0) {
        if (zb != (nz - 1) * n[0] * n[1]) return false;
        mask |= 4;
    }
    const int dims[3] = {n[0], n[1], nz};
    for (int e = 0; e < nelt; ++e) {
        const int ex = e % dims[0], ey = (e / dims[0]) % dims[1], ez = e / (dims[0] * dims[1]);
        for (int f = 0; f < 6; ++f)
            if (conn[6 * static_cast<size_t>(e) + f] != box_conn(ex, ey, ez, f, dims, mask)) return false;
    }
    for (int d = 0; d < 3; ++d) nel[d] = dims[d];
    *pm = mask;
    return true;
}

// Allocates and uploads a solver from analysed geometry.  m supplies the
// per-node arrays of the general class and may be null for the affine classes.
nwb_status create_solver(const nwb_mesh_desc* m, int N, int nelt, const double* D, const double* w3,
                         Analysis& A, double c0, nwb_precision prec, nwb_solver** out,
                         bool true_pmc) {
    const int N2 = N * N, N3 = N2 * N;
    const long long npts = static_cast<long long>(nelt) * N3;
    nwb_solver* s = new (std::nothrow) nwb_solver();
    if (!s) return fail(NWB_ENOMEM, "nwb_solver_create: out of host memory");
    auto bail = [&](nwb_status r) {
        s->release();
        delete s;
        return r;
    };
    cudaError_t ce = cudaGetDevice(&s->device);
    if (ce != cudaSuccess) {
        delete s;
        return fail(NWB_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(ce));
    }
    s->N = N;
    s->nelt = nelt;
    s->npts = npts;
    s->stride = (npts + 63) / 64 * 64;  // 512-byte aligned components
    s->nfp = static_cast<long long>(nelt) * 6 * N2;
    s->geo = A.geo;
    s->f32 = prec == NWB_FP32_BULK ? 1 : 0;
    s->c0 = c0;
    s->eblocks = nwb::energy_blocks(nelt);
    ce = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "cudaStreamCreate: %s", cudaGetErrorString(ce)));

    ce = nwb::launch_stage(N, s->geo, s->f32, s->variant, nullptr, nullptr, &s->cfg);
    if (ce != cudaSuccess)
        return bail(fail(NWB_ECUDA, "stage kernel set-up: %s", cudaGetErrorString(ce)));

    size_t& tot = s->device_bytes;
    nwb_status r = NWB_OK;
#define NWB_TRY(x)                  \
    do {                            \
        r = (x);                    \
        if (r != NWB_OK) return bail(r); \
    } while (0)
    NWB_TRY(dalloc(&s->u[0], 6 * static_cast<size_t>(s->stride), &tot));
    NWB_TRY(dalloc(&s->u[1], 6 * static_cast<size_t>(s->stride), &tot));
    NWB_TRY(dalloc(&s->k, 6 * static_cast<size_t>(s->stride), &tot));
    NWB_TRY(dalloc(&s->dD, static_cast<size_t>(N2), &tot));
    NWB_TRY(dalloc(&s->dw3, static_cast<size_t>(N3), &tot));
    // partial sums of the energy, or (max|E|, max|H|) pairs; energy, max|E|, max|H|
    NWB_TRY(dalloc(&s->dpartial, 2 * static_cast<size_t>(s->eblocks), &tot));
    NWB_TRY(dalloc(&s->denergy, 3, &tot));
    NWB_TRY(dalloc(&s->derr, 1, &tot));
    ce = cudaMemset(s->derr, 0, sizeof(int));
    if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "memset: %s", cudaGetErrorString(ce)));
#define NWB_H2D(dst, src, bytes) \
    do { ce = cudaMemcpy((dst), (src), (bytes), cudaMemcpyHostToDevice); \
         if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "upload: %s", cudaGetErrorString(ce))); } while (0)
    NWB_H2D(s->dD, D, sizeof(double) * N2);
    for (int x = 0; x < N2; ++x) s->hD[x] = D[x];
    nwb::line_coords(N, s->hD, s->hzl);
    NWB_H2D(s->dw3, w3, sizeof(double) * N3);
    if (s->geo != nwb::GEO_NODAL) {
        NWB_TRY(dalloc(&s->dgeo, static_cast<size_t>(nelt), &tot));
        // padded to a multiple of four entries: bulk copies of a tile's connections
        // are 16-byte aligned at both ends (stage_ws.cuh)
        NWB_TRY(dalloc(&s->dconn, 6 * static_cast<size_t>(nelt) + 4, &tot));
        NWB_TRY(dalloc(&s->djac_e, static_cast<size_t>(nelt), &tot));
        NWB_H2D(s->dgeo, A.egeo.data(), sizeof(nwb::ElemGeo) * nelt);
        NWB_H2D(s->dconn, A.conn.data(), sizeof(int) * 6 * static_cast<size_t>(nelt));
        ce = cudaMemset(s->dconn + 6 * static_cast<size_t>(nelt), 0, 4 * sizeof(int));
        if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "memset: %s", cudaGetErrorString(ce)));
        NWB_H2D(s->djac_e, A.jac_e.data(), sizeof(double) * nelt);
        detect_structure(A.conn, nelt, s->snel, &s->spmask);
    } else {
        const size_t nfp = static_cast<size_t>(s->nfp);
        try {
            std::vector<double> fn(3 * nfp), fl(nfp);
            std::vector<int> fpl(nfp);
            for (size_t fp = 0; fp < nfp; ++fp) {
                const int vm = m->vol_idx_minus[fp];
                const int wall = nwb::wall_code(m, static_cast<long long>(fp), true_pmc);
                fn[fp] = m->nx[fp];
                fn[nfp + fp] = m->ny[fp];
                fn[2 * nfp + fp] = m->nz[fp];
                fl[fp] = m->dA[fp] / (m->jac[vm] * m->w3[vm % N3]);
                fpl[fp] = wall ? wall : m->vol_idx_plus[fp];
            }
            NWB_TRY(dalloc(&s->dmet_n, 9 * static_cast<size_t>(s->stride), &tot));
            NWB_TRY(dalloc(&s->djac_n, static_cast<size_t>(npts), &tot));
            NWB_TRY(dalloc(&s->dfnrm, 3 * nfp, &tot));
            NWB_TRY(dalloc(&s->dflift, nfp, &tot));
            NWB_TRY(dalloc(&s->dfplus, nfp, &tot));
            for (int c = 0; c < 9; ++c) NWB_H2D(s->dmet_n + c * s->stride, m->met[c], sizeof(double) * npts);
            NWB_H2D(s->djac_n, m->jac, sizeof(double) * npts);
            NWB_H2D(s->dfnrm, fn.data(), sizeof(double) * 3 * nfp);
            NWB_H2D(s->dflift, fl.data(), sizeof(double) * nfp);
            NWB_H2D(s->dfplus, fpl.data(), sizeof(int) * nfp);
        } catch (const std::bad_alloc&) {
            return bail(fail(NWB_ENOMEM, "nwb_solver_create: out of host memory"));
        }
    }
    // state and LSRK register start at zero (src/dg_solver.cpp:122-125)
    for (int b = 0; b < 2; ++b) {
        ce = cudaMemset(s->u[b], 0, sizeof(double) * 6 * s->stride);
        if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "memset: %s", cudaGetErrorString(ce)));
    }
    ce = cudaMemset(s->k, 0, sizeof(double) * 6 * s->stride);
    if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "memset: %s", cudaGetErrorString(ce)));
    ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) return bail(fail(NWB_ECUDA, "set-up: %s", cudaGetErrorString(ce)));
#undef NWB_TRY
#undef NWB_H2D
    *out = s;
    return NWB_OK;
}

}  // namespace

extern "C" {

nwb_status nwb_solver_create_box(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                                 double ymin, double ymax, double zmin, double zmax,
                                 int periodic_mask, double c0, nwb_precision prec, nwb_solver** out) {
    if (!out) return fail(NWB_EINVAL, "nwb_solver_create_box: out is null");
    *out = nullptr;
    const long long nelt = static_cast<long long>(nelx) * nely * nelz;
    if (N < 2 || N > 10 || nelx < 1 || nely < 1 || nelz < 1 || nelt > (1 << 25) ||
        nelt * N * N * N > 0x7fffffffLL || !(xmax > xmin) || !(ymax > ymin) || !(zmax > zmin))
        return fail(NWB_EINVAL, "nwb_solver_create_box: bad box");
    if (prec != NWB_FP64 && prec != NWB_FP32_BULK)
        return fail(NWB_EINVAL, "nwb_solver_create_box: unknown precision %d", static_cast<int>(prec));
    if (!std::isfinite(c0)) return fail(NWB_EINVAL, "nwb_solver_create_box: c0 not finite");
    Analysis A;
    std::vector<double> z, w, D, w3(static_cast<size_t>(N) * N * N);
    const double lo[3] = {xmin, ymin, zmin}, hi[3] = {xmax, ymax, zmax};
    try {
        nwb::gll(N, z, w, D);
        nwb::box_geometry(N, nelx, nely, nelz, lo, hi, periodic_mask, z, w, A.egeo, A.conn);
    } catch (const std::bad_alloc&) {
        return fail(NWB_ENOMEM, "nwb_solver_create_box: out of host memory");
    }
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) w3[i + N * (j + N * k)] = w[i] * w[j] * w[k];
    A.jac_e.resize(A.egeo.size());
    bool box = true;
    for (size_t e = 0; e < A.egeo.size(); ++e) {
        A.jac_e[e] = A.egeo[e].jdet;
        double scale = 0;
        for (int c = 0; c < 9; ++c) scale = std::max(scale, std::abs(A.egeo[e].met[c]));
        for (int c : {1, 2, 3, 5, 6, 7})
            if (std::abs(A.egeo[e].met[c]) > 1e-13 * scale) box = false;
    }
    A.geo = box ? nwb::GEO_BOX : nwb::GEO_AFFINE;
    nwb_status r = create_solver(nullptr, N, static_cast<int>(nelt), D.data(), w3.data(), A, c0, prec, out,
                                 false);
    if (r != NWB_OK) return r;
    nwb_solver* s = *out;
    s->box.lo[0] = xmin; s->box.lo[1] = ymin; s->box.lo[2] = zmin;
    s->box.h[0] = (xmax - xmin) / nelx; s->box.h[1] = (ymax - ymin) / nely; s->box.h[2] = (zmax - zmin) / nelz;
    s->box.nel[0] = nelx; s->box.nel[1] = nely; s->box.nel[2] = nelz;
    s->box.N = N;
    for (int i = 0; i < N; ++i) s->box.z[i] = z[i];
    s->is_box = true;
    return NWB_OK;
}

nwb_status nwb_solver_init_pulse(nwb_solver* s, const double* pulse) {
    if (!s || !pulse) return fail(NWB_EINVAL, "nwb_solver_init_pulse: null argument");
    if (!s->is_box) return fail(NWB_EINVAL, "nwb_solver_init_pulse: solver was not created from a box");
    nwb::BoxPulse b = s->box;
    for (int i = 0; i < 30; ++i) b.pulse[i] = pulse[i];
    cudaError_t e = nwb::launch_box_pulse(b, s->u[s->cur], s->stride, s->st);
    if (e != cudaSuccess) return fail(NWB_ECUDA, "pulse kernel: %s", cudaGetErrorString(e));
    ++s->launches;
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_upload_state(nwb_solver* s, const double* h, size_t n) {
    if (!s || !h) return fail(NWB_EINVAL, "nwb_upload_state: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_upload_state: size %zu, expected 6*npts = %lld", n, 6 * s->npts);
    NWB_CU(cudaMemcpy2DAsync(s->u[s->cur], sizeof(double) * s->stride, h, sizeof(double) * s->npts,
                             sizeof(double) * s->npts, 6, cudaMemcpyHostToDevice, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_download_state(nwb_solver* s, double* h, size_t n) {
    if (!s || !h) return fail(NWB_EINVAL, "nwb_download_state: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_download_state: size %zu, expected 6*npts = %lld", n, 6 * s->npts);
    NWB_CU(cudaMemcpy2DAsync(h, sizeof(double) * s->npts, s->u[s->cur], sizeof(double) * s->stride,
                             sizeof(double) * s->npts, 6, cudaMemcpyDeviceToHost, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_download_nodes(nwb_solver* s, long long first, long long count, double* h, size_t n) {
    if (!s || !h) return fail(NWB_EINVAL, "nwb_download_nodes: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_download_nodes: size %zu, expected 6*npts = %lld", n, 6 * s->npts);
    if (first < 0 || count < 0 || first + count > s->npts)
        return fail(NWB_EINVAL, "nwb_download_nodes: nodes [%lld, %lld) outside [0, %lld)", first,
                    first + count, s->npts);
    if (count == 0) return NWB_OK;
    NWB_CU(cudaMemcpy2DAsync(h + first, sizeof(double) * s->npts, s->u[s->cur] + first,
                             sizeof(double) * s->stride, sizeof(double) * count, 6,
                             cudaMemcpyDeviceToHost, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_step(nwb_solver* s, double dt, int nsteps) {
    if (!s) return fail(NWB_EINVAL, "nwb_step: null solver");
    if (nsteps < 0 || !std::isfinite(dt)) return fail(NWB_EINVAL, "nwb_step: bad dt/nsteps");
    if (nsteps == 0) return NWB_OK;
    return s->run_steps(dt, nsteps, nsteps > 1);
}

nwb_status nwb_sync(nwb_solver* s) {
    if (!s) return fail(NWB_EINVAL, "nwb_sync: null solver");
    NWB_CU(cudaStreamSynchronize(s->st));
    // a bounded wait inside a stage kernel that expired (the warp-specialised form)
    int err = 0;
    NWB_CU(cudaMemcpy(&err, s->derr, sizeof(int), cudaMemcpyDeviceToHost));
    if (err != 0) {
        NWB_CU(cudaMemset(s->derr, 0, sizeof(int)));
        return fail(NWB_ETIMEOUT, "nwb_sync: a stage kernel's bounded wait expired (code %d); the "
                                  "state of the steps since the last sync is not valid", err);
    }
    return NWB_OK;
}

nwb_status nwb_eval_rhs(nwb_solver* s, double* h, size_t n) {
    if (!s || !h) return fail(NWB_EINVAL, "nwb_eval_rhs: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_eval_rhs: size %zu, expected 6*npts", n);
    // one stage with a = 0, b = 0, dt = 1 leaves k = rhs and copies u_in into the
    // spare buffer; the state itself (u[cur]) is untouched
    NWB_CU(cudaMemsetAsync(s->k, 0, sizeof(double) * 6 * s->stride, s->st));
    nwb::StageParams P = s->params(0, 1.0);
    P.a = 0.0;
    P.b = 0.0;
    cudaError_t e = nwb::launch_stage(s->N, s->geo, s->f32, s->variant, &P, s->st, nullptr);
    if (e != cudaSuccess) return fail(NWB_ECUDA, "stage kernel launch: %s", cudaGetErrorString(e));
    ++s->launches;
    NWB_CU(cudaMemcpy2DAsync(h, sizeof(double) * s->npts, s->k, sizeof(double) * s->stride,
                             sizeof(double) * s->npts, 6, cudaMemcpyDeviceToHost, s->st));
    NWB_CU(cudaMemsetAsync(s->k, 0, sizeof(double) * 6 * s->stride, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_energy(nwb_solver* s, double* out) {
    if (!s || !out) return fail(NWB_EINVAL, "nwb_energy: null argument");
    cudaError_t e = nwb::launch_energy(s->u[s->cur], s->stride, s->N, s->nelt, s->djac_e, s->djac_n,
                                       s->dw3, s->dpartial, s->eblocks, s->denergy, s->st);
    if (e != cudaSuccess) return fail(NWB_ECUDA, "energy kernel: %s", cudaGetErrorString(e));
    s->launches += 2;
    NWB_CU(cudaMemcpyAsync(out, s->denergy, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    if (!std::isfinite(*out)) return fail(NWB_ENONFINITE, "nwb_energy: state holds NaN/Inf");
    return NWB_OK;
}

nwb_status nwb_max_norms(nwb_solver* s, double* max_e, double* max_h) {
    if (!s || !max_e || !max_h) return fail(NWB_EINVAL, "nwb_max_norms: null argument");
    cudaError_t e = nwb::launch_max_norms(s->u[s->cur], s->stride, s->npts, s->dpartial, s->eblocks,
                                          s->denergy + 1, s->st);
    if (e != cudaSuccess) return fail(NWB_ECUDA, "max-norm kernel: %s", cudaGetErrorString(e));
    s->launches += 2;
    double h[2];
    NWB_CU(cudaMemcpyAsync(h, s->denergy + 1, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    *max_e = h[0];
    *max_h = h[1];
    if (!std::isfinite(h[0]) || !std::isfinite(h[1]))
        return fail(NWB_ENONFINITE, "nwb_max_norms: state holds Inf");
    return NWB_OK;
}

nwb_status nwb_probe_setup(nwb_solver* s, int nprobes, const long long* node_offset,
                           const double* weights) {
    if (!s) return fail(NWB_EINVAL, "nwb_probe_setup: null solver");
    if (nprobes < 0 || (nprobes > 0 && (!node_offset || !weights)))
        return fail(NWB_EINVAL, "nwb_probe_setup: bad probe arrays");
    const int N3 = s->N * s->N * s->N;
    for (int p = 0; p < nprobes; ++p)
        if (node_offset[p] < 0 || node_offset[p] % N3 != 0 || node_offset[p] + N3 > s->npts)
            return fail(NWB_EINVAL, "nwb_probe_setup: probe %d offset %lld is not an element start", p,
                        node_offset[p]);
    NWB_CU(cudaStreamSynchronize(s->st));
    for (void* q : {static_cast<void*>(s->dprobe_off), static_cast<void*>(s->dprobe_w),
                    static_cast<void*>(s->dprobe_out)})
        if (q) cudaFree(q);
    s->dprobe_off = nullptr;
    s->dprobe_w = nullptr;
    s->dprobe_out = nullptr;
    s->nprobes = 0;
    if (nprobes == 0) return NWB_OK;
    NWB_CU(cudaMalloc(&s->dprobe_off, sizeof(long long) * nprobes));
    NWB_CU(cudaMalloc(&s->dprobe_w, sizeof(double) * N3 * static_cast<size_t>(nprobes)));
    NWB_CU(cudaMalloc(&s->dprobe_out, sizeof(double) * 6 * nprobes));
    NWB_CU(cudaMemcpy(s->dprobe_off, node_offset, sizeof(long long) * nprobes, cudaMemcpyHostToDevice));
    NWB_CU(cudaMemcpy(s->dprobe_w, weights, sizeof(double) * N3 * static_cast<size_t>(nprobes),
                      cudaMemcpyHostToDevice));
    s->nprobes = nprobes;
    return NWB_OK;
}

nwb_status nwb_probe_read(nwb_solver* s, double* out) {
    if (!s || !out) return fail(NWB_EINVAL, "nwb_probe_read: null argument");
    if (s->nprobes == 0) return fail(NWB_EINVAL, "nwb_probe_read: no probes set up");
    cudaError_t e = nwb::launch_probes(s->u[s->cur], s->stride, s->N * s->N * s->N, s->dprobe_off,
                                       s->dprobe_w, s->nprobes, s->dprobe_out, s->st);
    if (e != cudaSuccess) return fail(NWB_ECUDA, "probe kernel: %s", cudaGetErrorString(e));
    ++s->launches;
    NWB_CU(cudaMemcpyAsync(out, s->dprobe_out, sizeof(double) * 6 * s->nprobes, cudaMemcpyDeviceToHost,
                           s->st));
    NWB_CU(cudaStreamSynchronize(s->st));
    return NWB_OK;
}

nwb_status nwb_snapshot_begin(nwb_solver* s, double* host, size_t n) {
    if (!s || !host) return fail(NWB_EINVAL, "nwb_snapshot_begin: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_snapshot_begin: size %zu, expected 6*npts = %lld", n, 6 * s->npts);
    if (!s->dsnap) {
        NWB_CU(cudaStreamSynchronize(s->st));
        NWB_CU(cudaMalloc(&s->dsnap, sizeof(double) * 6 * static_cast<size_t>(s->stride)));
        NWB_CU(cudaStreamCreateWithFlags(&s->snap_st, cudaStreamNonBlocking));
        NWB_CU(cudaEventCreateWithFlags(&s->snap_ev, cudaEventDisableTiming));
    }
    if (s->snap_pending) NWB_CU(cudaStreamSynchronize(s->snap_st));  // one snapshot in flight
    // device copy in stream order (after every step queued so far), then the host
    // copy on the snapshot stream, overlapping the steps queued after this call
    NWB_CU(cudaMemcpyAsync(s->dsnap, s->u[s->cur], sizeof(double) * 6 * s->stride,
                           cudaMemcpyDeviceToDevice, s->st));
    NWB_CU(cudaEventRecord(s->snap_ev, s->st));
    NWB_CU(cudaStreamWaitEvent(s->snap_st, s->snap_ev, 0));
    NWB_CU(cudaMemcpy2DAsync(host, sizeof(double) * s->npts, s->dsnap, sizeof(double) * s->stride,
                             sizeof(double) * s->npts, 6, cudaMemcpyDeviceToHost, s->snap_st));
    s->snap_pending = true;
    return NWB_OK;
}

nwb_status nwb_upload_begin(nwb_solver* s, const double* host, size_t n) {
    if (!s || !host) return fail(NWB_EINVAL, "nwb_upload_begin: null argument");
    if (n != 6 * static_cast<size_t>(s->npts))
        return fail(NWB_EINVAL, "nwb_upload_begin: size %zu, expected 6*npts = %lld", n, 6 * s->npts);
    const size_t bytes = sizeof(double) * 6 * static_cast<size_t>(s->stride);
    if (!s->dstage) {
        NWB_CU(cudaStreamSynchronize(s->st));
        NWB_CU(cudaMalloc(&s->dstage, bytes));
        // the rows' padding (npts..stride) is never written by the host copies:
        // zero, like the state's own padding
        NWB_CU(cudaMemset(s->dstage, 0, bytes));
        NWB_CU(cudaStreamCreateWithFlags(&s->up_st, cudaStreamNonBlocking));
        NWB_CU(cudaEventCreateWithFlags(&s->up_done, cudaEventDisableTiming));
        NWB_CU(cudaEventCreateWithFlags(&s->up_free, cudaEventDisableTiming));
        NWB_CU(cudaEventRecord(s->up_free, s->st));
    }
    // the staging buffer is reused once the solver stream has copied the previous
    // upload out of it; the host copy then overlaps the steps queued before this call
    NWB_CU(cudaStreamWaitEvent(s->up_st, s->up_free, 0));
    NWB_CU(cudaMemcpy2DAsync(s->dstage, sizeof(double) * s->stride, host, sizeof(double) * s->npts,
                             sizeof(double) * s->npts, 6, cudaMemcpyHostToDevice, s->up_st));
    NWB_CU(cudaEventRecord(s->up_done, s->up_st));
    // in the solver's stream order: steps queued later start from the uploaded state
    NWB_CU(cudaStreamWaitEvent(s->st, s->up_done, 0));
    NWB_CU(cudaMemcpyAsync(s->u[s->cur], s->dstage, bytes, cudaMemcpyDeviceToDevice, s->st));
    NWB_CU(cudaEventRecord(s->up_free, s->st));
    s->up_pending = true;
    return NWB_OK;
}

nwb_status nwb_upload_wait(nwb_solver* s) {
    if (!s) return fail(NWB_EINVAL, "nwb_upload_wait: null solver");
    if (s->up_pending) NWB_CU(cudaStreamSynchronize(s->up_st));
    s->up_pending = false;
    return NWB_OK;
}

nwb_status nwb_snapshot_wait(nwb_solver* s) {
    if (!s) return fail(NWB_EINVAL, "nwb_snapshot_wait: null solver");
    if (s->snap_pending) NWB_CU(cudaStreamSynchronize(s->snap_st));
    s->snap_pending = false;
    return NWB_OK;
}

nwb_status nwb_solver_destroy(nwb_solver* s) {
    if (!s) return NWB_OK;
    cudaStreamSynchronize(s->st);
    if (s->snap_st) cudaStreamSynchronize(s->snap_st);
    if (s->up_st) cudaStreamSynchronize(s->up_st);
    s->release();
    delete s;
    return NWB_OK;
}

nwb_status nwb_solver_get_info(const nwb_solver* s, nwb_solver_info* info) {
    if (!s || !info) return fail(NWB_EINVAL, "nwb_solver_get_info: null argument");
    info->N = s->N;
    info->nelt = s->nelt;
    info->npts = s->npts;
    info->stride = s->stride;
    info->geometry = s->geo;
    info->precision = s->f32;
    info->ks = s->cfg.ks;
    info->epb = s->cfg.epb;
    info->threads_per_block = s->cfg.threads;
    info->smem_bytes = s->cfg.smem;
    info->ksmem = s->cfg.ksmem;
    info->minb = s->cfg.minb;
    info->variant = s->variant;
    info->variant_count = nwb::stage_variant_count(s->N, s->geo, s->f32);
    info->device_bytes = static_cast<long long>(s->device_bytes);
    for (int d = 0; d < 3; ++d) info->structured[d] = s->snel[d];
    info->periodic_mask = s->spmask;
    return NWB_OK;
}

nwb_status nwb_solver_device_state(nwb_solver* s, double** d_state, void** stream) {
    if (!s) return fail(NWB_EINVAL, "nwb_solver_device_state: null solver");
    if (d_state) *d_state = s->u[s->cur];
    if (stream) *stream = s->st;
    return NWB_OK;
}

nwb_status nwb_solver_launch_count(const nwb_solver* s, long long* count) {
    if (!s || !count) return fail(NWB_EINVAL, "nwb_solver_launch_count: null argument");
    *count = s->launches;
    return NWB_OK;
}

nwb_status nwb_solver_set_variant(nwb_solver* s, int variant) {
    if (!s) return fail(NWB_EINVAL, "nwb_solver_set_variant: null solver");
    if (variant < 0 || variant >= nwb::stage_variant_count(s->N, s->geo, s->f32))
        return fail(NWB_EINVAL, "nwb_solver_set_variant: variant %d out of range", variant);
    nwb::StageConfig c{};
    cudaError_t e = nwb::launch_stage(s->N, s->geo, s->f32, variant, nullptr, nullptr, &c);
    if (e != cudaSuccess)
        return fail(NWB_ECUDA, "variant %d set-up: %s", variant, cudaGetErrorString(e));
    NWB_CU(cudaStreamSynchronize(s->st));
    s->variant = variant;
    s->cfg = c;
    s->drop_graphs();
    return NWB_OK;
}

// Times every launch shape of the stage kernel on this solver's mesh and keeps
// the fastest.  The timed launches use a = b = dt = 0, so they leave the state
// bit for bit as it was and reset the LSRK register to zero (which the first
// stage of every step multiplies by a = 0 anyway).
nwb_status nwb_solver_autotune(nwb_solver* s, int reps, int* best, float* ms_out, int ms_cap) {
    if (!s || reps < 1) return fail(NWB_EINVAL, "nwb_solver_autotune: bad argument");
    const int nv = nwb::stage_variant_count(s->N, s->geo, s->f32);
    cudaEvent_t a, b;
    NWB_CU(cudaEventCreate(&a));
    NWB_CU(cudaEventCreate(&b));
    int bestv = s->variant;
    float bestt = 1e30f, t0 = 1e30f;
    for (int v = 0; v < nv; ++v) {
        nwb::StageConfig c{};
        cudaError_t e = nwb::launch_stage(s->N, s->geo, s->f32, v, nullptr, nullptr, &c);
        if (e != cudaSuccess) return fail(NWB_ECUDA, "variant %d set-up: %s", v, cudaGetErrorString(e));
        nwb::StageParams P = s->params(0, 0.0);
        P.a = 0.0;
        P.b = 0.0;
        P.u_out = s->u[s->cur ^ 1];
        for (int w = 0; w < 2; ++w) {
            e = nwb::launch_stage(s->N, s->geo, s->f32, v, &P, s->st, nullptr);
            if (e != cudaSuccess) return fail(NWB_ECUDA, "autotune launch: %s", cudaGetErrorString(e));
        }
        NWB_CU(cudaEventRecord(a, s->st));
        for (int r = 0; r < reps; ++r) {
            e = nwb::launch_stage(s->N, s->geo, s->f32, v, &P, s->st, nullptr);
            if (e != cudaSuccess) return fail(NWB_ECUDA, "autotune launch: %s", cudaGetErrorString(e));
        }
        NWB_CU(cudaEventRecord(b, s->st));
        NWB_CU(cudaEventSynchronize(b));
        float t = 0.f;
        NWB_CU(cudaEventElapsedTime(&t, a, b));
        t /= reps;
        s->launches += reps + 2;
        if (ms_out && v < ms_cap) ms_out[v] = t;
        if (v == 0) t0 = t;
        if (t < bestt) {
            bestt = t;
            bestv = v;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // the default shape unless another beats it by more than the timing noise
    if (t0 <= 1.01f * bestt) bestv = 0;
    if (best) *best = bestv;
    return nwb_solver_set_variant(s, bestv);
}

nwb_status nwb_time_steps(nwb_solver* s, double dt, int nsteps, int use_graph, float* ms) {
    if (!s || !ms || nsteps < 1) return fail(NWB_EINVAL, "nwb_time_steps: bad argument");
    if (use_graph) {
        nwb_status r = s->ensure_graphs(dt);
        if (r != NWB_OK) return r;
    }
    cudaEvent_t a, b;
    NWB_CU(cudaEventCreate(&a));
    NWB_CU(cudaEventCreate(&b));
    NWB_CU(cudaStreamSynchronize(s->st));
    NWB_CU(cudaEventRecord(a, s->st));
    nwb_status r = s->run_steps(dt, nsteps, use_graph != 0);
    NWB_CU(cudaEventRecord(b, s->st));
    NWB_CU(cudaEventSynchronize(b));
    NWB_CU(cudaEventElapsedTime(ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return r;
}

nwb_status nwb_time_stage_kernel(nwb_solver* s, double dt, int nstages, float* ms) {
    if (!s || !ms || nstages < 1) return fail(NWB_EINVAL, "nwb_time_stage_kernel: bad argument");
    cudaEvent_t a, b;
    NWB_CU(cudaEventCreate(&a));
    NWB_CU(cudaEventCreate(&b));
    NWB_CU(cudaStreamSynchronize(s->st));
    NWB_CU(cudaEventRecord(a, s->st));
    nwb_status r = NWB_OK;
    for (int i = 0; i < nstages && r == NWB_OK; ++i) r = s->launch_stage(i % 5, dt);
    NWB_CU(cudaEventRecord(b, s->st));
    NWB_CU(cudaEventSynchronize(b));
    float t = 0.f;
    NWB_CU(cudaEventElapsedTime(&t, a, b));
    *ms = t / nstages;
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return r;
}

}  // extern "C"
