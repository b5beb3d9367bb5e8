/*
 * nwb.h -- C ABI of libnwb, the B200-native (sm_100a) DG-SEM Maxwell right-hand
 * side and LSRK45 time step of NekWave.
 *
 * The library is a drop-in for the reference's DgSolver (src/dg_solver.hpp:35-102)
 * and the single-rank kernel launchers behind it (src/device/dg_kernels.hpp:13-88):
 * it takes the same mesh arrays DgSolver::initialize reads from Mesh
 * (src/dg_solver.cpp:40-241), the same SoA state [Ex,Ey,Ez,Hx,Hy,Hz][npts], and
 * advances it with the same method.  Signatures use plain pointers and sizes only.
 *
 * Errors: every entry point returns an nwb_status.  nwb_last_error() gives a
 * thread-local message for the last failure on the calling thread.  The
 * reference aborts on any CUDA error (src/device/gpu_runtime.hpp:146-153); the
 * DgSolver shim in nekwave_b200/ref_shim/ keeps that behaviour on top of these
 * status codes.
 *
 * Terms: N is the number of GLL points per direction (the reference's Mesh::getN,
 * polynomial degree N-1); nelt the number of hexahedral elements; npts = nelt*N^3;
 * nfp = 6*N*N*nelt face points.
 */
#ifndef NWB_H
#define NWB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NWB_VERSION 1

typedef enum nwb_status {
    NWB_OK = 0,
    NWB_EINVAL = 1,      /* bad argument, size mismatch, unsupported mesh        */
    NWB_ENOMEM = 2,      /* device or host allocation failed                      */
    NWB_ECUDA = 3,       /* a CUDA runtime call failed                            */
    NWB_ETIMEOUT = 4,    /* a bounded device wait gave up                         */
    NWB_ENONFINITE = 5,  /* the state holds NaN or Inf                            */
    NWB_EBUSY = 6,       /* admission refused: over the memory budget / no slot   */
    NWB_ENOTFOUND = 7    /* unknown request or instance id                        */
} nwb_status;

typedef enum nwb_precision {
    NWB_FP64 = 0,        /* all arithmetic in FP64 (the reference's precision)     */
    NWB_FP32_BULK = 1    /* volume and flux arithmetic in FP32; solution, LSRK      */
                         /* register, geometry, inverse mass and energy in FP64    */
} nwb_precision;

/* Mesh arrays exactly as the reference's DgSolver::initialize consumes them
 * (src/dg_solver.cpp:76-112, 141-205).  All pointers are host pointers and are
 * only read during nwb_solver_create.  Face points must be in the reference's
 * canonical order: element-major, faces 0..5, then q, then p
 * (Mesh::setupFaceData, src/mesh.cpp:985-1080) -- the order createBoxMesh
 * produces; vol_idx_minus[fp] must equal Mesh::getFaceNodeVolIndex(e,f,p,q)
 * (src/mesh.cpp:955-981). */
typedef struct nwb_mesh_desc {
    int N;                        /* GLL points per direction, 2..10               */
    int nelt;                     /* number of elements                            */
    const double* D;              /* [N*N] column-major, Mesh::getD                */
    const double* w3;             /* [N^3] Mesh::getW3                             */
    const double* jac;            /* [npts] Mesh::getJac                           */
    const double* met[9];         /* [npts] each: rx,sx,tx,ry,sy,ty,rz,sz,tz       */
    const int* vol_idx_minus;     /* [nfp] FacePointData::volIdxMinus              */
    const int* vol_idx_plus;      /* [nfp] FacePointData::volIdxPlus (-1: none)    */
    const int* bc_type;           /* [nfp] 0 interior/periodic, 1 PEC, 2 PMC       */
                                  /* (nonzero is a PEC mirror, as the reference's */
                                  /* flux kernel does, src/device/dg_kernels.cu:244; */
                                  /* nwb_solver_create_ex can make 2 a PMC mirror) */
    const double* nx;             /* [nfp] outward unit normal                     */
    const double* ny;
    const double* nz;
    const double* dA;             /* [nfp] surface metric J_face w_p w_q           */
} nwb_mesh_desc;

typedef struct nwb_solver nwb_solver;
typedef struct nwb_box_mesh nwb_box_mesh;

/* ---- errors / version ------------------------------------------------------ */
const char* nwb_last_error(void);
const char* nwb_status_string(nwb_status s);
int nwb_version(void);
/* Makes device the current CUDA device of libnwb's own runtime for the calling
 * thread (libnwb links the CUDA runtime statically).  The reference picks the
 * device in Comm::init (src/comm.cpp:35-47); the DgSolver shim forwards it. */
nwb_status nwb_set_device(int device);

/* ---- box mesh builder ---------------------------------------------------------
 * Replaces Mesh::createBoxMesh (src/mesh.cpp:683-843) with its geometry
 * (src/mesh.cpp:188-314) and face data (src/mesh.cpp:985-1080), built with
 * structural O(faces*N^2) connectivity instead of coordinate matching.
 * periodic_mask: bit 0 = x, bit 1 = y, bit 2 = z.  The mesh owns host arrays
 * that nwb_box_mesh_desc exposes through an nwb_mesh_desc. */
nwb_status nwb_box_mesh_create(int N, int nelx, int nely, int nelz,
                               double xmin, double xmax, double ymin, double ymax,
                               double zmin, double zmax, int periodic_mask,
                               nwb_box_mesh** out);
nwb_status nwb_box_mesh_desc(const nwb_box_mesh* m, nwb_mesh_desc* out);
/* Node coordinates [npts] each (Mesh::getCoordX/Y/Z) and GLL nodes/weights [N]. */
nwb_status nwb_box_mesh_coords(const nwb_box_mesh* m, const double** x,
                               const double** y, const double** z);
nwb_status nwb_box_mesh_gll(const nwb_box_mesh* m, const double** z, const double** w);
/* Smallest GLL node spacing, Mesh::computeMinNodeDistance (src/mesh.cpp:883-930). */
nwb_status nwb_box_mesh_dxmin(const nwb_box_mesh* m, double* dxmin);
void nwb_box_mesh_destroy(nwb_box_mesh* m);
/* ProbeManager::init (src/probe.cpp:33-96) on the box mesh of these parameters,
 * on the host: for probe q at xyz[3q..3q+2], elem[q] = the first element whose box
 * is nearest (reference coordinates clamped to [-1,1]) and weights[(3q+a)*N + i]
 * the 1-D Lagrange weights along axis a (r, s, t); the tensor weight of node
 * (i,j,k) is w_r[i] w_s[j] w_t[k], the reference's interpWeights.  This is how
 * nwb_pool_add_box places its probes. */
nwb_status nwb_box_probes(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                          double ymin, double ymax, double zmin, double zmax, int nprobes,
                          const double* xyz, int* elem, double* weights);

/* ---- single-mesh solver: DgSolver (src/dg_solver.hpp:35-102) -----------------
 * nwb_solver_create     <- DgSolver::initialize(mesh, c0)   (src/dg_solver.cpp:40)
 * nwb_upload_state      <- DgSolver::uploadState            (src/dg_solver.cpp:243)
 * nwb_download_state    <- DgSolver::downloadState          (src/dg_solver.cpp:264)
 * nwb_step              <- DgSolver::step, nsteps times     (src/dg_solver.cpp:306)
 * nwb_solver_destroy    <- DgSolver::finalize               (src/dg_solver.cpp:529)
 * c0 = 0 central flux, 1 upwind (src/device/dg_kernels.cu:206-212).
 * The solver runs on the current CUDA device, on its own stream. */
nwb_status nwb_solver_create(const nwb_mesh_desc* mesh, double c0,
                             nwb_precision precision, nwb_solver** out);
/* nwb_solver_create with option flags (0: the same solver).  No counterpart in the
 * reference, which mirrors PMC/SYM faces (bc_type 2) as PEC walls
 * (src/dg_solver.cpp:92-98, src/device/dg_kernels.cu:243-251).
 * NWB_SOLVER_TRUE_PMC: bc_type 2 face points become true PMC mirrors,
 * [[E]] = 0 and [[H]] = -2 H^-, in the numerical flux; bc_type 1 and
 * neighbourless points stay PEC mirrors.  Without it (the default, parity mode)
 * the solver reproduces the reference. */
#define NWB_SOLVER_TRUE_PMC 1u
nwb_status nwb_solver_create_ex(const nwb_mesh_desc* mesh, double c0,
                                nwb_precision precision, unsigned flags, nwb_solver** out);
/* Solver on a box mesh built inside the library: the geometry of
 * Mesh::createBoxMesh (src/mesh.cpp:683-843) computed per element from the box
 * parameters, without per-node host arrays (large boxes need no host memory
 * beyond the state).  periodic_mask as in nwb_box_mesh_create. */
nwb_status nwb_solver_create_box(int N, int nelx, int nely, int nelz, double xmin, double xmax,
                                 double ymin, double ymax, double zmin, double zmax,
                                 int periodic_mask, double c0, nwb_precision precision,
                                 nwb_solver** out);
/* Device-generated initial state of a box solver: component c is
 * pulse[5c] * exp(-|x - (pulse[5c+1..5c+3])|^2 / pulse[5c+4]^2), 0 where
 * pulse[5c+4] <= 0. */
nwb_status nwb_solver_init_pulse(nwb_solver* s, const double* pulse /* [30] */);
/* n must be 6*npts (the reference asserts the same, src/dg_solver.cpp:244). */
nwb_status nwb_upload_state(nwb_solver* s, const double* host_state, size_t n);
nwb_status nwb_download_state(nwb_solver* s, double* host_state, size_t n);
/* Part of DgSolver::downloadState (src/dg_solver.cpp:264-283): nodes
 * [first, first+count) of all six components into their places of the
 * 6*npts-double host state (n = 6*npts); the rest of host_state is left as it
 * is.  For a front end that needs only some elements every step (the probe
 * elements of ProbeManager::record, src/probe.cpp:192-216) instead of the full
 * per-step download of Case::simulate (src/case.cpp:588).  Synchronous. */
nwb_status nwb_download_nodes(nwb_solver* s, long long first, long long count, double* host_state,
                              size_t n);
/* Enqueues nsteps LSRK45 steps of size dt on the solver's stream and returns
 * without waiting (the reference's step blocks; nwb_sync restores that). */
nwb_status nwb_step(nwb_solver* s, double dt, int nsteps);
nwb_status nwb_sync(nwb_solver* s);
/* Right-hand side M^{-1}(K u + F*) of the current state into host memory [6*npts]:
 * the quantity the reference's kernels leave in d_rhs_ before the LSRK update
 * (src/dg_solver.cpp:487).  Does not change the state. */
nwb_status nwb_eval_rhs(nwb_solver* s, double* host_rhs, size_t n);
/* Discrete energy 1/2 sum J w_i w_j w_k (|E|^2+|H|^2) of the current state,
 * FP64, on the device (src/case.cpp:733-766).  Returns NWB_ENONFINITE (and the
 * non-finite energy) when the state holds NaN/Inf. */
nwb_status nwb_energy(nwb_solver* s, double* energy);
/* Largest |E| and |H| over the nodes of the current state, on the device:
 * Case::getMaxE / Case::getMaxH (src/case.cpp:768-794), which the reference
 * computes on the host from a full download every output step.  Same roundings
 * as the host loop (no contraction, correctly rounded sqrt), so the values are
 * equal bit for bit; NaN nodes are passed over as the host's comparison does.
 * Synchronous; NWB_ENONFINITE when a maximum is infinite. */
nwb_status nwb_max_norms(nwb_solver* s, double* max_e, double* max_h);
/* Point probes on the device: ProbeManager::init's data (src/probe.cpp:33-96) --
 * per probe the first node of its element (e*N^3) and its N^3 tensor Lagrange
 * weights -- replace any earlier set; nprobes = 0 removes them. */
nwb_status nwb_probe_setup(nwb_solver* s, int nprobes, const long long* node_offset,
                           const double* weights /* [nprobes][N^3] */);
/* ProbeManager::record (src/probe.cpp:192-216) on the current state, on the
 * device, with the reference's summation order and roundings: out[p*6 + c] for
 * c = Ex, Ey, Ez, Hx, Hy, Hz.  Synchronous; the reference computes these on the
 * host from a full download of the state every step (src/case.cpp:588-600). */
nwb_status nwb_probe_read(nwb_solver* s, double* out);
/* Asynchronous snapshot of the current state into host memory (6*npts doubles, in
 * the reference's [6][npts] layout; pinned memory lets the copy overlap later
 * steps).  The state is first copied on the device in stream order, after every
 * step already queued, so steps queued afterwards may run while the host copy is
 * in flight; nwb_snapshot_wait returns when the host buffer is complete.  One
 * snapshot is in flight at a time (a second begin waits for the first).  Replaces
 * the synchronous per-step download of Case::simulate (src/case.cpp:588) where
 * the caller only needs the state at save steps. */
nwb_status nwb_snapshot_begin(nwb_solver* s, double* host, size_t n);
nwb_status nwb_snapshot_wait(nwb_solver* s);
/* Asynchronous upload, the reverse of the snapshot: replaces DgSolver::uploadState
 * (src/dg_solver.cpp:243-262) where the caller streams states in.  The host state
 * (6*npts doubles, [6][npts]; pinned memory lets the copy overlap) is copied on an
 * upload stream into a device staging buffer while the steps already queued run,
 * then, in the solver's stream order, into the current state: steps queued after
 * this call start from it.  The host buffer must stay unchanged until
 * nwb_upload_wait returns.  A second begin reuses the staging buffer once the
 * first upload has been copied out of it (on the device, without a host wait).
 * With nwb_snapshot_begin this pipelines upload, step and download of successive
 * states: the host link carries one state in and one out while the GPU steps. */
nwb_status nwb_upload_begin(nwb_solver* s, const double* host, size_t n);
nwb_status nwb_upload_wait(nwb_solver* s);
nwb_status nwb_solver_destroy(nwb_solver* s);

/* Introspection used by tests and the benchmark. */
typedef struct nwb_solver_info {
    int N, nelt;
    long long npts, stride;       /* component stride of the device state          */
    int geometry;                 /* 0 axis-aligned affine, 1 affine, 2 per-node   */
    int precision;
    int ks, epb;                  /* threads per node column, elements per block   */
    int threads_per_block;
    int smem_bytes;
    long long device_bytes;       /* device memory the solver holds                */
    int ksmem;                    /* 1: LSRK register staged in shared memory      */
    int minb;                     /* resident blocks the launch shape asks for     */
    int variant;                  /* current launch shape                          */
    int variant_count;            /* launch shapes available for this mesh         */
    int structured[3];            /* elements per axis when the connections are those
                                     of a structured box (x fastest, faces meeting
                                     without rotation; neighbours then follow from
                                     the element index), else 0                     */
    int periodic_mask;            /* structured box: periodic axes, bit 0 x .. 2 z  */
} nwb_solver_info;
nwb_status nwb_solver_get_info(const nwb_solver* s, nwb_solver_info* info);
/* Energy of a device-resident state without allocating device memory.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc: a
 * server that admits work against a fixed HBM budget, a host framework whose own
 * allocator owns all device memory, or a loop where cudaMalloc's implicit device
 * synchronisation is not acceptable.  Same quantity as nwb_energy, on any state
 * laid out as [6][stride] doubles (d_state), with J per element (jac_per_node = 0,
 * d_jac[nelt]) or per node (jac_per_node = 1, d_jac[nelt*N^3]) and w3[N^3], all
 * device pointers; the energy is written to the device double d_energy, on
 * stream (a cudaStream_t, 0 = default stream), without waiting.
 * Scratch: a fixed array of NWB_ENERGY_NOALLOC_MAX_ELEMENTS doubles (1 MiB) in
 * the library's device memory, present on every GPU that loads the library
 * until the process exits; meshes with more elements are refused with
 * NWB_EINVAL.  The first call on a device looks up that array's device address
 * (once per device, with the device current); make that first call before any
 * stream capture.  All calls share the array: calls that overlap on the GPU race
 * and must be ordered by the caller.  Every pointer must be device (or managed)
 * memory of the current device (nwb_set_device), and stream a stream of that
 * device; a pointer of another device or of the host is refused with NWB_EINVAL. */
#define NWB_ENERGY_NOALLOC_MAX_ELEMENTS 131072
nwb_status nwb_energy_noalloc(const double* d_state, long long stride, int N, int nelt,
                              const double* d_jac, int jac_per_node, const double* d_w3,
                              double* d_energy, void* stream);

/* Launch shape of the fused stage kernel.  nwb_solver_autotune times every
 * shape for this mesh (reps launches each, with a = b = dt = 0 so the state is
 * left as it was) and keeps the fastest, or the default shape (variant 0) when
 * it is within 1% of the fastest (timing noise); ms_out (optional, ms_cap entries)
 * receives the per-shape average launch time.  Neither call has a counterpart
 * in the reference, which has one fixed launch shape per kernel. */
nwb_status nwb_solver_set_variant(nwb_solver* s, int variant);
nwb_status nwb_solver_autotune(nwb_solver* s, int reps, int* best, float* ms_out, int ms_cap);
/* Device pointer of the current state ([6][stride] doubles) and the solver's
 * CUDA stream (a cudaStream_t), for callers that keep data on the device. */
nwb_status nwb_solver_device_state(nwb_solver* s, double** d_state, void** stream);
/* Number of kernels the solver has launched since it was created. */
nwb_status nwb_solver_launch_count(const nwb_solver* s, long long* count);
/* Times nsteps steps on the device with CUDA events on the solver's stream;
 * *ms receives the elapsed device time.  use_graph replays CUDA graphs. */
nwb_status nwb_time_steps(nwb_solver* s, double dt, int nsteps, int use_graph, float* ms);
/* Per-stage-kernel average device time over nstages stage launches (ms). */
nwb_status nwb_time_stage_kernel(nwb_solver* s, double dt, int nstages, float* ms);

/* ---- cavity pool: many independent cavities resident on one GPU ----------------
 * No counterpart in the reference, which solves one mesh per process
 * (Case::simulate, src/case.cpp:529-660).  A pool owns a fixed HBM arena of
 * hbm_budget_bytes, allocated once at creation; every cavity ("slot") is
 * sub-allocated from it, so nwb_pool_add never calls cudaMalloc and returns
 * NWB_EBUSY when the cavity does not fit (admission by HBM budget).  Outside the
 * arena the pool holds its slot table and two work lists (sized at creation for
 * any admissible set of cavities: 16 bytes each per 18 KB of budget at most) and
 * a pinned host staging area (2 x 48 MB).  nwb_pool_add, _add_box, _init_pulse,
 * _upload (states up to 48 MB), _remove and _step queue their device work in
 * stream order and return without waiting for the steps already in flight.
 * nwb_pool_step advances every uploaded, unfinished slot by up to nsteps steps
 * with one launch per LSRK stage and N present (or one persistent launch for
 * every N, nwb_pool_set_mode), replayed from one CUDA graph per step; a slot stops
 * by itself after its own nsteps.  Slots take axis-aligned box meshes (nwb_mesh_desc as above),
 * their own c0 and dt, up to 8 probes given as (element, tensor Lagrange
 * weights [3][N]) as ProbeManager builds them (src/probe.cpp:33-189), and record
 * the energy every energy_every steps (index 0 = initial state, NaN where not
 * recorded) and all six probe components every step.  Each slot's arithmetic is
 * the single-mesh stage kernel's, independent of the other slots. */
typedef struct nwb_pool nwb_pool;
nwb_status nwb_pool_create(size_t hbm_budget_bytes, int max_slots, nwb_precision precision,
                           nwb_pool** out);
nwb_status nwb_pool_add(nwb_pool* p, const nwb_mesh_desc* mesh, double c0, double dt, int nsteps,
                        int nprobes, const int* probe_elem, const double* probe_w,
                        int energy_every, int* slot);
/* Box cavity built inside the library: the geometry of Mesh::createBoxMesh
 * (src/mesh.cpp:683-843) computed per element from the box parameters (no
 * per-node arrays on the host), probes given as physical points located as
 * ProbeManager::init does (src/probe.cpp:33-96). */
nwb_status nwb_pool_add_box(nwb_pool* p, int N, int nelx, int nely, int nelz, double xmin,
                            double xmax, double ymin, double ymax, double zmin, double zmax,
                            int periodic_mask, double c0, double dt, int nsteps, int nprobes,
                            const double* probe_xyz, int energy_every, int* slot);
/* Initial state of a box cavity generated on the device: component c is
 * pulse[5c] * exp(-|x - (pulse[5c+1], pulse[5c+2], pulse[5c+3])|^2 / pulse[5c+4]^2)
 * (0 where pulse[5c+4] <= 0).  Like nwb_pool_upload, it starts the slot. */
nwb_status nwb_pool_init_pulse(nwb_pool* p, int slot, const double* pulse /* [30] */);
/* Initial state [6*npts]; the slot starts stepping with the next nwb_pool_step. */
nwb_status nwb_pool_upload(nwb_pool* p, int slot, const double* host_state, size_t n);
nwb_status nwb_pool_step(nwb_pool* p, int nsteps);      /* asynchronous */
nwb_status nwb_pool_sync(nwb_pool* p);
/* status[s]: -1 free, 0 added (no state yet), 1 running, 2 finished; done[s]:
 * steps taken.  Synchronises the pool's stream. */
nwb_status nwb_pool_query(nwb_pool* p, int* status, int* done, int cap);
/* Any of state [6*npts], energy [nsteps+1], probes [(nsteps+1)*nprobes*6] may be NULL. */
nwb_status nwb_pool_results(nwb_pool* p, int slot, double* state, double* energy, double* probes);
/* The same status without waiting for the steps in flight: nwb_pool_query_begin
 * queues a copy of the device slot table after everything queued so far and
 * returns; nwb_pool_query_end waits for that copy only (later steps keep
 * running) and reports the status as of that point, as nwb_pool_query does.
 * Slots admitted after the begin are reported as not yet started (0) or running
 * (1).  One snapshot is in flight at a time.  No counterpart in the reference. */
nwb_status nwb_pool_query_begin(nwb_pool* p);
nwb_status nwb_pool_query_end(nwb_pool* p, int* status, int* done, int cap);
/* nwb_pool_results without waiting: queues the copies of a slot that the last
 * nwb_pool_query_end reported finished and returns.  The buffers (pinned host
 * memory for the copies to be asynchronous) are complete when a later
 * nwb_pool_query_end or nwb_pool_sync returns; the slot may be removed at once
 * (its memory is reused only by work queued after the copies). */
nwb_status nwb_pool_results_async(nwb_pool* p, int slot, double* state, double* energy,
                                  double* probes);
nwb_status nwb_pool_remove(nwb_pool* p, int slot);
nwb_status nwb_pool_info(const nwb_pool* p, size_t* used_bytes, size_t* budget_bytes,
                         int* slots_used, long long* launches);
/* Stage launch mode: 0 = one persistent launch per stage for every N (tiles
 * handed out by an atomic counter, largest first), 1 = one launch per N present,
 * each with that N's tuned single-mesh launch shape, as parallel branches of the
 * step graph (the default of a new pool).  nwb_pool_autotune times both on the resident cavities (timing
 * launches with a = b = dt = 0 leave every state as it is) and keeps the faster;
 * ms_out (optional) receives the two per-step stage times. */
nwb_status nwb_pool_set_mode(nwb_pool* p, int mode);
nwb_status nwb_pool_autotune(nwb_pool* p, int reps, int* best_mode, float* ms_out);
/* Device time (ms, CUDA events on the pool's stream) of nsteps pool steps. */
nwb_status nwb_pool_time_steps(nwb_pool* p, int nsteps, float* ms);
nwb_status nwb_pool_destroy(nwb_pool* p);

#ifdef __cplusplus
}
#endif
#endif /* NWB_H */
