// batch.cuh -- device-side types of the multi-cavity pool (pool.cpp, batch.cu).
#pragma once

#include "nwb_internal.h"

namespace nwb {

constexpr int kBatchThreads = 128;  // block size of the persistent batch kernel
constexpr int kMaxProbes = 8;

// One resident cavity ("slot") as the device sees it.  All pointers are
// sub-allocations of the pool's HBM arena.
struct SlotDev {
    double* u[2];           // ping-pong state [6][stride]
    double* k;              // LSRK register [6][stride]
    const double* D;        // [N*N]
    const double* w3;       // [N^3]
    const ElemGeo* geo;     // [nelt]
    const int* conn;        // [6*nelt]
    double* partial;        // [ntiles] energy partial sums
    double* energy;         // [nsteps+1] energy history (index 0 = initial state)
    double* probes;         // [(nsteps+1) * nprobes * 6] probe history
    const int* probe_elem;  // [nprobes]
    const double* probe_w;  // [nprobes][3][N] tensor-product Lagrange weights
    long long stride;
    double c0, dt;
    double zl[10];          // line coordinates of D (nwb::line_coords)
    int N, nelt, ntiles, epb;
    int nprobes, energy_every;
    int nsteps;             // steps this cavity must take
    int done;               // steps taken
    int par;                // ping-pong parity at the start of the next step
    int active;             // 1 while done < nsteps
    int energy_now;         // set by the diagnostics when this step records energy
    int _pad;
};

// One tile of work: EPB consecutive elements of one slot.
struct WorkItem {
    int slot;
    int e0;
    int N;
    int tile;  // index of the tile within its slot (energy partial slot)
};

struct BatchShape {
    int ks, epb;
};

// Batch launchers (batch.cu).
// stage: 0..4.  counters[stage] is the dynamic tile counter of that stage.
// dry = 1 runs the stage with a = b = dt = 0 (timing only: u_out = u_in, k = 0).
cudaError_t launch_batch_stage(int f32, int stage, const SlotDev* slots, const WorkItem* work,
                               const int* ntiles, int* counters, int grid, int smem, int dry,
                               cudaStream_t st);
// Per-N mode: one block per tile of the given N (work points at that N's tiles,
// which must have been cut with batch_epb_n(N, f32) elements each).  Dh: that N's D on
// the host when every resident cavity of that N shares it (lets the kernel take D
// from its parameters), else null.
cudaError_t launch_batch_stage_n(int N, int f32, int stage, const SlotDev* slots,
                                 const WorkItem* work, int ntiles, int dry, const double* Dh,
                                 cudaStream_t st);
int batch_epb_n(int N, int f32);
// Diagnostics after a step (post = 1) or of the initial state (post = 0):
// energy partials per tile and probe values into the slots' history buffers.
// only_slot >= 0 restricts the work to one slot (initial-state diagnostics).
cudaError_t launch_batch_diag(SlotDev* slots, const WorkItem* work, const int* ntiles, int post,
                              int only_slot, int grid, cudaStream_t st);
// End of step: per-slot energy sum (fixed order), parity flip, step count,
// completion; resets the stage counters.
cudaError_t launch_batch_epilogue(SlotDev* slots, int nslots, int post, int only_slot,
                                  int* counters, cudaStream_t st);
// Gaussian pulses on the nodes of an axis-aligned box cavity: component c gets
// pulse[c*5+0] * exp(-|x - (pulse[c*5+1..3])|^2 / pulse[c*5+4]^2) (zero where
// pulse[c*5+4] <= 0), node positions from the box's uniform element grid.
struct BoxPulse {
    double lo[3], h[3];
    int nel[3];
    int N;
    double pulse[30];
    double z[10];  // GLL nodes
};
cudaError_t launch_box_pulse(const BoxPulse& b, double* u, long long stride, cudaStream_t st);

// Shape per N used by the batch kernel and its dynamic shared memory need.
BatchShape batch_shape(int N, int f32);
int batch_smem(int N, int f32);
cudaError_t batch_prepare(int f32, int smem);

}  // namespace nwb
