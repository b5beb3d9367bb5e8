// stage_variants.h -- launch shapes of the fused stage kernel per N.
// Each entry X(KS, EPB, KSMEM, MINB, ALG): KS threads per node column, EPB
// elements per block, KSMEM = stage k in shared memory (1) or read it from L2
// after a prefetch (0), MINB = resident blocks the register allocator must
// allow, ALG = 0 for the SIMT tile (stage_kernel.cuh) or 1 for the FP64
// tensor-core tile (stage_mma.cuh: N = 8, FP64 only; such entries come last).
// Entry 0 is the default (the fastest on B200 in a sweep over 2-4 M-node box
// meshes, FP64 and FP32-bulk); the autotuner (nwb_solver_autotune) times them
// all for the axis-aligned geometry class on the caller's own mesh.
#pragma once

#define NWB_VARIANTS_2(X) X(2, 16, 1, 1, 0) X(2, 32, 0, 2, 0) X(1, 32, 0, 2, 0)
#define NWB_VARIANTS_3(X) X(1, 16, 0, 4, 0) X(3, 8, 1, 1, 0) X(3, 8, 0, 3, 0)
#define NWB_VARIANTS_4(X) X(1, 8, 0, 4, 0) X(2, 4, 1, 1, 0) X(2, 4, 0, 4, 0) X(4, 4, 0, 2, 0)
#define NWB_VARIANTS_5(X) X(1, 4, 0, 4, 0) X(1, 4, 1, 1, 0) X(5, 2, 0, 2, 0) X(1, 8, 0, 2, 0)
#define NWB_VARIANTS_6(X) X(2, 2, 0, 3, 0) X(2, 2, 1, 1, 0) X(3, 2, 0, 2, 0) X(6, 1, 0, 2, 0) X(2, 4, 0, 1, 0)
#define NWB_VARIANTS_7(X) X(1, 2, 0, 3, 0) X(1, 2, 1, 1, 0) X(7, 1, 0, 2, 0) X(1, 4, 0, 1, 0)
#define NWB_VARIANTS_8(X) X(2, 1, 0, 4, 0) X(2, 1, 1, 1, 0) X(4, 1, 0, 2, 0) X(8, 1, 0, 1, 0) X(1, 2, 0, 2, 0) X(2, 2, 0, 2, 0) X(2, 1, 0, 3, 1)
#define NWB_VARIANTS_9(X) X(3, 1, 0, 2, 0) X(1, 1, 1, 1, 0) X(1, 1, 0, 2, 0) X(9, 1, 0, 1, 0)
#define NWB_VARIANTS_10(X) X(2, 1, 0, 2, 0) X(1, 1, 1, 1, 0) X(1, 1, 0, 2, 0) X(5, 1, 0, 1, 0)
