// stage_variants.h -- launch shapes of the fused stage kernel per N.
// Each entry X(KS, EPB, KSMEM, MINB, ALG): KS threads per node column, EPB
// elements per block, KSMEM = stage k in shared memory (1) or read it from L2
// after a prefetch (0), MINB = resident blocks the register allocator must
// allow, ALG = 0 for the SIMT tile (stage_kernel.cuh), 1 for the FP64
// tensor-core tile (stage_mma.cuh: N = 8, FP64 only), 200 / 201 (one / two warps
// per field) for the field-split FP64 tensor-core tile (stage_dmma.cuh: N = 8,
// axis-aligned class, FP64 only), or 2 + flags for the second family (stage_pipe.cuh; KSMEM must be 0) with flags
// 1 = PIPE (persistent, double-buffered), 2 = SPLIT (residual split by field
// between the two threads of a column, KS = 2), 4 = PAD (row pitch N+1),
// 8 = CONSTD (with SPLIT: t-derivative coefficients from the parameter bank; FP64),
// 16 = EARLY (without PIPE: neighbour traces requested before the tile wait),
// 32 = FACEFIRST (without PIPE: the face phase from global memory before the wait),
// 64 = DSMEM (with SPLIT: D rows from shared memory, fewer registers).
// ALG >= 1000: the bulk-copy one-tile form (stage_bulk.cuh: FP64, axis-aligned class)
// with second-family flags ALG - 1000 (SPLIT required; CONSTD; 16 = EARLY; 32 = KSM, k
// staged in shared memory by the bulk copies; DSMEM; 1 = ZCOL, tiles in z-column
// order on structured boxes; 4 = VROW, the r-derivative's rows read with 16-byte
// loads; 128 = ILP2, two partial sums per derivative; 256 / 512 = AHEAD, each block
// pulls into L2 the tile of the block half / one wave of resident blocks after it)
// and MINB resident blocks.  ALG 211 / 212: the field-split FP64 tensor-core tile with
// two warps per field (as 201) and that L2 pull half / one wave ahead.
// Entry 0 is the default (the fastest FP64 shape on B200 in a sweep over 8 M-node
// box meshes; for 5, 6, 7 and 9 points the bulk-copy form with k in shared memory
// and the neighbour traces requested while the tile's copies fly: one element per
// block at 5 points, and at 6 and 9 points with the L2 pull half a wave ahead, at 9
// points in z-column tile order).
// Variant numbers skip the FP64-only entries for FP32-bulk and for the other
// geometry classes, whose default is the first entry that is not FP64-only and
// which have that one variant.  The autotuner (nwb_solver_autotune) times every
// variant of the axis-aligned class on the caller's own mesh.  The pool's per-N
// kernels (batch.cu NShape/BShape) use the same arithmetic as the default.
#pragma once

#define NWB_VARIANTS_2(X) X(2, 16, 1, 1, 0) X(2, 32, 0, 2, 0) X(1, 32, 0, 2, 0)
#define NWB_VARIANTS_3(X) X(1, 16, 0, 4, 0) X(3, 8, 1, 1, 0) X(3, 8, 0, 3, 0)
#define NWB_VARIANTS_4(X) X(2, 4, 0, 3, 13) X(2, 4, 0, 3, 5) X(1, 8, 0, 4, 0) X(2, 4, 1, 1, 0) X(2, 4, 0, 4, 0) X(4, 4, 0, 2, 0) X(2, 4, 0, 4, 4) X(2, 8, 0, 2, 4) X(2, 4, 0, 4, 12) X(2, 4, 0, 4, 20) X(2, 4, 0, 4, 28) X(2, 4, 0, 3, 1042) X(2, 4, 0, 3, 1058) X(2, 4, 0, 3, 1062)
#define NWB_VARIANTS_5(X) X(2, 1, 0, 8, 1058) X(2, 2, 0, 4, 1034) X(2, 2, 0, 5, 68) X(2, 2, 0, 4, 4) X(1, 4, 0, 4, 0) X(1, 4, 1, 1, 0) X(5, 2, 0, 2, 0) X(1, 8, 0, 2, 0) X(2, 4, 0, 2, 4) X(2, 2, 0, 4, 8) X(2, 2, 0, 4, 12) X(2, 2, 0, 5, 4) X(2, 2, 0, 4, 20) X(2, 2, 0, 4, 1050) X(2, 2, 0, 5, 1098) X(2, 2, 0, 4, 1035) X(2, 2, 0, 4, 1026) X(2, 2, 0, 5, 1058) X(2, 2, 0, 3, 1058) X(2, 2, 0, 4, 1058) X(2, 1, 0, 8, 1034) X(2, 2, 0, 4, 1062) X(2, 2, 0, 4, 1186) X(2, 1, 0, 8, 1314) X(2, 1, 0, 8, 1570)
#define NWB_VARIANTS_6(X) X(2, 2, 0, 3, 1314) X(2, 2, 0, 3, 1058) X(2, 2, 0, 3, 1042) X(2, 2, 0, 3, 4) X(2, 2, 0, 3, 0) X(2, 2, 1, 1, 0) X(3, 2, 0, 2, 0) X(6, 1, 0, 2, 0) X(2, 4, 0, 1, 0) X(6, 1, 0, 3, 3) X(2, 2, 0, 3, 8) X(2, 2, 0, 3, 5) X(2, 2, 0, 3, 9) X(2, 4, 0, 2, 4) X(2, 2, 0, 3, 12) X(2, 2, 0, 3, 16) X(2, 2, 0, 4, 4) X(2, 2, 0, 5, 4) X(2, 4, 0, 2, 12) X(2, 2, 0, 3, 20) X(2, 2, 0, 3, 28) X(2, 2, 0, 3, 36) X(2, 2, 0, 3, 44) X(2, 2, 0, 3, 1034) X(2, 2, 0, 3, 1059) X(2, 2, 0, 3, 1062) X(2, 2, 0, 3, 1186) X(2, 2, 0, 3, 1570) X(2, 2, 0, 3, 1315)
#define NWB_VARIANTS_7(X) X(2, 1, 0, 4, 1058) X(2, 1, 0, 4, 1042) X(2, 1, 0, 4, 12) X(2, 1, 0, 4, 4) X(1, 2, 0, 3, 0) X(1, 2, 1, 1, 0) X(7, 1, 0, 2, 0) X(1, 4, 0, 1, 0) X(2, 2, 0, 3, 4) X(2, 2, 0, 3, 8) X(2, 1, 0, 5, 4) X(2, 1, 0, 6, 4) X(2, 1, 0, 4, 20) X(2, 1, 0, 3, 1042) X(2, 1, 0, 4, 1059) X(2, 1, 0, 4, 1026) X(2, 1, 0, 4, 1062) X(2, 1, 0, 4, 1186) X(2, 1, 0, 4, 1314) X(2, 1, 0, 4, 1570)
#define NWB_VARIANTS_8(X) X(2, 1, 0, 4, 201) X(2, 1, 0, 4, 12) X(2, 1, 0, 4, 8) X(2, 1, 0, 4, 0) X(2, 1, 1, 1, 0) X(4, 1, 0, 2, 0) X(8, 1, 0, 1, 0) X(1, 2, 0, 2, 0) X(2, 2, 0, 2, 0) X(4, 1, 0, 2, 3) X(2, 1, 0, 4, 4) X(2, 1, 0, 3, 5) X(2, 1, 0, 3, 9) X(2, 1, 0, 4, 6) X(2, 1, 0, 4, 16) X(2, 1, 0, 4, 28) X(2, 1, 0, 4, 20) X(2, 1, 0, 4, 44) X(2, 1, 0, 4, 36) X(1, 1, 0, 5, 200) X(2, 1, 0, 3, 201) X(2, 1, 0, 3, 1) X(2, 1, 0, 3, 1042) X(2, 1, 0, 3, 1058) X(2, 1, 0, 3, 1062) X(2, 1, 0, 4, 211) X(2, 1, 0, 4, 212)
#define NWB_VARIANTS_9(X) X(2, 1, 0, 2, 1315) X(2, 1, 0, 2, 1059) X(2, 1, 0, 2, 1042) X(2, 1, 0, 2, 12) X(2, 1, 0, 2, 4) X(3, 1, 0, 2, 0) X(1, 1, 1, 1, 0) X(1, 1, 0, 2, 0) X(9, 1, 0, 1, 0) X(2, 1, 0, 3, 4) X(2, 1, 0, 3, 8) X(2, 1, 0, 3, 12) X(2, 1, 0, 2, 1034) X(2, 1, 0, 2, 1058) X(2, 1, 0, 2, 1026) X(2, 1, 0, 2, 1062) X(2, 1, 0, 2, 1186) X(2, 1, 0, 2, 1571) X(2, 1, 0, 2, 1314)
#define NWB_VARIANTS_10(X) X(2, 1, 0, 2, 0) X(1, 1, 1, 1, 0) X(1, 1, 0, 2, 0) X(5, 1, 0, 1, 0) X(2, 1, 0, 3, 4) X(2, 1, 0, 3, 8) X(2, 1, 0, 2, 4) X(2, 1, 0, 2, 12)
