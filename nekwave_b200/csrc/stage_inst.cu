// stage_inst.cu -- instantiations of the fused stage kernel for one N.
// Compiled once per N (2..10) with -DNWB_N=<N> so the objects build in parallel.
#include "stage_kernel.cuh"
#include "stage_mma.cuh"
#include "stage_pipe.cuh"
#include "stage_dmma.cuh"
#include "stage_bulk.cuh"
#include "stage_variants.h"

#ifndef NWB_N
#error "compile with -DNWB_N=<points per direction>"
#endif

#define NWB_CAT2(a, b) a##b
#define NWB_CAT(a, b) NWB_CAT2(a, b)
#define NWB_VLIST NWB_CAT(NWB_VARIANTS_, NWB_N)

namespace nwb {
namespace stage {
// Everything below depends on NWB_N and differs between the per-N objects, so
// it must have internal linkage (one-definition rule across the objects).
namespace {

struct Shape {
    int ks, epb, ksm, minb, alg;
};
#define NWB_X(ks, epb, ksm, minb, alg) Shape{ks, epb, ksm, minb, alg},
constexpr Shape kShapes[] = {NWB_VLIST(NWB_X)};
#undef NWB_X
constexpr int kNumShapes = static_cast<int>(sizeof(kShapes) / sizeof(Shape));
// FP64 tensor-core shapes and the bulk-copy form: axis-aligned class, FP64 only
constexpr bool fp64_only(int alg) {
    return alg == 1 || alg == 200 || alg == 201 || alg == 211 || alg == 212 || alg >= 1000;
}
constexpr int count_simt() {
    int n = 0;
    for (int i = 0; i < kNumShapes; ++i) n += !fp64_only(kShapes[i].alg);
    return n;
}
constexpr int kNumSimt = count_simt();  // every shape but the FP64-only ones
// Shape index of variant v among the shapes that are not FP64-only.
constexpr int nth_general(int v) {
    int c = 0;
    for (int i = 0; i < kNumShapes; ++i)
        if (!fp64_only(kShapes[i].alg)) {
            if (c == v) return i;
            ++c;
        }
    return -1;
}
constexpr int kFirstGeneral = nth_general(0);
// Variant numbers: the axis-aligned class in FP64 has every shape in list order;
// the axis-aligned class in FP32-bulk has the shapes that are not FP64-only, in
// order; the other classes have one variant, the first such shape.
inline int shape_index(int geo, int f32, int variant) {
    return (geo == GEO_BOX && !f32) ? variant : nth_general(variant);
}

// vid: shape index (shape_index)
template <int GEO, bool F32, int I>
cudaError_t launch_variant(int vid, const StageParams* p, cudaStream_t st, StageConfig* cfg) {
    if constexpr (I < kNumShapes) {
        if (vid == I) {
            constexpr Shape v = kShapes[I];
            if constexpr (v.alg == 1) {
                if constexpr (GEO == GEO_BOX && !F32 && NWB_N == 8)
                    return launch_mma8<v.minb>(p, st, cfg);
                else
                    return cudaErrorInvalidValue;
            } else if constexpr (v.alg == 200 || v.alg == 201) {
                if constexpr (GEO == GEO_BOX && !F32 && NWB_N == 8)
                    return launch_dmma8<v.minb, v.alg - 199>(p, st, cfg);
                else
                    return cudaErrorInvalidValue;
            } else if constexpr (v.alg == 211 || v.alg == 212) {
                // two warps per field, each block pulling a later block's element into
                // L2 half (211) or one (212) wave of resident blocks ahead
                if constexpr (GEO == GEO_BOX && !F32 && NWB_N == 8)
                    return launch_dmma8<v.minb, 2, v.alg - 210>(p, st, cfg);
                else
                    return cudaErrorInvalidValue;
            } else if constexpr (v.alg >= 2 && v.alg <= 129) {
                static_assert(v.ksm == 0, "second family: k from L2");
                constexpr int fl = v.alg - 2;
                // the constant-bank D is an FP64 form; FP32-bulk runs the same shape without it
                constexpr bool cd = (fl & 8) != 0 && !F32;
                if constexpr (GEO == GEO_BOX || I == kFirstGeneral)
                    return launch2<NWB_N, GEO, F32, v.ks, v.epb, v.minb, (fl & 1) != 0, (fl & 2) != 0,
                                   (fl & 4) != 0, cd, (fl & 16) != 0, (fl & 32) != 0,
                                   (fl & 64) != 0>(p, st, cfg);
                else
                    return cudaErrorInvalidValue;
            } else if constexpr (v.alg >= 1000) {
                // the bulk-copy one-tile form (stage_bulk.cuh), second-family flags
                // ALG - 1000: 2 SPLIT (required), 8 CONSTD, 16 EARLY, 32 KSM, 64 DSMEM,
                // 1 ZCOL (z-column tile order on structured boxes), 4 VROW (16-byte row
                // loads), 128 ILP2 (two partial sums per derivative), 256 / 512 AHEAD
                // (the tile of a block half / one wave of resident blocks later pulled
                // into L2)
                constexpr int fl = v.alg - 1000;
                static_assert((fl & 2) != 0 && v.ks == 2 && fl < 1024 && (fl & 768) != 768, "the field split");
                if constexpr (GEO == GEO_BOX && !F32)
                    return launch_bulk<NWB_N, GEO, v.ks, v.epb, v.minb, (fl & 8) != 0, (fl & 64) != 0,
                                       (fl & 32) != 0, (fl & 16) != 0, (fl & 1) != 0, (fl & 4) != 0,
                                       (fl & 128) != 0, (fl & 512) ? 2 : ((fl & 256) ? 1 : 0)>(p, st, cfg);
                else
                    return cudaErrorInvalidValue;
            } else if constexpr (GEO == GEO_BOX || I == kFirstGeneral) {
                return launch_cfg<NWB_N, GEO, F32, v.ks, v.epb, (v.ksm != 0), v.minb>(p, st, cfg);
            } else {
                return cudaErrorInvalidValue;
            }
        }
        return launch_variant<GEO, F32, I + 1>(vid, p, st, cfg);
    } else {
        return cudaErrorInvalidValue;
    }
}

template <int GEO>
int count_variants(int f32) {
    return GEO == GEO_BOX ? (f32 ? kNumSimt : kNumShapes) : 1;
}

}  // namespace
}  // namespace stage

template <>
cudaError_t launch_stage_n<NWB_N>(int geo, int f32, int variant, const StageParams* p,
                                  cudaStream_t st, StageConfig* cfg) {
    using namespace stage;
    const int nv = geo == GEO_BOX ? count_variants<GEO_BOX>(f32) : 1;
    if (variant < 0 || variant >= nv) return cudaErrorInvalidValue;
    const int vid = shape_index(geo, f32, variant);
    switch (geo) {
        case GEO_BOX:
            return f32 ? launch_variant<GEO_BOX, true, 0>(vid, p, st, cfg)
                       : launch_variant<GEO_BOX, false, 0>(vid, p, st, cfg);
        case GEO_AFFINE:
            return f32 ? launch_variant<GEO_AFFINE, true, 0>(vid, p, st, cfg)
                       : launch_variant<GEO_AFFINE, false, 0>(vid, p, st, cfg);
        case GEO_NODAL:
            return f32 ? launch_variant<GEO_NODAL, true, 0>(vid, p, st, cfg)
                       : launch_variant<GEO_NODAL, false, 0>(vid, p, st, cfg);
        default:
            return cudaErrorInvalidValue;
    }
}

template <>
int stage_variant_count_n<NWB_N>(int geo, int f32) {
    switch (geo) {
        case GEO_BOX: return stage::count_variants<GEO_BOX>(f32);
        case GEO_AFFINE: return stage::count_variants<GEO_AFFINE>(f32);
        case GEO_NODAL: return stage::count_variants<GEO_NODAL>(f32);
        default: return 0;
    }
}

}  // namespace nwb
