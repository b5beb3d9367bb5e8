// stage_dispatch.cu -- runtime dispatch of the fused stage kernel on N.
#include "nwb_internal.h"

namespace nwb {

cudaError_t launch_stage(int N, int geo, int f32, int variant, const StageParams* p,
                         cudaStream_t st, StageConfig* cfg) {
    switch (N) {
        case 2: return launch_stage_n<2>(geo, f32, variant, p, st, cfg);
        case 3: return launch_stage_n<3>(geo, f32, variant, p, st, cfg);
        case 4: return launch_stage_n<4>(geo, f32, variant, p, st, cfg);
        case 5: return launch_stage_n<5>(geo, f32, variant, p, st, cfg);
        case 6: return launch_stage_n<6>(geo, f32, variant, p, st, cfg);
        case 7: return launch_stage_n<7>(geo, f32, variant, p, st, cfg);
        case 8: return launch_stage_n<8>(geo, f32, variant, p, st, cfg);
        case 9: return launch_stage_n<9>(geo, f32, variant, p, st, cfg);
        case 10: return launch_stage_n<10>(geo, f32, variant, p, st, cfg);
        default: return cudaErrorInvalidValue;
    }
}

int stage_variant_count(int N, int geo, int f32) {
    switch (N) {
        case 2: return stage_variant_count_n<2>(geo, f32);
        case 3: return stage_variant_count_n<3>(geo, f32);
        case 4: return stage_variant_count_n<4>(geo, f32);
        case 5: return stage_variant_count_n<5>(geo, f32);
        case 6: return stage_variant_count_n<6>(geo, f32);
        case 7: return stage_variant_count_n<7>(geo, f32);
        case 8: return stage_variant_count_n<8>(geo, f32);
        case 9: return stage_variant_count_n<9>(geo, f32);
        case 10: return stage_variant_count_n<10>(geo, f32);
        default: return 0;
    }
}

}  // namespace nwb
