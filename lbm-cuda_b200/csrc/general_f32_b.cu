// General-solver kernels, FP32 storage: plain MRT (with and without a moving
// wall) and BGK variants, and the FP32 dispatcher.
#include "dispatch.cuh"

namespace lbm {

int general_launch_f32_mrt_smag(int variant, const WaveParams &p, int T, cudaStream_t s);

int general_launch_f32(int variant, const WaveParams &p, int T, cudaStream_t s)
{
    switch (variant) {
    case VAR_MRT_SMAG_CLAMP:
    case VAR_MRT_SMAG:
        return general_launch_f32_mrt_smag(variant, p, T, s);
    case VAR_MRT:
        return launch_step<PhysMrt, StoreF32, MODE_GENERAL>(p, T, s);
    case VAR_MRT_LID:
        return launch_step<PhysMrt, StoreF32, MODE_GENERAL, true>(p, T, s);
    case VAR_BGK:
        return launch_step<PhysBgk, StoreF32, MODE_GENERAL>(p, T, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

} // namespace lbm
