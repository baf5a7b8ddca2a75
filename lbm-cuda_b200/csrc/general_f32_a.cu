// General-solver kernels, FP32 storage: MRT + Smagorinsky variants.
#include "dispatch.cuh"

namespace lbm {

int general_launch_f32_mrt_smag(int variant, const WaveParams &p, int T, cudaStream_t s)
{
    if (variant == VAR_MRT_SMAG_CLAMP)
        return launch_step<PhysMrtSmagClamp, StoreF32, MODE_GENERAL>(p, T, s);
    return launch_step<PhysMrtSmag, StoreF32, MODE_GENERAL>(p, T, s);
}

} // namespace lbm
