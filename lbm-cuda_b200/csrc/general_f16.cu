// General-solver kernels, 16-bit deviation storage (StoreF16Dev): MRT variants.
#include "dispatch.cuh"

namespace lbm {

int general_launch_f16(int variant, const WaveParams &p, int T, cudaStream_t s)
{
    switch (variant) {
    case VAR_MRT_SMAG_CLAMP:
        return launch_step<PhysMrtSmagClamp, StoreF16Dev, MODE_GENERAL>(p, T, s);
    case VAR_MRT_SMAG:
        return launch_step<PhysMrtSmag, StoreF16Dev, MODE_GENERAL>(p, T, s);
    case VAR_MRT:
        return launch_step<PhysMrt, StoreF16Dev, MODE_GENERAL>(p, T, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

} // namespace lbm
