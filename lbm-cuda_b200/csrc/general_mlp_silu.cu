// General-solver kernels with the learned closure (MRT + MLP eddy viscosity),
// SiLU network, every storage format.
#include "dispatch.cuh"

namespace lbm {

int general_launch_mlp_silu(int storage, const WaveParams &p, int T, cudaStream_t s)
{
    switch (storage) {
    case LBM_STORE_F32:
        return launch_step_mlp<PhysMrtMlpSilu, StoreF32>(p, T, s);
    case LBM_STORE_F16DEV:
        return launch_step_mlp<PhysMrtMlpSilu, StoreF16Dev>(p, T, s);
    case LBM_STORE_BF16DEV:
        return launch_step_mlp<PhysMrtMlpSilu, StoreBF16Dev>(p, T, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

} // namespace lbm
