// Kernel selection for one launch of T fused steps: the 128-bit streaming
// kernel for aligned single steps, the register wavefront kernel for
// TMA-aligned even T <= 6, the shared-memory wavefront kernel otherwise.
#pragma once

#include "rwave.cuh"
#include "stream.cuh"
#include "wave_launch.cuh"

namespace lbm {

// General-solver physics variants (lbm_params -> compile-time choices).
enum : int {
    VAR_MRT_SMAG_CLAMP = 0,
    VAR_MRT_SMAG = 1,
    VAR_MRT = 2,
    VAR_MRT_LID = 3,
    VAR_BGK = 4,
    VAR_MRT_MLP = 5,      // learned closure, ReLU network
    VAR_MRT_MLP_SILU = 6, // learned closure, SiLU network
};

template <class C> int launch_stream(WaveParams p, cudaStream_t s)
{
    if (!p.err)
        p.err = device_error_word();
    dim3 grid((p.W + 127) / 128, (p.H + 3) / 4);
    dim3 block(32, 4);
    return status(launch_pdl(stream_kernel<C>, grid, block, 0, s, p));
}

inline bool stream_ok(const WaveParams &p)
{
    auto a4 = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 3u) == 0; };
    bool ok = p.W % 4 == 0 && p.pitch % 4 == 0 && p.plane % 4 == 0 && aligned16(p.f_in) && aligned16(p.f_out) &&
              a4(p.mask) && p.mask_pitch % 4 == 0;
    if (p.ux)
        ok = ok && aligned16(p.ux) && aligned16(p.uy) && aligned16(p.rho);
    return ok;
}

// The learned closure runs in the register wavefront kernel only (1 <= T <= 4,
// TMA-aligned planes, x not periodic).  Ph: PhysMrtMlp or PhysMrtMlpSilu.
template <class Ph, class St> int launch_step_mlp(const WaveParams &p, int T, cudaStream_t s)
{
    if (!p.k.mlp || !rwave_ok<typename St::T>(p, T, MODE_GENERAL, true))
        return LBM_ERR_UNSUPPORTED;
    switch (T) {
    case 1:
        return launch_rwave<RwCfg<1, 1, 1, Ph, St, MODE_GENERAL>>(p, s);
    case 2:
        return launch_rwave<RwCfg<2, 1, 1, Ph, St, MODE_GENERAL>>(p, s);
    case 3:
        return launch_rwave<RwCfg<3, 1, 2, Ph, St, MODE_GENERAL>>(p, s);
    case 4:
        return launch_rwave<RwCfg<4, 1, 2, Ph, St, MODE_GENERAL>>(p, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

// Tuning of the T = 2 register wavefront (build-time, for experiments): the
// resident warps per SM its registers are sized for (0: the RwCfg default), the
// row lag between its two time levels and its TMA prefetch distance.  Measured
// on the 4096 x 1024 cylinder (FP32, GLUPS): 16 warps 112, 14 warps 113, 12
// warps 102; lag 2 at 12 / 14 warps 97 / 65; prefetch 2 rows at 16 / 14 warps
// 106 / 106, 3 rows at 12 warps 107: the defaults (16 warps, lag 1, one row
// ahead) are the fastest.
#ifndef LBM_RW2_MINB
#define LBM_RW2_MINB 0
#endif
#ifndef LBM_RW2_LAG
#define LBM_RW2_LAG 1
#endif
#ifndef LBM_RW2_P
#define LBM_RW2_P 1 // rows of TMA prefetch ahead of the row being consumed
#endif

template <class Ph, class St, int MODE, bool LID = false>
int launch_step(const WaveParams &p, int T, cudaStream_t s)
{
    if (T == 1 && stream_ok(p))
        return launch_stream<StreamCfg<Ph, St, MODE, LID>>(p, s);
    if (T >= 2 && rwave_ok<typename St::T>(p, T, MODE)) {
        switch (T) {
        case 2:
            return launch_rwave<RwCfg<2, 1, LBM_RW2_P, Ph, St, MODE, LID, true, LBM_RW2_MINB, LBM_RW2_LAG>>(p, s);
        case 3:
            return launch_rwave<RwCfg<3, 1, 2, Ph, St, MODE, LID, true>>(p, s);
        case 4:
            return launch_rwave<RwCfg<4, 1, 2, Ph, St, MODE, LID, false>>(p, s);
        case 5:
            return launch_rwave<RwCfg<5, 1, 2, Ph, St, MODE, LID, false>>(p, s);
        default:
            return launch_rwave<RwCfg<6, 1, 2, Ph, St, MODE, LID, false>>(p, s);
        }
    }
    switch (T) {
    case 1:
        return launch_wave<WaveCfg<1, 224, Ph, St, MODE, LID>>(p, s);
    case 2:
        return launch_wave<WaveCfg<2, 128, Ph, St, MODE, LID>>(p, s);
    case 3:
        return launch_wave<WaveCfg<3, 128, Ph, St, MODE, LID>>(p, s);
    case 4:
        return launch_wave<WaveCfg<4, 128, Ph, St, MODE, LID>>(p, s);
    case 5:
        return launch_wave<WaveCfg<5, 128, Ph, St, MODE, LID>>(p, s);
    case 6:
        return launch_wave<WaveCfg<6, 128, Ph, St, MODE, LID>>(p, s);
    case 7:
        return launch_wave<WaveCfg<7, 128, Ph, St, MODE, LID>>(p, s);
    case 8:
        return launch_wave<WaveCfg<8, 128, Ph, St, MODE, LID>>(p, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

// Defined in general_*.cu (one translation unit per storage format; the learned
// closure in general_mlp.cu (ReLU) and general_mlp_silu.cu).
int general_launch_mlp(int storage, const WaveParams &p, int T, cudaStream_t s);
int general_launch_mlp_silu(int storage, const WaveParams &p, int T, cudaStream_t s);
int general_launch_f32(int variant, const WaveParams &p, int T, cudaStream_t s);
int general_launch_f16(int variant, const WaveParams &p, int T, cudaStream_t s);
int general_launch_bf16(int variant, const WaveParams &p, int T, cudaStream_t s);

} // namespace lbm
