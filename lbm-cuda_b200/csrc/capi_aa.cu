// C-ABI drop-ins for the shared-memory AA kernels of the reference:
// lbm_core_smemaa.cu (lbm_smemaa_step) and lbm_core_smemaa_policy.cu /
// lbm_core_smemaa_endfused.cu (lbm_blocked_step).
#include <stdlib.h>
#include <string.h>

#include "aa_tile.cuh"
#include "host.h"

namespace lbm {

int *device_error_word();

template <class C> int launch_aa(AaParams p, cudaStream_t s)
{
    static int attr_done[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr_done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(aa_tile_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
        if (e != cudaSuccess)
            return status(e);
        attr_done[dev] = 1;
    }
    if (!p.err)
        p.err = device_error_word();
    CUtensorMap tmf, tmm;
    memset(&tmf, 0, sizeof(tmf));
    memset(&tmm, 0, sizeof(tmm));
    bool tma = p.use_tma && aligned16(p.f_in) && aligned16(p.mask) && (p.W % 16) == 0;
    if (tma)
        tma = make_map_planes(&tmf, p.f_in, 4, p.W, p.H, p.W, (long long)p.W * p.H, C::SW, C::SY) &&
              make_map_mask(&tmm, p.mask, p.W, p.H, p.W, C::MW, C::SY);
    p.use_tma = tma ? 1 : 0;
    dim3 grid((p.W + C::CX - 1) / C::CX, (p.H + C::CY - 1) / C::CY);
    aa_tile_kernel<C><<<grid, C::NT, C::SMEM, s>>>(p, tmf, tmm);
    return status(cudaGetLastError());
}

// Tile shapes: (SX, SY, threads, cells per batch, CTAs per SM).  Shape 0 is a
// 64 x 32 tile (less halo recomputation), shape 1 a 32 x 32 tile with more
// CTAs per SM (more warps to hide latency).
template <int VAR, int SHAPE> static int aa_dispatch_shape(const AaParams &p, int T, cudaStream_t s)
{
    constexpr int SX = SHAPE == 0 ? 64 : 32, SY = 32, NT = SHAPE == 0 ? 256 : 256, NB = SHAPE == 0 ? 4 : 2;
    constexpr int MB = SHAPE == 0 ? 2 : 3;
    switch (T) {
    case 2:
        return launch_aa<AaCfg<2, VAR, SX, SY, NT, NB, MB>>(p, s);
    case 4:
        return launch_aa<AaCfg<4, VAR, SX, SY, NT, NB, MB>>(p, s);
    case 6:
        return launch_aa<AaCfg<6, VAR, SX, SY, NT, NB, MB>>(p, s);
    case 8:
        return launch_aa<AaCfg<8, VAR, SX, 48, NT, NB, MB>>(p, s);
    default:
        return LBM_ERR_UNSUPPORTED;
    }
}

template <int VAR> static int aa_dispatch(const AaParams &p, int T, cudaStream_t s)
{
    static int shape = -1;
    if (shape < 0) {
        const char *e = getenv("LBM_AA_SHAPE"); // tuning override for experiments
        shape = (e && atoi(e) == 0) ? 0 : 1;
    }
    return shape == 0 ? aa_dispatch_shape<VAR, 0>(p, T, s) : aa_dispatch_shape<VAR, 1>(p, T, s);
}

static AaParams aa_params(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho,
                          int W, int H, float tau_inv, float u_in)
{
    AaParams p;
    memset(&p, 0, sizeof(p));
    p.f_in = f_now;
    p.f_out = f_out;
    p.mask = mask;
    p.ux = ux;
    p.uy = uy;
    p.rho = rho;
    p.W = W;
    p.H = H;
    p.use_tma = 1;
    p.k.s_nu = tau_inv;
    p.k.u_in = u_in;
    p.k.H = H;
    p.k.ramp = 1;
    return p;
}

} // namespace lbm

using namespace lbm;

extern "C" {

int lbm_smemaa_step(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho, int W,
                    int H, float tau_inv, float u_in, int T, void *stream)
{
    if (!mask || !f_now || !f_out || !ux || !uy || !rho || f_now == f_out || W < 3 || H < 3)
        return LBM_ERR_ARG;
    if (T < 2 || T > 8 || (T & 1))
        return LBM_ERR_UNSUPPORTED;
    AaParams p = aa_params(mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in);
    return aa_dispatch<VARIANT_SMEMAA>(p, T, static_cast<cudaStream_t>(stream));
}

int lbm_blocked_step(const uint8_t *mask, const float *f_now, float *f_out, int W, int H, float tau_inv, float u_in,
                     int T, void *stream)
{
    if (!mask || !f_now || !f_out || f_now == f_out || W < 3 || H < 3)
        return LBM_ERR_ARG;
    if (T < 2 || T > 8 || (T & 1))
        return LBM_ERR_UNSUPPORTED;
    AaParams p = aa_params(mask, f_now, f_out, nullptr, nullptr, nullptr, W, H, tau_inv, u_in);
    return aa_dispatch<VARIANT_POLICY>(p, T, static_cast<cudaStream_t>(stream));
}

} // extern "C"
