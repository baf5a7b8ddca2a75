// Host-side launcher of wave_kernel.
#pragma once

#include <stdlib.h>

#include "host.h"
#include "wave.cuh"

namespace lbm {

// Device-side error word for bounded waits (bit 0 = a wait gave up).  A
// file-scope __device__ variable, so the drop-ins need no allocation.
int *device_error_word();

template <class C> int wave_occupancy()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && cache[dev])
        return cache[dev];
    int n = 0;
    cudaFuncSetAttribute(wave_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wave_kernel<C>, C::NX, C::SMEM);
    if (n < 1)
        n = 1;
    if (dev >= 0 && dev < 64)
        cache[dev] = n;
    return n;
}

// Rows per CTA: enough CTAs to fill every resident slot once when possible,
// never fewer than max(8, 2T) rows (the row halo costs 2T/chunk).
template <class C> int default_chunk(int W, int H)
{
    // Tuning override for experiments: LBM_WAVE_CHUNK=<rows per CTA>.
    if (const char *e = getenv("LBM_WAVE_CHUNK")) {
        const int v = atoi(e);
        if (v >= 1)
            return v;
    }
    const int strips = (W + C::CW - 1) / C::CW;
    const int slots = sm_count() * wave_occupancy<C>();
    int nch = slots / strips;
    if (nch < 1)
        nch = 1;
    const int minch = (2 * C::T > 8) ? 2 * C::T : 8;
    if (nch > H / minch)
        nch = H / minch > 0 ? H / minch : 1;
    return (H + nch - 1) / nch;
}

template <class C> int launch_wave(WaveParams p, cudaStream_t s)
{
    using E = typename C::E;
    (void)wave_occupancy<C>(); // also raises the dynamic shared-memory limit
    if (p.chunk <= 0)
        p.chunk = default_chunk<C>(p.W, p.H);
    if (!p.err)
        p.err = device_error_word();
    CUtensorMap tmf, tmm;
    memset(&tmf, 0, sizeof(tmf));
    memset(&tmm, 0, sizeof(tmm));
    bool tma = p.use_tma != 0;
    if (C::MODE == MODE_GENERAL && p.bc_left == LBM_BC_PERIODIC)
        tma = false; // wrapped columns are gathered by the plain loader
    tma = tma && aligned16(p.f_in) && ((long long)p.pitch * C::ES) % 16 == 0 && (p.plane * C::ES) % 16 == 0 &&
          aligned16(p.mask) && p.mask_pitch % 16 == 0;
    if (tma)
        tma = make_map_planes(&tmf, p.f_in, C::ES, p.W, p.H, p.pitch, p.plane, C::RW) &&
              make_map_mask(&tmm, p.mask, p.W, p.H, p.mask_pitch, C::RWM);
    p.use_tma = tma ? 1 : 0;
    dim3 grid((p.W + C::CW - 1) / C::CW, (p.H + p.chunk - 1) / p.chunk);
    return status(launch_pdl(wave_kernel<C>, grid, dim3(C::NX), (size_t)C::SMEM, s, p, tmf, tmm));
}

} // namespace lbm
