// C-ABI drop-ins for the shared-memory AA kernels of the reference:
// lbm_core_smemaa.cu (lbm_smemaa_step) and lbm_core_smemaa_policy.cu /
// lbm_core_smemaa_endfused.cu (lbm_blocked_step).
#include <stdlib.h>
#include <string.h>

#include "aa_tile.cuh"
#include "host.h"
#include "rwave.cuh"

namespace lbm {

int *device_error_word();

template <class C> int launch_aa(AaParams p, cudaStream_t s)
{
    static std::atomic<int> attr_done[64];
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
    return status(launch_pdl(aa_tile_kernel<C>, grid, dim3(C::NT), (size_t)C::SMEM, s, p, tmf, tmm));
}

// The tile kernel on an explicit 1-D grid (edge-only launches).
template <class C> int launch_aa_grid(AaParams p, int nblocks, cudaStream_t s)
{
    static std::atomic<int> attr_done[64];
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
    return status(launch_pdl(aa_tile_kernel<C>, dim3(nblocks), dim3(C::NT), (size_t)C::SMEM, s, p, tmf, tmm));
}

template <class Cfg, int MODE> static int aa_split(AaParams p, int T, cudaStream_t s, bool &done);

// Tile shapes: (SX, SY, threads, cells per batch, CTAs per SM).  Measured on the
// drivers' 2048 x 512 and on 4096 x 1024 (GLUPS, lbm_smemaa_step T = 4 /
// lbm_blocked_step T = 6): 64 x 40 tiles, 512 threads, one cell per batch, two
// CTAs per SM (shape 5) are fastest where the tile kernel runs alone (85.2 /
// 72.3 at 2048 x 512, against 74.9 / 62.4 for 64 x 32 tiles with two-cell
// batches); on domains of at least 4 M cells, where the tiles only cover the
// edge band of the split launch, the thinner 64 x 32 tiles with one-cell
// batches (shape 6) are (86.9 / 71.1 at 4096 x 1024).  Batches of one cell
// beat two in both (fewer registers per thread under the 64-register cap of
// two 512-thread CTAs).  Shape 1 (32 x 32, 256 threads, four CTAs per SM) and
// shape 2 (64 x 32, two-cell batches) stay selectable for experiments.
template <int VAR, int SHAPE> static int aa_dispatch_shape(const AaParams &p, int T, cudaStream_t s)
{
    constexpr int SX = SHAPE == 1 ? 32 : 64, SY = SHAPE == 5 ? 40 : 32;
    constexpr int NT = SHAPE == 1 ? 256 : 512, NB = (SHAPE >= 5) ? 1 : 2;
    constexpr int MB = SHAPE == 1 ? 4 : 2;
    constexpr int MODE = VAR == VARIANT_SMEMAA ? MODE_PRE_SMEMAA : MODE_PRE_POLICY;
    bool done = false;
    int rc = LBM_OK;
    if (T == 2)
        rc = aa_split<AaCfg<2, VAR, SX, SY, NT, NB, MB>, MODE>(p, T, s, done);
    else if (T == 4)
        rc = aa_split<AaCfg<4, VAR, SX, SY, NT, NB, MB>, MODE>(p, T, s, done);
    else if (T == 6)
        rc = aa_split<AaCfg<6, VAR, SX, SY, NT, NB, MB>, MODE>(p, T, s, done);
    if (rc || done)
        return rc;
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
    static const int forced = []() { // tuning override for experiments
        const char *e = getenv("LBM_AA_SHAPE");
        return e ? atoi(e) : -1;
    }();
    const int shape = forced >= 0 ? forced : ((long long)p.W * p.H >= (4ll << 20) ? 6 : 5);
    switch (shape) {
    case 1:
        return aa_dispatch_shape<VAR, 1>(p, T, s);
    case 2:
        return aa_dispatch_shape<VAR, 2>(p, T, s);
    case 6:
        return aa_dispatch_shape<VAR, 6>(p, T, s);
    default:
        return aa_dispatch_shape<VAR, 5>(p, T, s);
    }
}

// Split launch for T = 2, 4, 6 on TMA-aligned buffers: the reference's AA slot
// semantics differ from plain collide-then-stream only near x = 0 (Zou-He and the
// stale inlet slots), x = W-2 / W-1 (stale outlet slots, the ghost copy) and the
// first and last rows; the shared-memory AA tile kernel runs on the tiles of that
// edge band, and the register wavefront kernel in pre-collision mode on the
// interior rectangle (tile-aligned, at least T + 2 cells from every edge), where
// both give the same values.  LBM_AA_SPLIT=0 runs the tile kernel everywhere.
// Side stream and events for running the edge-band kernel beside the interior
// kernel (fork on an event of the caller's stream, join on another); event waits
// keep the pair capturable into a CUDA graph.  They are owned by the calling host
// thread, one set per device: two threads splitting at the same time never
// re-record each other's fork event between its record and the side stream's
// wait, and a thread capturing a graph never pulls another thread's edge-band
// launch into it (a side stream that joined a capture stays in it until the
// capture ends).  The set is released when its thread exits.
struct SplitStreams {
    cudaStream_t side = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
struct ThreadSplitStreams {
    SplitStreams per_dev[64];
    ~ThreadSplitStreams()
    {
        for (auto &ss : per_dev) {
            if (ss.side)
                cudaStreamDestroy(ss.side);
            if (ss.fork)
                cudaEventDestroy(ss.fork);
            if (ss.join)
                cudaEventDestroy(ss.join);
        }
    }
};
static int split_streams(SplitStreams **out)
{
    static thread_local ThreadSplitStreams mine;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return status(e);
    if (dev < 0 || dev >= 64)
        return LBM_ERR_DEVICE;
    SplitStreams &ss = mine.per_dev[dev];
    if (!ss.side) {
        SplitStreams n;
        if ((e = cudaStreamCreateWithFlags(&n.side, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&n.fork, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&n.join, cudaEventDisableTiming)) != cudaSuccess) {
            if (n.side)
                cudaStreamDestroy(n.side);
            if (n.fork)
                cudaEventDestroy(n.fork);
            return status(e);
        }
        ss = n;
    }
    *out = &ss;
    return LBM_OK;
}

template <class Cfg, int MODE>
static int aa_split(AaParams p, int T, cudaStream_t s, bool &done)
{
    done = false;
    // LBM_AA_SPLIT=0: never split; =2: split at any size (tuning experiments)
    int force = 0;
    if (const char *e = getenv("LBM_AA_SPLIT")) {
        if (atoi(e) == 0)
            return LBM_OK;
        force = atoi(e) == 2;
    }
    constexpr int CX = Cfg::CX, CY = Cfg::CY;
    const int W = p.W, H = p.H;
    const bool al = aligned16(p.f_in) && aligned16(p.f_out) && aligned16(p.mask) && W % 16 == 0 &&
                    (!p.ux || (aligned16(p.ux) && aligned16(p.uy) && aligned16(p.rho)));
    const int nx = (W + CX - 1) / CX, ny = (H + CY - 1) / CY;
    const int etx0 = (T + 2 + CX - 1) / CX, etx1 = (W - T - 3) / CX;
    const int ety0 = (T + 2 + CY - 1) / CY, ety1 = (H - T - 2) / CY;
    // the split pays on domains larger than the L2 cache (measured: 1.3x the tile
    // kernel at 4096 x 1024, 0.8x at 2048 x 512 where the interior is too small to
    // fill the GPU with full-length work items)
    if (!al || etx1 - etx0 < 2 || ety1 - ety0 < 1 || (CX & 1) || (!force && (long long)W * H < (4ll << 20)))
        return LBM_OK;
    // edge band: the tile kernel on the tiles outside the interior block
    p.edge_only = 1;
    p.etx0 = etx0;
    p.etx1 = etx1;
    p.ety0 = ety0;
    p.ety1 = ety1;
    p.nx = nx;
    const int nedge = nx * ny - (etx1 - etx0) * (ety1 - ety0);
    SplitStreams *ss = nullptr;
    int rc = split_streams(&ss);
    if (rc)
        return rc;
    cudaError_t e;
    if ((e = cudaEventRecord(ss->fork, s)) != cudaSuccess || (e = cudaStreamWaitEvent(ss->side, ss->fork, 0)) != cudaSuccess)
        return status(e);
    rc = launch_aa_grid<Cfg>(p, nedge, ss->side);
    if (rc)
        return rc;
    if ((e = cudaEventRecord(ss->join, ss->side)) != cudaSuccess)
        return status(e);
    // interior: pre-collision register wavefront
    WaveParams w;
    memset(&w, 0, sizeof(w));
    w.f_in = p.f_in;
    w.f_out = p.f_out;
    w.mask = p.mask;
    w.ux = p.ux;
    w.uy = p.uy;
    w.rho = p.rho;
    w.W = W;
    w.H = H;
    w.pitch = W;
    w.plane = (long long)W * H;
    w.mask_pitch = W;
    w.bc_left = w.bc_right = w.bc_y = LBM_BC_WALL;
    w.use_tma = 1;
    w.k = p.k;
    w.rx0 = etx0 * CX;
    w.rx1 = etx1 * CX;
    w.ry0 = ety0 * CY;
    w.ry1 = ety1 * CY;
    switch (T) {
    case 2:
        rc = launch_rwave<RwCfg<2, 1, 1, PhysBgkRef, StoreF32, MODE>>(w, s);
        break;
    case 4:
        rc = launch_rwave<RwCfg<4, 1, 2, PhysBgkRef, StoreF32, MODE>>(w, s);
        break;
    case 6:
        rc = launch_rwave<RwCfg<6, 1, 2, PhysBgkRef, StoreF32, MODE>>(w, s);
        break;
    default:
        rc = LBM_ERR_UNSUPPORTED;
    }
    // join: the caller's stream continues after both kernels
    e = cudaStreamWaitEvent(s, ss->join, 0);
    done = true;
    return rc ? rc : status(e);
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
    NvtxRange nvtx_range("lbm_smemaa_step");
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
    NvtxRange nvtx_range("lbm_blocked_step");
    if (!mask || !f_now || !f_out || f_now == f_out || W < 3 || H < 3)
        return LBM_ERR_ARG;
    if (T < 2 || T > 8 || (T & 1))
        return LBM_ERR_UNSUPPORTED;
    AaParams p = aa_params(mask, f_now, f_out, nullptr, nullptr, nullptr, W, H, tau_inv, u_in);
    return aa_dispatch<VARIANT_POLICY>(p, T, static_cast<cudaStream_t>(stream));
}

} // extern "C"
