// C-ABI drop-ins for lbm_core4.cu (MRT + Smagorinsky pull step) and the
// per-cell auxiliary kernels (macro extraction, vorticity colour map).
#include <string.h>

#include "dispatch.cuh"

namespace lbm {

__device__ int g_error_word;

int *device_error_word()
{
    static std::atomic<int *> ptr[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64)
        return nullptr;
    if (!ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_error_word) != cudaSuccess)
            return nullptr;
        ptr[dev] = static_cast<int *>(p);
    }
    return ptr[dev];
}

// The reference's compile-time constants: Cs (lbm_core4.cu:123) and the MRT
// rates si[] (lbm_core4.cu:6).
constexpr float kCore4Cs = 0.20f;
constexpr float kCore4Si = 1.1f;

static WaveParams core4_params(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho,
                               int W, int H, float tau_inv, float u_in)
{
    WaveParams p;
    memset(&p, 0, sizeof(p));
    p.f_in = f_now;
    p.f_out = f_out;
    p.mask = mask;
    p.ux = ux;
    p.uy = uy;
    p.rho = rho;
    p.W = W;
    p.H = H;
    p.pitch = W;
    p.plane = (long long)W * H;
    p.mask_pitch = W;
    p.chunk = 0;
    p.use_tma = 1;
    p.k.s_nu = tau_inv;
    p.k.s_e = kCore4Si;
    p.k.s_eps = kCore4Si;
    p.k.s_q = kCore4Si;
    p.k.tau0 = 1.0f / tau_inv;
    p.k.cs2x18 = 18.0f * kCore4Cs * kCore4Cs;
    p.k.u_in = u_in;
    p.k.u_lid = 0.0f;
    p.k.H = H;
    p.k.ramp = 1;
    return p;
}

static int core4_launch(const WaveParams &p, int T, cudaStream_t s)
{
    return launch_step<PhysCore4, StoreF32, MODE_CORE4>(p, T, s);
}

// macro_kernel semantics (lbm_core_smemaa_policy.cu:431-476).
__global__ void macro_kernel(const float *__restrict__ f, float *__restrict__ ux, float *__restrict__ uy,
                             float *__restrict__ rho, const uint8_t *__restrict__ mask, int W, int H, Phys k)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W - 1 || y <= 0 || y >= H - 1)
        return;
    const long long pid = (long long)y * W + x;
    if (mask[pid])
        return;
    const long long N = (long long)W * H;
    float fl[9];
#pragma unroll
    for (int q = 0; q < 9; ++q)
        fl[q] = f[q * N + pid];
    float r, u, v;
    moments_seq(fl, r, u, v);
    if (x == 0) {
        const float lu = inlet_u(k, y);
        r = zou_he(fl, lu);
        u = lu;
        v = 0.0f;
    }
    ux[pid] = u;
    uy[pid] = v;
    rho[pid] = r;
}

// visualizekernel semantics (lbm_core4.cu:214-255).
__global__ void visualize_kernel(const float *__restrict__ ux, const float *__restrict__ uy,
                                 uint8_t *__restrict__ image, const uint8_t *__restrict__ mask, int W, int H,
                                 float vort_scale)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x <= 0 || x >= W - 1 || y <= 0 || y >= H - 1)
        return;
    const long long pid = (long long)y * W + x;
    uchar4 px;
    if (mask[pid]) {
        px = make_uchar4(0, 0, 0, 255);
    } else {
        const float vort = ((uy[pid + 1] - uy[pid - 1]) - (ux[pid + W] - ux[pid - W])) * vort_scale;
        const float r = fminf(fmaxf(1.0f + vort, 0.0f), 1.0f);
        const float g = fminf(fmaxf(1.0f - fabsf(vort), 0.0f), 1.0f);
        const float b = fminf(fmaxf(1.0f - vort, 0.0f), 1.0f);
        px = make_uchar4((uint8_t)(r * 255), (uint8_t)(g * 255), (uint8_t)(b * 255), 255);
    }
    reinterpret_cast<uchar4 *>(image)[pid] = px;
}

} // namespace lbm

using namespace lbm;

extern "C" {

int lbm_core4_step(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho, int W,
                   int H, float tau_inv, float u_in, float tau_inv_bnd, void *stream)
{
    NvtxRange nvtx_range("lbm_core4_step");
    (void)tau_inv_bnd; // unused by the reference too (lbm_core4.cu:12)
    if (!mask || !f_now || !f_out || !ux || !uy || !rho || f_now == f_out || W < 3 || H < 3 || !(tau_inv > 0.0f))
        return LBM_ERR_ARG;
    WaveParams p = core4_params(mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in);
    return core4_launch(p, 1, static_cast<cudaStream_t>(stream));
}

int lbm_core4_run(const uint8_t *mask, float *f_a, float *f_b, float *ux, float *uy, float *rho, int W, int H,
                  float tau_inv, float u_in, int n_steps, int T, void *stream, int *result_in_b)
{
    NvtxRange nvtx_range("lbm_core4_run");
    if (!mask || !f_a || !f_b || !ux || !uy || !rho || f_a == f_b || W < 3 || H < 3 || !(tau_inv > 0.0f) ||
        n_steps < 0 || T < 1 || T > 8)
        return LBM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    float *src = f_a, *dst = f_b;
    int launches = 0;
    for (int done = 0; done < n_steps;) {
        const int t = (n_steps - done < T) ? (n_steps - done) : T;
        WaveParams p = core4_params(mask, src, dst, ux, uy, rho, W, H, tau_inv, u_in);
        int rc = core4_launch(p, t, s);
        if (rc)
            return rc;
        done += t;
        ++launches;
        float *tmp = src;
        src = dst;
        dst = tmp;
    }
    if (result_in_b)
        *result_in_b = launches & 1;
    return LBM_OK;
}

int lbm_macro(const float *f, float *ux, float *uy, float *rho, const uint8_t *mask, int W, int H, float u_in,
              void *stream)
{
    if (!f || !ux || !uy || !rho || !mask || W < 3 || H < 3)
        return LBM_ERR_ARG;
    Phys k;
    memset(&k, 0, sizeof(k));
    k.u_in = u_in;
    k.H = H;
    k.ramp = 1;
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8);
    macro_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(f, ux, uy, rho, mask, W, H, k);
    return status(cudaGetLastError());
}

int lbm_visualize(const float *ux, const float *uy, const float *rho, uint8_t *image, const uint8_t *mask, int W,
                  int H, float vort_scale, void *stream)
{
    (void)rho; // accepted for signature parity; the colour map does not use it (lbm_core4.cu:238)
    if (!ux || !uy || !image || !mask || W < 3 || H < 3)
        return LBM_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(image) & 3u)
        return LBM_ERR_ARG;
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8);
    visualize_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(ux, uy, image, mask, W, H, vort_scale);
    return status(cudaGetLastError());
}

const char *lbm_error_string(int st)
{
    switch (st) {
    case LBM_OK:
        return "ok";
    case LBM_ERR_ARG:
        return "invalid argument";
    case LBM_ERR_UNSUPPORTED:
        return "unsupported configuration";
    case LBM_ERR_DEVICE:
        return "no usable sm_100 device";
    case LBM_ERR_TIMEOUT:
        return "a bounded device-side wait gave up";
    case LBM_ERR_TOO_LARGE:
        return "domain exceeds the fixed scratch of lbm_diag_fp64_noalloc (LBM_NOALLOC_MAX_CELLS cells)";
    default:
        return (st > 0 && st < 1000) ? cudaGetErrorString(static_cast<cudaError_t>(st)) : "unknown status";
    }
}

int lbm_version(void)
{
    return 100;
}

} // extern "C"
