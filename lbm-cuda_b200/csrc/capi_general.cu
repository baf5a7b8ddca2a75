// C-ABI of the general solver: lbm_params / lbm_create / lbm_run, equilibrium
// initialisation, FP64 diagnostics (mass, momentum, momentum-exchange forces)
// and storage-format conversion.
#include <stdlib.h>
#include <string.h>

#include "dispatch.cuh"

namespace lbm {
struct PairGraph {
    cudaGraphExec_t exec;
    const void *a, *b, *mask;
    int T;
    unsigned long long last_use;
};
} // namespace lbm

struct lbm_handle {
    lbm_params p;
    lbm::Phys k;
    int variant;      // VAR_* compile-time physics variant
    double *partials; // reduction scratch: kRedBlocks x 3 doubles
    // lbm_run's CUDA graphs of one ping-pong pair of launches (a -> b -> a), captured
    // on a private stream; two slots, so that a caller alternating (f_a, f_b) and
    // (f_b, f_a) keeps both
    cudaStream_t cap;
    lbm::PairGraph graphs[2];
    unsigned long long uses;
    std::atomic<int> g_busy; // held by the lbm_run call using the graphs (others launch plainly)
    // Domains whose planes suit the register wavefront's TMA row loads but whose width
    // is not a multiple of 16 (the mask rows' stride cannot be a TMA stride): lbm_run
    // copies the mask into this buffer of 16-byte aligned rows first
    uint8_t *mask_pad;
    int mask_pad_pitch;
};

namespace lbm {

constexpr int kRedBlocks = 296; // fixed, so that the FP64 reductions are deterministic
constexpr int kRedThreads = 256;

static int elem_bytes(int storage)
{
    return storage == LBM_STORE_F64 ? 8 : (storage == LBM_STORE_F32 ? 4 : 2);
}

template <class St> __device__ __forceinline__ typename St::R ld(const void *f, long long i, int q)
{
    return St::load(reinterpret_cast<const typename St::T *>(f)[i], q);
}

template <class St>
__global__ void equilibrium_kernel(void *f, const float *rho, const float *ux, const float *uy, long long N)
{
    using R = typename St::R;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const R r = rho ? rho[i] : 1.0f;
        const R u = ux ? ux[i] : 0.0f;
        const R v = uy ? uy[i] : 0.0f;
        const R usq = u * u + v * v;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const R cu = (R)cx(q) * u + (R)cy(q) * v;
            const R w = q == 0 ? R(4) / R(9) : (q <= 4 ? R(1) / R(9) : R(1) / R(36));
            const R feq = w * r * (R(1) + R(3) * cu + R(4.5) * cu * cu - R(1.5) * usq);
            reinterpret_cast<typename St::T *>(f)[q * N + i] = St::store(feq, q);
        }
    }
}

template <class Si, class So> __global__ void convert_kernel(const void *src, void *dst, long long n9, long long N)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n9; i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / N);
        const auto v = Si::load(reinterpret_cast<const typename Si::T *>(src)[i], q);
        reinterpret_cast<typename So::T *>(dst)[i] = So::store(v, q);
    }
}

// Fixed-shape block reduction of NV doubles (same order on every run).
template <int NV> __device__ void block_reduce(double (&v)[NV], double *out)
{
    __shared__ double red[kRedThreads / 32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NV; ++c)
        for (int o = 16; o > 0; o >>= 1)
            v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
    if (lane == 0)
#pragma unroll
        for (int c = 0; c < NV; ++c)
            red[warp][c] = v[c];
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            double s = 0.0;
            for (int w = 0; w < kRedThreads / 32; ++w)
                s += red[w][c];
            out[c] = s;
        }
    }
}

template <class St>
__global__ void __launch_bounds__(kRedThreads) diag_partial_kernel(const void *f, const uint8_t *mask, long long N,
                                                                    double *part)
{
    double v[3] = {0.0, 0.0, 0.0};
    for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < N; i += (long long)gridDim.x * kRedThreads) {
        if (mask[i])
            continue;
        typename St::R fl[9];
#pragma unroll
        for (int q = 0; q < 9; ++q)
            fl[q] = ld<St>(f, q * N + i, q);
        double m = 0.0, jx = 0.0, jy = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            m += (double)fl[q];
            jx += (double)(cx(q) * fl[q]);
            jy += (double)(cy(q) * fl[q]);
        }
        v[0] += m;
        v[1] += jx;
        v[2] += jy;
    }
    block_reduce<3>(v, part + 3 * blockIdx.x);
}

template <class St>
__global__ void __launch_bounds__(kRedThreads) forces_partial_kernel(const void *f, const uint8_t *mask, int W, int H,
                                                                      double *part)
{
    const long long N = (long long)W * H;
    double v[2] = {0.0, 0.0};
    for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < N; i += (long long)gridDim.x * kRedThreads) {
        if (mask[i])
            continue;
        const int x = (int)(i % W), y = (int)(i / W);
#pragma unroll
        for (int q = 1; q < 9; ++q) {
            const int nx = x + cx(q), ny = y + cy(q);
            if (nx < 0 || nx >= W || ny < 0 || ny >= H)
                continue;
            if (mask[(long long)ny * W + nx] != LBM_MASK_OBSTACLE)
                continue;
            const double fq = (double)ld<St>(f, q * N + i, q);
            v[0] += 2.0 * cx(q) * fq;
            v[1] += 2.0 * cy(q) * fq;
        }
    }
    block_reduce<2>(v, part + 3 * blockIdx.x);
}

template <int NV> __global__ void __launch_bounds__(kRedThreads) final_reduce_kernel(const double *part, int n, double *out)
{
    double v[NV];
#pragma unroll
    for (int c = 0; c < NV; ++c)
        v[c] = 0.0;
    for (int b = threadIdx.x; b < n; b += kRedThreads)
#pragma unroll
        for (int c = 0; c < NV; ++c)
            v[c] += part[3 * b + c];
    block_reduce<NV>(v, out);
}

template <class F> static int by_storage(int storage, F &&fn)
{
    switch (storage) {
    case LBM_STORE_F32:
        return fn(StoreF32{});
    case LBM_STORE_F16DEV:
        return fn(StoreF16Dev{});
    case LBM_STORE_BF16DEV:
        return fn(StoreBF16Dev{});
    case LBM_STORE_F64:
        return fn(StoreF64{});
    default:
        return LBM_ERR_ARG;
    }
}

// Compile-time physics variant of a parameter set, or -1 if none is built.
static int variant_of(const lbm_params &p)
{
    int v = -1;
    if (p.collision == LBM_COLL_MRT && p.closure == LBM_CLOSURE_SMAG)
        v = (p.u_lid != 0.0f) ? -1 : (p.ref_clamps ? VAR_MRT_SMAG_CLAMP : VAR_MRT_SMAG);
    else if (p.collision == LBM_COLL_MRT && p.closure == LBM_CLOSURE_NONE && !p.ref_clamps)
        v = (p.u_lid != 0.0f) ? VAR_MRT_LID : VAR_MRT;
    else if (p.collision == LBM_COLL_BGK && p.closure == LBM_CLOSURE_NONE && !p.ref_clamps && p.u_lid == 0.0f)
        v = VAR_BGK;
    else if (p.collision == LBM_COLL_MRT && (p.closure == LBM_CLOSURE_MLP || p.closure == LBM_CLOSURE_MLP_SILU) &&
             !p.ref_clamps && p.u_lid == 0.0f && p.mlp != nullptr)
        return p.closure == LBM_CLOSURE_MLP ? VAR_MRT_MLP : VAR_MRT_MLP_SILU;
    if ((p.storage == LBM_STORE_F16DEV || p.storage == LBM_STORE_BF16DEV) && (v == VAR_MRT_LID || v == VAR_BGK))
        v = -1;
    return v;
}

static int validate(const lbm_params *p)
{
    if (!p || p->W < 3 || p->H < 3)
        return LBM_ERR_ARG;
    if ((long long)p->W * p->H * 9 > (1ll << 40))
        return LBM_ERR_ARG;
    if (p->storage < LBM_STORE_F32 || p->storage > LBM_STORE_F64)
        return LBM_ERR_ARG;
    if (p->collision != LBM_COLL_BGK && p->collision != LBM_COLL_MRT)
        return LBM_ERR_ARG;
    const bool mlp = p->closure == LBM_CLOSURE_MLP || p->closure == LBM_CLOSURE_MLP_SILU;
    if (p->closure != LBM_CLOSURE_NONE && p->closure != LBM_CLOSURE_SMAG && !mlp)
        return LBM_ERR_UNSUPPORTED;
    if (mlp && (!p->mlp || (reinterpret_cast<uintptr_t>(p->mlp) & 15u) != 0))
        return LBM_ERR_ARG;
    if (!(p->s_nu > 0.0f && p->s_nu < 2.0f))
        return LBM_ERR_ARG;
    const int l = p->bc_left, r = p->bc_right, y = p->bc_y;
    if (l != LBM_BC_WALL && l != LBM_BC_PERIODIC && l != LBM_BC_ZOUHE && l != LBM_BC_ZOUHE_RAMP)
        return LBM_ERR_ARG;
    if (r != LBM_BC_WALL && r != LBM_BC_PERIODIC && r != LBM_BC_OUTFLOW)
        return LBM_ERR_ARG;
    if ((l == LBM_BC_PERIODIC) != (r == LBM_BC_PERIODIC))
        return LBM_ERR_ARG;
    if (y != LBM_BC_WALL && y != LBM_BC_PERIODIC)
        return LBM_ERR_ARG;
    if (variant_of(*p) < 0)
        return LBM_ERR_UNSUPPORTED;
    if (p->storage == LBM_STORE_F64 && mlp)
        return LBM_ERR_UNSUPPORTED;
    return LBM_OK;
}

static Phys make_phys(const lbm_params &p)
{
    Phys k;
    memset(&k, 0, sizeof(k));
    k.s_nu = p.s_nu;
    k.s_e = p.s_e;
    k.s_eps = p.s_eps;
    k.s_q = p.s_q;
    k.tau0 = 1.0f / p.s_nu;
    k.cs2x18 = 18.0f * p.cs_smag * p.cs_smag;
    k.u_in = p.u_in;
    k.u_lid = p.u_lid;
    k.H = p.H;
    k.ramp = p.bc_left == LBM_BC_ZOUHE_RAMP;
    k.mlp = (p.closure == LBM_CLOSURE_MLP || p.closure == LBM_CLOSURE_MLP_SILU) ? p.mlp : nullptr;
    k.flags = (p.collision == LBM_COLL_MRT ? PF_MRT : 0) | (p.closure == LBM_CLOSURE_SMAG ? PF_SMAG : 0) |
              (p.ref_clamps ? (PF_CLAMPU | PF_CLAMPF) : 0);
    return k;
}

// Periodic halo refresh of a local domain of `width` columns: columns [0, halo)
// take the owned columns [width - 2 halo, width - halo), columns [width - halo,
// width) take [halo, 2 halo); every plane, every row.  Element type of 2 or 4 bytes.
template <class E> __global__ void periodic_halo_kernel(E *f, int width, int H, int halo, long long plane)
{
    const long long n = 9ll * H * (2 * halo);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % (2 * halo));
        const long long r = i / (2 * halo); // plane * H + row
        const int q = (int)(r / H), y = (int)(r % H);
        E *row = f + q * plane + (long long)y * width;
        if (c < halo)
            row[c] = row[width - 2 * halo + c];
        else
            row[width - halo + (c - halo)] = row[halo + (c - halo)];
    }
}

// Halo columns of both sides of a state of `width` columns into (or from) one
// contiguous buffer buf[side][q][y][c] (side 0: columns [xl, xl + ncols), side
// 1: [xr, xr + ncols); a side with a negative start is skipped).  Element type of
// 2, 4 or 8 bytes.
template <class E, bool PACK>
__global__ void halo_copy_kernel(E *f, int width, int H, int xl, int xr, int ncols, E *buf)
{
    const long long per_side = 9ll * H * ncols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 2 * per_side;
         i += (long long)gridDim.x * blockDim.x) {
        const int side = (int)(i / per_side);
        const int x = side == 0 ? xl : xr;
        if (x < 0)
            continue;
        const long long j = i - side * per_side;
        const int c = (int)(j % ncols);
        const long long r = j / ncols; // q * H + y
        E *cell = f + r * width + x + c;   // plane q, row y: (q * H + y) * width
        if (PACK)
            buf[i] = *cell;
        else
            *cell = buf[i];
    }
}

static int grid_for(long long n)
{
    long long g = (n + 255) / 256;
    const long long cap = 16ll * sm_count();
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

struct InplaceParams {
    void *f;
    const uint8_t *mask;
    float *ux, *uy, *rho;
    int W, H;
    int bc_left, bc_right, bc_y;
    Phys k;
};
int inplace_step(int variant, int storage, const InplaceParams &p, bool local, cudaStream_t s);
int general_step_f64(const lbm_params &lp, const void *src, void *dst, const uint8_t *mask, float *ux, float *uy,
                     float *rho, cudaStream_t s);

} // namespace lbm

using namespace lbm;

extern "C" {

void lbm_params_default(lbm_params *p, int W, int H)
{
    if (!p)
        return;
    memset(p, 0, sizeof(*p));
    p->W = W;
    p->H = H;
    p->storage = LBM_STORE_F32;
    p->collision = LBM_COLL_MRT;
    p->closure = LBM_CLOSURE_SMAG;
    p->s_nu = 1.8f;
    p->s_e = p->s_eps = p->s_q = 1.1f;
    p->cs_smag = 0.2f;
    p->bc_left = LBM_BC_ZOUHE_RAMP;
    p->bc_right = LBM_BC_OUTFLOW;
    p->bc_y = LBM_BC_WALL;
    p->u_in = 0.1f;
    p->u_lid = 0.0f;
    p->ref_clamps = 1;
}

int lbm_create(const lbm_params *p, lbm_handle **out)
{
    if (!out)
        return LBM_ERR_ARG;
    *out = nullptr;
    int rc = validate(p);
    if (rc)
        return rc;
    lbm_handle *h = static_cast<lbm_handle *>(calloc(1, sizeof(lbm_handle)));
    if (!h)
        return LBM_ERR_ARG;
    h->p = *p;
    h->k = make_phys(*p);
    h->variant = variant_of(*p);
    cudaError_t e = cudaMalloc(&h->partials, sizeof(double) * 3 * kRedBlocks);
    if (e != cudaSuccess) {
        free(h);
        return status(e);
    }
    const int es = elem_bytes(p->storage);
    if (p->storage != LBM_STORE_F64 && p->bc_left != LBM_BC_PERIODIC && (p->W * es) % 16 == 0 && p->W % 16 != 0) {
        h->mask_pad_pitch = (p->W + 15) / 16 * 16;
        e = cudaMalloc(&h->mask_pad, (size_t)h->mask_pad_pitch * p->H);
        if (e != cudaSuccess) {
            cudaFree(h->partials);
            free(h);
            return status(e);
        }
    }
    *out = h;
    return LBM_OK;
}

int lbm_destroy(lbm_handle *h)
{
    if (!h)
        return LBM_ERR_ARG;
    for (auto &g : h->graphs)
        if (g.exec)
            cudaGraphExecDestroy(g.exec);
    if (h->cap)
        cudaStreamDestroy(h->cap);
    cudaError_t e = cudaFree(h->partials);
    if (h->mask_pad) {
        const cudaError_t e2 = cudaFree(h->mask_pad);
        if (e == cudaSuccess)
            e = e2;
    }
    free(h);
    return status(e);
}

size_t lbm_state_bytes(const lbm_handle *h)
{
    return h ? (size_t)h->p.W * h->p.H * 9 * elem_bytes(h->p.storage) : 0;
}

int lbm_init_equilibrium(lbm_handle *h, void *f, const float *rho, const float *ux, const float *uy, void *stream)
{
    if (!h || !f)
        return LBM_ERR_ARG;
    const long long N = (long long)h->p.W * h->p.H;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return by_storage(h->p.storage, [&](auto st) {
        using St = decltype(st);
        equilibrium_kernel<St><<<grid_for(N), 256, 0, s>>>(f, rho, ux, uy, N);
        return status(cudaGetLastError());
    });
}

} // extern "C"

namespace lbm {

// One launch of t steps from src to dst (u, v, rho written when non-null).
// FP64 storage has one step per launch (lbm_run passes t = 1).
// With x1 > 0 only the columns [x0, x1) of dst are written (the register
// wavefront kernel's output rectangle; other kernels cannot restrict their
// output, so such a launch is LBM_ERR_UNSUPPORTED where they would run).
static int run_launch(lbm_handle *h, void *src, void *dst, const uint8_t *mask, int t, float *ux, float *uy,
                      float *rho, cudaStream_t s, int x0 = 0, int x1 = 0)
{
    if (h->p.storage == LBM_STORE_F64)
        return (t == 1 && x1 == 0) ? general_step_f64(h->p, src, dst, mask, ux, uy, rho, s) : LBM_ERR_UNSUPPORTED;
    WaveParams wp;
    memset(&wp, 0, sizeof(wp));
    wp.f_in = src;
    wp.f_out = dst;
    wp.mask = mask;
    wp.ux = ux;
    wp.uy = uy;
    wp.rho = rho;
    wp.W = h->p.W;
    wp.H = h->p.H;
    wp.pitch = h->p.W;
    wp.plane = (long long)h->p.W * h->p.H;
    wp.mask_pitch = (h->mask_pad && mask == h->mask_pad) ? h->mask_pad_pitch : h->p.W;
    wp.chunk = 0;
    wp.bc_left = h->p.bc_left;
    wp.bc_right = h->p.bc_right;
    wp.bc_y = h->p.bc_y;
    wp.use_tma = 1;
    wp.k = h->k;
    if (x1 > 0) {
        const bool mlp = h->variant == VAR_MRT_MLP || h->variant == VAR_MRT_MLP_SILU;
        const bool ok = h->p.storage == LBM_STORE_F32 ? rwave_ok<float>(wp, t, MODE_GENERAL, mlp)
                                                      : rwave_ok<uint16_t>(wp, t, MODE_GENERAL, mlp);
        if (!ok || (mlp && t > 4))
            return LBM_ERR_UNSUPPORTED;
        wp.rx0 = x0;
        wp.rx1 = x1;
    }
    if (h->variant == VAR_MRT_MLP)
        return general_launch_mlp(h->p.storage, wp, t, s);
    if (h->variant == VAR_MRT_MLP_SILU)
        return general_launch_mlp_silu(h->p.storage, wp, t, s);
    if (h->p.storage == LBM_STORE_F32)
        return general_launch_f32(h->variant, wp, t, s);
    if (h->p.storage == LBM_STORE_F16DEV)
        return general_launch_f16(h->variant, wp, t, s);
    if (h->p.storage == LBM_STORE_BF16DEV)
        return general_launch_bf16(h->variant, wp, t, s);
    return LBM_ERR_ARG;
}

// The cached graph of the pair a -> b -> a, or null.
static PairGraph *find_pair(lbm_handle *h, const void *a, const void *b, const void *mask, int T)
{
    for (auto &g : h->graphs)
        if (g.exec && g.a == a && g.b == b && g.mask == mask && g.T == T) {
            g.last_use = ++h->uses;
            return &g;
        }
    return nullptr;
}

// Captures the pair a -> b -> a of T-step launches on the handle's private
// stream into the least recently used slot and instantiates it (the launches
// are recorded, not run).
static PairGraph *capture_pair(lbm_handle *h, void *a, void *b, const uint8_t *mask, int T)
{
    cudaError_t e;
    if (!h->cap && cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    PairGraph *slot = &h->graphs[0];
    for (auto &g : h->graphs)
        if (!g.exec || g.last_use < slot->last_use)
            slot = &g;
    if (slot->exec) {
        cudaGraphExecDestroy(slot->exec);
        slot->exec = nullptr;
    }
    if (cudaStreamBeginCapture(h->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    int rc = run_launch(h, a, b, mask, T, nullptr, nullptr, nullptr, h->cap);
    if (!rc)
        rc = run_launch(h, b, a, mask, T, nullptr, nullptr, nullptr, h->cap);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(h->cap, &g);
    if (!rc && e == cudaSuccess && g)
        e = cudaGraphInstantiate(&slot->exec, g, 0);
    if (g)
        cudaGraphDestroy(g);
    if (rc || e != cudaSuccess || !slot->exec) {
        slot->exec = nullptr;
        cudaGetLastError();
        return nullptr;
    }
    slot->a = a;
    slot->b = b;
    slot->mask = mask;
    slot->T = T;
    slot->last_use = ++h->uses;
    return slot;
}

} // namespace lbm

extern "C" {

int lbm_run(lbm_handle *h, void *f_a, void *f_b, const uint8_t *mask, int n_steps, int T, float *ux, float *uy,
            float *rho, void *stream, int *result_in_b)
{
    NvtxRange nvtx_range("lbm_run");
    if (!h || !f_a || !f_b || !mask || f_a == f_b || n_steps < 0 || T < 1 || T > 8)
        return LBM_ERR_ARG;
    if ((ux || uy || rho) && !(ux && uy && rho))
        return LBM_ERR_ARG;
    if (h->p.storage == LBM_STORE_F64)
        T = 1; // the FP64 kernel advances one step per launch
    // Periodic in x the temporally blocked kernel is the shared-memory wavefront
    // (the register wavefront's TMA rows do not wrap), and one streaming step per
    // launch is faster than it: MRT, FP32, GLUPS at T = 1 / 2 / 4: 68 / 35 / 41 on
    // 1024^2, 85 / 38 / 47 on 4096^2.  (The slab layer instead pads the domain with
    // halo columns and runs the register wavefront: 82 and 146 at T = 4.)
    const bool mlp = h->variant == VAR_MRT_MLP || h->variant == VAR_MRT_MLP_SILU;
    if (T > 1 && !mlp && h->p.bc_left == LBM_BC_PERIODIC && h->p.W % 4 == 0 && aligned16(f_a) && aligned16(f_b) &&
        (reinterpret_cast<uintptr_t>(mask) & 3u) == 0 && (!ux || (aligned16(ux) && aligned16(uy) && aligned16(rho))))
        T = 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int launches = 0, done = 0, rc = LBM_OK;
    if (h->mask_pad && n_steps > 0) {
        // rows of 16-byte aligned pitch for the TMA row loads (one copy per call)
        cudaError_t e = cudaMemcpy2DAsync(h->mask_pad, h->mask_pad_pitch, mask, h->p.W, h->p.W, h->p.H,
                                          cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess)
            return status(e);
        mask = h->mask_pad;
    }
    // Whole pairs of T-step launches before the last launch replay from a CUDA
    // graph captured once per (f_a, f_b, mask, T): the host loop of small domains
    // costs a launch per pair instead of two kernel launches.  The first pair runs
    // eagerly (it makes the per-device setup calls), and a caller whose stream is
    // being captured gets the plain launches in its own graph.
    const int full = n_steps / T;
    int pairs = (full - (n_steps % T == 0 ? 1 : 0)) / 2;
    // LBM_RUN_GRAPH=0 turns the replay off (plain launches only).
    static const bool graphs = [] {
        const char *e = getenv("LBM_RUN_GRAPH");
        return !(e && e[0] == '0');
    }();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusActive;
    int idle = 0;
    if (graphs && pairs >= 1 && cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone &&
        h->g_busy.compare_exchange_strong(idle, 1)) {
        PairGraph *pg = find_pair(h, f_a, f_b, mask, T);
        if (!pg && pairs >= 3) {
            if ((rc = run_launch(h, f_a, f_b, mask, T, nullptr, nullptr, nullptr, s)) ||
                (rc = run_launch(h, f_b, f_a, mask, T, nullptr, nullptr, nullptr, s))) {
                h->g_busy = 0;
                return rc;
            }
            done += 2 * T;
            launches += 2;
            --pairs;
            pg = capture_pair(h, f_a, f_b, mask, T); // on failure: plain launches below
        }
        if (pg) {
            for (int i = 0; i < pairs; ++i) {
                cudaError_t e = cudaGraphLaunch(pg->exec, s);
                if (e != cudaSuccess) {
                    h->g_busy = 0;
                    return status(e);
                }
            }
            done += 2 * T * pairs;
            launches += 2 * pairs;
        }
        h->g_busy = 0;
    }
    void *src = (launches & 1) ? f_b : f_a, *dst = (launches & 1) ? f_a : f_b;
    for (; done < n_steps;) {
        const int t = (n_steps - done < T) ? (n_steps - done) : T;
        const bool last = done + t == n_steps;
        if ((rc = run_launch(h, src, dst, mask, t, last ? ux : nullptr, last ? uy : nullptr, last ? rho : nullptr,
                             s)))
            return rc;
        done += t;
        ++launches;
        void *tmp = src;
        src = dst;
        dst = tmp;
    }
    if (result_in_b)
        *result_in_b = launches & 1;
    return LBM_OK;
}

int lbm_run_columns(lbm_handle *h, const void *src, void *dst, const uint8_t *mask, int T, int x0, int x1,
                    void *stream)
{
    NvtxRange nvtx_range("lbm_run_columns");
    if (!h || !src || !dst || !mask || src == dst || T < 1 || T > 8)
        return LBM_ERR_ARG;
    if (x0 < 0 || x1 > h->p.W || x0 >= x1 || ((x0 | x1) & 1))
        return LBM_ERR_ARG;
    return run_launch(h, const_cast<void *>(src), dst, mask, T, nullptr, nullptr, nullptr,
                      static_cast<cudaStream_t>(stream), x0, x1);
}

int lbm_run_graph_reset(lbm_handle *h)
{
    if (!h)
        return LBM_ERR_ARG;
    int idle = 0;
    if (!h->g_busy.compare_exchange_strong(idle, 1))
        return LBM_ERR_ARG; // an lbm_run on another thread is replaying them
    cudaError_t e = cudaSuccess;
    for (auto &g : h->graphs) {
        if (g.exec) {
            cudaError_t r = cudaGraphExecDestroy(g.exec);
            if (r != cudaSuccess && e == cudaSuccess)
                e = r;
        }
        g = PairGraph{};
    }
    h->g_busy = 0;
    return status(e);
}

int lbm_run_inplace(lbm_handle *h, void *f, const uint8_t *mask, int n_steps, float *ux, float *uy, float *rho,
                    void *stream)
{
    NvtxRange nvtx_range("lbm_run_inplace");
    if (!h || !f || !mask || n_steps < 0 || (n_steps & 1))
        return LBM_ERR_ARG;
    if ((ux || uy || rho) && !(ux && uy && rho))
        return LBM_ERR_ARG;
    if (h->variant == VAR_MRT_MLP || h->variant == VAR_MRT_MLP_SILU || h->p.storage == LBM_STORE_F64)
        return LBM_ERR_UNSUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    InplaceParams ip;
    memset(&ip, 0, sizeof(ip));
    ip.f = f;
    ip.mask = mask;
    ip.W = h->p.W;
    ip.H = h->p.H;
    ip.bc_left = h->p.bc_left;
    ip.bc_right = h->p.bc_right;
    ip.bc_y = h->p.bc_y;
    ip.k = h->k;
    for (int done = 0; done < n_steps; done += 2) {
        ip.ux = ip.uy = ip.rho = nullptr;
        int rc = inplace_step(h->variant, h->p.storage, ip, false, s);
        if (rc)
            return rc;
        if (done + 2 == n_steps) {
            ip.ux = ux;
            ip.uy = uy;
            ip.rho = rho;
        }
        rc = inplace_step(h->variant, h->p.storage, ip, true, s);
        if (rc)
            return rc;
    }
    return LBM_OK;
}

int lbm_diag_fp64(lbm_handle *h, const void *f, const uint8_t *mask, double *d_out, void *stream)
{
    if (!h || !f || !mask || !d_out)
        return LBM_ERR_ARG;
    const long long N = (long long)h->p.W * h->p.H;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return by_storage(h->p.storage, [&](auto st) {
        using St = decltype(st);
        diag_partial_kernel<St><<<kRedBlocks, kRedThreads, 0, s>>>(f, mask, N, h->partials);
        final_reduce_kernel<3><<<1, kRedThreads, 0, s>>>(h->partials, kRedBlocks, d_out);
        return status(cudaGetLastError());
    });
}

int lbm_forces_fp64(lbm_handle *h, const void *f, const uint8_t *mask, double *d_out, void *stream)
{
    if (!h || !f || !mask || !d_out)
        return LBM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return by_storage(h->p.storage, [&](auto st) {
        using St = decltype(st);
        forces_partial_kernel<St><<<kRedBlocks, kRedThreads, 0, s>>>(f, mask, h->p.W, h->p.H, h->partials);
        final_reduce_kernel<2><<<1, kRedThreads, 0, s>>>(h->partials, kRedBlocks, d_out);
        return status(cudaGetLastError());
    });
}

} // extern "C"

namespace lbm {
template <bool PACK>
static int halo_copy(void *f, int width, int H, int storage, int xl, int xr, int ncols, void *buf, cudaStream_t s)
{
    if (!f || !buf || width < 1 || H < 1 || ncols < 1 || (xl < 0 && xr < 0))
        return LBM_ERR_ARG;
    if (xl + ncols > width || xr + ncols > width)
        return LBM_ERR_ARG;
    if (storage < LBM_STORE_F32 || storage > LBM_STORE_F64)
        return LBM_ERR_ARG;
    const long long n = 2ll * 9 * H * ncols;
    if (storage == LBM_STORE_F64)
        halo_copy_kernel<double, PACK><<<grid_for(n), 256, 0, s>>>(static_cast<double *>(f), width, H, xl, xr, ncols,
                                                                   static_cast<double *>(buf));
    else if (storage == LBM_STORE_F32)
        halo_copy_kernel<float, PACK><<<grid_for(n), 256, 0, s>>>(static_cast<float *>(f), width, H, xl, xr, ncols,
                                                                  static_cast<float *>(buf));
    else
        halo_copy_kernel<uint16_t, PACK><<<grid_for(n), 256, 0, s>>>(static_cast<uint16_t *>(f), width, H, xl, xr,
                                                                     ncols, static_cast<uint16_t *>(buf));
    return status(cudaGetLastError());
}
} // namespace lbm

extern "C" {

int lbm_halo_pack(const void *f, int width, int H, int storage, int xl, int xr, int ncols, void *buf, void *stream)
{
    return halo_copy<true>(const_cast<void *>(f), width, H, storage, xl, xr, ncols, buf,
                           static_cast<cudaStream_t>(stream));
}

int lbm_halo_unpack(void *f, int width, int H, int storage, int xl, int xr, int ncols, const void *buf, void *stream)
{
    return halo_copy<false>(f, width, H, storage, xl, xr, ncols, const_cast<void *>(buf),
                            static_cast<cudaStream_t>(stream));
}

int lbm_periodic_halo_x(void *f, int width, int H, int halo, int storage, void *stream)
{
    if (!f || H < 1 || halo < 1 || width < 3 * halo)
        return LBM_ERR_ARG;
    if (storage < LBM_STORE_F32 || storage > LBM_STORE_F64)
        return LBM_ERR_ARG;
    const long long n = 9ll * H * 2 * halo;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long plane = (long long)width * H;
    if (storage == LBM_STORE_F64)
        periodic_halo_kernel<double><<<grid_for(n), 256, 0, s>>>(static_cast<double *>(f), width, H, halo, plane);
    else if (storage == LBM_STORE_F32)
        periodic_halo_kernel<float><<<grid_for(n), 256, 0, s>>>(static_cast<float *>(f), width, H, halo, plane);
    else
        periodic_halo_kernel<uint16_t><<<grid_for(n), 256, 0, s>>>(static_cast<uint16_t *>(f), width, H, halo, plane);
    return status(cudaGetLastError());
}

int lbm_convert_state(int W, int H, const void *src, int src_storage, void *dst, int dst_storage, void *stream)
{
    if (!src || !dst || W < 1 || H < 1 || src == dst)
        return LBM_ERR_ARG;
    const long long N = (long long)W * H;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return by_storage(src_storage, [&](auto si) {
        return by_storage(dst_storage, [&](auto so) {
            convert_kernel<decltype(si), decltype(so)><<<grid_for(9 * N), 256, 0, s>>>(src, dst, 9 * N, N);
            return status(cudaGetLastError());
        });
    });
}

int lbm_device_error_flags(int *flags, int clear)
{
    if (!flags)
        return LBM_ERR_ARG;
    int *w = device_error_word();
    if (!w)
        return LBM_ERR_DEVICE;
    cudaError_t e = cudaMemcpy(flags, w, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && clear)
        e = cudaMemset(w, 0, sizeof(int));
    return status(e);
}

} // extern "C"
