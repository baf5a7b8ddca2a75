// Batched independent domains: one launch advances every domain T steps, so
// domains of uneven size share the GPU without one launch per domain.  Two
// engines: when every domain is TMA-aligned (and T is 1, 2 or 4), the register
// wavefront kernel runs one warp per (domain, window, row range) item of a
// host-built list (edge windows first); otherwise a persistent kernel whose CTAs
// take (domain, strip, row-chunk) items from a device counter and run the
// shared-memory wavefront tile of wave.cuh.  Launch pairs (ping-pong) are
// captured once into a CUDA graph and replayed.
//
// Tile shape: an item is one window (64 columns, register wavefront) or strip
// (shared-memory wavefront) of a domain by `rows` rows, and `rows` is chosen per
// domain size class (LBM_BATCH_SIZE_CLASSES classes by cell count): small
// domains want short items to spread over the GPU, large ones long items that
// waste less of their wavefront warm-up.  The autotuner searches the depth T,
// then the rows of every class in turn.
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "dispatch.cuh"

namespace lbm {

struct __align__(64) BatchDomain {
    CUtensorMap tmf[2]; // input map when f_a (0) / f_b (1) is the source
    CUtensorMap tmm;
    CUtensorMap rtmf[2]; // the same for the register wavefront's row boxes
    CUtensorMap rtmm;
    WaveParams p;
    void *f[2];
    int rw; // 1: the register wavefront can run this domain (TMA-aligned, x not periodic)
};

// Register-wavefront batch: one warp per (domain, window, row range) item of a
// host-built list; every domain's inlet / outlet windows come first (see rw_items).
template <class C>
__global__ void __launch_bounds__(32 * C::NW, C::MINB)
    rbatch_kernel(const BatchDomain *__restrict__ doms, const int4 *__restrict__ items, int n_items, int parity)
{
    const int it = blockIdx.x * C::NW + (threadIdx.x >> 5);
    if (it >= n_items)
        return;
    const int4 item = items[it]; // domain, window, ya, yb
    const BatchDomain &d = doms[item.x];
    WaveParams p = d.p;
    p.f_in = d.f[parity];
    p.f_out = d.f[parity ^ 1];
    rwave_run<C>(p, &d.rtmf[parity], &d.rtmm, item.y, item.z, item.w);
}

template <class Ph, class St, int T> using RBCfg = RwCfg<T, 1, (T <= 2 ? 1 : 2), Ph, St, MODE_GENERAL>;

template <class C> static int rbatch_launch(const BatchDomain *d, const int4 *items, int n_items, int parity,
                                            cudaStream_t s)
{
    static std::atomic<int> attr[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !attr[dev]) {
        cudaFuncSetAttribute(rbatch_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
        attr[dev] = 1;
    }
    if (n_items < 1)
        return LBM_OK;
    rbatch_kernel<C><<<(n_items + C::NW - 1) / C::NW, 32 * C::NW, C::SMEM, s>>>(d, items, n_items, parity);
    return status(cudaGetLastError());
}

template <template <class> class F, class... A> static int with_rcfg(int clamps, int storage, int T, A &&...a)
{
    auto go = [&](auto ph, auto st) -> int {
        using Ph = decltype(ph);
        using St = decltype(st);
        switch (T) {
        case 1:
            return F<RBCfg<Ph, St, 1>>::run(a...);
        case 2:
            return F<RBCfg<Ph, St, 2>>::run(a...);
        case 4:
            return F<RBCfg<Ph, St, 4>>::run(a...);
        default:
            return LBM_ERR_UNSUPPORTED;
        }
    };
    if (storage == LBM_STORE_F32)
        return clamps ? go(PhysMrtSmagClamp{}, StoreF32{}) : go(PhysMrtSmag{}, StoreF32{});
    if (storage == LBM_STORE_F16DEV)
        return clamps ? go(PhysMrtSmagClamp{}, StoreF16Dev{}) : go(PhysMrtSmag{}, StoreF16Dev{});
    return LBM_ERR_UNSUPPORTED;
}

template <class C> struct RLaunchOp {
    static int run(const BatchDomain *d, const int4 *items, int n_items, int parity, cudaStream_t s)
    {
        return rbatch_launch<C>(d, items, n_items, parity, s);
    }
};
template <class C> struct RGeomOp {
    static int run(int *cw, int *padl)
    {
        *cw = C::CW;
        *padl = C::PADL;
        return LBM_OK;
    }
};

constexpr int kBatchNX = 128;

template <class C> struct BatchSmem {
    static constexpr int OFF_PRM = round_up(C::SMEM, 16);
    static constexpr int OFF_ITEM = OFF_PRM + round_up((int)sizeof(WaveParams), 16);
    static constexpr int SMEM = OFF_ITEM + 16;
};

template <class C>
__global__ void __launch_bounds__(C::NX, C::MINB)
    batch_kernel(const BatchDomain *__restrict__ doms, const int4 *__restrict__ items, int n_items, int *counter,
                 int parity)
{
    extern __shared__ __align__(128) unsigned char smem[];
    WaveParams *sp = reinterpret_cast<WaveParams *>(smem + BatchSmem<C>::OFF_PRM);
    volatile int *s_item = reinterpret_cast<volatile int *>(smem + BatchSmem<C>::OFF_ITEM);
    bool first = true;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0)
            *s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int it = *s_item;
        if (it >= n_items)
            break;
        const int4 item = items[it];
        const BatchDomain &d = doms[item.x];
        if (threadIdx.x == 0) {
            WaveParams w = d.p;
            w.f_in = d.f[parity];
            w.f_out = d.f[parity ^ 1];
            *sp = w;
        }
        __syncthreads();
        wave_tile<C>(*sp, &d.tmf[parity], &d.tmm, item.y, item.z, !first);
        first = false;
    }
}

template <class Ph, class St, int T> using BCfg = WaveCfg<T, kBatchNX, Ph, St, MODE_GENERAL>;

// Resident CTAs per SM of a batch configuration (also raises the smem limit).
template <class C> static int batch_occupancy()
{
    const int smem = BatchSmem<C>::SMEM;
    cudaFuncSetAttribute(batch_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<C>, C::NX, smem);
    return n < 1 ? 1 : n;
}

template <class C>
static int batch_launch(const BatchDomain *d, const int4 *items, int n_items, int *counter, int parity,
                        cudaStream_t s)
{
    const int grid = sm_count() * batch_occupancy<C>();
    cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(int), s);
    if (e != cudaSuccess)
        return status(e);
    batch_kernel<C><<<grid, C::NX, BatchSmem<C>::SMEM, s>>>(d, items, n_items, counter, parity);
    return status(cudaGetLastError());
}

// Dispatch on (clamps, storage, T).
template <template <class> class F, class... A> static int with_cfg(int clamps, int storage, int T, A &&...a)
{
    auto go = [&](auto ph, auto st) -> int {
        using Ph = decltype(ph);
        using St = decltype(st);
        switch (T) {
        case 1:
            return F<BCfg<Ph, St, 1>>::run(a...);
        case 2:
            return F<BCfg<Ph, St, 2>>::run(a...);
        case 4:
            return F<BCfg<Ph, St, 4>>::run(a...);
        case 8:
            return F<BCfg<Ph, St, 8>>::run(a...);
        default:
            return LBM_ERR_UNSUPPORTED;
        }
    };
    if (storage == LBM_STORE_F32)
        return clamps ? go(PhysMrtSmagClamp{}, StoreF32{}) : go(PhysMrtSmag{}, StoreF32{});
    if (storage == LBM_STORE_F16DEV)
        return clamps ? go(PhysMrtSmagClamp{}, StoreF16Dev{}) : go(PhysMrtSmag{}, StoreF16Dev{});
    return LBM_ERR_UNSUPPORTED;
}

template <class C> struct LaunchOp {
    static int run(const BatchDomain *d, const int4 *items, int n_items, int *counter, int parity, cudaStream_t s)
    {
        return batch_launch<C>(d, items, n_items, counter, parity, s);
    }
};
template <class C> struct CwOp {
    static int run(int *cw)
    {
        *cw = C::CW;
        return LBM_OK;
    }
};
template <class C> struct RwOp {
    static int run(int *rw, int *rwm)
    {
        *rw = C::RW;
        *rwm = C::RWM;
        return LBM_OK;
    }
};
// One launch per domain through the single-domain dispatcher (streaming, register
// or shared-memory wavefront kernel, whichever fits the domain and T).
static int separate_launch(int clamps, int storage, const WaveParams &w, int T, cudaStream_t s)
{
    if (storage == LBM_STORE_F32)
        return clamps ? launch_step<PhysMrtSmagClamp, StoreF32, MODE_GENERAL>(w, T, s)
                      : launch_step<PhysMrtSmag, StoreF32, MODE_GENERAL>(w, T, s);
    if (storage == LBM_STORE_F16DEV)
        return clamps ? launch_step<PhysMrtSmagClamp, StoreF16Dev, MODE_GENERAL>(w, T, s)
                      : launch_step<PhysMrtSmag, StoreF16Dev, MODE_GENERAL>(w, T, s);
    return LBM_ERR_UNSUPPORTED;
}

} // namespace lbm

using namespace lbm;

namespace lbm {
// Rows per work item for each domain size class.
struct Rows {
    int r[LBM_BATCH_SIZE_CLASSES];
    bool operator==(const Rows &o) const
    {
        for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c)
            if (r[c] != o.r[c])
                return false;
        return true;
    }
    bool operator!=(const Rows &o) const
    {
        return !(*this == o);
    }
};
inline Rows uniform_rows(int v)
{
    Rows x;
    for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c)
        x.r[c] = v;
    return x;
}
// Size class of a domain of W x H cells: < 2^17 cells, < 2^19, larger.
inline int size_class(int W, int H)
{
    const long long n = (long long)W * H;
    return n < (1ll << 17) ? 0 : (n < (1ll << 19) ? 1 : 2);
}
} // namespace lbm

struct lbm_batch {
    lbm_params p;
    std::vector<lbm_domain> doms;
    std::vector<BatchDomain> hdoms;
    BatchDomain *d_doms = nullptr;
    int4 *d_items = nullptr;
    int max_items = 0;
    int n_items = 0;
    int *d_counter = nullptr;
    int cur_T = 0;                    // configuration the device item list holds
    Rows cur_rows = uniform_rows(0);
    std::vector<int4> h_items;
    int tuned_T = 4;
    Rows tuned_rows = uniform_rows(64);
    int class_count[LBM_BATCH_SIZE_CLASSES] = {0};
    bool rw_all = false; // every domain can take the register wavefront
    int cur_engine = 0;  // engine the device item list is for: 0 shared-memory wavefront, 1 register
    int tuned_engine = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
    int exec_T = 0;
    Rows exec_rows = uniform_rows(0);
};

static int rows_of(const lbm_batch *b, const Rows &rows, int d)
{
    return rows.r[size_class(b->doms[d].W, b->doms[d].H)];
}

static int batch_items(lbm_batch *b, int T, const Rows &rows, cudaStream_t s)
{
    if (b->cur_engine == 0 && b->cur_T == T && b->cur_rows == rows)
        return LBM_OK;
    int cw = 0;
    int rc = with_cfg<CwOp>(b->p.ref_clamps, b->p.storage, T, &cw);
    if (rc)
        return rc;
    b->h_items.clear();
    for (int d = 0; d < (int)b->doms.size(); ++d) {
        const int chunk = rows_of(b, rows, d);
        const int strips = (b->doms[d].W + cw - 1) / cw;
        const int chunks = (b->doms[d].H + chunk - 1) / chunk;
        for (int by = 0; by < chunks; ++by)
            for (int bx = 0; bx < strips; ++bx)
                b->h_items.push_back(make_int4(d, bx, by, 0));
    }
    if ((int)b->h_items.size() > b->max_items)
        return LBM_ERR_ARG;
    for (int d = 0; d < (int)b->hdoms.size(); ++d)
        b->hdoms[d].p.chunk = rows_of(b, rows, d);
    cudaError_t e = cudaMemcpyAsync(b->d_items, b->h_items.data(), sizeof(int4) * b->h_items.size(),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_doms, b->hdoms.data(), sizeof(BatchDomain) * b->hdoms.size(),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s); // the host vectors may change before the copies run otherwise
    if (e != cudaSuccess)
        return status(e);
    b->n_items = (int)b->h_items.size();
    b->cur_T = T;
    b->cur_rows = rows;
    return LBM_OK;
}

static bool rw_engine(const lbm_batch *b, int T)
{
    return b->rw_all && (T == 1 || T == 2 || T == 4);
}

// Item list of the register wavefront for (T, chunk): the edge windows of every
// domain first (half-height items), then all other windows.
static int rbatch_items(lbm_batch *b, int T, const Rows &rows, cudaStream_t s)
{
    if (b->cur_engine == 1 && b->cur_T == T && b->cur_rows == rows)
        return LBM_OK;
    int cw = 0, padl = 0;
    int rc = with_rcfg<RGeomOp>(b->p.ref_clamps, b->p.storage, T, &cw, &padl);
    if (rc)
        return rc;
    b->h_items.clear();
    std::vector<int4> mid;
    for (int d = 0; d < (int)b->doms.size(); ++d) {
        const int chunk = rows_of(b, rows, d);
        const RwItems it = rw_items(b->doms[d].W, b->doms[d].H, cw, padl, chunk);
        for (int i = 0; i < it.n_items; ++i) {
            int win, ya, yb;
            rw_item(it, i, b->doms[d].H, chunk, win, ya, yb);
            (i < it.n_edge_items ? b->h_items : mid).push_back(make_int4(d, win, ya, yb));
        }
    }
    b->h_items.insert(b->h_items.end(), mid.begin(), mid.end());
    if ((int)b->h_items.size() > b->max_items)
        return LBM_ERR_ARG;
    cudaError_t e = cudaMemcpyAsync(b->d_items, b->h_items.data(), sizeof(int4) * b->h_items.size(),
                                    cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->d_doms, b->hdoms.data(), sizeof(BatchDomain) * b->hdoms.size(),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
        return status(e);
    b->n_items = (int)b->h_items.size();
    b->cur_T = T;
    b->cur_rows = rows;
    b->cur_engine = 1;
    return LBM_OK;
}

static int prepare(lbm_batch *b, int T, const Rows &rows, cudaStream_t s)
{
    if (rw_engine(b, T))
        return rbatch_items(b, T, rows, s);
    if (b->cur_engine != 0) {
        b->cur_T = 0; // force a rebuild of the shared-memory wavefront's list
        b->cur_engine = 0;
    }
    return batch_items(b, T, rows, s);
}

static bool prepared(const lbm_batch *b, int T, const Rows &rows)
{
    return b->cur_T == T && b->cur_rows == rows && b->cur_engine == (rw_engine(b, T) ? 1 : 0);
}

// Rows per item a configuration may use with depth T on the batch's engine.
static bool rows_ok(const lbm_batch *b, int T, int ch)
{
    return ch >= 8 && ch >= 2 * T && ch <= 128 && (rw_engine(b, T) ? ch <= 32 : ch >= 16);
}

static int batch_launch_one(lbm_batch *b, int T, int parity, cudaStream_t s)
{
    if (rw_engine(b, T))
        return with_rcfg<RLaunchOp>(b->p.ref_clamps, b->p.storage, T, (const BatchDomain *)b->d_doms,
                                    (const int4 *)b->d_items, b->n_items, parity, s);
    return with_cfg<LaunchOp>(b->p.ref_clamps, b->p.storage, T, (const BatchDomain *)b->d_doms,
                              (const int4 *)b->d_items, b->n_items, b->d_counter, parity, s);
}

extern "C" {

int lbm_batch_create(const lbm_params *common, const lbm_domain *domains, int n, lbm_batch **out)
{
    if (!common || !domains || n < 1 || !out)
        return LBM_ERR_ARG;
    *out = nullptr;
    if (common->collision != LBM_COLL_MRT || common->closure != LBM_CLOSURE_SMAG || common->u_lid != 0.0f ||
        (common->storage != LBM_STORE_F32 && common->storage != LBM_STORE_F16DEV))
        return LBM_ERR_UNSUPPORTED;
    if ((common->bc_left == LBM_BC_PERIODIC) != (common->bc_right == LBM_BC_PERIODIC))
        return LBM_ERR_ARG;
    lbm_batch *b = new lbm_batch();
    b->p = *common;
    b->doms.assign(domains, domains + n);
    const int es = common->storage == LBM_STORE_F32 ? 4 : 2;
    int rw = 0, rwm = 0;
    with_cfg<RwOp>(common->ref_clamps, common->storage, 4, &rw, &rwm);
    b->hdoms.resize(n);
    int max_items = 0;
    for (int d = 0; d < n; ++d) {
        lbm_domain dm = domains[d];
        if (dm.W < 3 || dm.H < 3 || !dm.f_a || !dm.f_b || !dm.mask || dm.f_a == dm.f_b) {
            delete b;
            return LBM_ERR_ARG;
        }
        if (!dm.pitch)
            dm.pitch = dm.W;
        if (!dm.mask_pitch)
            dm.mask_pitch = dm.W;
        b->doms[d] = dm;
        BatchDomain &hd = b->hdoms[d];
        memset(&hd, 0, sizeof(hd));
        WaveParams &w = hd.p;
        w.mask = dm.mask;
        w.W = dm.W;
        w.H = dm.H;
        w.pitch = dm.pitch;
        w.plane = (long long)dm.pitch * dm.H;
        w.mask_pitch = dm.mask_pitch;
        w.bc_left = common->bc_left;
        w.bc_right = common->bc_right;
        w.bc_y = common->bc_y;
        w.err = device_error_word();
        w.k.s_nu = common->s_nu;
        w.k.s_e = common->s_e;
        w.k.s_eps = common->s_eps;
        w.k.s_q = common->s_q;
        w.k.tau0 = 1.0f / common->s_nu;
        w.k.cs2x18 = 18.0f * common->cs_smag * common->cs_smag;
        w.k.u_in = dm.u_in;
        w.k.H = dm.H;
        w.k.ramp = common->bc_left == LBM_BC_ZOUHE_RAMP;
        hd.f[0] = dm.f_a;
        hd.f[1] = dm.f_b;
        bool tma = common->bc_left != LBM_BC_PERIODIC && aligned16(dm.f_a) && aligned16(dm.f_b) &&
                   aligned16(dm.mask) && ((long long)dm.pitch * es) % 16 == 0 && (w.plane * es) % 16 == 0 &&
                   dm.mask_pitch % 16 == 0;
        if (tma)
            tma = make_map_planes(&hd.tmf[0], dm.f_a, es, dm.W, dm.H, dm.pitch, w.plane, rw) &&
                  make_map_planes(&hd.tmf[1], dm.f_b, es, dm.W, dm.H, dm.pitch, w.plane, rw) &&
                  make_map_mask(&hd.tmm, dm.mask, dm.W, dm.H, dm.mask_pitch, rwm);
        w.use_tma = tma ? 1 : 0;
        // register wavefront: row boxes of 64 + 16 / es elements and 80 mask bytes
        hd.rw = tma && make_map_planes(&hd.rtmf[0], dm.f_a, es, dm.W, dm.H, dm.pitch, w.plane, 64 + 16 / es) &&
                make_map_planes(&hd.rtmf[1], dm.f_b, es, dm.W, dm.H, dm.pitch, w.plane, 64 + 16 / es) &&
                make_map_mask(&hd.rtmm, dm.mask, dm.W, dm.H, dm.mask_pitch, 80);
        b->class_count[size_class(dm.W, dm.H)] += 1;
        // bound on the work items of any (T, rows >= 8 or >= 4) configuration of either engine
        max_items += ((dm.W + (kBatchNX - 16) - 1) / (kBatchNX - 16)) * ((dm.H + 7) / 8) +
                     ((dm.W + 51) / 52) * ((dm.H + 3) / 4);
    }
    b->max_items = max_items;
    b->rw_all = true;
    for (const auto &hd : b->hdoms)
        b->rw_all = b->rw_all && hd.rw;
    if (b->rw_all) {
        b->tuned_T = 2;
        b->tuned_rows = uniform_rows(16);
    }
    cudaError_t e = cudaMalloc(&b->d_doms, sizeof(BatchDomain) * n);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_items, sizeof(int4) * max_items);
    if (e == cudaSuccess)
        e = cudaMalloc(&b->d_counter, sizeof(int));
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        lbm_batch_destroy(b);
        return status(e);
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_destroy(lbm_batch *b)
{
    if (!b)
        return LBM_ERR_ARG;
    if (b->exec)
        cudaGraphExecDestroy(b->exec);
    if (b->cap)
        cudaStreamDestroy(b->cap);
    cudaFree(b->d_doms);
    cudaFree(b->d_items);
    cudaFree(b->d_counter);
    delete b;
    return LBM_OK;
}

int lbm_batch_run(lbm_batch *b, int n_steps, int T, void *stream, int *result_in_b)
{
    NvtxRange nvtx_range("lbm_batch_run");
    if (!b || n_steps < 0 || T < 0 || T > 8)
        return LBM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (T == 0)
        T = b->tuned_T;
    if (T != 1 && T != 2 && T != 4 && T != 8)
        return LBM_ERR_UNSUPPORTED;
    // the tuned rows per class where they suit T and the engine, else the default
    Rows chunk = b->tuned_rows;
    for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c)
        if (!rows_ok(b, T, chunk.r[c]))
            chunk.r[c] = rw_engine(b, T) ? (T <= 2 ? 16 : 24) : 64;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(s, &cs);
    const bool capturing = cs != cudaStreamCaptureStatusNone;
    if (!prepared(b, T, chunk)) {
        if (capturing)
            return LBM_ERR_ARG; // the item list must be prepared outside a capture (run once first)
        int rc = prepare(b, T, chunk, s);
        if (rc)
            return rc;
    }
    int done = 0, parity = 0;
    const int pairs = n_steps / (2 * T);
    if (pairs > 0 && !capturing) {
        if (!b->exec || b->exec_T != T || b->exec_rows != chunk) {
            if (b->exec) {
                cudaGraphExecDestroy(b->exec);
                b->exec = nullptr;
            }
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess)
                return status(e);
            int rc = batch_launch_one(b, T, 0, b->cap);
            if (!rc)
                rc = batch_launch_one(b, T, 1, b->cap);
            e = cudaStreamEndCapture(b->cap, &g);
            if (rc || e != cudaSuccess) {
                if (g)
                    cudaGraphDestroy(g);
                return rc ? rc : status(e);
            }
            e = cudaGraphInstantiate(&b->exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess)
                return status(e);
            b->exec_T = T;
            b->exec_rows = chunk;
        }
        for (int i = 0; i < pairs; ++i) {
            cudaError_t e = cudaGraphLaunch(b->exec, s);
            if (e != cudaSuccess)
                return status(e);
        }
        done = pairs * 2 * T;
    }
    while (done < n_steps) {
        // remaining steps: launches of depth T, then the largest supported depth that fits
        const int left = n_steps - done;
        const int t = left >= T ? T : (left >= 4 ? 4 : (left >= 2 ? 2 : 1));
        Rows ct = chunk;
        for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c)
            if (!rows_ok(b, t, ct.r[c]))
                ct.r[c] = rw_engine(b, t) ? (t <= 2 ? 16 : 24) : 64;
        if (!prepared(b, t, ct)) {
            if (capturing)
                return LBM_ERR_ARG;
            int rc = prepare(b, t, ct, s);
            if (rc)
                return rc;
        }
        int rc = batch_launch_one(b, t, parity, s);
        if (rc)
            return rc;
        done += t;
        parity ^= 1;
    }
    if (result_in_b)
        *result_in_b = parity;
    return LBM_OK;
}

int lbm_batch_run_separate(lbm_batch *b, int n_steps, int T, void *stream, int *result_in_b)
{
    NvtxRange nvtx_range("lbm_batch_run_separate");
    if (!b || n_steps < 0 || T < 1 || T > 8)
        return LBM_ERR_ARG;
    if (T != 1 && T != 2 && T != 4 && T != 8)
        return LBM_ERR_UNSUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int parity = 0;
    for (int done = 0; done < n_steps;) {
        const int t = (n_steps - done >= T) ? T : ((n_steps - done) >= 4 ? 4 : ((n_steps - done) >= 2 ? 2 : 1));
        for (size_t d = 0; d < b->hdoms.size(); ++d) {
            WaveParams w = b->hdoms[d].p;
            w.f_in = b->hdoms[d].f[parity];
            w.f_out = b->hdoms[d].f[parity ^ 1];
            w.chunk = 0;
            int rc = separate_launch(b->p.ref_clamps, b->p.storage, w, t, s);
            if (rc)
                return rc;
        }
        done += t;
        parity ^= 1;
    }
    if (result_in_b)
        *result_in_b = parity;
    return LBM_OK;
}

} // extern "C"

namespace lbm {
// Device time of one step of configuration (T, rows): two warm-up launches, then
// `n` timed launches (ms per step), or a negative status.
static float time_config(lbm_batch *b, int T, const Rows &rows, cudaStream_t s, cudaEvent_t e0, cudaEvent_t e1,
                         int n, int *rc_out)
{
    int rc = prepare(b, T, rows, s);
    for (int w = 0; !rc && w < 2; ++w)
        rc = batch_launch_one(b, T, w & 1, s);
    cudaEventRecord(e0, s);
    for (int w = 0; !rc && w < n; ++w)
        rc = batch_launch_one(b, T, w & 1, s);
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    if (!rc && e != cudaSuccess)
        rc = status(e);
    *rc_out = rc;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    return ms / ((float)n * T);
}
} // namespace lbm

extern "C" {

int lbm_batch_autotune(lbm_batch *b, void *stream, int *best_T, int *best_chunk)
{
    if (!b)
        return LBM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int Ts[] = {1, 2, 4, 8};
    const int chunks[] = {8, 16, 24, 32, 64, 128};
    float best = 1e30f;
    int bT = b->tuned_T;
    Rows bR = b->tuned_rows;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = LBM_OK;
    for (int T : Ts) {
        // one height for every class first
        float bt = 1e30f;
        Rows br = uniform_rows(0);
        for (int ch : chunks) {
            if (!rows_ok(b, T, ch))
                continue;
            const float t = time_config(b, T, uniform_rows(ch), s, e0, e1, 4, &rc);
            if (rc)
                break;
            if (t < bt) {
                bt = t;
                br = uniform_rows(ch);
            }
        }
        if (rc)
            break;
        if (br.r[0] == 0)
            continue;
        // then each populated size class in turn, the others held at their best
        for (int c = 0; c < LBM_BATCH_SIZE_CLASSES && !rc; ++c) {
            if (b->class_count[c] == 0)
                continue;
            for (int ch : chunks) {
                if (!rows_ok(b, T, ch) || ch == br.r[c])
                    continue;
                Rows cand = br;
                cand.r[c] = ch;
                const float t = time_config(b, T, cand, s, e0, e1, 4, &rc);
                if (rc)
                    break;
                if (t < 0.98f * bt) { // a clear gain: the class is a part of the launch
                    bt = t;
                    br = cand;
                }
            }
        }
        if (!rc && bt < best) {
            best = bt;
            bT = T;
            bR = br;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc)
        return rc;
    b->tuned_T = bT;
    b->tuned_rows = bR;
    if (best_T)
        *best_T = bT;
    if (best_chunk) { // rows of the largest populated class
        int c = LBM_BATCH_SIZE_CLASSES - 1;
        while (c > 0 && b->class_count[c] == 0)
            --c;
        *best_chunk = bR.r[c];
    }
    return LBM_OK;
}

int lbm_batch_get_tiles(const lbm_batch *b, int *T, int *rows)
{
    if (!b || !T || !rows)
        return LBM_ERR_ARG;
    *T = b->tuned_T;
    for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c)
        rows[c] = b->tuned_rows.r[c];
    return LBM_OK;
}

int lbm_batch_set_tiles(lbm_batch *b, int T, const int *rows)
{
    if (!b || !rows || (T != 1 && T != 2 && T != 4 && T != 8))
        return LBM_ERR_ARG;
    Rows r;
    for (int c = 0; c < LBM_BATCH_SIZE_CLASSES; ++c) {
        if (!rows_ok(b, T, rows[c]))
            return LBM_ERR_ARG;
        r.r[c] = rows[c];
    }
    b->tuned_T = T;
    b->tuned_rows = r;
    return LBM_OK;
}

} // extern "C"
