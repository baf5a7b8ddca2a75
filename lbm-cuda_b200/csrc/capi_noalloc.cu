// lbm_diag_fp64_noalloc: the FP64 mass / momentum reduction of lbm_diag_fp64
// for callers that cannot allocate device memory.
//
// Who cannot allocate: code that runs inside a host that owns the whole device
// heap (a pooled allocator that must see every byte, an embedded solver whose
// memory budget is fixed when it is set up), code that must not make a call
// that can synchronise the device or fail for lack of memory in the middle of a
// time loop, and code reached from a foreign runtime that only hands over
// buffers it already owns.  lbm_diag_fp64 needs a handle from lbm_create, which
// allocates its scratch with cudaMalloc; this entry point takes no handle and
// keeps its scratch in a fixed array that is part of the loaded library.
//
// Scratch: one file-scope __device__ array of kNoallocScratchBytes (about
// 384 KiB) per device: a 256-byte header whose first word counts finished
// blocks, then one FP64 partial (mass, jx, jy) per block of kCellsPerPart
// cells.  That bounds the domain at LBM_NOALLOC_MAX_CELLS cells; larger
// domains are rejected with LBM_ERR_TOO_LARGE before anything is launched.
//
// Every call on a device shares that device's array, and the array keeps what
// the last call left in it.  The block counter must start at zero, so each call
// clears it on its stream before the kernel; the partials need no clearing
// (every partial the final pass reads was written by the same call).  Calls
// whose work overlaps on the GPU (two streams, or two host threads without
// ordering between their streams) race on the array and give wrong sums.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (with that device current) and caches it; later
// calls on that device reuse it.  Make that first call before any stream
// capture begins.
#include <mutex>

#include "common.cuh"

namespace lbm {
namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 32;
constexpr long long kCellsPerPart = (long long)kThreads * kCellsPerThread; // 8192 cells per block
constexpr int kMaxParts = 16384;
constexpr int kHeaderDoubles = 32; // 256 bytes: block counter, then padding
constexpr size_t kNoallocScratchBytes = sizeof(double) * (kHeaderDoubles + 3 * (size_t)kMaxParts);
static_assert(kCellsPerPart * kMaxParts == LBM_NOALLOC_MAX_CELLS, "limit in the header");

static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchBytes / sizeof(double)];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
double *g_scratch_ptr[kMaxDevices];

int scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return (int)e;
    if (dev < 0 || dev >= kMaxDevices)
        return LBM_ERR_DEVICE;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return (int)e;
        g_scratch_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_ptr[dev];
    return LBM_OK;
}

// Sums NV doubles over the block in a fixed order; thread 0 gets the result.
template <int NV> __device__ void block_sum(double (&v)[NV])
{
    __shared__ double red[kThreads / 32][NV];
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
    if (threadIdx.x == 0)
#pragma unroll
        for (int c = 0; c < NV; ++c) {
            double s = 0.0;
            for (int w = 0; w < kThreads / 32; ++w)
                s += red[w][c];
            v[c] = s;
        }
    __syncthreads(); // red[] is reused by the final pass
}

// One pass: block b reduces cells [b * kCellsPerPart, (b + 1) * kCellsPerPart)
// to a partial; the block that finishes last sums the n_parts partials in
// block order and writes d_out, so the result does not depend on scheduling.
template <class St>
__global__ void __launch_bounds__(kThreads) diag_noalloc_kernel(const void *f, const uint8_t *mask, long long N,
                                                                 int n_parts, double *scratch, double *d_out)
{
    __shared__ bool s_last;
    unsigned int *counter = reinterpret_cast<unsigned int *>(scratch);
    double *part = scratch + kHeaderDoubles;
    const typename St::T *fs = reinterpret_cast<const typename St::T *>(f);

    double v[3] = {0.0, 0.0, 0.0};
    const long long c0 = (long long)blockIdx.x * kCellsPerPart;
    const long long c1 = c0 + kCellsPerPart < N ? c0 + kCellsPerPart : N;
    for (long long i = c0 + threadIdx.x; i < c1; i += kThreads) {
        if (mask[i])
            continue;
        double m = 0.0, jx = 0.0, jy = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float fq = St::load(fs[q * N + i], q);
            m += (double)fq;
            jx += (double)(cx(q) * fq);
            jy += (double)(cy(q) * fq);
        }
        v[0] += m;
        v[1] += jx;
        v[2] += jy;
    }
    block_sum<3>(v);
    if (threadIdx.x == 0) {
        if (blockIdx.x < kMaxParts)
#pragma unroll
            for (int c = 0; c < 3; ++c)
                part[3 * blockIdx.x + c] = v[c];
        __threadfence();
        s_last = atomicAdd(counter, 1u) == (unsigned)(n_parts - 1);
    }
    __syncthreads();
    if (!s_last)
        return;
    __threadfence();
    double t[3] = {0.0, 0.0, 0.0};
    const int n = n_parts < kMaxParts ? n_parts : kMaxParts;
    for (int b = threadIdx.x; b < n; b += kThreads)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            t[c] += __ldcg(part + 3 * b + c);
    block_sum<3>(t);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c)
            d_out[c] = t[c];
        *counter = 0u;
    }
}

template <class F> int with_storage(int storage, F &&fn)
{
    switch (storage) {
    case LBM_STORE_F32:
        return fn(StoreF32{});
    case LBM_STORE_F16DEV:
        return fn(StoreF16Dev{});
    case LBM_STORE_BF16DEV:
        return fn(StoreBF16Dev{});
    default:
        return LBM_ERR_ARG;
    }
}

} // namespace
} // namespace lbm

extern "C" int lbm_diag_fp64_noalloc(int W, int H, int storage, const void *f, const uint8_t *mask, double *d_out,
                                     void *stream)
{
    using namespace lbm;
    if (!f || !mask || !d_out || W < 1 || H < 1)
        return LBM_ERR_ARG;
    if (storage != LBM_STORE_F32 && storage != LBM_STORE_F16DEV && storage != LBM_STORE_BF16DEV)
        return LBM_ERR_ARG;
    const long long N = (long long)W * H;
    if (N > LBM_NOALLOC_MAX_CELLS)
        return LBM_ERR_TOO_LARGE;
    double *scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != LBM_OK)
        return rc;
    const int n_parts = (int)((N + kCellsPerPart - 1) / kCellsPerPart);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned int), s); // the block counter
    if (e != cudaSuccess)
        return (int)e;
    return with_storage(storage, [&](auto st) {
        diag_noalloc_kernel<decltype(st)><<<n_parts, kThreads, 0, s>>>(f, mask, N, n_parts, scratch, d_out);
        return (int)cudaGetLastError();
    });
}
