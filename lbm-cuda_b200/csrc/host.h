// Host helpers shared by the entry points: TMA descriptors, launch plumbing.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <stdlib.h>

#include <atomic>

#include "lbm_b200.h"

namespace lbm {

// NVTX range around an entry point (header-only NVTX 3: a no-op unless a
// profiler is attached), so that a capture can be restricted to one call
// (ncu --nvtx --nvtx-include "lbm_run/").
struct NvtxRange {
    explicit NvtxRange(const char *name)
    {
        nvtxRangePushA(name);
    }
    ~NvtxRange()
    {
        nvtxRangePop();
    }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// cuTensorMapEncodeTiled through the runtime's driver entry point, so that the
// library itself does not link libcuda (it loads on machines without a GPU).
// (Looked up once; the static's initialisation is thread-safe.)
inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return nullptr;
    }();
    return fn;
}

inline bool aligned16(const void *p)
{
    return (reinterpret_cast<uintptr_t>(p) & 15u) == 0;
}

// 3-D map over population planes: dims (W, H, 9), box (box_w, box_h, 9).
inline bool make_map_planes(CUtensorMap *m, const void *base, int elem_bytes, int W, int H, int pitch,
                            long long plane, int box_w, int box_h = 1)
{
    auto fn = encode_fn();
    if (!fn)
        return false;
    CUtensorMapDataType dt = elem_bytes == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    cuuint64_t dims[3] = {(cuuint64_t)W, (cuuint64_t)H, 9};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * elem_bytes, (cuuint64_t)plane * elem_bytes};
    cuuint32_t box[3] = {(cuuint32_t)box_w, (cuuint32_t)box_h, 9};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = fn(m, dt, 3, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// 2-D byte map over the mask: dims (W, H), box (box_w, box_h).
inline bool make_map_mask(CUtensorMap *m, const void *base, int W, int H, int pitch, int box_w, int box_h = 1)
{
    auto fn = encode_fn();
    if (!fn)
        return false;
    cuuint64_t dims[2] = {(cuuint64_t)W, (cuuint64_t)H};
    cuuint64_t strides[1] = {(cuuint64_t)pitch};
    cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Launch with programmatic dependent launch: the kernel may be scheduled while
// the previous kernel in the stream drains; it must execute griddepcontrol.wait
// (pdl_wait) before touching anything that kernel writes.  LBM_PDL=0 in the
// environment launches plainly.
template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args)
{
    static const bool on = [] {
        const char *e = getenv("LBM_PDL");
        return !(e && e[0] == '0');
    }();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = on ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args &&>(args)...);
}

inline int status(cudaError_t e)
{
    return e == cudaSuccess ? LBM_OK : (int)e;
}

// Number of SMs of the current device (cached per device; the per-device
// caches in this library are atomics, as several host threads may call in).
inline int sm_count()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64)
        return 148;
    if (!cache[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

} // namespace lbm
