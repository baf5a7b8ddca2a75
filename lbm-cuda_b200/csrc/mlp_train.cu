// Training kernels of the learned closure: a 5 -> 32 -> 32 -> 1 MLP (ReLU or
// SiLU hidden layers, softplus output) mapping per-cell features to an eddy
// viscosity.  FP32 master weights,
// one thread per sample; the weight gradient is reduced deterministically
// (per-block partial sums in a fixed order, then a fixed-order sum over blocks).
//
// Parameter vector (LBM_MLP_NPARAM floats): W1[32][5], b1[32], W2[32][32],
// b2[32], w3[32], b3.
#include <math.h>

#include "host.h"
#include "mlp.cuh"

namespace lbm {
namespace {

constexpr int NI = LBM_MLP_IN, NH = LBM_MLP_HID;
constexpr int OW1 = 0, OB1 = OW1 + NH * NI, OW2 = OB1 + NH, OB2 = OW2 + NH * NH, OW3 = OB2 + NH, OB3 = OW3 + NH;
static_assert(OB3 + 1 == LBM_MLP_NPARAM, "parameter layout");
constexpr int BT = 64; // samples per block (static shared memory < 48 KB)

__device__ __forceinline__ float sigm(float x)
{
    return 1.0f / (1.0f + expf(-x));
}
// ReLU and its derivative (1 for a > 0, else 0)
__device__ __forceinline__ float relu(float a)
{
    return fmaxf(a, 0.0f);
}
__device__ __forceinline__ float relu_grad(float a)
{
    return a > 0.0f ? 1.0f : 0.0f;
}
// SiLU a sigmoid(a) and its derivative sigmoid(a) (1 + a (1 - sigmoid(a)))
__device__ __forceinline__ float silu(float a)
{
    return a * sigm(a);
}
__device__ __forceinline__ float silu_grad(float a)
{
    const float s = sigm(a);
    return s * (1.0f + a * (1.0f - s));
}
template <int ACT> __device__ __forceinline__ float act(float a)
{
    return ACT == LBM_MLP_ACT_SILU ? silu(a) : relu(a);
}
template <int ACT> __device__ __forceinline__ float act_grad(float a)
{
    return ACT == LBM_MLP_ACT_SILU ? silu_grad(a) : relu_grad(a);
}
__device__ __forceinline__ float softplus(float x)
{
    return x > 20.0f ? x : log1pf(expf(x));
}

// Forward of one sample; keeps pre-activations for the backward pass.
template <int ACT>
__device__ __forceinline__ float forward1(const float *P, const float *x, float (&a1)[NH], float (&h1)[NH],
                                          float (&a2)[NH], float (&h2)[NH], float &z)
{
#pragma unroll
    for (int i = 0; i < NH; ++i) {
        float s = P[OB1 + i];
#pragma unroll
        for (int k = 0; k < NI; ++k)
            s = fmaf(P[OW1 + i * NI + k], x[k], s);
        a1[i] = s;
        h1[i] = act<ACT>(s);
    }
#pragma unroll
    for (int i = 0; i < NH; ++i) {
        float s = P[OB2 + i];
#pragma unroll
        for (int k = 0; k < NH; ++k)
            s = fmaf(P[OW2 + i * NH + k], h1[k], s);
        a2[i] = s;
        h2[i] = act<ACT>(s);
    }
    float s = P[OB3];
#pragma unroll
    for (int k = 0; k < NH; ++k)
        s = fmaf(P[OW3 + k], h2[k], s);
    z = s;
    return softplus(s);
}

template <int ACT>
__global__ void __launch_bounds__(BT) mlp_forward_kernel(const float *params, const float *x, float *y, int n)
{
    __shared__ float P[LBM_MLP_NPARAM];
    for (int i = threadIdx.x; i < LBM_MLP_NPARAM; i += BT)
        P[i] = params[i];
    __syncthreads();
    const int s = blockIdx.x * BT + threadIdx.x;
    if (s >= n)
        return;
    float xi[NI], a1[NH], h1[NH], a2[NH], h2[NH], z;
#pragma unroll
    for (int k = 0; k < NI; ++k)
        xi[k] = x[(long long)s * NI + k];
    y[s] = forward1<ACT>(P, xi, a1, h1, a2, h2, z);
}

// Per-block partial gradient of L = sum_s w_s (y_s - t_s)^2 / sum_s w_s
// (w_s = 1 when weights are null), and the partial loss sum.
template <int ACT>
__global__ void __launch_bounds__(BT) mlp_grad_kernel(const float *params, const float *x, const float *t,
                                                      const float *w, int n, float inv_norm, float *partial)
{
    __shared__ float P[LBM_MLP_NPARAM];
    __shared__ float sh1[BT][NH + 1], sd2[BT][NH + 1]; // per-sample h1 and dL/da2
    __shared__ float sx[BT][NI], sd1[BT][NH + 1];
    __shared__ float sdz[BT], sloss[BT];
    for (int i = threadIdx.x; i < LBM_MLP_NPARAM; i += BT)
        P[i] = params[i];
    __syncthreads();
    const int tid = threadIdx.x;
    const int s = blockIdx.x * BT + tid;
    float xi[NI], a1[NH], h1[NH], a2[NH], h2[NH], z;
    float dz = 0.0f, loss = 0.0f;
    if (s < n) {
#pragma unroll
        for (int k = 0; k < NI; ++k)
            xi[k] = x[(long long)s * NI + k];
        const float yv = forward1<ACT>(P, xi, a1, h1, a2, h2, z);
        const float ws = w ? w[s] : 1.0f;
        const float e = yv - t[s];
        loss = ws * e * e * inv_norm;
        dz = 2.0f * ws * e * inv_norm * sigm(z); // d softplus / dz = sigmoid
    } else {
#pragma unroll
        for (int k = 0; k < NI; ++k)
            xi[k] = 0.0f;
#pragma unroll
        for (int i = 0; i < NH; ++i)
            a1[i] = h1[i] = a2[i] = h2[i] = 0.0f;
    }
    // dL/da2 = dz * w3 * act'(a2)
    float d2[NH];
#pragma unroll
    for (int i = 0; i < NH; ++i)
        d2[i] = dz * P[OW3 + i] * act_grad<ACT>(a2[i]);
    // dL/da1 = (W2^T d2) * act'(a1)
#pragma unroll
    for (int k = 0; k < NH; ++k) {
        float g = 0.0f;
#pragma unroll
        for (int i = 0; i < NH; ++i)
            g = fmaf(P[OW2 + i * NH + k], d2[i], g);
        sd1[tid][k] = g * act_grad<ACT>(a1[k]);
    }
#pragma unroll
    for (int i = 0; i < NH; ++i) {
        sh1[tid][i] = h1[i];
        sd2[tid][i] = d2[i];
    }
#pragma unroll
    for (int k = 0; k < NI; ++k)
        sx[tid][k] = xi[k];
    sdz[tid] = dz;
    sloss[tid] = loss;
    __syncthreads();
    float *out = partial + (long long)blockIdx.x * (LBM_MLP_NPARAM + 1);
    // W2 (NH x NH) and b2: thread p sums parameter p over the block's samples in order
    for (int p = tid; p < NH * NH + NH; p += BT) {
        float acc = 0.0f;
        if (p < NH * NH) {
            const int i = p / NH, k = p % NH;
            for (int j = 0; j < BT; ++j)
                acc = fmaf(sd2[j][i], sh1[j][k], acc);
            out[OW2 + p] = acc;
        } else {
            const int i = p - NH * NH;
            for (int j = 0; j < BT; ++j)
                acc += sd2[j][i];
            out[OB2 + i] = acc;
        }
    }
    // W1 (NH x NI) and b1
    for (int p = tid; p < NH * NI + NH; p += BT) {
        float acc = 0.0f;
        if (p < NH * NI) {
            const int i = p / NI, k = p % NI;
            for (int j = 0; j < BT; ++j)
                acc = fmaf(sd1[j][i], sx[j][k], acc);
            out[OW1 + p] = acc;
        } else {
            const int i = p - NH * NI;
            for (int j = 0; j < BT; ++j)
                acc += sd1[j][i];
            out[OB1 + i] = acc;
        }
    }
    __syncthreads();
    // w3 and b3: dz * h2 (store h2 into sh1 now that the W2 pass is done)
#pragma unroll
    for (int i = 0; i < NH; ++i)
        sh1[tid][i] = h2[i];
    __syncthreads();
    for (int p = tid; p < NH + 2; p += BT) {
        float acc = 0.0f;
        if (p < NH) {
            for (int j = 0; j < BT; ++j)
                acc = fmaf(sdz[j], sh1[j][p], acc);
            out[OW3 + p] = acc;
        } else if (p == NH) {
            for (int j = 0; j < BT; ++j)
                acc += sdz[j];
            out[OB3] = acc;
        } else {
            for (int j = 0; j < BT; ++j)
                acc += sloss[j];
            out[LBM_MLP_NPARAM] = acc;
        }
    }
}

// grad[p] = sum over blocks of partial[b][p] (fixed order); loss likewise.
__global__ void mlp_reduce_kernel(const float *partial, int nblocks, float *grad, float *loss)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > LBM_MLP_NPARAM)
        return;
    float acc = 0.0f;
    for (int b = 0; b < nblocks; ++b)
        acc += partial[(long long)b * (LBM_MLP_NPARAM + 1) + p];
    if (p < LBM_MLP_NPARAM)
        grad[p] = acc;
    else if (loss)
        *loss = acc;
}

__global__ void mlp_adam_kernel(float *params, const float *grad, float *m, float *v, int np, float lr, float b1,
                                float b2, float eps, float c1, float c2)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np)
        return;
    const float g = grad[p];
    const float mm = b1 * m[p] + (1.0f - b1) * g;
    const float vv = b2 * v[p] + (1.0f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    params[p] -= lr * (mm * c1) / (sqrtf(vv * c2) + eps);
}

// Packing: W1 with in_scale folded in and b1 as column 5, W2, w3 in BF16; b2, b3
// and out_scale in FP32.  For SiLU the first two layers are halved (the
// inference kernel evaluates silu(a) = h (1 + tanh h) on h = a / 2).
__global__ void mlp_pack_kernel(const float *P, int act, const float *in_scale, float out_scale, MlpPacked *W)
{
    const int tid = threadIdx.x;
    const float hs = act == LBM_MLP_ACT_SILU ? 0.5f : 1.0f;
    for (int i = tid; i < 32 * 16; i += blockDim.x) {
        const int n = i / 16, k = i % 16;
        float v = 0.0f;
        if (k < NI)
            v = P[OW1 + n * NI + k] * in_scale[k];
        else if (k == NI)
            v = P[OB1 + n];
        W->w1[n][k] = __float2bfloat16_rn(hs * v);
    }
    for (int i = tid; i < 32 * 32; i += blockDim.x)
        W->w2[i / 32][i % 32] = __float2bfloat16_rn(hs * P[OW2 + i]);
    for (int i = tid; i < 8 * 32; i += blockDim.x)
        W->w3[i / 32][i % 32] = __float2bfloat16_rn(i < 32 ? P[OW3 + i] : 0.0f);
    for (int i = tid; i < 32; i += blockDim.x)
        W->b2[i] = hs * P[OB2 + i];
    if (tid == 0) {
        W->b3 = P[OB3];
        W->out_scale = out_scale;
        W->act = act;
    }
}

bool act_ok(int act)
{
    return act == LBM_MLP_ACT_RELU || act == LBM_MLP_ACT_SILU;
}

} // namespace
} // namespace lbm

using namespace lbm;

extern "C" {

size_t lbm_mlp_workspace_bytes(int n)
{
    if (n < 1)
        return 0;
    const size_t nb = (size_t)(n + BT - 1) / BT;
    return nb * (LBM_MLP_NPARAM + 1) * sizeof(float);
}

int lbm_mlp_forward_act(const float *params, int act, const float *x, float *y, int n, void *stream)
{
    if (!params || !x || !y || n < 0 || !act_ok(act))
        return LBM_ERR_ARG;
    if (n == 0)
        return LBM_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (act == LBM_MLP_ACT_SILU)
        mlp_forward_kernel<LBM_MLP_ACT_SILU><<<(n + BT - 1) / BT, BT, 0, s>>>(params, x, y, n);
    else
        mlp_forward_kernel<LBM_MLP_ACT_RELU><<<(n + BT - 1) / BT, BT, 0, s>>>(params, x, y, n);
    return status(cudaGetLastError());
}

int lbm_mlp_forward(const float *params, const float *x, float *y, int n, void *stream)
{
    return lbm_mlp_forward_act(params, LBM_MLP_ACT_RELU, x, y, n, stream);
}

int lbm_mlp_grad_act(const float *params, int act, const float *x, const float *target, const float *weight, int n,
                     float *grad, float *loss, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!params || !x || !target || !grad || !workspace || n < 1 || !act_ok(act))
        return LBM_ERR_ARG;
    if (workspace_bytes < lbm_mlp_workspace_bytes(n))
        return LBM_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = (n + BT - 1) / BT;
    float *part = static_cast<float *>(workspace);
    // the loss is normalised by the number of samples (or the sum of the weights,
    // which the caller passes through by scaling them); 1/n here
    if (act == LBM_MLP_ACT_SILU)
        mlp_grad_kernel<LBM_MLP_ACT_SILU><<<nb, BT, 0, s>>>(params, x, target, weight, n, 1.0f / (float)n, part);
    else
        mlp_grad_kernel<LBM_MLP_ACT_RELU><<<nb, BT, 0, s>>>(params, x, target, weight, n, 1.0f / (float)n, part);
    mlp_reduce_kernel<<<(LBM_MLP_NPARAM + 1 + 255) / 256, 256, 0, s>>>(part, nb, grad, loss);
    return status(cudaGetLastError());
}

int lbm_mlp_grad(const float *params, const float *x, const float *target, const float *weight, int n, float *grad,
                 float *loss, void *workspace, size_t workspace_bytes, void *stream)
{
    return lbm_mlp_grad_act(params, LBM_MLP_ACT_RELU, x, target, weight, n, grad, loss, workspace, workspace_bytes,
                            stream);
}

int lbm_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float beta1, float beta2,
                 float eps, void *stream)
{
    if (!params || !grad || !m || !v || step < 1)
        return LBM_ERR_ARG;
    const float c1 = 1.0f / (1.0f - powf(beta1, (float)step));
    const float c2 = 1.0f / (1.0f - powf(beta2, (float)step));
    mlp_adam_kernel<<<(LBM_MLP_NPARAM + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        params, grad, m, v, LBM_MLP_NPARAM, lr, beta1, beta2, eps, c1, c2);
    return status(cudaGetLastError());
}

int lbm_mlp_pack_act(const float *params, int act, const float *in_scale, float out_scale, void *packed,
                     void *stream)
{
    if (!params || !in_scale || !packed || !(out_scale > 0.0f) || !act_ok(act))
        return LBM_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(packed) & 15u) != 0)
        return LBM_ERR_ARG;
    mlp_pack_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, act, in_scale, out_scale,
                                                                      static_cast<MlpPacked *>(packed));
    return status(cudaGetLastError());
}

int lbm_mlp_pack(const float *params, const float *in_scale, float out_scale, void *packed, void *stream)
{
    return lbm_mlp_pack_act(params, LBM_MLP_ACT_RELU, in_scale, out_scale, packed, stream);
}

} // extern "C"
