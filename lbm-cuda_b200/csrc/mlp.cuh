// Learned closure, inference side: the 5 -> 32 -> 32 -> 1 MLP (ReLU or SiLU
// hidden layers, softplus output) evaluated by one warp for 64 cells (two per
// lane) on the tensor cores with mma.sync.m16n8k16 (BF16 inputs, FP32
// accumulation).
//
// Packed weights (MlpPacked, written by lbm_mlp_pack_act):
//   w1[32][16]  first layer, feature k (k < 5) pre-multiplied by in_scale[k],
//               column 5 holds b1 (the staged features carry a constant 1
//               there), columns 6..15 zero;
//   w2[32][32], w3[8][32] (row 0 = w3, rows 1..7 zero), b2[32], b3, out_scale;
//   act: the activation the block was packed for;
//   BF16 weights; b2, b3 and out_scale FP32.  For SiLU the first two layers
//   (w1 with its bias column, w2, b2) are packed halved, see below.
//
// Per warp: the 64 feature rows are staged as BF16 in 1 KB of shared memory
// (row c = cell c = 2 lane + n, 8 values: 5 features, 1, 0, 0) and read as A
// fragments; a layer's accumulators become the next layer's A fragments in
// registers (the m16n8k16 accumulator layout of two adjacent 8-column tiles is
// the A layout of one 16-wide k tile).  The activation is applied while the
// FP32 accumulators are packed to BF16x2:
//   ReLU: the packing conversion itself (cvt.rn.relu.bf16x2.f32), no extra
//         instruction;
//   SiLU: the accumulators hold h = a / 2 (halved weights), and
//         silu(a) = a sigmoid(a) = h (1 + tanh h): the packing, one
//         tanh.approx.bf16x2 and one fma.rn.bf16x2 per pair.  The tanh runs on
//         the transcendental unit (8 per clock per SM against about 60 for the
//         conversion), which bounds the SiLU kernel.
// The accumulators start from the bias (or zero) passed as the MMA's C operand.
// The output z of a cell is nu_t = out_scale softplus(z).
#pragma once

#include "collide.cuh"

namespace lbm {

struct MlpPacked {
    __nv_bfloat16 w1[32][16];
    __nv_bfloat16 w2[32][32];
    __nv_bfloat16 w3[8][32];
    float b2[32];
    float b3;
    float out_scale;
    int act; // LBM_MLP_ACT_* the block was packed for
};
static_assert(sizeof(MlpPacked) <= LBM_MLP_PACKED_BYTES, "packed MLP size");

// Per-thread B fragments and biases (loaded once per warp).
struct MlpFrag {
    uint32_t b1[4][2];    // [n tile][reg]
    uint32_t b2[4][2][2]; // [n tile][k tile][reg]
    uint32_t b3[2][2];    // [k tile][reg]
    float c2[4][2];       // b2 at this thread's two columns of each n tile
    float b3v, out_scale;
};

__device__ __forceinline__ uint32_t ld_bf16x2(const __nv_bfloat16 *p)
{
    return *reinterpret_cast<const uint32_t *>(p);
}

__device__ __forceinline__ void mlp_load_frag(const MlpPacked *W, MlpFrag &F, int lane)
{
    const int g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
        const int n = nt * 8 + g;
        F.b1[nt][0] = ld_bf16x2(&W->w1[n][2 * t]);
        F.b1[nt][1] = ld_bf16x2(&W->w1[n][2 * t + 8]);
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            F.b2[nt][kt][0] = ld_bf16x2(&W->w2[n][kt * 16 + 2 * t]);
            F.b2[nt][kt][1] = ld_bf16x2(&W->w2[n][kt * 16 + 2 * t + 8]);
        }
        F.c2[nt][0] = W->b2[nt * 8 + 2 * t];
        F.c2[nt][1] = W->b2[nt * 8 + 2 * t + 1];
    }
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
        F.b3[kt][0] = ld_bf16x2(&W->w3[g][kt * 16 + 2 * t]);
        F.b3[kt][1] = ld_bf16x2(&W->w3[g][kt * 16 + 2 * t + 8]);
    }
    F.b3v = W->b3;
    F.out_scale = W->out_scale;
}

// d = a b + c (m16n8k16, BF16 inputs, FP32 accumulators)
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1, float c0,
                                         float c1, float c2, float c3)
{
    asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, "
        "{%8, %9}, {%10, %11, %12, %13};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1), "f"(c0), "f"(c1), "f"(c2), "f"(c3));
}

// BF16 pair {lo, hi} (lo in the low half).
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// BF16 pair {relu(lo), relu(hi)}: the activation and the packing in one conversion.
__device__ __forceinline__ uint32_t relu_bf16x2(float lo, float hi)
{
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
    return d;
}

// The next layer's A fragment from two accumulators: the activation and the
// packing to BF16x2 (lo in the low half).
template <int ACT> __device__ __forceinline__ uint32_t act_bf16x2(float lo, float hi)
{
    if constexpr (ACT == LBM_MLP_ACT_SILU) {
        const uint32_t h = pack_bf16x2(lo, hi); // h = a / 2
        uint32_t t, d;
        asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
        asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(d) : "r"(h), "r"(t)); // h tanh h + h
        return d;
    } else {
        return relu_bf16x2(lo, hi);
    }
}

// Eddy viscosity of the lane's two cells from their features x[n][5].  Warp-
// collective: every lane of the warp calls it together.  stage: 64 x 8 BF16
// (1 KB) and zbuf: 64 floats of this warp's shared memory.
template <int ACT>
__device__ __forceinline__ void mlp_nu_t(const MlpFrag &F, const float (&x)[2][5], __nv_bfloat16 *stage, float *zbuf,
                                         int lane, float (&nu)[2])
{
    const int g = lane >> 2, t = lane & 3;
    // stage rows 2 lane and 2 lane + 1: features, the constant 1, zeros
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        uint4 v;
        v.x = pack_bf16x2(x[n][0], x[n][1]);
        v.y = pack_bf16x2(x[n][2], x[n][3]);
        v.z = pack_bf16x2(x[n][4], 1.0f);
        v.w = 0u;
        *reinterpret_cast<uint4 *>(stage + (2 * lane + n) * 8) = v;
    }
    __syncwarp();
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
        // layer 1: A = staged rows (k 0..7 from the stage, 8..15 zero)
        uint32_t a[4];
        const int r0 = mt * 16 + g;
        a[0] = ld_bf16x2(stage + r0 * 8 + 2 * t);
        a[1] = ld_bf16x2(stage + (r0 + 8) * 8 + 2 * t);
        a[2] = 0u;
        a[3] = 0u;
        float h1[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
            mma_bf16(h1[nt], a, F.b1[nt][0], F.b1[nt][1], 0.0f, 0.0f, 0.0f, 0.0f);
        // activation -> layer-2 A fragments (k tile kt = hidden 16 kt .. 16 kt + 15)
        uint32_t a2[2][4];
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            a2[kt][0] = act_bf16x2<ACT>(h1[2 * kt][0], h1[2 * kt][1]);
            a2[kt][1] = act_bf16x2<ACT>(h1[2 * kt][2], h1[2 * kt][3]);
            a2[kt][2] = act_bf16x2<ACT>(h1[2 * kt + 1][0], h1[2 * kt + 1][1]);
            a2[kt][3] = act_bf16x2<ACT>(h1[2 * kt + 1][2], h1[2 * kt + 1][3]);
        }
        float h2[4][4];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            float t2[4];
            mma_bf16(t2, a2[0], F.b2[nt][0][0], F.b2[nt][0][1], F.c2[nt][0], F.c2[nt][1], F.c2[nt][0], F.c2[nt][1]);
            mma_bf16(h2[nt], a2[1], F.b2[nt][1][0], F.b2[nt][1][1], t2[0], t2[1], t2[2], t2[3]);
        }
        uint32_t a3[2][4];
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            a3[kt][0] = act_bf16x2<ACT>(h2[2 * kt][0], h2[2 * kt][1]);
            a3[kt][1] = act_bf16x2<ACT>(h2[2 * kt][2], h2[2 * kt][3]);
            a3[kt][2] = act_bf16x2<ACT>(h2[2 * kt + 1][0], h2[2 * kt + 1][1]);
            a3[kt][3] = act_bf16x2<ACT>(h2[2 * kt + 1][2], h2[2 * kt + 1][3]);
        }
        float z0[4], z[4];
        mma_bf16(z0, a3[0], F.b3[0][0], F.b3[0][1], F.b3v, 0.0f, F.b3v, 0.0f);
        mma_bf16(z, a3[1], F.b3[1][0], F.b3[1][1], z0[0], z0[1], z0[2], z0[3]);
        if (t == 0) { // column 0 of rows g and g + 8
            zbuf[r0] = z[0];
            zbuf[r0 + 8] = z[2];
        }
    }
    __syncwarp();
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        const float zz = zbuf[2 * lane + n];
        const float sp = zz > 20.0f ? zz : __logf(1.0f + __expf(zz));
        nu[n] = F.out_scale * sp;
    }
    __syncwarp(); // the stage and zbuf are reused by the next call
}

// Collision of a lane's two cells with the learned eddy viscosity (warp-
// collective): Zou-He where inlet0 / inlet1 (kZh), the moments and the reference
// clamps as collide_pair, the MLP features of both cells, then MRT with the
// stress-moment rate 1 / (tau0 + 3 nu_t) (s_nu at the inlet, as Smagorinsky).
template <class Ph, bool kZh>
__device__ __forceinline__ void collide_pair_mlp(float2 (&f)[9], bool inlet0, bool inlet1, float lu, const Phys &k,
                                                 const MlpFrag &F, __nv_bfloat16 *stage, float *zbuf, int lane,
                                                 float2 &r, float2 &u, float2 &v)
{
    static_assert(Ph::kMlp && Ph::kMrt && !Ph::kRefOrder, "MRT with the learned closure");
    float2 rz = bc2(1.0f);
    if (kZh) {
        float zr[2];
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            const bool in = n == 0 ? inlet0 : inlet1;
            float g[9];
#pragma unroll
            for (int q = 0; q < 9; ++q)
                g[q] = n == 0 ? f[q].x : f[q].y;
            const float rr = (g[0] + g[2] + g[4] + 2.0f * (g[3] + g[6] + g[7])) / (1.0f - lu);
            const float a = 0.16666666666f * rr * lu;
            const float h = 0.5f * (g[2] - g[4]);
            const float z1 = g[3] + 0.666666667f * rr * lu, z5 = g[7] - h + a, z8 = g[6] + h + a;
            if (n == 0) {
                f[1].x = in ? z1 : f[1].x;
                f[5].x = in ? z5 : f[5].x;
                f[8].x = in ? z8 : f[8].x;
            } else {
                f[1].y = in ? z1 : f[1].y;
                f[5].y = in ? z5 : f[5].y;
                f[8].y = in ? z8 : f[8].y;
            }
            zr[n] = rr;
        }
        rz = make_float2(zr[0], zr[1]);
    }
    const float2 a13 = add2(f[1], f[3]), a24 = add2(f[2], f[4]), a57 = add2(f[5], f[7]), a68 = add2(f[6], f[8]);
    const float2 b13 = sub2(f[1], f[3]), b24 = sub2(f[2], f[4]), b57 = sub2(f[5], f[7]), b68 = sub2(f[6], f[8]);
    const float2 s14 = add2(a13, a24), s58 = add2(a57, a68);
    const float2 rho = add2(add2(f[0], s14), s58);
    const float2 e = sub2(b57, b68), g = add2(b57, b68);
    const float2 jx = add2(b13, e), jy = add2(b24, g);
    const float2 rinv = rcp2(rho);
    u = mul2(jx, rinv);
    v = mul2(jy, rinv);
    r = rho;
    if (Ph::kClampU) {
        u.x = fminf(0.4f, fmaxf(-0.4f, u.x));
        u.y = fminf(0.4f, fmaxf(-0.4f, u.y));
        v.x = fminf(0.4f, fmaxf(-0.4f, v.x));
        v.y = fminf(0.4f, fmaxf(-0.4f, v.y));
        r.x = fminf(1.5f, fmaxf(0.0f, rho.x));
        r.y = fminf(1.5f, fmaxf(0.0f, rho.y));
    }
    if (kZh) {
        r.x = inlet0 ? rz.x : r.x;
        r.y = inlet1 ? rz.y : r.y;
        u.x = inlet0 ? lu : u.x;
        u.y = inlet1 ? lu : u.y;
        v.x = inlet0 ? 0.0f : v.x;
        v.y = inlet1 ? 0.0f : v.y;
    }
    const float2 uu = mul2(u, u), vv = mul2(v, v);
    const float2 m3 = mul2(r, u), m5 = mul2(r, v);
    const float2 n7 = fma2(r, sub2(vv, uu), sub2(a13, a24));
    const float2 n8 = sub2(sub2(a57, a68), mul2(m3, v));
    const float2 t3 = mul2(bc2(3.0f), add2(uu, vv));
    const float2 m1 = fma2(bc2(-4.0f), f[0], sub2(add2(s58, s58), s14));
    const float2 ne = fma2(r, sub2(bc2(2.0f), t3), m1);
    // features: n7, n8, ne, |(n7, n8)|, rho - 1
    const float2 qq = fma2(n7, n7, mul2(n8, n8));
    float x[2][5];
    x[0][0] = n7.x, x[0][1] = n8.x, x[0][2] = ne.x, x[0][3] = sqrtf(qq.x), x[0][4] = r.x - 1.0f;
    x[1][0] = n7.y, x[1][1] = n8.y, x[1][2] = ne.y, x[1][3] = sqrtf(qq.y), x[1][4] = r.y - 1.0f;
    float nu[2];
    mlp_nu_t<Ph::kMlpAct>(F, x, stage, zbuf, lane, nu);
    float2 s = make_float2(__fdividef(1.0f, k.tau0 + 3.0f * nu[0]), __fdividef(1.0f, k.tau0 + 3.0f * nu[1]));
    if (kZh) {
        s.x = inlet0 ? k.s_nu : s.x;
        s.y = inlet1 ? k.s_nu : s.y;
    }
    float2 d0 = bc2(0.0f), d3 = bc2(0.0f), d5 = bc2(0.0f);
    if (Ph::kClampU || kZh) {
        d0 = sub2(rho, r);
        d3 = sub2(jx, m3);
        d5 = sub2(jy, m5);
    }
    const float2 m2 = fma2(bc2(4.0f), f[0], fma2(bc2(-2.0f), s14, s58));
    const float2 d1 = mul2(bc2(k.s_e), ne);
    const float2 d2 = mul2(bc2(k.s_eps), fma2(r, add2(t3, bc2(-1.0f)), m2));
    const float2 d4 = mul2(bc2(k.s_q), add2(fma2(bc2(-2.0f), b13, e), m3));
    const float2 d6 = mul2(bc2(k.s_q), add2(fma2(bc2(-2.0f), b24, g), m5));
    const float2 d7 = mul2(s, n7), d8 = mul2(s, n8);
    const float2 Z = mul2(add2(sub2(d0, d1), d2), bc2(0.1111111111f));
    const float2 A = mul2(fma2(bc2(4.0f), d0, fma2(bc2(-2.0f), d2, mul2(d1, bc2(-1.0f)))), bc2(0.02777777778f));
    const float2 D = mul2(fma2(bc2(4.0f), d0, fma2(bc2(2.0f), d1, d2)), bc2(0.02777777778f));
    const float2 Bx = mul2(sub2(d3, d4), bc2(0.16666666666f));
    const float2 By = mul2(sub2(d5, d6), bc2(0.16666666666f));
    const float2 Ex = mul2(fma2(bc2(2.0f), d3, d4), bc2(0.08333333333f));
    const float2 Ey = mul2(fma2(bc2(2.0f), d5, d6), bc2(0.08333333333f));
    const float2 AP = fma2(bc2(0.25f), d7, A), AM = fma2(bc2(-0.25f), d7, A);
    const float2 DP = fma2(bc2(0.25f), d8, D), DM = fma2(bc2(-0.25f), d8, D);
    const float2 EP = add2(Ex, Ey), EM = sub2(Ex, Ey);
    f[0] = sub2(f[0], Z);
    f[1] = sub2(f[1], add2(AP, Bx));
    f[3] = sub2(f[3], sub2(AP, Bx));
    f[2] = sub2(f[2], add2(AM, By));
    f[4] = sub2(f[4], sub2(AM, By));
    f[5] = sub2(f[5], add2(DP, EP));
    f[7] = sub2(f[7], sub2(DP, EP));
    f[6] = sub2(f[6], sub2(DM, EM));
    f[8] = sub2(f[8], add2(DM, EM));
    if (Ph::kClampF) {
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            f[q].x = fminf(10.0f, fmaxf(0.0f, f[q].x));
            f[q].y = fminf(10.0f, fmaxf(0.0f, f[q].y));
        }
    }
}

} // namespace lbm
