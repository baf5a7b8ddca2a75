// Per-cell D2Q9 physics: Zou-He inlet, moments, Smagorinsky, MRT and BGK relaxation.
//
// The arithmetic follows the reference kernels (the library is compiled with
// -use_fast_math, as the reference drivers compile theirs, lbm_mine2.py:69):
//   Zou-He with the cosine ramp      lbm_core4.cu:46-57
//   moments, clamps                  lbm_core4.cu:129-144
//   Smagorinsky tau_eff              lbm_core4.cu:171-177
//   MRT relax + inverse transform    lbm_core4.cu:150-199
//   BGK                              lbm_core_smemaa.cu:206-212
#pragma once

#include "common.cuh"

namespace lbm {

// Runtime constants of one launch.
struct Phys {
    float s_nu;   // stress relaxation rate 1/tau (tau_inv of the reference)
    float s_e;    // energy
    float s_eps;  // energy square
    float s_q;    // heat flux
    float tau0;   // 1 / s_nu
    float cs2x18; // 18 Cs^2 (Smagorinsky)
    float u_in;   // inlet velocity
    float u_lid;  // moving-wall x velocity (Ladd)
    int H;        // domain height (ramp profile)
    int ramp;     // 1: cosine-ramped inlet profile (reference), 0: flat
    int flags;    // PF_* (used by PhysRuntime only)
    const void *mlp; // packed MLP weights (Physics::kMlp)
};

enum : int { PF_MRT = 1, PF_SMAG = 2, PF_CLAMPU = 4, PF_CLAMPF = 8, PF_INLET_SMAG = 16 };

// Compile-time physics variant.
//   kMrt       MRT (else BGK)
//   kSmag      Smagorinsky-corrected stress rate in the interior
//   kClampU    the reference's velocity/density clamps |u| <= 0.4, rho in [0, 1.5]
//              (lbm_core4.cu:142-144)
//   kClampF    the reference's population clamp f in [0, 10] (lbm_core4.cu:203,
//              lbm_core_smemaa.cu:220)
//   kInletSmag Smagorinsky also at the Zou-He inlet (the reference does not)
//   kRefOrder  evaluate in the reference's order (drop-ins: rounding closest to the
//              reference kernels); otherwise the leaner order of collide_bf
//   kMlpAct    activation of the learned closure's hidden layers (LBM_MLP_ACT_*)
template <bool kMrt_, bool kSmag_, bool kClampU_, bool kClampF_, bool kInletSmag_, bool kRefOrder_ = false,
          bool kMlp_ = false, int kMlpAct_ = LBM_MLP_ACT_RELU>
struct Physics {
    static constexpr bool kRuntime = false;
    static constexpr bool kMlp = kMlp_; // learned eddy viscosity in place of Smagorinsky
    static constexpr int kMlpAct = kMlpAct_;
    static constexpr bool kRefOrder = kRefOrder_;
    static constexpr bool kMrt = kMrt_;
    static constexpr bool kSmag = kSmag_;
    static constexpr bool kClampU = kClampU_;
    static constexpr bool kClampF = kClampF_;
    static constexpr bool kInletSmag = kInletSmag_;
};

// lbm_core4.cu semantics: MRT + Smagorinsky, clamps, plain MRT at the inlet.
using PhysCore4 = Physics<true, true, true, true, false, true>;
// lbm_core_smemaa*.cu semantics: BGK, population clamp only.
using PhysBgkRef = Physics<false, false, false, true, false, true>;
// General solver variants.
using PhysMrtSmagClamp = Physics<true, true, true, true, false>; // = PhysCore4 with runtime rates and Cs
using PhysMrtSmag = Physics<true, true, false, false, false>;
using PhysMrt = Physics<true, false, false, false, false>;
using PhysBgk = Physics<false, false, false, false, false>;
using PhysMrtMlp = Physics<true, false, false, false, false, false, true>; // MRT + learned closure (ReLU)
using PhysMrtMlpSilu = Physics<true, false, false, false, false, false, true, LBM_MLP_ACT_SILU>; // SiLU network
// The same choices read from Phys::flags (uniform branches; non-hot paths).
struct PhysRuntime {
    static constexpr bool kRuntime = true;
    static constexpr bool kMlp = false;
    static constexpr int kMlpAct = LBM_MLP_ACT_RELU;
    static constexpr bool kRefOrder = true;
    static constexpr bool kMrt = true, kSmag = true, kClampU = true, kClampF = true, kInletSmag = true;
};

__device__ __forceinline__ float inlet_u(const Phys &k, int y)
{
    if (!k.ramp)
        return k.u_in;
    float d = fminf((float)y, (float)(k.H - 1 - y));
    float sm = 1.0f;
    if (d < 50.0f)
        sm = 0.5f * (1.0f - cosf(3.14159f * d / 50.0f));
    return k.u_in * sm;
}

// Zou-He velocity inlet: overwrites f1, f5, f8 and returns rho (lbm_core4.cu:54-57).
__device__ __forceinline__ float zou_he(float (&f)[9], float lu)
{
    float rho = (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7])) / (1.0f - lu);
    float a = 0.16666666666f * rho * lu;
    float h = 0.5f * (f[2] - f[4]);
    f[1] = f[3] + 0.666666667f * rho * lu;
    f[5] = f[7] - h + a;
    f[8] = f[6] + h + a;
    return rho;
}

// Smagorinsky stress relaxation rate from the non-equilibrium stress moments.
__device__ __forceinline__ float smag_rate(const float (&f)[9], float r, float u, float v, const Phys &k)
{
    float n7 = (f[1] - f[2] + f[3] - f[4]) - r * (u * u - v * v);
    float n8 = (f[5] - f[6] + f[7] - f[8]) - r * u * v;
    float Q = sqrtf(n7 * n7 + n8 * n8 + 1e-8f);
    float tau_eff = 0.5f * (k.tau0 + sqrtf(k.tau0 * k.tau0 + k.cs2x18 * Q / r));
    return 1.0f / tau_eff;
}

// MRT relaxation in the Lallemand-Luo basis and inverse transform.  m0 = r,
// m3 = r u and m5 = r v are the values chosen by the caller.
__device__ __forceinline__ void mrt_relax(float (&f)[9], float r, float u, float v, float s_e, float s_eps, float s_q,
                                          float s_nu)
{
    const float f14 = f[1] + f[2] + f[3] + f[4];
    const float f58 = f[5] + f[6] + f[7] + f[8];
    float m1 = -4.0f * f[0] + 2.0f * f58 - f14;
    float m2 = 4.0f * f[0] + f58 - 2.0f * f14;
    const float m3 = r * u;
    float m4 = -2.0f * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
    const float m5 = r * v;
    float m6 = -2.0f * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
    float m7 = f[1] - f[2] + f[3] - f[4];
    float m8 = f[5] - f[6] + f[7] - f[8];
    const float usq = u * u + v * v;
    m1 -= s_e * (m1 - (3.0f * usq - 2.0f) * r);
    m2 -= s_eps * (m2 - (1.0f - 3.0f * usq) * r);
    m4 -= s_q * (m4 + m3);
    m6 -= s_q * (m6 + m5);
    m7 -= s_nu * (m7 - r * (u * u - v * v));
    m8 -= s_nu * (m8 - r * u * v);
    const float inv9 = 0.1111111111f, inv36 = 0.02777777778f;
    const float t0 = r - m1 + m2;
    const float t1 = 4.0f * r - m1 - 2.0f * m2;
    const float t2 = 4.0f * r + 2.0f * m1 + m2;
    f[0] = t0 * inv9;
    f[1] = (t1 + 6.0f * m3 - 6.0f * m4 + 9.0f * m7) * inv36;
    f[2] = (t1 + 6.0f * m5 - 6.0f * m6 - 9.0f * m7) * inv36;
    f[3] = (t1 - 6.0f * m3 + 6.0f * m4 + 9.0f * m7) * inv36;
    f[4] = (t1 - 6.0f * m5 + 6.0f * m6 - 9.0f * m7) * inv36;
    f[5] = (t2 + 6.0f * m3 + 3.0f * m4 + 6.0f * m5 + 3.0f * m6 + 9.0f * m8) * inv36;
    f[6] = (t2 - 6.0f * m3 - 3.0f * m4 + 6.0f * m5 + 3.0f * m6 - 9.0f * m8) * inv36;
    f[7] = (t2 - 6.0f * m3 - 3.0f * m4 - 6.0f * m5 - 3.0f * m6 + 9.0f * m8) * inv36;
    f[8] = (t2 + 6.0f * m3 + 3.0f * m4 - 6.0f * m5 - 3.0f * m6 - 9.0f * m8) * inv36;
}

__device__ __forceinline__ void bgk_relax(float (&f)[9], float r, float u, float v, float s_nu)
{
    const float usq = u * u + v * v;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        float cu = (float)cx(q) * u + (float)cy(q) * v;
        float feq = wgt(q) * r * (1.0f + 3.0f * cu + 4.5f * cu * cu - 1.5f * usq);
        f[q] += s_nu * (feq - f[q]);
    }
}

// rho, u, v with the reference's summation order (sequential over q,
// lbm_core4.cu:130-141), so that FP32 rounding follows the reference.
__device__ __forceinline__ void moments_seq(const float (&f)[9], float &r, float &u, float &v)
{
    r = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    const float jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    const float jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    u = jx / r;
    v = jy / r;
}

// Full collision of one updated cell.  `inlet` selects the Zou-He branch
// (x = 0, prescribed velocity); r/u/v receive the macroscopic values the
// reference writes to its rho/ux/uy arrays.
template <class Ph>
__device__ __forceinline__ void collide(float (&f)[9], bool inlet, int y, const Phys &k, float &r, float &u, float &v)
{
    const bool kMrt = Ph::kRuntime ? (k.flags & PF_MRT) != 0 : Ph::kMrt;
    const bool kSmag = Ph::kRuntime ? (k.flags & PF_SMAG) != 0 : Ph::kSmag;
    const bool kClampU = Ph::kRuntime ? (k.flags & PF_CLAMPU) != 0 : Ph::kClampU;
    const bool kClampF = Ph::kRuntime ? (k.flags & PF_CLAMPF) != 0 : Ph::kClampF;
    const bool kInletSmag = Ph::kRuntime ? (k.flags & PF_INLET_SMAG) != 0 : Ph::kInletSmag;
    moments_seq(f, r, u, v);
    if (kClampU) {
        u = fminf(0.4f, fmaxf(-0.4f, u));
        v = fminf(0.4f, fmaxf(-0.4f, v));
        r = fminf(1.5f, fmaxf(0.0f, r));
    }
    if (inlet) {
        const float lu = inlet_u(k, y);
        r = zou_he(f, lu);
        u = lu;
        v = 0.0f;
    }
    float s = k.s_nu;
    if (kSmag) {
        if (kInletSmag || !inlet)
            s = smag_rate(f, r, u, v, k);
    }
    if (kMrt)
        mrt_relax(f, r, u, v, k.s_e, k.s_eps, k.s_q, s);
    else
        bgk_relax(f, r, u, v, s);
    if (kClampF) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
            f[q] = fminf(10.0f, fmaxf(0.0f, f[q]));
    }
}

// Branch-free collision for the hot loops (wavefront and streaming kernels).
// Same physics as collide() with fewer instructions:
//   * moments from shared pair sums/differences of opposite populations;
//   * one reciprocal of rho, square roots as x * rsqrt(x) (x > 0 here);
//   * MRT applied as f -= M^-1 d, d = m - m' (m' the post-collision moments;
//     for the conserved moments d0 = rho - rho', d3 = j_x - rho'u', d5 = j_y - rho'v',
//     nonzero only when the clamps engage or at the inlet), using the structure
//     of the Lallemand-Luo inverse (lbm_core4.cu:187-199).
// The Zou-He values (kZh) are computed for every cell and selected where
// `inlet` holds; `lu` is the inlet velocity of the cell's row.  Rounding
// differs from the reference's evaluation order at the 1e-7 level.
// Branch-free collision in the reference's evaluation order (moments summed
// over q in sequence, MRT through the explicit moment vector).
template <class Ph, bool kZh>
__device__ __forceinline__ void collide_ref_bf(float (&f)[9], bool inlet, float lu, const Phys &k, float &r, float &u,
                                               float &v)
{
    moments_seq(f, r, u, v);
    if (Ph::kClampU) {
        u = fminf(0.4f, fmaxf(-0.4f, u));
        v = fminf(0.4f, fmaxf(-0.4f, v));
        r = fminf(1.5f, fmaxf(0.0f, r));
    }
    if (kZh) {
        const float rz = (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7])) / (1.0f - lu);
        const float a = 0.16666666666f * rz * lu;
        const float h = 0.5f * (f[2] - f[4]);
        const float z1 = f[3] + 0.666666667f * rz * lu;
        const float z5 = f[7] - h + a;
        const float z8 = f[6] + h + a;
        f[1] = inlet ? z1 : f[1];
        f[5] = inlet ? z5 : f[5];
        f[8] = inlet ? z8 : f[8];
        r = inlet ? rz : r;
        u = inlet ? lu : u;
        v = inlet ? 0.0f : v;
    }
    float s = k.s_nu;
    if (Ph::kSmag) {
        const float sm = smag_rate(f, r, u, v, k);
        s = (kZh && inlet && !Ph::kInletSmag) ? k.s_nu : sm;
    }
    if (Ph::kMrt)
        mrt_relax(f, r, u, v, k.s_e, k.s_eps, k.s_q, s);
    else
        bgk_relax(f, r, u, v, s);
    if (Ph::kClampF) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
            f[q] = fminf(10.0f, fmaxf(0.0f, f[q]));
    }
}

template <class Ph, bool kZh>
__device__ __forceinline__ void collide_bf(float (&f)[9], bool inlet, float lu, const Phys &k, float &r, float &u,
                                           float &v)
{
    static_assert(!Ph::kRuntime, "compile-time physics only");
    if constexpr (Ph::kRefOrder) {
        collide_ref_bf<Ph, kZh>(f, inlet, lu, k, r, u, v);
        return;
    }
    float rz = 0.0f;
    if (kZh) {
        rz = (f[0] + f[2] + f[4] + 2.0f * (f[3] + f[6] + f[7])) / (1.0f - lu);
        const float a = 0.16666666666f * rz * lu;
        const float h = 0.5f * (f[2] - f[4]);
        const float z1 = f[3] + 0.666666667f * rz * lu;
        f[1] = inlet ? z1 : f[1];
        f[5] = inlet ? f[7] - h + a : f[5];
        f[8] = inlet ? f[6] + h + a : f[8];
    }
    const float a13 = f[1] + f[3], a24 = f[2] + f[4], a57 = f[5] + f[7], a68 = f[6] + f[8];
    const float b13 = f[1] - f[3], b24 = f[2] - f[4], b57 = f[5] - f[7], b68 = f[6] - f[8];
    const float s14 = a13 + a24, s58 = a57 + a68;
    const float rho = (f[0] + s14) + s58;
    const float e = b57 - b68, g = b57 + b68;
    const float jx = b13 + e, jy = b24 + g;
    const float rinv = __fdividef(1.0f, rho);
    u = jx * rinv;
    v = jy * rinv;
    r = rho;
    float rcinv = rinv;
    if (Ph::kClampU) {
        u = fminf(0.4f, fmaxf(-0.4f, u));
        v = fminf(0.4f, fmaxf(-0.4f, v));
        r = fminf(1.5f, fmaxf(0.0f, rho));
        rcinv = __fdividef(1.0f, r);
    }
    if (kZh) {
        r = inlet ? rz : r;
        u = inlet ? lu : u;
        v = inlet ? 0.0f : v;
        rcinv = inlet ? __fdividef(1.0f, rz) : rcinv;
    }
    const float uu = u * u, vv = v * v;
    const float m3 = r * u, m5 = r * v;
    const float m7 = a13 - a24, m8 = a57 - a68;
    const float n7 = m7 - r * (uu - vv);
    const float n8 = m8 - m3 * v;
    float s = k.s_nu;
    if (Ph::kSmag) {
        const float q2 = fmaf(n7, n7, fmaf(n8, n8, 1e-8f));
        const float Q = q2 * rsqrtf(q2);
        const float X = fmaf(k.cs2x18 * Q, rcinv, k.tau0 * k.tau0);
        const float Sx = X * rsqrtf(X);
        const float sm = __fdividef(2.0f, k.tau0 + Sx);
        s = (kZh && inlet && !Ph::kInletSmag) ? k.s_nu : sm;
    }
    if (Ph::kMrt) {
        // conserved moments replaced by the clamps or the Zou-He inlet; without
        // them d0 = d3 = d5 = 0 exactly, as in collide_multi, so that a cell
        // gets the same bits from either function
        const bool cons = Ph::kClampU || (kZh && inlet);
        const float d0 = cons ? rho - r : 0.0f;
        const float d3 = cons ? jx - m3 : 0.0f;
        const float d5 = cons ? jy - m5 : 0.0f;
        const float t3 = 3.0f * (uu + vv);
        const float m1 = fmaf(2.0f, s58, -s14) - 4.0f * f[0];
        const float m2 = fmaf(-2.0f, s14, s58) + 4.0f * f[0];
        const float m4 = fmaf(-2.0f, b13, e);
        const float m6 = fmaf(-2.0f, b24, g);
        const float d1 = k.s_e * (m1 - r * (t3 - 2.0f));
        const float d2 = k.s_eps * (m2 - r * (1.0f - t3));
        const float d4 = k.s_q * (m4 + m3);
        const float d6 = k.s_q * (m6 + m5);
        const float d7 = s * n7;
        const float d8 = s * n8;
        const float Z = (d0 - d1 + d2) * 0.1111111111f;
        const float A = (4.0f * d0 - d1 - 2.0f * d2) * 0.02777777778f;
        const float D = (4.0f * d0 + 2.0f * d1 + d2) * 0.02777777778f;
        const float Bx = (d3 - d4) * 0.16666666666f;
        const float By = (d5 - d6) * 0.16666666666f;
        const float Ex = (2.0f * d3 + d4) * 0.08333333333f;
        const float Ey = (2.0f * d5 + d6) * 0.08333333333f;
        const float AP = fmaf(0.25f, d7, A), AM = fmaf(-0.25f, d7, A);
        const float DP = fmaf(0.25f, d8, D), DM = fmaf(-0.25f, d8, D);
        const float EP = Ex + Ey, EM = Ex - Ey;
        f[0] -= Z;
        f[1] -= AP + Bx;
        f[3] -= AP - Bx;
        f[2] -= AM + By;
        f[4] -= AM - By;
        f[5] -= DP + EP;
        f[7] -= DP - EP;
        f[6] -= DM - EM;
        f[8] -= DM + EM;
    } else {
        bgk_relax(f, r, u, v, s);
    }
    if (Ph::kClampF) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
            f[q] = fminf(10.0f, fmaxf(0.0f, f[q]));
    }
}

// The fast-order collision of N independent cells at once (no Zou-He, no
// per-cell branches).  Every statement is applied to all N cells before the
// next one, so the N dependency chains reach the scheduler interleaved.
template <class Ph, int N>
__device__ __forceinline__ void collide_multi(float (&f)[N][9], const Phys &k, float (&r)[N], float (&u)[N],
                                              float (&v)[N])
{
    static_assert(!Ph::kRuntime && !Ph::kRefOrder, "fast-order compile-time physics only");
    float a13[N], a24[N], a57[N], a68[N], b13[N], b24[N], b57[N], b68[N], s14[N], s58[N], rho[N], e[N], g[N];
    float jx[N], jy[N], rinv[N], rcinv[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        a13[n] = f[n][1] + f[n][3];
        a24[n] = f[n][2] + f[n][4];
        a57[n] = f[n][5] + f[n][7];
        a68[n] = f[n][6] + f[n][8];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        b13[n] = f[n][1] - f[n][3];
        b24[n] = f[n][2] - f[n][4];
        b57[n] = f[n][5] - f[n][7];
        b68[n] = f[n][6] - f[n][8];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        s14[n] = a13[n] + a24[n];
        s58[n] = a57[n] + a68[n];
        e[n] = b57[n] - b68[n];
        g[n] = b57[n] + b68[n];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        rho[n] = (f[n][0] + s14[n]) + s58[n];
        jx[n] = b13[n] + e[n];
        jy[n] = b24[n] + g[n];
    }
#pragma unroll
    for (int n = 0; n < N; ++n)
        rinv[n] = __fdividef(1.0f, rho[n]);
#pragma unroll
    for (int n = 0; n < N; ++n) {
        u[n] = jx[n] * rinv[n];
        v[n] = jy[n] * rinv[n];
        r[n] = rho[n];
        rcinv[n] = rinv[n];
    }
    if (Ph::kClampU) {
#pragma unroll
        for (int n = 0; n < N; ++n) {
            u[n] = fminf(0.4f, fmaxf(-0.4f, u[n]));
            v[n] = fminf(0.4f, fmaxf(-0.4f, v[n]));
            r[n] = fminf(1.5f, fmaxf(0.0f, rho[n]));
        }
#pragma unroll
        for (int n = 0; n < N; ++n)
            rcinv[n] = __fdividef(1.0f, r[n]);
    }
    float uu[N], vv[N], m3[N], m5[N], n7[N], n8[N], s[N];
#pragma unroll
    for (int n = 0; n < N; ++n) {
        uu[n] = u[n] * u[n];
        vv[n] = v[n] * v[n];
        m3[n] = r[n] * u[n];
        m5[n] = r[n] * v[n];
    }
#pragma unroll
    for (int n = 0; n < N; ++n) {
        n7[n] = (a13[n] - a24[n]) - r[n] * (uu[n] - vv[n]);
        n8[n] = (a57[n] - a68[n]) - m3[n] * v[n];
    }
    if (Ph::kSmag) {
        float X[N];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const float q2 = fmaf(n7[n], n7[n], fmaf(n8[n], n8[n], 1e-8f));
            X[n] = q2 * rsqrtf(q2);
        }
#pragma unroll
        for (int n = 0; n < N; ++n)
            X[n] = fmaf(k.cs2x18 * X[n], rcinv[n], k.tau0 * k.tau0);
#pragma unroll
        for (int n = 0; n < N; ++n)
            X[n] = X[n] * rsqrtf(X[n]);
#pragma unroll
        for (int n = 0; n < N; ++n)
            s[n] = __fdividef(2.0f, k.tau0 + X[n]);
    } else {
#pragma unroll
        for (int n = 0; n < N; ++n)
            s[n] = k.s_nu;
    }
    if (Ph::kMrt) {
        float d0[N], d1[N], d2[N], d3[N], d4[N], d5[N], d6[N], d7[N], d8[N];
#pragma unroll
        for (int n = 0; n < N; ++n) {
            d0[n] = Ph::kClampU ? rho[n] - r[n] : 0.0f;
            d3[n] = Ph::kClampU ? jx[n] - m3[n] : 0.0f;
            d5[n] = Ph::kClampU ? jy[n] - m5[n] : 0.0f;
        }
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const float t3 = 3.0f * (uu[n] + vv[n]);
            const float m1 = fmaf(2.0f, s58[n], -s14[n]) - 4.0f * f[n][0];
            const float m2 = fmaf(-2.0f, s14[n], s58[n]) + 4.0f * f[n][0];
            d1[n] = k.s_e * (m1 - r[n] * (t3 - 2.0f));
            d2[n] = k.s_eps * (m2 - r[n] * (1.0f - t3));
        }
#pragma unroll
        for (int n = 0; n < N; ++n) {
            d4[n] = k.s_q * (fmaf(-2.0f, b13[n], e[n]) + m3[n]);
            d6[n] = k.s_q * (fmaf(-2.0f, b24[n], g[n]) + m5[n]);
            d7[n] = s[n] * n7[n];
            d8[n] = s[n] * n8[n];
        }
#pragma unroll
        for (int n = 0; n < N; ++n) {
            const float Z = (d0[n] - d1[n] + d2[n]) * 0.1111111111f;
            const float A = (4.0f * d0[n] - d1[n] - 2.0f * d2[n]) * 0.02777777778f;
            const float D = (4.0f * d0[n] + 2.0f * d1[n] + d2[n]) * 0.02777777778f;
            const float Bx = (d3[n] - d4[n]) * 0.16666666666f;
            const float By = (d5[n] - d6[n]) * 0.16666666666f;
            const float Ex = (2.0f * d3[n] + d4[n]) * 0.08333333333f;
            const float Ey = (2.0f * d5[n] + d6[n]) * 0.08333333333f;
            const float AP = fmaf(0.25f, d7[n], A), AM = fmaf(-0.25f, d7[n], A);
            const float DP = fmaf(0.25f, d8[n], D), DM = fmaf(-0.25f, d8[n], D);
            const float EP = Ex + Ey, EM = Ex - Ey;
            f[n][0] -= Z;
            f[n][1] -= AP + Bx;
            f[n][3] -= AP - Bx;
            f[n][2] -= AM + By;
            f[n][4] -= AM - By;
            f[n][5] -= DP + EP;
            f[n][7] -= DP - EP;
            f[n][6] -= DM - EM;
            f[n][8] -= DM + EM;
        }
    } else {
#pragma unroll
        for (int n = 0; n < N; ++n)
            bgk_relax(f[n], r[n], u[n], v[n], s[n]);
    }
    if (Ph::kClampF) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
#pragma unroll
            for (int n = 0; n < N; ++n)
                f[n][q] = fminf(10.0f, fmaxf(0.0f, f[n][q]));
    }
}

// ---------------------------------------------------------------------------
// Two cells at once on Blackwell's packed FP32 pipe (FFMA2 / FADD2 / FMUL2:
// one instruction updates both halves of a float2, each half rounded as the
// scalar operation would be).  Same physics and evaluation order as
// collide_multi; reciprocals and square roots stay scalar.  The reference's
// clamps are applied only when a value is outside its range: the check works
// on the IEEE bit patterns (for x >= +0, bits(x) <= bits(hi) <=> x <= hi;
// negative values, -0 and NaN compare above every positive bound), so a value
// inside the range is returned unchanged and any other value goes through the
// same fminf / fmaxf as before -- the result equals the unconditional clamp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 bc2(float s)
{
    return make_float2(s, s);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    return __fadd2_rn(a, b);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) // a - b, one rounding
{
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    return __fmul2_rn(a, b);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 rcp2(float2 a)
{
    return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y));
}
__device__ __forceinline__ float2 rsqrt2(float2 a)
{
    return make_float2(rsqrtf(a.x), rsqrtf(a.y));
}
__device__ __forceinline__ uint32_t fbits(float x)
{
    return __float_as_uint(x);
}

template <class Ph>
__device__ __forceinline__ void collide_pair(float2 (&f)[9], const Phys &k, float2 &r, float2 &u, float2 &v)
{
    static_assert(!Ph::kRuntime && !Ph::kRefOrder, "fast-order compile-time physics only");
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
    float2 rcinv = rinv;
    if (Ph::kClampU) {
        const uint32_t mu = max(max(fbits(u.x) & 0x7fffffffu, fbits(u.y) & 0x7fffffffu),
                                max(fbits(v.x) & 0x7fffffffu, fbits(v.y) & 0x7fffffffu));
        const uint32_t mr = max(fbits(r.x), fbits(r.y));
        if (mu > fbits(0.4f) || mr > fbits(1.5f)) {
            u.x = fminf(0.4f, fmaxf(-0.4f, u.x));
            u.y = fminf(0.4f, fmaxf(-0.4f, u.y));
            v.x = fminf(0.4f, fmaxf(-0.4f, v.x));
            v.y = fminf(0.4f, fmaxf(-0.4f, v.y));
            r.x = fminf(1.5f, fmaxf(0.0f, rho.x));
            r.y = fminf(1.5f, fmaxf(0.0f, rho.y));
            rcinv = rcp2(r);
        }
    }
    const float2 uu = mul2(u, u), vv = mul2(v, v);
    const float2 m3 = mul2(r, u), m5 = mul2(r, v);
    const float2 n7 = fma2(r, sub2(vv, uu), sub2(a13, a24));
    const float2 n8 = sub2(sub2(a57, a68), mul2(m3, v));
    float2 s = bc2(k.s_nu);
    if (Ph::kSmag) {
        const float2 q2 = fma2(n7, n7, fma2(n8, n8, bc2(1e-8f)));
        const float2 Q = mul2(q2, rsqrt2(q2));
        const float2 X = fma2(mul2(bc2(k.cs2x18), Q), rcinv, bc2(k.tau0 * k.tau0));
        const float2 Sx = mul2(X, rsqrt2(X));
        s = mul2(bc2(2.0f), rcp2(add2(bc2(k.tau0), Sx)));
    }
    if (Ph::kMrt) {
        float2 d0 = bc2(0.0f), d3 = bc2(0.0f), d5 = bc2(0.0f);
        if (Ph::kClampU) {
            d0 = sub2(rho, r);
            d3 = sub2(jx, m3);
            d5 = sub2(jy, m5);
        }
        const float2 t3 = mul2(bc2(3.0f), add2(uu, vv));
        const float2 m1 = fma2(bc2(-4.0f), f[0], sub2(add2(s58, s58), s14));
        const float2 m2 = fma2(bc2(4.0f), f[0], fma2(bc2(-2.0f), s14, s58));
        const float2 d1 = mul2(bc2(k.s_e), fma2(r, sub2(bc2(2.0f), t3), m1));
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
    } else {
        const float2 usq = add2(uu, vv);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float2 cu = fma2(bc2((float)cx(q)), u, mul2(bc2((float)cy(q)), v));
            const float2 poly = fma2(mul2(bc2(4.5f), cu), cu, fma2(bc2(3.0f), cu, fma2(bc2(-1.5f), usq, bc2(1.0f))));
            const float2 feq = mul2(mul2(bc2(wgt(q)), r), poly);
            f[q] = fma2(s, sub2(feq, f[q]), f[q]);
        }
    }
    if (Ph::kClampF) {
        // max of the 18 bit patterns with three-input integer max: 9 operations
        uint32_t m3[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float a = (3 * k) % 2 ? f[(3 * k) / 2].y : f[(3 * k) / 2].x;
            const float b = (3 * k + 1) % 2 ? f[(3 * k + 1) / 2].y : f[(3 * k + 1) / 2].x;
            const float c = (3 * k + 2) % 2 ? f[(3 * k + 2) / 2].y : f[(3 * k + 2) / 2].x;
            m3[k] = __vimax3_u32(fbits(a), fbits(b), fbits(c));
        }
        const uint32_t mx = max(__vimax3_u32(m3[0], m3[1], m3[2]), __vimax3_u32(m3[3], m3[4], m3[5]));
        if (mx > fbits(10.0f)) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                f[q].x = fminf(10.0f, fmaxf(0.0f, f[q].x));
                f[q].y = fminf(10.0f, fmaxf(0.0f, f[q].y));
            }
        }
    }
}

// Two cells on the packed FP32x2 pipe in the reference's evaluation order:
// collide_ref_bf without the Zou-He inlet (the inlet window keeps the scalar
// form).  The sequential sums of moments_seq and the sums and products of
// smag_rate, mrt_relax and bgk_relax are FADD2 / FMUL2 / FFMA2 in the same
// order; the divisions and square roots stay per cell.  Rounding can differ
// from the scalar form where the compiler contracts a product and a sum into
// one FMA differently.  The clamps are applied only when a value is outside
// its range, as in collide_pair.
template <class Ph>
__device__ __forceinline__ void collide_ref_pair(float2 (&f)[9], const Phys &k, float2 &r, float2 &u, float2 &v)
{
    static_assert(!Ph::kRuntime && Ph::kRefOrder, "reference-order compile-time physics only");
    // moments_seq
    float2 rr = f[0];
#pragma unroll
    for (int q = 1; q < 9; ++q)
        rr = add2(rr, f[q]);
    const float2 jx = add2(sub2(sub2(add2(sub2(f[1], f[3]), f[5]), f[6]), f[7]), f[8]);
    const float2 jy = sub2(sub2(add2(add2(sub2(f[2], f[4]), f[5]), f[6]), f[7]), f[8]);
    u = make_float2(jx.x / rr.x, jx.y / rr.y);
    v = make_float2(jy.x / rr.x, jy.y / rr.y);
    r = rr;
    if (Ph::kClampU) {
        const uint32_t mu = max(max(fbits(u.x) & 0x7fffffffu, fbits(u.y) & 0x7fffffffu),
                                max(fbits(v.x) & 0x7fffffffu, fbits(v.y) & 0x7fffffffu));
        const uint32_t mr = max(fbits(r.x), fbits(r.y));
        if (mu > fbits(0.4f) || mr > fbits(1.5f)) {
            u.x = fminf(0.4f, fmaxf(-0.4f, u.x));
            u.y = fminf(0.4f, fmaxf(-0.4f, u.y));
            v.x = fminf(0.4f, fmaxf(-0.4f, v.x));
            v.y = fminf(0.4f, fmaxf(-0.4f, v.y));
            r.x = fminf(1.5f, fmaxf(0.0f, r.x));
            r.y = fminf(1.5f, fmaxf(0.0f, r.y));
        }
    }
    const float2 uu = mul2(u, u), vv = mul2(v, v);
    float2 s = bc2(k.s_nu);
    if (Ph::kSmag) {
        // smag_rate
        const float2 n7 = sub2(sub2(add2(sub2(f[1], f[2]), f[3]), f[4]), mul2(r, sub2(uu, vv)));
        const float2 n8 = sub2(sub2(add2(sub2(f[5], f[6]), f[7]), f[8]), mul2(mul2(r, u), v));
        const float2 q2 = add2(fma2(n7, n7, mul2(n8, n8)), bc2(1e-8f));
        const float2 cq = mul2(bc2(k.cs2x18), make_float2(sqrtf(q2.x), sqrtf(q2.y)));
        const float2 X = add2(bc2(k.tau0 * k.tau0), make_float2(cq.x / r.x, cq.y / r.y));
        const float2 te = mul2(bc2(0.5f), add2(bc2(k.tau0), make_float2(sqrtf(X.x), sqrtf(X.y))));
        s = make_float2(1.0f / te.x, 1.0f / te.y);
    }
    if (Ph::kMrt) {
        // mrt_relax
        const float2 f14 = add2(add2(add2(f[1], f[2]), f[3]), f[4]);
        const float2 f58 = add2(add2(add2(f[5], f[6]), f[7]), f[8]);
        float2 m1 = sub2(fma2(bc2(-4.0f), f[0], mul2(bc2(2.0f), f58)), f14);
        float2 m2 = sub2(fma2(bc2(4.0f), f[0], f58), mul2(bc2(2.0f), f14));
        const float2 m3 = mul2(r, u);
        float2 m4 = add2(sub2(sub2(fma2(bc2(-2.0f), sub2(f[1], f[3]), f[5]), f[6]), f[7]), f[8]);
        const float2 m5 = mul2(r, v);
        float2 m6 = sub2(sub2(add2(fma2(bc2(-2.0f), sub2(f[2], f[4]), f[5]), f[6]), f[7]), f[8]);
        float2 m7 = sub2(add2(sub2(f[1], f[2]), f[3]), f[4]);
        float2 m8 = sub2(add2(sub2(f[5], f[6]), f[7]), f[8]);
        const float2 usq = add2(uu, vv);
        m1 = sub2(m1, mul2(bc2(k.s_e), sub2(m1, mul2(fma2(bc2(3.0f), usq, bc2(-2.0f)), r))));
        m2 = sub2(m2, mul2(bc2(k.s_eps), sub2(m2, mul2(fma2(bc2(-3.0f), usq, bc2(1.0f)), r))));
        m4 = sub2(m4, mul2(bc2(k.s_q), add2(m4, m3)));
        m6 = sub2(m6, mul2(bc2(k.s_q), add2(m6, m5)));
        m7 = sub2(m7, mul2(s, sub2(m7, mul2(r, sub2(uu, vv)))));
        m8 = sub2(m8, mul2(s, sub2(m8, mul2(mul2(r, u), v))));
        const float2 inv9 = bc2(0.1111111111f), inv36 = bc2(0.02777777778f);
        const float2 t0 = add2(sub2(r, m1), m2);
        const float2 t1 = sub2(sub2(mul2(bc2(4.0f), r), m1), mul2(bc2(2.0f), m2));
        const float2 t2 = add2(fma2(bc2(4.0f), r, mul2(bc2(2.0f), m1)), m2);
        const float2 a3 = mul2(bc2(6.0f), m3), a4 = mul2(bc2(6.0f), m4), a5 = mul2(bc2(6.0f), m5),
                     a6 = mul2(bc2(6.0f), m6), a7 = mul2(bc2(9.0f), m7), a8 = mul2(bc2(9.0f), m8);
        const float2 b4 = mul2(bc2(3.0f), m4), b6 = mul2(bc2(3.0f), m6);
        f[0] = mul2(t0, inv9);
        f[1] = mul2(add2(sub2(add2(t1, a3), a4), a7), inv36);
        f[2] = mul2(sub2(sub2(add2(t1, a5), a6), a7), inv36);
        f[3] = mul2(add2(add2(sub2(t1, a3), a4), a7), inv36);
        f[4] = mul2(sub2(add2(sub2(t1, a5), a6), a7), inv36);
        f[5] = mul2(add2(add2(add2(add2(add2(t2, a3), b4), a5), b6), a8), inv36);
        f[6] = mul2(sub2(add2(add2(sub2(sub2(t2, a3), b4), a5), b6), a8), inv36);
        f[7] = mul2(add2(sub2(sub2(sub2(sub2(t2, a3), b4), a5), b6), a8), inv36);
        f[8] = mul2(sub2(sub2(sub2(add2(add2(t2, a3), b4), a5), b6), a8), inv36);
    } else {
        // bgk_relax
        const float2 usq = add2(uu, vv);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const float2 cu = add2(mul2(bc2((float)cx(q)), u), mul2(bc2((float)cy(q)), v));
            const float2 poly =
                sub2(add2(add2(bc2(1.0f), mul2(bc2(3.0f), cu)), mul2(mul2(bc2(4.5f), cu), cu)), mul2(bc2(1.5f), usq));
            const float2 feq = mul2(mul2(bc2(wgt(q)), r), poly);
            f[q] = fma2(s, sub2(feq, f[q]), f[q]);
        }
    }
    if (Ph::kClampF) {
        uint32_t m3[6];
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const float a = (3 * j) % 2 ? f[(3 * j) / 2].y : f[(3 * j) / 2].x;
            const float b = (3 * j + 1) % 2 ? f[(3 * j + 1) / 2].y : f[(3 * j + 1) / 2].x;
            const float c = (3 * j + 2) % 2 ? f[(3 * j + 2) / 2].y : f[(3 * j + 2) / 2].x;
            m3[j] = __vimax3_u32(fbits(a), fbits(b), fbits(c));
        }
        const uint32_t mx = max(__vimax3_u32(m3[0], m3[1], m3[2]), __vimax3_u32(m3[3], m3[4], m3[5]));
        if (mx > fbits(10.0f)) {
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                f[q].x = fminf(10.0f, fmaxf(0.0f, f[q].x));
                f[q].y = fminf(10.0f, fmaxf(0.0f, f[q].y));
            }
        }
    }
}

} // namespace lbm
