// General solver in FP64: double-precision populations in HBM and double
// arithmetic, one pull step per launch.  It is the high-precision judge of the
// 16-bit and FP32 storage formats at sizes where a CPU FP64 run would take hours
// (8192 x 2048 for 50 000 steps), and it runs every lbm_params configuration of
// the FP32 general solver except the learned closure.
//
// The per-cell update is the general solver's (MRT in the Lallemand-Luo basis or
// BGK, optional Smagorinsky rate and the reference's clamps, Zou-He inlet with
// or without the cosine ramp, Ladd moving walls, outflow ghost column, periodic
// sides), i.e. the physics of lbm_core4.cu:29-211 with the choices of
// lbm_params, evaluated in double.  Constants that the reference writes as
// single-precision literals (the ramp's 3.14159, the Zou-He 2/3 and 1/6, the
// 1e-8 under the Smagorinsky square root) are those float values widened to
// double, so that this kernel and an FP64 restatement of the reference agree to
// rounding.  No fast-math: the library's -use_fast_math changes only float
// operations; double division and square root here are IEEE.
//
// Layout: planes f[q * W * H + y * W + x] of doubles, the same SoA as the other
// formats.  One thread per cell, a warp on 32 consecutive cells of a row, so
// every plane access is one coalesced 256-byte segment and the x-shifted pulls
// are served from L1.  HBM traffic: 144 B per lattice update (9 doubles in, 9
// out) plus the mask bytes.
#include <string.h>

#include "dispatch.cuh"

namespace lbm {
namespace {

struct F64Step {
    const double *fin;
    double *fout;
    const uint8_t *mask;
    float *ux, *uy, *rho; // written when non-null (float: the macro arrays of the API)
    int W, H;
    long long N;
    int px, py;           // periodic in x / y
    int inlet, ramp;      // Zou-He at x = 0; cosine-ramped profile
    int outflow;          // ghost column W-1 (zero gradient)
    int mrt, smag, clamps;
    double s_nu, s_e, s_eps, s_q, tau0, cs2x18, u_in, u_lid;
};

__device__ __forceinline__ double w64(int q)
{
    return q == 0 ? 4.0 / 9.0 : (q <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
}

__device__ __forceinline__ double clamp64(double v, double lo, double hi)
{
    return fmin(hi, fmax(lo, v));
}

// MRT relaxation toward the equilibrium moments of (r, u, v) and the inverse
// transform (Lallemand-Luo basis; the structure of lbm_core4.cu:150-199).
__device__ __forceinline__ void mrt64(double (&f)[9], double r, double u, double v, double s_e, double s_eps,
                                      double s_q, double s_nu)
{
    const double a = f[1] + f[2] + f[3] + f[4];
    const double d = f[5] + f[6] + f[7] + f[8];
    double e = -4.0 * f[0] + 2.0 * d - a;
    double eps = 4.0 * f[0] + d - 2.0 * a;
    const double jx = r * u, jy = r * v;
    double qx = -2.0 * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
    double qy = -2.0 * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
    double pxx = f[1] - f[2] + f[3] - f[4];
    double pxy = f[5] - f[6] + f[7] - f[8];
    const double uu = u * u + v * v;
    e -= s_e * (e - (3.0 * uu - 2.0) * r);
    eps -= s_eps * (eps - (1.0 - 3.0 * uu) * r);
    qx -= s_q * (qx + jx);
    qy -= s_q * (qy + jy);
    pxx -= s_nu * (pxx - r * (u * u - v * v));
    pxy -= s_nu * (pxy - r * u * v);
    const double i9 = 1.0 / 9.0, i36 = 1.0 / 36.0;
    const double t0 = r - e + eps;
    const double t1 = 4.0 * r - e - 2.0 * eps;
    const double t2 = 4.0 * r + 2.0 * e + eps;
    f[0] = t0 * i9;
    f[1] = (t1 + 6.0 * jx - 6.0 * qx + 9.0 * pxx) * i36;
    f[2] = (t1 + 6.0 * jy - 6.0 * qy - 9.0 * pxx) * i36;
    f[3] = (t1 - 6.0 * jx + 6.0 * qx + 9.0 * pxx) * i36;
    f[4] = (t1 - 6.0 * jy + 6.0 * qy - 9.0 * pxx) * i36;
    f[5] = (t2 + 6.0 * jx + 3.0 * qx + 6.0 * jy + 3.0 * qy + 9.0 * pxy) * i36;
    f[6] = (t2 - 6.0 * jx - 3.0 * qx + 6.0 * jy + 3.0 * qy - 9.0 * pxy) * i36;
    f[7] = (t2 - 6.0 * jx - 3.0 * qx - 6.0 * jy - 3.0 * qy + 9.0 * pxy) * i36;
    f[8] = (t2 + 6.0 * jx + 3.0 * qx - 6.0 * jy - 3.0 * qy - 9.0 * pxy) * i36;
}

__device__ __forceinline__ void bgk64(double (&f)[9], double r, double u, double v, double s)
{
    const double uu = 1.5 * (u * u + v * v);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double cu = (double)cx(q) * u + (double)cy(q) * v;
        const double feq = w64(q) * r * (1.0 + 3.0 * cu + 4.5 * cu * cu - uu);
        f[q] += s * (feq - f[q]);
    }
}

__global__ void __launch_bounds__(256) f64_step_kernel(F64Step p)
{
    const int x = blockIdx.x * 32 + threadIdx.x;
    const int y = blockIdx.y * 8 + threadIdx.y;
    if (x >= p.W || y >= p.H)
        return;
    const long long c = (long long)y * p.W + x;
    if (p.mask[c] != 0 || (p.outflow && x == p.W - 1))
        return;

    // Pull with half-way bounce-back: a solid source (or a wall outside the
    // domain) returns this cell's own opposite population, plus the Ladd
    // momentum term when the source is a moving wall.
    double f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        int sx = x - cx(q), sy = y - cy(q);
        bool wall = false;
        if (p.px)
            sx = sx < 0 ? sx + p.W : (sx >= p.W ? sx - p.W : sx);
        else
            wall = sx < 0 || sx >= p.W;
        if (p.py)
            sy = sy < 0 ? sy + p.H : (sy >= p.H ? sy - p.H : sy);
        else
            wall = wall || sy < 0 || sy >= p.H;
        const int m = wall ? LBM_MASK_SOLID : p.mask[(long long)sy * p.W + sx];
        if (m == LBM_MASK_FLUID) {
            f[q] = p.fin[q * p.N + (long long)sy * p.W + sx];
        } else {
            double b = p.fin[opp(q) * p.N + c];
            if (m == LBM_MASK_MOVING)
                b += 6.0 * w64(q) * (double)cx(q) * p.u_lid;
            f[q] = b;
        }
    }

    double r, u, v, s = p.s_nu;
    if (p.inlet && x == 0) {
        // Zou-He velocity inlet (lbm_core4.cu:46-57).
        double lu = p.u_in;
        if (p.ramp) {
            const double dwall = fmin((double)y, (double)(p.H - 1 - y));
            if (dwall < 50.0)
                lu *= 0.5 * (1.0 - cos((double)3.14159f * dwall / 50.0));
        }
        r = (f[0] + f[2] + f[4] + 2.0 * (f[3] + f[6] + f[7])) / (1.0 - lu);
        const double h = 0.5 * (f[2] - f[4]);
        f[1] = f[3] + (double)0.666666667f * r * lu;
        f[5] = f[7] - h + (double)0.16666666666f * r * lu;
        f[8] = f[6] + h + (double)0.16666666666f * r * lu;
        u = lu;
        v = 0.0;
    } else {
        r = 0.0;
        u = 0.0;
        v = 0.0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            r += f[q];
            u += (double)cx(q) * f[q];
            v += (double)cy(q) * f[q];
        }
        u /= r;
        v /= r;
        if (p.clamps) {
            u = clamp64(u, -0.4, 0.4);
            v = clamp64(v, -0.4, 0.4);
            r = clamp64(r, 0.0, 1.5);
        }
        if (p.smag) {
            // Smagorinsky stress rate (lbm_core4.cu:171-177).
            const double n7 = (f[1] - f[2] + f[3] - f[4]) - r * (u * u - v * v);
            const double n8 = (f[5] - f[6] + f[7] - f[8]) - r * u * v;
            const double Q = sqrt(n7 * n7 + n8 * n8 + (double)1e-8f);
            s = 1.0 / (0.5 * (p.tau0 + sqrt(p.tau0 * p.tau0 + p.cs2x18 * Q / r)));
        }
    }
    if (p.ux) {
        p.ux[c] = (float)u;
        p.uy[c] = (float)v;
        p.rho[c] = (float)r;
    }
    if (p.mrt)
        mrt64(f, r, u, v, p.s_e, p.s_eps, p.s_q, s);
    else
        bgk64(f, r, u, v, s);
    const bool ghost = p.outflow && x == p.W - 2;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const double o = p.clamps ? clamp64(f[q], 0.0, 10.0) : f[q];
        p.fout[q * p.N + c] = o;
        if (ghost)
            p.fout[q * p.N + c + 1] = o;
    }
}

} // namespace

// One FP64 step src -> dst with the parameters of an lbm_params set (the learned
// closure is rejected when the handle is created).
int general_step_f64(const lbm_params &lp, const void *src, void *dst, const uint8_t *mask, float *ux, float *uy,
                     float *rho, cudaStream_t s)
{
    F64Step p;
    memset(&p, 0, sizeof(p));
    p.fin = static_cast<const double *>(src);
    p.fout = static_cast<double *>(dst);
    p.mask = mask;
    p.ux = ux;
    p.uy = uy;
    p.rho = rho;
    p.W = lp.W;
    p.H = lp.H;
    p.N = (long long)lp.W * lp.H;
    p.px = lp.bc_left == LBM_BC_PERIODIC;
    p.py = lp.bc_y == LBM_BC_PERIODIC;
    p.inlet = lp.bc_left == LBM_BC_ZOUHE || lp.bc_left == LBM_BC_ZOUHE_RAMP;
    p.ramp = lp.bc_left == LBM_BC_ZOUHE_RAMP;
    p.outflow = lp.bc_right == LBM_BC_OUTFLOW;
    p.mrt = lp.collision == LBM_COLL_MRT;
    p.smag = lp.closure == LBM_CLOSURE_SMAG;
    p.clamps = lp.ref_clamps != 0;
    p.s_nu = lp.s_nu;
    p.s_e = lp.s_e;
    p.s_eps = lp.s_eps;
    p.s_q = lp.s_q;
    p.tau0 = 1.0 / (double)lp.s_nu;
    p.cs2x18 = 18.0 * (double)lp.cs_smag * (double)lp.cs_smag;
    p.u_in = lp.u_in;
    p.u_lid = lp.u_lid;
    dim3 block(32, 8);
    dim3 grid((lp.W + 31) / 32, (lp.H + 7) / 8);
    f64_step_kernel<<<grid, block, 0, s>>>(p);
    return status(cudaGetLastError());
}

} // namespace lbm
