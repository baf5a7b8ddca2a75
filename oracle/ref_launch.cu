// Host launchers for the reference's own CUDA kernels.
//
// TEST INFRASTRUCTURE ONLY (the parity oracle on the GPU and the reference arm of
// bench.py).  oracle/Makefile compiles this file once per reference source,
// passing the source's path in REF_SRC and its family in REF_KIND, and writes the
// result to oracle/_ref/.  The reference sources are included where they lie and
// are not copied into this repository.  Launch shapes follow the reference
// drivers:
//   lbm_mine2.py:77-80                block (32,8),  grid ceil(W/32) x ceil(H/8)
//   lbm_smemaa_main.py:205-207        block (32,8),  grid ceil(W/24) x ceil(H/24)
//   lbm_smemaa_endfused_main.py:60-63 block (32,16), grid ceil(W/24) x ceil(H/24)
//   lbm_smemaa_endfused_main.py:98    macro / visualize: block (16,16)
#include <cuda_runtime.h>

#include REF_SRC

#define REF_CORE4 1
#define REF_SMEMAA 2
#define REF_BLOCKED 3

extern "C" {

int ref_kind(void)
{
    return REF_KIND;
}

#if REF_KIND == REF_CORE4
int ref_T(void)
{
    return 1;
}

int ref_core4_step(const unsigned char *mask, float *f_now, float *f_out, float *ux, float *uy, float *rho, int W,
                   int H, float tau_inv, float u_in, float tau_inv_bnd, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((W + 31) / 32, (H + 7) / 8);
    fused_lbmkernel<<<grid, block, 0, s>>>((bool *)mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in, tau_inv_bnd);
    return (int)cudaGetLastError();
}
#elif REF_KIND == REF_SMEMAA
int ref_T(void)
{
    return T;
}

int ref_smemaa_step(const unsigned char *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho,
                    int W, int H, float tau_inv, float u_in, cudaStream_t s)
{
    dim3 block(32, 8);
    dim3 grid((W + SQUARE_A - 1) / SQUARE_A, (H + SQUARE_A - 1) / SQUARE_A);
    fused_lbmkernel<<<grid, block, 0, s>>>((bool *)mask, f_now, f_out, ux, uy, rho, W, H, tau_inv, u_in);
    return (int)cudaGetLastError();
}
#elif REF_KIND == REF_BLOCKED
int ref_T(void)
{
    return T;
}

int ref_blocked_step(const unsigned char *mask, const float *f_now, float *f_out, int W, int H, float tau_inv,
                     float u_in, cudaStream_t s)
{
    dim3 block(32, 16);
    dim3 grid((W + SQUARE_A - 1) / SQUARE_A, (H + SQUARE_A - 1) / SQUARE_A);
    fused_lbmkernel<<<grid, block, 0, s>>>((const bool *)mask, f_now, f_out, W, H, tau_inv, u_in);
    return (int)cudaGetLastError();
}

int ref_macro(const float *f, float *ux, float *uy, float *rho, const unsigned char *mask, int W, int H, float u_in,
              cudaStream_t s)
{
    dim3 block(16, 16);
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    macro_kernel<<<grid, block, 0, s>>>(f, ux, uy, rho, (const bool *)mask, W, H, u_in);
    return (int)cudaGetLastError();
}
#endif

int ref_visualize(const float *ux, const float *uy, const float *rho, unsigned char *img, const unsigned char *mask,
                  int W, int H, float vort_scale, cudaStream_t s)
{
    dim3 block(16, 16);
    dim3 grid((W + 15) / 16, (H + 15) / 16);
    visualizekernel<<<grid, block, 0, s>>>(ux, uy, rho, img, (const bool *)mask, W, H, vort_scale);
    return (int)cudaGetLastError();
}

} // extern "C"
