/*
 * lbm_b200.h - C ABI of liblbm_b200.so, a B200 (sm_100a) D2Q9 lattice-Boltzmann
 * collide-stream library that drops in for the kernels of Qianyv-Li8262/LBM-CUDA.
 *
 * Conventions shared by every entry point (they follow the reference kernels):
 *   - populations are SoA float planes f[q*W*H + y*W + x], q in the order
 *     c_x = {0,1,0,-1,0,1,-1,-1,1}, c_y = {0,0,1,0,-1,1,1,-1,-1} (lbm_core4.cu:1-3);
 *   - the mask is one byte per cell, row-major y*W + x, nonzero = solid
 *     (the reference passes a bool array, lbm_mine2.py:55-56);
 *   - every pointer is device memory owned by the caller; apart from lbm_create,
 *     no entry point allocates;
 *   - work is enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream)
 *     and nothing synchronises, so calls can be captured into a CUDA graph as the
 *     reference drivers do (lbm_mine2.py:75-81);
 *   - the return value is 0 on success, the cudaError_t of a failing CUDA call
 *     (1..999), or one of the LBM_ERR_* validation codes below.  The reference
 *     kernels return nothing; their launch errors surface asynchronously;
 *   - the library keeps a few per-device objects for the life of the process (the
 *     addresses of its __device__ arrays, TMA entry points, side streams); a
 *     device reset (cudaDeviceReset) while the library is loaded is not supported.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_OK 0
#define LBM_ERR_ARG 1001         /* null pointer, size or parameter out of range */
#define LBM_ERR_UNSUPPORTED 1002 /* configuration not built (e.g. temporal depth T) */
#define LBM_ERR_DEVICE 1003      /* no usable sm_100 device or driver entry point */
#define LBM_ERR_TIMEOUT 1004     /* a bounded device-side wait gave up */
#define LBM_ERR_TOO_LARGE 1005   /* domain larger than lbm_diag_fp64_noalloc's fixed scratch */

/* Storage formats of the population planes (general solver). */
#define LBM_STORE_F32 0
#define LBM_STORE_F16DEV 1  /* IEEE half of f_q - w_q, FP32 arithmetic */
#define LBM_STORE_BF16DEV 2 /* bfloat16 of f_q - w_q, FP32 arithmetic */
#define LBM_STORE_F64 3     /* IEEE double and FP64 arithmetic, one step per launch: the
                               high-precision judge of the other formats (general solver only) */

/* Mask byte values of the general solver (the drop-ins treat nonzero as solid). */
#define LBM_MASK_FLUID 0
#define LBM_MASK_SOLID 1
#define LBM_MASK_MOVING 2   /* wall moving with (u_lid, 0): Ladd bounce-back, rho_w = 1 */
#define LBM_MASK_OBSTACLE 3 /* solid, included in the drag/lift momentum exchange */

/* Domain sides of the general solver. */
#define LBM_BC_WALL 0       /* stationary half-way bounce-back wall outside the domain */
#define LBM_BC_PERIODIC 1   /* left: both x sides periodic; bc_y: both y sides periodic */
#define LBM_BC_ZOUHE 2      /* left only: Zou-He velocity inlet, flat profile u_in */
#define LBM_BC_ZOUHE_RAMP 3 /* left only: Zou-He with the reference's cosine ramp (lbm_core4.cu:46-51) */
#define LBM_BC_OUTFLOW 4    /* right only: zero-gradient ghost column W-1 (lbm_core4.cu:114-116) */

/* ------------------------------------------------------------------------
 * Reference drop-ins.  Same argument order and meaning as the reference
 * kernels, plus the stream and an int status.
 * ------------------------------------------------------------------------ */

/* One MRT + Smagorinsky pull step, f_now -> f_out, writing u, v, rho of every
 * updated cell.  Replaces fused_lbmkernel of lbm_core4.cu:7-13 (launched at
 * lbm_mine2.py:77-80).  Cs = 0.20 and s_e = s_eps = s_q = 1.1 as in the
 * reference; tau_inv_bnd is accepted and unused, as in the reference (:12). */
int lbm_core4_step(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho, int W,
                   int H, float tau_inv, float u_in, float tau_inv_bnd, void *stream);

/* n_steps of lbm_core4_step in ping-pong order starting from f_a, fused T
 * steps per launch (temporal blocking, 1 <= T <= 8).  The final state is in
 * f_b when *result_in_b is set to 1, else in f_a.  u, v, rho are those of the
 * last step.  Identical results to n_steps calls of lbm_core4_step when cells
 * that are never updated (solid cells, rows 0 and H-1) are not fluid sources,
 * which holds for the reference drivers' masks (lbm_mine2.py:49-53). */
int lbm_core4_run(const uint8_t *mask, float *f_a, float *f_b, float *ux, float *uy, float *rho, int W, int H,
                  float tau_inv, float u_in, int n_steps, int T, void *stream, int *result_in_b);

/* T BGK steps (T even, 2..8) with the shared-memory AA pattern, f_now -> f_out,
 * writing u, v, rho from the final canonical populations.  Replaces
 * fused_lbmkernel of lbm_core_smemaa.cu:12-15 (T = 4 there, :8). */
int lbm_smemaa_step(const uint8_t *mask, const float *f_now, float *f_out, float *ux, float *uy, float *rho, int W,
                    int H, float tau_inv, float u_in, int T, void *stream);

/* T BGK steps (T even, 2..8), first step read from f_now, last step scattered
 * straight into f_out.  Replaces fused_lbmkernel of
 * lbm_core_smemaa_policy.cu:78-80 and lbm_core_smemaa_endfused.cu:12-14
 * (T = 6 there).  Entries of f_out that the final scatter does not reach keep
 * their previous contents, as in the reference. */
int lbm_blocked_step(const uint8_t *mask, const float *f_now, float *f_out, int W, int H, float tau_inv, float u_in,
                     int T, void *stream);

/* u, v, rho from canonical populations, Zou-He at x = 0.  Replaces macro_kernel
 * of lbm_core_smemaa_policy.cu:431-433. */
int lbm_macro(const float *f, float *ux, float *uy, float *rho, const uint8_t *mask, int W, int H, float u_in,
              void *stream);

/* Vorticity colour map into an RGBA8 device buffer (W*H*4 bytes).  Replaces
 * visualizekernel of lbm_core4.cu:214-217; the buffer replaces the OpenGL
 * pixel buffer of zero_copy_window.py:119-155. */
int lbm_visualize(const float *ux, const float *uy, const float *rho, uint8_t *image, const uint8_t *mask, int W,
                  int H, float vort_scale, void *stream);

/* ------------------------------------------------------------------------
 * General solver (no reference counterpart: the reference hard-codes these
 * choices in its kernels, lbm_core4.cu:6,123).  Same SoA layout; the storage
 * format selects 4-byte or 2-byte elements per population.
 * ------------------------------------------------------------------------ */

#define LBM_COLL_BGK 0
#define LBM_COLL_MRT 1
#define LBM_CLOSURE_NONE 0
#define LBM_CLOSURE_SMAG 1
#define LBM_CLOSURE_MLP 2      /* learned eddy viscosity (lbm_params.mlp), ReLU network; see the MLP section */
#define LBM_CLOSURE_MLP_SILU 3 /* the same with the SiLU network (the configured activation, slower) */

typedef struct lbm_params {
    int W, H;
    int storage;   /* LBM_STORE_* */
    int collision; /* LBM_COLL_* */
    int closure;   /* LBM_CLOSURE_* */
    float s_nu;    /* stress relaxation rate 1/tau, tau = 3 nu + 1/2 */
    float s_e, s_eps, s_q; /* MRT rates of the energy, energy-square and heat-flux moments */
    float cs_smag; /* Smagorinsky constant (LBM_CLOSURE_SMAG) */
    int bc_left, bc_right, bc_y; /* LBM_BC_* */
    float u_in;    /* Zou-He inlet velocity */
    float u_lid;   /* x velocity of LBM_MASK_MOVING cells */
    int ref_clamps; /* 1: the reference's stabilisers |u| <= 0.4, rho in [0,1.5], f in [0,10] */
    const void *mlp; /* LBM_CLOSURE_MLP(_SILU): device pointer to LBM_MLP_PACKED_BYTES from lbm_mlp_pack_act */
} lbm_params;

typedef struct lbm_handle lbm_handle;

/* Defaults: the lbm_core4.cu choices (MRT, s_e = s_eps = s_q = 1.1, Smagorinsky
 * Cs = 0.2, Zou-He inlet with the ramp, outflow, walls in y, clamps on) with
 * s_nu = 1.8 and u_in = 0.1 as in lbm_mine2.py:77-78. */
void lbm_params_default(lbm_params *p, int W, int H);

/* Validate the parameters and allocate the handle and its small reduction
 * scratch (the only entry point that allocates device memory); lbm_destroy
 * frees them and lbm_run's cached graph.  When the planes' rows are a multiple
 * of 16 bytes but W is not a multiple of 16 (and x is not periodic, storage not
 * FP64), the handle also holds a copy of the mask with rows padded to a multiple
 * of 16 bytes (H * roundup(W, 16) bytes): the register wavefront kernel's TMA row
 * loads need that stride. */
int lbm_create(const lbm_params *p, lbm_handle **out);
int lbm_destroy(lbm_handle *h);

/* Bytes of one population state (9 planes of W*H elements of the storage format). */
size_t lbm_state_bytes(const lbm_handle *h);

/* f := equilibrium of (rho, ux, uy) (device arrays of W*H floats; NULL = 1, 0, 0). */
int lbm_init_equilibrium(lbm_handle *h, void *f, const float *rho, const float *ux, const float *uy, void *stream);

/* n_steps pull steps in ping-pong order starting from f_a, fused T per launch
 * (1 <= T <= 8; FP64 storage, and x-periodic domains without the learned
 * closure whose buffers suit the streaming kernel, one step per launch whatever
 * T: it is the faster kernel there).  The stored
 * state is post-collision populations (the lbm_core4.cu convention).  u, v, rho
 * of the last step are written when the pointers are non-NULL.  *result_in_b =
 * 1 when the final state is in f_b.  A handle with a padded mask copy (see
 * lbm_create) copies the mask into it first, on `stream`: two lbm_run calls on
 * such a handle must not overlap on the GPU.
 * Graph cache: when at least three whole pairs of T-step launches precede the
 * last launch, the handle captures one pair as a CUDA graph and replays it, so
 * a small domain pays one graph launch per pair; the results are bit-identical
 * to the plain launches, which a stream under capture by the caller always
 * gets.  Up to two graphs are kept, keyed by the ADDRESSES of f_a, f_b and mask
 * and by T (the handle's W, H and parameters are fixed), until another key
 * evicts them, lbm_run_graph_reset or lbm_destroy.  A caller that frees its
 * state buffers and allocates new ones (which may reuse the same addresses)
 * calls lbm_run_graph_reset first; LBM_RUN_GRAPH=0 in the environment turns
 * the cache off. */
int lbm_run(lbm_handle *h, void *f_a, void *f_b, const uint8_t *mask, int n_steps, int T, float *ux, float *uy,
            float *rho, void *stream, int *result_in_b);

/* One launch of T steps from src to dst that writes only the columns [x0, x1)
 * of dst (x0, x1 even, 0 <= x0 < x1 <= W); every other column of dst keeps its
 * contents (no counterpart in the reference, whose kernels cover the whole
 * domain).  The x-slab decomposition computes a rank's edge columns with it
 * first, sends them while the interior columns compute, then fills its halos.
 * Needs the register wavefront kernel: 2 <= T <= 6 (1 .. 4 with the learned
 * closure), TMA-aligned buffers (16-byte bases, W a multiple of 4 elements and
 * of 16 mask bytes) and x not periodic; otherwise LBM_ERR_UNSUPPORTED. */
int lbm_run_columns(lbm_handle *h, const void *src, void *dst, const uint8_t *mask, int T, int x0, int x1,
                    void *stream);

/* Halo columns of a state of `width` columns (9 planes of H rows, elements of
 * `storage`) to and from one contiguous buffer buf[2][9][H][ncols], in one
 * launch each (no counterpart in the reference): side 0 holds columns [xl, xl +
 * ncols), side 1 columns [xr, xr + ncols); a negative xl or xr skips that side
 * (its part of buf is neither read nor written).  The x-slab decomposition packs
 * the owned edge columns it sends and unpacks the halo columns it receives. */
int lbm_halo_pack(const void *f, int width, int H, int storage, int xl, int xr, int ncols, void *buf, void *stream);
int lbm_halo_unpack(void *f, int width, int H, int storage, int xl, int xr, int ncols, const void *buf, void *stream);

/* Drops lbm_run's cached graphs (no counterpart in the reference).  Returns
 * LBM_ERR_ARG while an lbm_run on another thread is replaying them. */
int lbm_run_graph_reset(lbm_handle *h);

/* n_steps steps in ONE state buffer (no counterpart in the reference, whose
 * drivers ping-pong two buffers, lbm_mine2.py:77-80): half the state memory of
 * lbm_run.  The AA access pattern: a pull-and-push step, then a step local to
 * each cell, so that within each step every location is read and written by a
 * single cell.  f holds the same post-collision state as lbm_run's buffers
 * before and after; n_steps must be even (LBM_ERR_ARG otherwise), and the
 * result equals lbm_run's for the same parameters (both of lbm_run's buffers
 * initialised with the same state).  u, v, rho of the last step are written
 * when the pointers are non-NULL.  The learned closure is not supported here
 * (LBM_ERR_UNSUPPORTED). */
int lbm_run_inplace(lbm_handle *h, void *f, const uint8_t *mask, int n_steps, float *ux, float *uy, float *rho,
                    void *stream);

/* Total mass and momentum sum_x sum_q f, c_x f, c_y f over cells with mask == 0,
 * accumulated in FP64 with a fixed-order two-pass reduction (deterministic).
 * d_out: 3 doubles of device memory. */
int lbm_diag_fp64(lbm_handle *h, const void *f, const uint8_t *mask, double *d_out, void *stream);

/* lbm_diag_fp64 without a handle and without allocating: no counterpart in the
 * reference.  For callers that cannot call cudaMalloc (a host whose allocator
 * owns the device heap, a time loop that must not make a call that can
 * synchronise or run out of memory, a foreign runtime that only lends its own
 * buffers).  Its scratch is a fixed array of about 384 KiB inside the library,
 * one per device; domains of more than LBM_NOALLOC_MAX_CELLS cells return
 * LBM_ERR_TOO_LARGE.  The first call on a device looks up that array's address
 * (make it before any stream capture).  All calls on a device share the array:
 * calls whose work overlaps on the GPU race and must be ordered by the caller.
 * f: W*H*9 elements of `storage`; d_out: 3 doubles (mass, jx, jy). */
#define LBM_NOALLOC_MAX_CELLS 134217728LL /* 16384 blocks x 8192 cells, e.g. 16384 x 8192 */
int lbm_diag_fp64_noalloc(int W, int H, int storage, const void *f, const uint8_t *mask, double *d_out,
                          void *stream);

/* Momentum-exchange force on LBM_MASK_OBSTACLE cells, sum 2 c_q f_q(x) over fluid
 * x and directions q with x + c_q an obstacle cell, in FP64 (deterministic).
 * d_out: 2 doubles (Fx = drag, Fy = lift) of device memory. */
int lbm_forces_fp64(lbm_handle *h, const void *f, const uint8_t *mask, double *d_out, void *stream);

/* Periodic halo refresh in x of one state of `width` columns (no counterpart in
 * the reference, which has no periodic sides): columns [0, halo) take columns
 * [width - 2 halo, width - halo) and columns [width - halo, width) take
 * [halo, 2 halo), in all 9 planes and H rows; one launch.  The single-rank
 * periodic slab uses it between launches. */
int lbm_periodic_halo_x(void *f, int width, int H, int halo, int storage, void *stream);

/* Convert a state between storage formats (W*H*9 elements each). */
int lbm_convert_state(int W, int H, const void *src, int src_storage, void *dst, int dst_storage, void *stream);

/* ------------------------------------------------------------------------
 * Batched independent domains (no reference counterpart): many domains of
 * uneven size advance together in one persistent launch per T steps; the
 * CTAs take (domain, strip, row-chunk) work items from a device counter.
 * ------------------------------------------------------------------------ */

typedef struct lbm_domain {
    int W, H;
    int pitch;       /* elements between rows of a plane (0 = W); multiples of 16 enable TMA */
    int mask_pitch;  /* bytes between mask rows (0 = W) */
    void *f_a, *f_b; /* ping-pong states, 9 planes of pitch*H elements of the batch's storage */
    const uint8_t *mask;
    float u_in;      /* inlet velocity of this domain */
} lbm_domain;

typedef struct lbm_batch lbm_batch;

/* Copies the domain table (and a per-domain tensor-map table) to the device.
 * common->W/H are ignored; the physics variant must be MRT + Smagorinsky
 * with FP32 or FP16-deviation storage. */
int lbm_batch_create(const lbm_params *common, const lbm_domain *domains, int n, lbm_batch **out);
int lbm_batch_destroy(lbm_batch *b);

/* n_steps steps of every domain, T per launch (T = 0: the autotuned choice,
 * else 1..8).  Launch pairs are replayed from a captured CUDA graph unless the
 * stream is itself capturing.  *result_in_b = 1 when the states end in f_b. */
int lbm_batch_run(lbm_batch *b, int n_steps, int T, void *stream, int *result_in_b);

/* The same steps with one ordinary launch per domain (the comparison point). */
int lbm_batch_run_separate(lbm_batch *b, int n_steps, int T, void *stream, int *result_in_b);

/* Tile shape: a work item is one 64-column window (register wavefront) or one
 * strip (shared-memory wavefront) of a domain by `rows` rows, with `rows` chosen
 * per domain size class: class 0 below 2^17 cells, class 1 below 2^19, class 2
 * the rest.  Rows: 8 .. 32 for the register wavefront, 16 .. 128 otherwise, and
 * at least 2 T. */
#define LBM_BATCH_SIZE_CLASSES 3

/* Time candidate configurations on the batch and keep the fastest for T = 0:
 * for every depth T, one row count for all classes first, then each populated
 * size class's rows in turn with the others held.  *best_chunk receives the rows
 * of the largest populated class.  Advances every domain by an even number of
 * steps per candidate (states end in f_a).  Synchronous. */
int lbm_batch_autotune(lbm_batch *b, void *stream, int *best_T, int *best_chunk);

/* The configuration T = 0 runs (tuned, or the default before lbm_batch_autotune):
 * the depth and rows[LBM_BATCH_SIZE_CLASSES]. */
int lbm_batch_get_tiles(const lbm_batch *b, int *T, int *rows);
/* Sets that configuration (LBM_ERR_ARG for a depth or row count out of range). */
int lbm_batch_set_tiles(lbm_batch *b, int T, const int *rows);

/* ------------------------------------------------------------------------
 * Learned closure (no reference counterpart): a 5 -> 32 -> 32 -> 1 MLP (ReLU or
 * SiLU hidden layers, softplus output) maps per-cell features to an eddy
 * viscosity nu_t >= 0; the collision then relaxes the stress moments with
 * 1 / (1/s_nu + 3 nu_t) in place of the Smagorinsky rate.  Features of a cell,
 * from its pre-collision populations: the non-equilibrium stress moments n7 =
 * P_xx - P_yy - rho (u^2 - v^2), n8 = P_xy - rho u v and ne = e - rho (3 |u|^2 -
 * 2) (the energy moment), their magnitude sqrt(n7^2 + n8^2), and rho - 1.
 * Training runs on the GPU through the kernels below (FP32 master weights);
 * inference uses BF16 weights packed by lbm_mlp_pack_act, on the tensor cores.
 * The closure kind selects the hidden activation of inference:
 * LBM_CLOSURE_MLP runs a ReLU network, LBM_CLOSURE_MLP_SILU a SiLU one; the
 * block in lbm_params.mlp must be packed for the same activation (a kernel that
 * finds another sets bit 1 of the device error word).
 * ------------------------------------------------------------------------ */
#define LBM_MLP_IN 5
#define LBM_MLP_HID 32
#define LBM_MLP_NPARAM (LBM_MLP_HID * LBM_MLP_IN + LBM_MLP_HID + LBM_MLP_HID * LBM_MLP_HID + LBM_MLP_HID + \
                        LBM_MLP_HID + 1) /* W1[32][5], b1[32], W2[32][32], b2[32], w3[32], b3 */
#define LBM_MLP_PACKED_BYTES 4096
#define LBM_MLP_ACT_RELU 0 /* relu(a) */
#define LBM_MLP_ACT_SILU 1 /* silu(a) = a / (1 + exp(-a)) */

/* y[i] = softplus(MLP(x[i])) for n samples x[n][5] (FP32, device), with the
 * hidden activation act (LBM_MLP_ACT_*). */
int lbm_mlp_forward_act(const float *params, int act, const float *x, float *y, int n, void *stream);
/* lbm_mlp_forward_act with ReLU. */
int lbm_mlp_forward(const float *params, const float *x, float *y, int n, void *stream);
/* Bytes of workspace lbm_mlp_grad needs for n samples. */
size_t lbm_mlp_workspace_bytes(int n);
/* Gradient of L = (1/n) sum_i w_i (y_i - target_i)^2 (w = NULL: all 1) with
 * respect to the parameters, and L; deterministic (fixed-order reductions). */
int lbm_mlp_grad_act(const float *params, int act, const float *x, const float *target, const float *weight, int n,
                     float *grad, float *loss, void *workspace, size_t workspace_bytes, void *stream);
/* lbm_mlp_grad_act with ReLU. */
int lbm_mlp_grad(const float *params, const float *x, const float *target, const float *weight, int n, float *grad,
                 float *loss, void *workspace, size_t workspace_bytes, void *stream);
/* One Adam update of the parameters (step >= 1 for the bias corrections). */
int lbm_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float beta1, float beta2,
                 float eps, void *stream);
/* BF16 inference block for lbm_params.mlp, for the hidden activation act: the
 * features are multiplied by in_scale[5] before the first layer and nu_t =
 * out_scale * softplus(z). */
int lbm_mlp_pack_act(const float *params, int act, const float *in_scale, float out_scale, void *packed,
                     void *stream);
/* lbm_mlp_pack_act with ReLU. */
int lbm_mlp_pack(const float *params, const float *in_scale, float out_scale, void *packed, void *stream);

/* Read (and optionally clear) the device error word of the current device:
 * bit 0 = a bounded device-side wait gave up (the kernel then stopped its work
 * and returned; the launch itself reports success); bit 1 = a learned-closure
 * block packed for another activation than the closure kind.  Synchronises the
 * device. */
int lbm_device_error_flags(int *flags, int clear);

/* Self-test of the give-up path of the bounded device-side waits (no reference
 * counterpart): one CTA initialises an mbarrier and waits on it with a limit of
 * limit_cycles SM cycles (1 .. 2^31).  With arrive = 0 nothing arrives and no
 * copy is issued, so the wait runs out, the kernel sets bit 0 of the device
 * error word and returns; with arrive = 1 the CTA arrives first and the wait
 * succeeds.  d_cycles (optional, one device int64) receives the cycles the
 * wait took.  Nothing faults or hangs either way. */
int lbm_selftest_wait_timeout(long long limit_cycles, int arrive, long long *d_cycles, void *stream);

/* Human-readable text for a status code (static storage). */
const char *lbm_error_string(int status);

/* Library version, major*10000 + minor*100 + patch. */
int lbm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LBM_B200_H */
