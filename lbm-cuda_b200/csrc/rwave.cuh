// Register wavefront kernel: T fused pull steps (1 <= T <= 6; the general
// solver uses it for 2 <= T <= 6, the learned closure for 1 <= T <= 4) with the
// intermediate time levels held in registers.
//
// Same state convention, boundary rules and per-cell codes as the shared-
// memory wavefront kernel (wave.cuh): stored populations are post-collision
// values, one step pulls f_q(x) = f*_q(x - c_q) (or bounces back from solid
// sources) and collides.
//
// Decomposition.  Every warp is independent (no CTA barrier anywhere).  A warp
// owns a window of 64 columns, two adjacent columns per lane, and a chunk of
// output rows [ya, yb) (one work item, see rw_items); it sweeps rows
// ya - T .. yb + T - 1 upwards once:
//   level 0   the input row of the iteration, brought by TMA (one 3-D box
//             [64 + pad, 1, 9] plus the mask row) into a private ring of D
//             rows with one mbarrier per slot, P rows ahead;
//   level t   (1 <= t < T) computed for row yk - t at iteration yk, lag one
//             row per level, and kept in registers: the row just computed
//             (all 9 populations), the one before (all 9: its own values are
//             needed for bounce-back) and q = 2, 5, 6 of the one before that;
//   level T   row yk - T, stored to HBM for the window's core columns
//             [T, 64 - T) and the chunk's rows.
// The x-neighbours of a lane's two columns come from the adjacent lanes by
// warp shuffle (six per level).  Level t is valid on window columns
// [t, 64 - t) and rows [ya - T + t, yb + T - t); values outside that cone are
// never stored and never feed a valid value, and the rows below the cone are
// not computed at all.
//
// Cells needing more than the plain pull + collide (solid or moving-wall
// neighbours, the Zou-He inlet, the outlet ghost, cells that are not updated,
// domain edges) are found per row from the mask: a row of the window is
// "special" when any lane sees a nonzero mask byte in its 3 x 4 neighbourhood
// or touches a domain edge.  Codes (wave.cuh's C_* bits) are built, bit-
// parallel from the mask bytes, only for special rows; a per-warp history
// bit-mask tells each iteration whether all T rows it works on are plain (fast
// body) or not (generic body: bounce-back by selects, then the same two-cell
// collision; the Zou-He and outlet-ghost work only in the windows that hold
// the inlet or outlet column).
#pragma once

#include "mlp.cuh"
#include "wave_launch.cuh"

namespace lbm {

#ifndef LBM_MLP_WARPS
#define LBM_MLP_WARPS 12 // resident warps per SM the learned-closure kernels are sized for
#endif

template <int T_, int NW_, int P_, class Ph_, class St_, int MODE_, bool LID_ = false, bool PACKED_ = true,
          int MINB_ = 0, int LAG_ = 1>
struct RwCfg {
    static constexpr int T = T_;
    static constexpr int NW = NW_; // warps (windows) per CTA
    static constexpr int P = P_;   // TMA prefetch distance in rows
    static constexpr int D = P + 3; // ring depth: rows yk-2, yk-1, yk in use + P in flight
    // Rows between consecutive time levels: 1 (level t at row yk - t) or 2 (level t
    // at row yk - 1 - 2 (t - 1): the levels of an iteration no longer depend on
    // each other, at the cost of one more carried row per level).  Lag 2 passed the
    // parity tests but measured slower at T = 2 (64 against 113 GLUPS FP32 on the
    // 4096 x 1024 cylinder: the extra row spills at 128 registers), so the
    // dispatchers use lag 1.
    static constexpr int LAG = LAG_;
    static_assert(LAG == 1 || LAG == 2, "lag");
    // Left pad of the window: T rounded up to even, so that a lane's column pair
    // stays 8-byte aligned; CW output columns [PADL, 64 - PADL).
    static constexpr int PADL = T_ + (T_ & 1);
    static constexpr int CW = 64 - 2 * PADL;
    static constexpr int MODE = MODE_;
    static constexpr bool LID = LID_;
    // two-cell collision on the packed FP32x2 pipe (collide_pair; collide_ref_pair for
    // the reference's evaluation order, up to T = 3 only: its moment vector costs
    // registers the deeper kernels do not have) or scalar (collide_multi, collide_bf)
    static constexpr bool PACKED = PACKED_ && (!Ph_::kRefOrder || T_ <= 3);
    using Ph = Ph_;
    using St = St_;
    using E = typename St::T;
    static constexpr int ES = (int)sizeof(E);
    static constexpr int AE = 16 / ES;  // TMA x alignment in elements
    static constexpr int BW = 64 + AE;  // population box width (elements)
    static constexpr int BWM = 80;      // mask box width (bytes)
    static constexpr int SLOT_F = round_up(9 * BW * ES, 128);
    static constexpr int SLOT = SLOT_F + 128;
    static constexpr int CR = 8; // code ring rows
    static constexpr bool MLP = Ph_::kMlp;
    static constexpr int MLP_BYTES = MLP ? 64 * 8 * 2 + 64 * 4 : 0; // feature stage + outputs
    static constexpr int WARP_BYTES = 128 + D * SLOT + CR * 32 * 8 + MLP_BYTES;
    static constexpr int SMEM = NW * WARP_BYTES;
    static constexpr uint32_t TX_BYTES = 9 * BW * ES + BWM;
    // resident warps per SM the registers are sized for: 16 / 12 / 8 (<= 128 / 170 / 255 registers)
    static constexpr int MINB_R =
        (MLP ? LBM_MLP_WARPS : ((T <= 2) ? (LAG_ == 2 ? 14 : 16) : ((T <= 4) ? 12 : 8))) / NW;
    static constexpr int MINB_S = (227 * 1024) / (SMEM + 1024);
    static constexpr int MINB_A = MINB_ > 0 ? MINB_ : MINB_R; // blocks per SM the registers are sized for
    static constexpr int MINB = MINB_A < MINB_S ? MINB_A : MINB_S;
    static_assert(T >= 1 && T <= 6 && CR >= LAG_ * (T - 1) + 2, "temporal depth / code ring rows");
    static_assert(D * 8 <= 128, "mbarriers");
    static_assert(MINB >= 1, "shared memory");
};

// Two adjacent stored populations <-> float2 (16-bit formats hold f - w).
__device__ __forceinline__ float2 ld2(const float *p, int)
{
    return *reinterpret_cast<const float2 *>(p);
}
// 16-bit deviations: the weight is added (subtracted on store) on the packed
// FP32x2 pipe, one instruction for both cells.
__device__ __forceinline__ float2 ld2(const __half *p, int q)
{
    return add2(__half22float2(*reinterpret_cast<const __half2 *>(p)), bc2(wgt(q)));
}
__device__ __forceinline__ float2 ld2(const __nv_bfloat16 *p, int q)
{
    return add2(__bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(p)), bc2(wgt(q)));
}
__device__ __forceinline__ void st2(float *p, float2 v, int)
{
    *reinterpret_cast<float2 *>(p) = v;
}
__device__ __forceinline__ void st2(__half *p, float2 v, int q)
{
    const float2 d = sub2(v, bc2(wgt(q)));
    *reinterpret_cast<__half2 *>(p) = __floats2half2_rn(d.x, d.y);
}
__device__ __forceinline__ void st2(__nv_bfloat16 *p, float2 v, int q)
{
    const float2 d = sub2(v, bc2(wgt(q)));
    *reinterpret_cast<__nv_bfloat162 *>(p) = __floats2bfloat162_rn(d.x, d.y);
}

// Pull of both cells of a lane from the three source rows of the previous
// level: S = row y-1 (q 2, 5, 6 used), O = row y (q 0, 1, 3), N = row y+1
// (q 4, 7, 8).  g[q].x / .y are the pulled values of columns x / x+1.
__device__ __forceinline__ void pull2(const float2 (&S)[9], const float2 (&O)[9], const float2 (&N)[9], float2 (&g)[9])
{
    const unsigned M = 0xffffffffu;
    g[0] = O[0];
    g[1] = make_float2(__shfl_up_sync(M, O[1].y, 1), O[1].x);
    g[2] = S[2];
    g[3] = make_float2(O[3].y, __shfl_down_sync(M, O[3].x, 1));
    g[4] = N[4];
    g[5] = make_float2(__shfl_up_sync(M, S[5].y, 1), S[5].x);
    g[6] = make_float2(S[6].y, __shfl_down_sync(M, S[6].x, 1));
    g[7] = make_float2(N[7].y, __shfl_down_sync(M, N[7].x, 1));
    g[8] = make_float2(__shfl_up_sync(M, N[8].y, 1), N[8].x);
}

// 0x01 in every byte of w that is nonzero.
__host__ __device__ __forceinline__ uint32_t nz_bytes(uint32_t w)
{
    w |= w >> 4;
    w |= w >> 2;
    w |= w >> 1;
    return w & 0x01010101u;
}
// Gathers the low bits of the four bytes of b (each 0 or 1) into bits 0..3.
__host__ __device__ __forceinline__ uint32_t gather4(uint32_t b)
{
    return ((b * 0x01020408u) >> 24) & 0xfu; // byte k -> bit 24 + k, no overlapping terms
}
// Bounce bits (bit q set: the pull source of q is solid) of the cell at bit
// position 1 of the solid nibbles s0, s1, s2 (rows y-1, y, y+1; bit k <->
// column x-1+k): the source of q is column 1 - c_x of row 1 - c_y.
__host__ __device__ __forceinline__ uint32_t bounce_bits(uint32_t s0, uint32_t s1, uint32_t s2)
{
    return ((s1 & 5u) << 1)         // q1 <- (x-1, y), q3 <- (x+1, y)
           | ((s0 & 2u) << 1)       // q2 <- (x, y-1)
           | ((s2 & 2u) << 3)       // q4 <- (x, y+1)
           | ((s0 & 1u) << 5)       // q5 <- (x-1, y-1)
           | ((s0 & 4u) << 4)       // q6 <- (x+1, y-1)
           | ((s2 & 4u) << 5)       // q7 <- (x+1, y+1)
           | ((s2 & 1u) << 8);      // q8 <- (x-1, y+1)
}

// Codes of the two cells x, x+1 of row R from the mask bytes of columns
// x-1 .. x+2 (raw[d], byte b <-> column x-1+b, rows R-1+d), bit-parallel.
// Equal to build_code_general / build_code_core4 (wave.cuh) for non-periodic x
// when out-of-domain mask bytes read zero; oob_cols has 0x01 in the bytes of
// columns outside [0, W).
template <int MODE, bool LID>
__host__ __device__ __forceinline__ void codes_from_bytes(const uint32_t (&raw)[3], uint32_t oob_cols, int x, int R,
                                                          int W, int H, int bc_left, int bc_right, bool py,
                                                          uint32_t (&code)[2])
{
    const uint32_t own0 = (raw[1] >> 8) & 0xffu, own1 = (raw[1] >> 16) & 0xffu;
    const uint32_t left0 = raw[1] & 0xffu;
    if (MODE == MODE_CORE4) {
        // lbm_core4.cu rules: out-of-domain sources are never consulted by updated cells
        const uint32_t n0 = gather4(nz_bytes(raw[0])), n1 = gather4(nz_bytes(raw[1])), n2 = gather4(nz_bytes(raw[2]));
        const bool rowin = R >= 1 && R <= H - 2;
#pragma unroll
        for (int n = 0; n < 2; ++n) {
            const int xn = x + n;
            const bool own = (n == 0 ? own0 : own1) != 0u;
            const bool upd = rowin && xn >= 0 && xn <= W - 2 && (xn == 0 || !own);
            uint32_t c;
            if (!upd) {
                c = C_SKIP;
                if (xn == W - 1 && rowin && (n == 0 ? left0 : own0) == 0u)
                    c |= C_GHOST_SKIP;
            } else {
                c = bounce_bits(n0 >> n, n1 >> n, n2 >> n);
                if (xn == 0)
                    c = (c & ~((1u << 1) | (1u << 5) | (1u << 8))) | C_INLET; // x = -1 sources read zero
                if (xn == W - 2)
                    c |= C_GHOST_SRC;
            }
            code[n] = c;
        }
        return;
    }
    const bool outflow = bc_right == LBM_BC_OUTFLOW;
    const bool zh = bc_left == LBM_BC_ZOUHE || bc_left == LBM_BC_ZOUHE_RAMP;
    uint32_t sn[3], mv[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const int r = R - 1 + d;
        const bool row_oob = !py && (r < 0 || r >= H);
        sn[d] = row_oob ? 0xfu : gather4(nz_bytes(raw[d]) | oob_cols);
        // a moving wall is a mask byte of value 2 inside the domain
        mv[d] = LID ? gather4(0x01010101u & ~nz_bytes(raw[d] ^ 0x02020202u)) : 0u;
    }
    const bool rowin = py || (R >= 0 && R < H);
#pragma unroll
    for (int n = 0; n < 2; ++n) {
        const int xn = x + n;
        const bool in_dom = rowin && xn >= 0 && xn < W;
        const bool own = (n == 0 ? own0 : own1) != 0u;
        const bool upd = in_dom && !own && !(outflow && xn == W - 1);
        uint32_t c;
        if (!upd) {
            c = C_SKIP;
            if (outflow && in_dom && xn == W - 1 && (n == 0 ? left0 : own0) == 0u)
                c |= C_GHOST_SKIP;
        } else {
            c = bounce_bits(sn[0] >> n, sn[1] >> n, sn[2] >> n);
            if (LID)
                c |= bounce_bits(mv[0] >> n, mv[1] >> n, mv[2] >> n) << C_MOVING_SHIFT;
            if (zh && xn == 0)
                c |= C_INLET;
            if (outflow && xn == W - 2)
                c |= C_GHOST_SRC;
        }
        code[n] = c;
    }
}

// Work items of a launch: (window, row range).  The windows at the domain's
// left and right ends take the generic body on every row (inlet, outlet, out-
// of-domain columns), so they come first in launch order and in chunks of half
// the height; the hardware starts CTAs in index order as earlier ones finish,
// which lets the cheaper items fill in behind them.  The other items follow
// window by window (vertically adjacent chunks of a window run at about the
// same time): on the 4096 x 1024 cylinder at T = 2, 118.3 GLUPS against 115.3
// with the chunks of a row band consecutive, at the same DRAM traffic.
struct RwItems {
    int nwin, wr, nedge, che, nche, nch, n_edge_items, n_items;
};
__host__ __device__ __forceinline__ RwItems rw_items(int W, int H, int CW, int PADL, int chunk)
{
    RwItems it;
    it.nwin = (W + CW - 1) / CW;
    // first window whose columns reach W - 3 (xs + 63 >= W - 3, xs = w CW - PADL)
    int wr = (W - 66 + PADL + CW - 1) / CW;
    if (wr < 1)
        wr = 1;
    if (wr > it.nwin)
        wr = it.nwin;
    it.wr = wr;
    it.nedge = 1 + (it.nwin - wr);
    it.che = (chunk + 1) / 2;
    it.nche = (H + it.che - 1) / it.che;
    it.nch = (H + chunk - 1) / chunk;
    it.n_edge_items = it.nedge * it.nche;
    it.n_items = it.n_edge_items + (it.nwin - it.nedge) * it.nch;
    return it;
}
__host__ __device__ __forceinline__ void rw_item(const RwItems &it, int item, int H, int chunk, int &win, int &ya,
                                                 int &yb)
{
    if (item < it.n_edge_items) {
        const int e = item % it.nedge, k = item / it.nedge;
        win = e == 0 ? 0 : it.wr + e - 1;
        ya = k * it.che;
        yb = min(H, ya + it.che);
    } else {
        // window by window: consecutive items are vertically adjacent row chunks
        // of one window
        const int j = item - it.n_edge_items;
        win = 1 + j / it.nch;
        ya = (j % it.nch) * chunk;
        yb = min(H, ya + chunk);
    }
}

// rho, u, v of a lane's two cells in the reference's summation order.
__device__ __forceinline__ void moments_pair(const float2 (&g)[9], float2 &r, float2 &u, float2 &v)
{
    float f0[9], f1[9], r0, u0, v0, r1, u1, v1;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        f0[q] = g[q].x;
        f1[q] = g[q].y;
    }
    moments_seq(f0, r0, u0, v0);
    moments_seq(f1, r1, u1, v1);
    r = make_float2(r0, r1);
    u = make_float2(u0, u1);
    v = make_float2(v0, v1);
}

// Per-warp state of the learned closure (unused by the other variants).
struct MlpCtx {
    MlpFrag F;
    __nv_bfloat16 *stage;
    float *zbuf;
    int lane;
};

// Collision of a lane's two cells without Zou-He: packed or scalar, or with the
// learned closure (warp-collective).
template <class C>
__device__ __forceinline__ void collide_two(float2 (&g)[9], const Phys &k, float2 &r, float2 &u, float2 &v,
                                            const MlpCtx &mc)
{
    using Ph = typename C::Ph;
    if constexpr (C::MLP) {
        collide_pair_mlp<Ph, false>(g, false, false, 0.0f, k, mc.F, mc.stage, mc.zbuf, mc.lane, r, u, v);
    } else if constexpr (C::PACKED) {
        if constexpr (Ph::kRefOrder)
            collide_ref_pair<Ph>(g, k, r, u, v);
        else
            collide_pair<Ph>(g, k, r, u, v);
    } else {
        float f[2][9], r_[2], u_[2], v_[2];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            f[0][q] = g[q].x;
            f[1][q] = g[q].y;
        }
        if constexpr (Ph::kRefOrder) {
#pragma unroll
            for (int n = 0; n < 2; ++n)
                collide_bf<Ph, false>(f[n], false, 0.0f, k, r_[n], u_[n], v_[n]);
        } else {
            collide_multi<Ph, 2>(f, k, r_, u_, v_);
        }
#pragma unroll
        for (int q = 0; q < 9; ++q)
            g[q] = make_float2(f[0][q], f[1][q]);
        r = make_float2(r_[0], r_[1]);
        u = make_float2(u_[0], u_[1]);
        v = make_float2(v_[0], v_[1]);
    }
}

// One work item: window `win` (columns rx0 + win CW - PADL ..) and output rows
// [ya, yb) of the domain p; run by one whole warp (lane = threadIdx.x % 32, the
// warp's shared memory at wi * WARP_BYTES).
template <class C>
__device__ __forceinline__ void rwave_run(const WaveParams &p, const CUtensorMap *tmf_, const CUtensorMap *tmm_,
                                          int win, int ya, int yb)
{
    using Ph = typename C::Ph;
    using St = typename C::St;
    using E = typename C::E;
    constexpr int T = C::T, D = C::D, P = C::P, BW = C::BW, CR = C::CR;
    constexpr unsigned M = 0xffffffffu;
    constexpr bool PRE = C::MODE == MODE_PRE_SMEMAA || C::MODE == MODE_PRE_POLICY;
    const CUtensorMap &tmf = *tmf_;
    const CUtensorMap &tmm = *tmm_;

    extern __shared__ __align__(128) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wi = threadIdx.x >> 5;
    const int rx0 = p.rx1 > 0 ? p.rx0 : 0, rx1 = p.rx1 > 0 ? p.rx1 : p.W;
    unsigned char *wbase = smem + wi * C::WARP_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(wbase);
    unsigned char *ring = wbase + 128;
    uint2 *cring = reinterpret_cast<uint2 *>(wbase + 128 + D * C::SLOT);
    MlpCtx mc;
    mc.lane = lane;
    if constexpr (C::MLP) {
        unsigned char *mb = wbase + 128 + D * C::SLOT + CR * 32 * 8;
        mc.stage = reinterpret_cast<__nv_bfloat16 *>(mb);
        mc.zbuf = reinterpret_cast<float *>(mb + 64 * 8 * 2);
        const MlpPacked *W = static_cast<const MlpPacked *>(p.k.mlp);
        mlp_load_frag(W, mc.F, lane);
        if (lane == 0 && p.err && W->act != Ph::kMlpAct)
            atomicOr(p.err, 2); // the block was packed for another activation
    }

    const int xs = rx0 + win * C::CW - C::PADL;
    const int x = xs + 2 * lane; // column of the lane's first cell
    const int row0 = ya - T;
    constexpr int LAG = C::LAG;
    const int nrows = yb - ya + T + LAG * (T - 1) + 1;
    const bool pyper = (C::MODE == MODE_GENERAL) && p.bc_y == LBM_BC_PERIODIC;
    const int xa = floor_div(xs, C::AE) * C::AE; // TMA box origins (aligned)
    const int xm = floor_div(xs, 16) * 16;
    const int offf = (xs - xa) + 2 * lane; // element offset of the lane's pair in a ring row
    const int offm = (xs - xm) + 2 * lane; // byte offset of the lane's mask pair
    // Columns at or next to the domain's left/right ends are always special
    // (for the whole window).
    const bool colspec = !PRE && (x <= 0 || x + 1 >= p.W - 2);
    const bool wcolspec = __any_sync(M, colspec);
    const bool core0 = 2 * lane >= C::PADL && 2 * lane < 64 - C::PADL;
    // Window-wide work of the generic body: Zou-He inlet and outlet ghost.
    const bool win_inlet =
        xs <= 0 && (C::MODE == MODE_CORE4 || p.bc_left == LBM_BC_ZOUHE || p.bc_left == LBM_BC_ZOUHE_RAMP);
    const bool win_ghost = xs + 63 >= p.W - 1 && (C::MODE == MODE_CORE4 || p.bc_right == LBM_BC_OUTFLOW);
    uint32_t oob_cols = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
        oob_cols |= ((x - 1 + b < 0 || x - 1 + b >= p.W) ? 1u : 0u) << (8 * b);

    if (lane == 0) {
        for (int s = 0; s < D; ++s)
            mbar_init(&bar[s], 1);
        mbar_fence_init();
        prefetch_tmap(&tmf);
        prefetch_tmap(&tmm);
    }
#pragma unroll
    for (int s = 0; s < CR; ++s)
        cring[s * 32 + lane] = make_uint2(0u, 0u);
    __syncwarp();

    auto issue = [&](int j) { // lane 0: ring row j = row0 + j into slot j % D
        const int s = j % D;
        const int r = row0 + j;
        const int ry = pyper ? wrap(r, p.H) : r;
        unsigned char *dst = ring + s * C::SLOT;
        mbar_arrive_expect_tx(&bar[s], C::TX_BYTES);
        tma_load_3d(dst, &tmf, &bar[s], xa, ry, 0);
        tma_load_2d(dst + C::SLOT_F, &tmm, &bar[s], xm, ry);
    };
    if (lane == 0) {
        fence_proxy_async();
        for (int j = 0; j < P && j < nrows; ++j)
            issue(j);
    }

    // Carried levels 1..T-1: pv = row yk-t-1 (all q), p2 = row yk-t-2 (q 2,5,6
    // stored at their own indices; the others unused), cu = row yk-t.
    constexpr int NL = T > 1 ? T - 1 : 1; // carried levels (one unused slot at T = 1)
    float2 pv[NL][9], p2[NL][9], p3[NL][9], cu[NL][9]; // p3: the LAG == 2 extra row
#pragma unroll
    for (int t = 0; t < NL; ++t)
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            pv[t][q] = make_float2(wgt(q), wgt(q));
            p2[t][q] = pv[t][q];
            p3[t][q] = pv[t][q];
            cu[t][q] = pv[t][q];
        }

    uint32_t hist = 0; // bit t-1: the row of level t in this iteration is special
    uint32_t rhist = 0; // bit d: ring row i - d has a nonzero mask byte in the window
    int s0 = 0, ph = 0; // slot and phase of ring row i
    int abort = 0, i_ab = 0;
    for (int i = 0; i < nrows; ++i) {
        const int yk = row0 + i;
        __syncwarp(); // every lane is done with the slot that is refilled next
        if (lane == 0 && i + P < nrows) {
            fence_proxy_async();
            issue(i + P);
        }
        bool ok = mbar_wait_bounded(&bar[s0], (uint32_t)ph);
        if (!__all_sync(M, ok)) {
            abort = 1;
            i_ab = i;
            break;
        }
        const int s1 = s0 == 0 ? D - 1 : s0 - 1;
        const int s2 = s1 == 0 ? D - 1 : s1 - 1;
        const E *rN = reinterpret_cast<const E *>(ring + s0 * C::SLOT) + offf;
        const E *rO = reinterpret_cast<const E *>(ring + s1 * C::SLOT) + offf;
        const E *rS = reinterpret_cast<const E *>(ring + s2 * C::SLOT) + offf;
        if constexpr (PRE) {
            // collide the new row in place (its own cells only): the ring then holds
            // post-collision values, which the levels above stream and collide
            float *rw = reinterpret_cast<float *>(ring + s0 * C::SLOT) + offf;
            const uint32_t om =
                *reinterpret_cast<const uint16_t *>(ring + s0 * C::SLOT + C::SLOT_F + offm); // own mask bytes
            float2 g[9];
#pragma unroll
            for (int q = 0; q < 9; ++q)
                g[q] = ld2(rw + q * BW, q);
            float2 rr, uu, vv;
            float2 c[9];
#pragma unroll
            for (int q = 0; q < 9; ++q)
                c[q] = g[q];
            collide_two<C>(c, p.k, rr, uu, vv, mc);
            const bool sk0 = (om & 0xffu) != 0u, sk1 = (om >> 8) != 0u;
#pragma unroll
            for (int q = 0; q < 9; ++q)
                st2(rw + q * BW, make_float2(sk0 ? g[q].x : c[q].x, sk1 ? g[q].y : c[q].y), q);
            fence_proxy_async(); // these generic writes precede the slot's next TMA refill
            __syncwarp();
        }

        // ---- codes of level 1's row (yk - 1) from mask rows yk-2 .. yk ----
        // The row is special when the window's columns hold a nonzero mask byte in
        // one of the three rows (one vote per new row, kept as a bit history), or
        // it lies at a domain end; the neighbourhood words and codes are built
        // only then.  (The window's 64 columns cover the neighbourhoods of every
        // cell whose value is used: columns 1 .. 62 at level 1.)
        {
            const uint32_t own_new = *reinterpret_cast<const uint16_t *>(ring + s0 * C::SLOT + C::SLOT_F + offm);
            rhist = (rhist << 1) | (__any_sync(M, own_new != 0u) ? 1u : 0u);
            const int R1 = yk - 1;
            const bool rowspec = !PRE && !pyper && (R1 <= 0 || R1 >= p.H - 1);
            const bool wspec = wcolspec || rowspec || (rhist & 7u) != 0u;
            hist = (hist << 1) | (wspec ? 1u : 0u);
            uint2 cc = make_uint2(0u, 0u);
            if (wspec) {
                uint32_t mw[3];
                const unsigned char *mb[3] = {ring + s2 * C::SLOT + C::SLOT_F, ring + s1 * C::SLOT + C::SLOT_F,
                                              ring + s0 * C::SLOT + C::SLOT_F};
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    const uint32_t own = *reinterpret_cast<const uint16_t *>(mb[d] + offm);
                    const uint32_t lft = __shfl_up_sync(M, own, 1);
                    const uint32_t rgt = __shfl_down_sync(M, own, 1);
                    mw[d] = ((lft >> 8) & 0xffu) | (own << 8) | ((rgt & 0xffu) << 24);
                }
                uint32_t c2[2];
                codes_from_bytes<PRE ? (int)MODE_GENERAL : C::MODE, C::LID>(mw, oob_cols, x, R1, p.W, p.H,
                                                                            PRE ? (int)LBM_BC_WALL : p.bc_left,
                                                                            PRE ? (int)LBM_BC_WALL : p.bc_right,
                                                                            pyper, c2);
                cc = make_uint2(c2[0], c2[1]);
            }
            cring[((i + CR - 1) & (CR - 1)) * 32 + lane] = cc;
        }

        constexpr uint32_t HMASK = [] {
            uint32_t m = 0;
            for (int t = 1; t <= C::T; ++t)
                m |= 1u << (C::LAG * (t - 1));
            return m;
        }();
        const bool fast = (hist & HMASK) == 0u;
        float2 out[9], mr, mu, mv;

        // Level t: sources S/O/N of level t-1, result into cu[t-1] (t < T) or out.
        static_for<1, T + 1>([&](auto tt) {
            constexpr int t = decltype(tt)::value;
            if (i < 1 + t + LAG * (t - 1))
                return; // below level t's cone: nothing valid to compute yet
            float2 S[9], O[9], N[9];
            if constexpr (t == 1) {
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    S[q] = (q == 2 || q == 5 || q == 6) ? ld2(rS + q * BW, q) : make_float2(0.f, 0.f);
                    N[q] = (q == 4 || q == 7 || q == 8) ? ld2(rN + q * BW, q) : make_float2(0.f, 0.f);
                    O[q] = (fast && !(q == 0 || q == 1 || q == 3)) ? make_float2(0.f, 0.f) : ld2(rO + q * BW, q);
                }
            } else {
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    if constexpr (LAG == 1) {
                        S[q] = p2[t - 2][q];
                        O[q] = pv[t - 2][q];
                        N[q] = cu[t - 2][q];
                    } else {
                        S[q] = p3[t - 2][q];
                        O[q] = p2[t - 2][q];
                        N[q] = pv[t - 2][q];
                    }
                }
            }
            float2 g[9];
            pull2(S, O, N, g);
            float2 r_, u_, v_;
            // pre-collision storage: the last level only streams (its result is the
            // canonical state); u, v, rho are the moments of that state
            constexpr bool STREAM_ONLY = PRE && t == T;
            if (fast && STREAM_ONLY) {
                moments_pair(g, r_, u_, v_);
            } else if (fast) {
                collide_two<C>(g, p.k, r_, u_, v_, mc);
            } else {
                const uint2 cc = cring[((i - 1 - LAG * (t - 1) + 2 * CR) & (CR - 1)) * 32 + lane];
                // half-way bounce-back (and Ladd's moving-wall term) by selects
#pragma unroll
                for (int q = 1; q < 9; ++q) {
                    float bx = O[opp(q)].x, by = O[opp(q)].y;
                    if (C::LID) {
                        const float du = 6.0f * wgt(q) * (float)cx(q) * p.k.u_lid;
                        bx += ((cc.x >> (C_MOVING_SHIFT + q)) & 1u) ? du : 0.0f;
                        by += ((cc.y >> (C_MOVING_SHIFT + q)) & 1u) ? du : 0.0f;
                    }
                    g[q].x = ((cc.x >> q) & 1u) ? bx : g[q].x;
                    g[q].y = ((cc.y >> q) & 1u) ? by : g[q].y;
                }
                if constexpr (STREAM_ONLY) {
                    moments_pair(g, r_, u_, v_);
                } else if (win_inlet) {
                    const int R = yk - 1 - LAG * (t - 1);
                    const float lu = inlet_u(p.k, pyper ? wrap(R, p.H) : R);
                    if constexpr (C::MLP) {
                        collide_pair_mlp<Ph, true>(g, (cc.x & C_INLET) != 0, (cc.y & C_INLET) != 0, lu, p.k, mc.F,
                                                   mc.stage, mc.zbuf, lane, r_, u_, v_);
                    } else {
                        float f0[9], f1[9], rr[2], uu[2], vv[2];
#pragma unroll
                        for (int q = 0; q < 9; ++q) {
                            f0[q] = g[q].x;
                            f1[q] = g[q].y;
                        }
                        collide_bf<Ph, true>(f0, (cc.x & C_INLET) != 0, lu, p.k, rr[0], uu[0], vv[0]);
                        collide_bf<Ph, true>(f1, (cc.y & C_INLET) != 0, lu, p.k, rr[1], uu[1], vv[1]);
#pragma unroll
                        for (int q = 0; q < 9; ++q)
                            g[q] = make_float2(f0[q], f1[q]);
                        r_ = make_float2(rr[0], rr[1]);
                        u_ = make_float2(uu[0], uu[1]);
                        v_ = make_float2(vv[0], vv[1]);
                    }
                } else {
                    collide_two<C>(g, p.k, r_, u_, v_, mc);
                }
                if (C::MODE != MODE_GENERAL) {
                    // cells that are not updated pass their values on (lbm_core4.cu's
                    // fluid rows 0 and H-1 are read by their neighbours).  With the
                    // general rules a cell that is not updated is solid, out of the
                    // domain or the outlet ghost: the first two are never read (their
                    // neighbours bounce back) and the ghost is overwritten below.
                    const bool sk0 = (cc.x & C_SKIP) != 0, sk1 = (cc.y & C_SKIP) != 0;
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        g[q].x = sk0 ? O[q].x : g[q].x;
                        g[q].y = sk1 ? O[q].y : g[q].y;
                    }
                }
                if (win_ghost) {
                    // outlet ghost: a C_GHOST_SKIP cell takes the result of its left neighbour
#pragma unroll
                    for (int q = 0; q < 9; ++q) {
                        const float left0 = __shfl_up_sync(M, g[q].y, 1);
                        const float keep0 = g[q].x;
                        g[q].x = (cc.x & C_GHOST_SKIP) ? left0 : g[q].x;
                        g[q].y = (cc.y & C_GHOST_SKIP) ? keep0 : g[q].y;
                    }
                }
            }
            if constexpr (t < T) {
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    cu[t - 1][q] = g[q];
            } else {
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    out[q] = g[q];
                mr = r_;
                mu = u_;
                mv = v_;
            }
        });

        // ---- level T: store row yk - T ----
        const int RT = yk - 1 - LAG * (T - 1);
        if (RT >= ya && RT < yb) {
            E *fo = reinterpret_cast<E *>(p.f_out) + (long long)RT * p.pitch + x;
            if (fast) {
                if (core0 && x + 1 < rx1) {
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        st2(fo + q * p.plane, out[q], q);
                    if (p.ux) {
                        const long long id = (long long)RT * p.W + x;
                        p.ux[id] = mu.x;
                        p.ux[id + 1] = mu.y;
                        p.uy[id] = mv.x;
                        p.uy[id + 1] = mv.y;
                        p.rho[id] = mr.x;
                        p.rho[id + 1] = mr.y;
                    }
                }
            } else {
                const uint2 cc = cring[((i - 1 - LAG * (T - 1) + 2 * CR) & (CR - 1)) * 32 + lane];
                const uint32_t cd[2] = {cc.x, cc.y};
#pragma unroll
                for (int n = 0; n < 2; ++n) {
                    const int xn = x + n;
                    const bool incore = core0 && xn < rx1;
                    const bool upd = !(cd[n] & C_SKIP);
                    // lbm_core_smemaa.cu stores every cell (solid ones unchanged)
                    const bool wr = incore && (upd || (cd[n] & C_GHOST_SKIP) || C::MODE == MODE_PRE_SMEMAA);
                    if (wr) {
#pragma unroll
                        for (int q = 0; q < 9; ++q)
                            fo[q * p.plane + n] = St::store(n == 0 ? out[q].x : out[q].y, q);
                    }
                    if (incore && upd && p.ux) {
                        const long long id = (long long)RT * p.W + xn;
                        p.ux[id] = n == 0 ? mu.x : mu.y;
                        p.uy[id] = n == 0 ? mv.x : mv.y;
                        p.rho[id] = n == 0 ? mr.x : mr.y;
                    }
                }
            }
        }

        // ---- rotate the carried rows ----
#pragma unroll
        for (int t = 0; t < T - 1; ++t) {
            if constexpr (LAG == 2) {
                p3[t][2] = p2[t][2];
                p3[t][5] = p2[t][5];
                p3[t][6] = p2[t][6];
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    p2[t][q] = pv[t][q];
            } else {
                p2[t][2] = pv[t][2];
                p2[t][5] = pv[t][5];
                p2[t][6] = pv[t][6];
            }
#pragma unroll
            for (int q = 0; q < 9; ++q)
                pv[t][q] = cu[t][q];
        }
        if (++s0 == D) {
            s0 = 0;
            ph ^= 1;
        }
    }

    if (abort) {
        if (lane == 0) {
            if (p.err)
                atomicOr(p.err, 1);
            // wait (bounded) for copies still in flight before the CTA may exit
            int s = s0, phase = ph;
            const int inflight = min(P + 1, nrows - i_ab); // rows i_ab .. i_ab + P were issued
            for (int i = 0; i < inflight; ++i) {
                if (!mbar_wait_bounded(&bar[s], (uint32_t)phase))
                    break;
                if (++s == D) {
                    s = 0;
                    phase ^= 1;
                }
            }
        }
        __syncwarp();
    }
}

template <class C>
__global__ void __launch_bounds__(32 * C::NW, C::MINB)
    rwave_kernel(const __grid_constant__ WaveParams p, const __grid_constant__ CUtensorMap tmf,
                 const __grid_constant__ CUtensorMap tmm)
{
    // launched with programmatic dependent launch: wait for the previous launch's
    // stores (its output is this launch's input) before the first row load
    pdl_trigger();
    pdl_wait();
    // output rectangle [rx0, rx1) x [ry0, ry1) (the whole domain unless set)
    const int rx0 = p.rx1 > 0 ? p.rx0 : 0, rx1 = p.rx1 > 0 ? p.rx1 : p.W;
    const int ry0 = p.ry1 > 0 ? p.ry0 : 0, ry1 = p.ry1 > 0 ? p.ry1 : p.H;
    const RwItems items = rw_items(rx1 - rx0, ry1 - ry0, C::CW, C::PADL, p.chunk);
    const int item = blockIdx.x * C::NW + (threadIdx.x >> 5);
    if (item >= items.n_items)
        return; // whole warp: no item left (nothing below waits on other warps)
    int win, ya, yb;
    rw_item(items, item, ry1 - ry0, p.chunk, win, ya, yb);
    rwave_run<C>(p, &tmf, &tmm, win, ya + ry0, yb + ry0);
}

// Launch constraints: TMA-aligned planes and mask (16-byte base, pitches and
// plane strides multiples of 16 bytes), no periodic x (the TMA boxes do not
// wrap), 2 <= T <= 6 (1 <= T <= 6 for the learned closure).
template <class E> inline bool rwave_ok(const WaveParams &p, int T, int mode, bool any_T = false)
{
    const int es = (int)sizeof(E);
    if (any_T ? !(T >= 1 && T <= 6) : !(T >= 2 && T <= 6))
        return false;
    if (!any_T)
        if (const char *e = getenv("LBM_KERNEL"))
            if (e[0] == 'w') // LBM_KERNEL=wave: shared-memory wavefront kernel instead
                return false;
    if (mode == MODE_GENERAL && p.bc_left == LBM_BC_PERIODIC)
        return false;
    bool ok = aligned16(p.f_in) && aligned16(p.f_out) && ((long long)p.pitch * es) % 16 == 0 &&
              (p.plane * es) % 16 == 0 && aligned16(p.mask) && p.mask_pitch % 16 == 0;
    if (p.ux)
        ok = ok && aligned16(p.ux) && aligned16(p.uy) && aligned16(p.rho);
    return ok;
}

template <class C> int rwave_occupancy()
{
    static std::atomic<int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && cache[dev])
        return cache[dev];
    int n = 0;
    cudaFuncSetAttribute(rwave_kernel<C>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, rwave_kernel<C>, 32 * C::NW, C::SMEM);
    if (n < 1)
        n = 1;
    if (dev >= 0 && dev < 64)
        cache[dev] = n;
    return n;
}

template <class C> int launch_rwave(WaveParams p, cudaStream_t s)
{
    const int occ = rwave_occupancy<C>(); // also raises the dynamic shared-memory limit
    // output rectangle (the whole domain unless set); its x bounds are even
    const int Wr = p.rx1 > 0 ? p.rx1 - p.rx0 : p.W;
    const int Hr = p.ry1 > 0 ? p.ry1 - p.ry0 : p.H;
    if (p.rx1 > 0 && ((p.rx0 | p.rx1) & 1))
        return LBM_ERR_ARG;
    if (p.chunk <= 0) {
        // Tuning override for experiments: LBM_RW_CHUNK=<rows per item>.
        int v = 0;
        if (const char *e = getenv("LBM_RW_CHUNK"))
            v = atoi(e);
        if (v < 1) {
            // Short items: several CTAs per resident slot, so the hardware's in-order
            // CTA dispatch balances the cost of the generic rows (measured on the
            // 4096 x 1024 cylinder channel: 16 rows at T = 2, 24 at T >= 4); fewer
            // items than resident warps only on small domains.
            v = C::T <= 2 ? 16 : 24;
            const int nwin = (Wr + C::CW - 1) / C::CW;
            const long long slots = (long long)sm_count() * occ * C::NW;
            if ((long long)nwin * ((Hr + v - 1) / v) < slots) {
                long long nch = slots / nwin;
                if (nch < 1)
                    nch = 1;
                v = (int)((Hr + nch - 1) / nch);
                if (v < 4 * C::T)
                    v = 4 * C::T;
            }
        }
        p.chunk = v;
    }
    if (!p.err)
        p.err = device_error_word();
    CUtensorMap tmf, tmm;
    memset(&tmf, 0, sizeof(tmf));
    memset(&tmm, 0, sizeof(tmm));
    if (!make_map_planes(&tmf, p.f_in, C::ES, p.W, p.H, p.pitch, p.plane, C::BW) ||
        !make_map_mask(&tmm, p.mask, p.W, p.H, p.mask_pitch, C::BWM))
        return LBM_ERR_DEVICE;
    p.use_tma = 1;
    const RwItems it = rw_items(Wr, Hr, C::CW, C::PADL, p.chunk);
    const int grid = (it.n_items + C::NW - 1) / C::NW;
    return status(launch_pdl(rwave_kernel<C>, dim3(grid), dim3(32 * C::NW), (size_t)C::SMEM, s, p, tmf, tmm));
}

} // namespace lbm
