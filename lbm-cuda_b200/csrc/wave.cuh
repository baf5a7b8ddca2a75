// Wavefront temporally-blocked pull kernel (the MRT + Smagorinsky hot path).
//
// State convention: the stored populations are post-collision values, as in
// lbm_core4.cu (f_out of one launch is f_now of the next).  One physical step
// pulls f_q(x) = f*_q(x - c_q), or f*_opp(q)(x) when x - c_q is solid
// (half-way bounce-back), then collides (lbm_core4.cu:120-211).
//
// Decomposition.  A CTA of NX threads owns a vertical strip of NX columns
// (thread i <-> column xs + i) and a chunk of output rows [ya, yb).  It sweeps
// the rows upwards once and advances T time levels in a wavefront:
//   level 0      input rows, streamed from HBM by TMA into a ring of DI rows
//                (one 3-D box [RW x 1 x 9] per row, zero-filled out of bounds);
//   level t      (1 <= t < T) post-collision rows kept in a 4-row ring in
//                shared memory; level t lags level t-1 by two rows, so the
//                three source rows it pulls from were written in earlier
//                iterations and one __syncthreads per row suffices;
//   level T      written straight to HBM for the strip's core columns
//                [x0, x0 + NX - 2T) and the chunk's rows.
// Each cell is read once and written once from HBM per T steps; halo columns
// (T per side) are recomputed by neighbouring strips, halo rows (T per side)
// by neighbouring chunks.
//
// Per-cell flags ("codes") are built once per row from a mask ring that is
// loaded with the input rows: which pull sources are solid (bounce-back),
// moving walls (Ladd), whether the cell is updated, the Zou-He inlet, and the
// zero-gradient outlet (the updated x = W-2 cell also writes the x = W-1 ghost,
// lbm_core4.cu:114-116).  Cells that are not updated pass their previous level
// through unchanged.
#pragma once

#include "collide.cuh"

namespace lbm {

enum : uint32_t {
    C_BOUNCE = 0x1FEu,      // bit q (1..8): the pull source of q is solid
    C_MOVING_SHIFT = 9,     // bit 9+q: that solid source is a moving wall
    C_SKIP = 1u << 20,      // cell is not updated (pass-through)
    C_GHOST_SKIP = 1u << 21, // not updated and its level slot is written by x = W-2
    C_INLET = 1u << 22,     // Zou-He velocity inlet cell
    C_GHOST_SRC = 1u << 23, // updated x = W-2 cell: also feeds the x = W-1 ghost
};

enum : int {
    MODE_CORE4 = 0,   // lbm_core4.cu boundary rules
    MODE_GENERAL = 1, // lbm_params boundary rules
    // Pre-collision storage (the AA kernels' canonical state): collide, then
    // stream; interior of the domain only (register wavefront kernel).  SMEMAA
    // writes every cell (solid ones unchanged) and u, v, rho of the fluid ones
    // (lbm_core_smemaa.cu:500-546); POLICY writes the fluid cells only
    // (lbm_core_smemaa_policy.cu:338-424).
    MODE_PRE_SMEMAA = 2,
    MODE_PRE_POLICY = 3,
};

struct WaveParams {
    const void *f_in;
    void *f_out;
    const uint8_t *mask;
    float *ux, *uy, *rho; // optional macroscopic outputs of the last level (null: skipped)
    int W, H;
    int pitch;          // elements between rows of a population plane
    long long plane;    // elements between population planes
    int mask_pitch;     // bytes between mask rows
    int chunk;          // output rows per CTA
    int bc_left, bc_right, bc_y; // LBM_BC_* (MODE_GENERAL)
    int use_tma;        // 1: TMA row loads; 0: plain loads (any alignment)
    int *err;           // device error word (bit 0: a bounded wait gave up)
    Phys k;
    int rx0, rx1, ry0, ry1; // register wavefront: output rectangle (0, W, 0, H when 0, 0, 0, 0)
};

template <int T_, int NX_, class Ph_, class St_, int MODE_, bool LID_ = false> struct WaveCfg {
    static constexpr int T = T_;
    static constexpr bool LID = LID_;
    static constexpr int NX = NX_;
    static constexpr int CW = NX - 2 * T;
    static constexpr int MODE = MODE_;
    using Ph = Ph_;
    using St = St_;
    using E = typename St::T;
    static constexpr int ES = (int)sizeof(E);
    static constexpr int AE = 16 / ES;              // TMA x alignment in elements
    static constexpr int RW = NX + 2 * AE;          // input row width (covers xs-1 .. xs+NX)
    static constexpr int RWM = NX + 32;             // mask row width (bytes)
    static constexpr int LW = NX + 2;               // level ring row width
    static constexpr int P = 4;                     // TMA prefetch distance (rows)
    static constexpr int DI = P + 4;                // input ring depth (power of two)
    static constexpr int DC = (2 * T <= 2) ? 2 : ((2 * T <= 4) ? 4 : ((2 * T <= 8) ? 8 : 16)); // code ring depth
    static_assert((DI & (DI - 1)) == 0 && DC >= 2 * T, "ring depths");
    static constexpr int NLV = (T > 1) ? (T - 1) : 0;
    static constexpr int SLOT_F = round_up(9 * RW * ES, 128); // bytes per input row
    static constexpr int SLOT_M = round_up(RWM, 128);
    static constexpr int OFF_BAR = 0;
    static constexpr int OFF_IN = 128;
    static constexpr int OFF_M = OFF_IN + DI * SLOT_F;
    static constexpr int OFF_L = OFF_M + DI * SLOT_M;
    static constexpr int OFF_C = OFF_L + NLV * 4 * 9 * LW * 4;
    static constexpr int OFF_LU = OFF_C + DC * NX * 4;
    static constexpr int OFF_DUM = OFF_LU + round_up(DC * 4, 16); // write-only sink, 2 x 9 x NX floats
    static constexpr int SMEM = OFF_DUM + 2 * 9 * NX * 4;
    static constexpr uint32_t TX_BYTES = 9 * RW * ES + RWM;
    static constexpr int MINB = (SMEM <= 74 * 1024) ? 3 : ((SMEM <= 112 * 1024) ? 2 : 1);
    static_assert(NX % 32 == 0 && CW > 0, "strip");
    static_assert(RW <= 256 && RWM <= 256, "TMA box dimension");
    static_assert(SMEM <= 227 * 1024, "shared memory");
    static_assert(DI * 8 <= 120, "mbarriers and the abort flag share the first 128 bytes");
};

template <int V> struct IntC {
    static constexpr int value = V;
};

// Compile-time loop: f(IntC<I>{}) for I in [I0, I1).
template <int I0, int I1, class F> __device__ __forceinline__ void static_for(F &&f)
{
    if constexpr (I0 < I1) {
        f(IntC<I0>{});
        static_for<I0 + 1, I1>(f);
    }
}

// Mask value of the 3x3 neighbourhood entry (dx, dy) in {-1,0,1}^2.
struct Nbhd {
    uint8_t m[3][3]; // [dy+1][dx+1]
};

__device__ __forceinline__ uint32_t build_code_core4(const Nbhd &n, int x, int y, int W, int H)
{
    const bool in_dom = x >= 0 && x < W && y >= 0 && y < H;
    const bool upd = in_dom && y >= 1 && y <= H - 2 && x <= W - 2 && (x == 0 || n.m[1][1] == 0);
    if (!upd) {
        uint32_t c = C_SKIP;
        if (x == W - 1 && y >= 1 && y <= H - 2 && n.m[1][0] == 0)
            c |= C_GHOST_SKIP;
        return c;
    }
    uint32_t c = 0;
#pragma unroll
    for (int q = 1; q < 9; ++q) {
        if (x == 0 && cx(q) == 1)
            continue; // pulled from x = -1, which reads zero (lbm_core4.cu:36-37)
        if (n.m[1 - cy(q)][1 - cx(q)])
            c |= 1u << q;
    }
    if (x == 0)
        c |= C_INLET;
    if (x == W - 2)
        c |= C_GHOST_SRC;
    return c;
}

// General boundary rules (lbm_params): out-of-domain sources are stationary
// walls unless the side is periodic; mask 0 fluid, 2 moving wall, other
// nonzero values solid; with an outflow right side column W-1 is the ghost.
__device__ __forceinline__ uint32_t build_code_general(const Nbhd &n, int x, int y, const WaveParams &p)
{
    const int W = p.W, H = p.H;
    const bool px = p.bc_left == LBM_BC_PERIODIC;
    const bool py = p.bc_y == LBM_BC_PERIODIC;
    const bool outflow = p.bc_right == LBM_BC_OUTFLOW;
    const int xw = px ? wrap(x, W) : x;
    const int yw = py ? wrap(y, H) : y;
    const bool in_dom = xw >= 0 && xw < W && yw >= 0 && yw < H;
    auto src = [&](int dx, int dy) -> int { // mask value of a neighbour, out of domain = solid
        int sx = xw + dx, sy = yw + dy;
        if (!px && (sx < 0 || sx >= W))
            return LBM_MASK_SOLID;
        if (!py && (sy < 0 || sy >= H))
            return LBM_MASK_SOLID;
        return n.m[dy + 1][dx + 1];
    };
    const bool upd = in_dom && n.m[1][1] == 0 && !(outflow && xw == W - 1);
    if (!upd) {
        uint32_t c = C_SKIP;
        if (outflow && in_dom && xw == W - 1 && n.m[1][0] == 0)
            c |= C_GHOST_SKIP;
        return c;
    }
    uint32_t c = 0;
#pragma unroll
    for (int q = 1; q < 9; ++q) {
        int v = src(-cx(q), -cy(q));
        if (v) {
            c |= 1u << q;
            if (v == LBM_MASK_MOVING)
                c |= 1u << (C_MOVING_SHIFT + q);
        }
    }
    if ((p.bc_left == LBM_BC_ZOUHE || p.bc_left == LBM_BC_ZOUHE_RAMP) && xw == 0)
        c |= C_INLET;
    if (outflow && xw == W - 2)
        c |= C_GHOST_SRC;
    return c;
}

// One tile (strip bx, chunk by) of the wavefront.  `reinit` re-initialises the
// mbarriers of a CTA that already ran a tile (persistent batch kernel).
template <class C>
__device__ __forceinline__ void wave_tile(const WaveParams &p, const CUtensorMap *tmf, const CUtensorMap *tmm, int bx,
                                          int by, bool reinit)
{
    using St = typename C::St;
    using E = typename C::E;
    using Ph = typename C::Ph;
    constexpr int T = C::T, NX = C::NX, CW = C::CW, DI = C::DI, RW = C::RW, LW = C::LW, DC = C::DC, P = C::P;

    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + C::OFF_BAR);
    unsigned char *in_base = smem + C::OFF_IN;
    unsigned char *m_base = smem + C::OFF_M;
    float *lvl = reinterpret_cast<float *>(smem + C::OFF_L);
    uint32_t *code = reinterpret_cast<uint32_t *>(smem + C::OFF_C);
    float *lu_ring = reinterpret_cast<float *>(smem + C::OFF_LU);
    volatile int &s_abort = *reinterpret_cast<int *>(smem + C::OFF_BAR + 124);

    const int i = threadIdx.x;
    const int x0 = bx * CW;
    const int xs = x0 - T;
    const int x = xs + i;
    const int ya = by * p.chunk;
    const int yb = min(p.H, ya + p.chunk);
    const int row0 = ya - T;
    const int nin = yb - ya + 2 * T;
    const int K = yb - ya + 3 * T - 3;
    const bool tma = p.use_tma != 0;
    const bool pyper = (C::MODE == MODE_GENERAL) && p.bc_y == LBM_BC_PERIODIC;
    const bool pxper = (C::MODE == MODE_GENERAL) && p.bc_left == LBM_BC_PERIODIC;
    // Ring entry 0 holds column xf0 (input) / xm0 (mask).
    const int xf0 = tma ? floor_div(xs - 1, C::AE) * C::AE : xs - 1;
    const int xm0 = tma ? floor_div(xs - 1, 16) * 16 : xs - 1;
    const int of = xs - xf0;
    const int om = xs - xm0;
    const bool colcore = i >= T && i < T + CW && x < p.W;

    auto in_row = [&](int r) -> E * { return reinterpret_cast<E *>(in_base + ((r - row0) & (DI - 1)) * C::SLOT_F); };
    auto m_row = [&](int r) -> uint8_t * { return m_base + ((r - row0) & (DI - 1)) * C::SLOT_M; };
    auto lv_row = [&](int t, int r) -> float * { return lvl + ((t - 1) * 4 + ((r - row0) & 3)) * 9 * LW; };

    if (i == 0) {
        s_abort = 0;
        if (tma) {
            for (int s = 0; s < DI; ++s) {
                if (reinit)
                    mbar_inval(&mbar[s]);
                mbar_init(&mbar[s], 1);
            }
            mbar_fence_init();
            prefetch_tmap(tmf);
            prefetch_tmap(tmm);
        }
    }
    for (int j = i; j < C::NLV * 4 * 9 * LW; j += NX)
        lvl[j] = 0.0f;
    __syncthreads();

    auto issue_row = [&](int r) { // thread 0, TMA path
        const int s = (r - row0) & (DI - 1);
        const int ry = pyper ? wrap(r, p.H) : r;
        mbar_arrive_expect_tx(&mbar[s], C::TX_BYTES);
        tma_load_3d(in_base + s * C::SLOT_F, tmf, &mbar[s], xf0, ry, 0);
        tma_load_2d(m_base + s * C::SLOT_M, tmm, &mbar[s], xm0, ry);
    };
    // Plain path: thread i loads ring entries i and (i < 2) NX + i, i.e. columns
    // xs - 1 + e; out-of-range columns/rows read zero unless periodic.
    auto plain_row = [&](int r) {
        E *dst = in_row(r);
        uint8_t *md = m_row(r);
        int ry = pyper ? wrap(r, p.H) : r;
        const bool rok = ry >= 0 && ry < p.H;
        for (int e = i; e < NX + 2; e += NX) {
            int cxl = xs - 1 + e;
            if (pxper)
                cxl = wrap(cxl, p.W);
            const bool ok = rok && cxl >= 0 && cxl < p.W;
            const E *src = reinterpret_cast<const E *>(p.f_in) + (long long)ry * p.pitch + cxl;
#pragma unroll
            for (int q = 0; q < 9; ++q)
                dst[q * RW + e] = ok ? src[q * p.plane] : E(0.0f);
            md[e] = ok ? p.mask[(long long)ry * p.mask_pitch + cxl] : (uint8_t)0;
        }
    };

    int next_wait = row0;  // next input row this thread waits for (TMA path)
    int issued_end = row0; // thread 0: one past the last issued row
    if (tma) {
        if (i == 0) {
            const int pro = min(nin, P + 3);
            fence_proxy_async();
            for (int j = 0; j < pro; ++j)
                issue_row(row0 + j);
            issued_end = row0 + pro;
        }
    } else {
        plain_row(row0);
        plain_row(row0 + 1);
    }

    auto build_code = [&](int r) {
        Nbhd n;
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const uint8_t *mr = m_row(r + dy);
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx)
                n.m[dy + 1][dx + 1] = mr[i + om + dx];
        }
        uint32_t c;
        if (C::MODE == MODE_CORE4)
            c = build_code_core4(n, x, r, p.W, p.H);
        else
            c = build_code_general(n, x, r, p);
        const int slot = (r - row0) & (DC - 1);
        code[slot * NX + i] = c;
        if (i == 0)
            lu_ring[slot] = inlet_u(p.k, pyper ? wrap(r, p.H) : r);
    };

    // ---- level computations ----
    // Level t at iteration k works on row r1 - 2(t-1).  All T levels are
    // computed in every iteration (levels outside their row range compute on
    // stale ring rows and do not store), so one straight-line body serves every
    // iteration and the T independent cells overlap in the scheduler.
    // Per iteration a warp vote picks the fast body (every lane's cell is
    // interior fluid at every level: code == 0) or the generic body (bounce-back
    // and moving walls, Zou-He inlet, pass-through of cells that are not
    // updated, outlet ghost).  Suppressed shared-memory writes go to a dummy row.
    float *dummy = reinterpret_cast<float *>(smem + C::OFF_DUM);

    auto main_loop = [&]() {
        for (int k = 0; k < K; ++k) {
            const int r1 = ya - T + 1 + k;
            const bool l1 = r1 <= yb + T - 2;
            if (tma) {
                if (l1) {
                    // Wait for every row up to r1 + 1 (rows arrive in order).
                    while (next_wait <= r1 + 1) {
                        const int rr = next_wait - row0;
                        if (!mbar_wait_bounded(&mbar[rr & (DI - 1)], (uint32_t)((rr / DI) & 1))) {
                            s_abort = 1;
                            if (p.err)
                                atomicOr(p.err, 1);
                            break;
                        }
                        ++next_wait;
                    }
                    build_code(r1);
                }
                __syncthreads();
                if (s_abort)
                    break;
                if (i == 0 && l1 && r1 + 2 + P < row0 + nin) {
                    fence_proxy_async();
                    issue_row(r1 + 2 + P);
                    issued_end = r1 + 3 + P;
                }
            } else {
                if (l1)
                    plain_row(r1 + 1);
                __syncthreads();
                if (l1)
                    build_code(r1);
                __syncthreads();
            }

            int rt[T];
            bool act[T];
            uint32_t cd[T];
            bool special = false;
#pragma unroll
            for (int t = 1; t <= T; ++t) {
                rt[t - 1] = r1 - 2 * (t - 1);
                act[t - 1] = rt[t - 1] >= ya - T + t && rt[t - 1] < yb + T - t;
                cd[t - 1] = code[((rt[t - 1] - row0) & (DC - 1)) * NX + i];
                special |= act[t - 1] && cd[t - 1] != 0;
            }
            const bool fast = !__any_sync(0xffffffffu, special);

            // Source row pointers of every level (rows rt-1, rt, rt+1 of level t-1),
            // already offset to this thread's column, so loads use immediate offsets.
            const E *ib[3];
            const float *lb[T][3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ib[d] = in_row(rt[0] - 1 + d) + i + of;
#pragma unroll
                for (int t = 2; t <= T; ++t)
                    lb[t - 1][d] = lv_row(t - 1, rt[t - 1] - 1 + d) + i + 1;
            }
            auto srcp = [&](auto t_tag, int dr, int q, int dc) -> float {
                constexpr int t = decltype(t_tag)::value;
                if constexpr (t == 1)
                    return St::load(ib[dr + 1][q * RW + dc], q);
                else
                    return lb[t - 1][dr + 1][q * LW + dc];
            };

            float f[T][9];
            float mr[T], mu[T], mv[T];
            if (fast) {
                static_for<1, T + 1>([&](auto tt) {
                    constexpr int t = decltype(tt)::value;
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        f[t - 1][q] = srcp(tt, -cy(q), q, -cx(q));
                });
                if constexpr (Ph::kRefOrder) {
#pragma unroll
                    for (int t = 0; t < T; ++t)
                        collide_bf<Ph, false>(f[t], false, 0.0f, p.k, mr[t], mu[t], mv[t]);
                } else {
                    collide_multi<Ph, T>(f, p.k, mr, mu, mv);
                }
            } else {
                float own[T][9];
                static_for<1, T + 1>([&](auto tt) {
                    constexpr int t = decltype(tt)::value;
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        own[t - 1][q] = srcp(tt, 0, q, 0);
                    f[t - 1][0] = own[t - 1][0];
#pragma unroll
                    for (int q = 1; q < 9; ++q)
                        f[t - 1][q] = srcp(tt, -cy(q), q, -cx(q));
                });
#pragma unroll
                for (int t = 0; t < T; ++t) {
                    const uint32_t c = cd[t];
#pragma unroll
                    for (int q = 1; q < 9; ++q) {
                        float bv = own[t][opp(q)];
                        if (C::LID)
                            bv += ((c >> (C_MOVING_SHIFT + q)) & 1u) ? 6.0f * wgt(q) * (float)cx(q) * p.k.u_lid : 0.0f;
                        f[t][q] = ((c >> q) & 1u) ? bv : f[t][q];
                    }
                    const int slot = (rt[t] - row0) & (DC - 1);
                    collide_bf<Ph, true>(f[t], (c & C_INLET) != 0, lu_ring[slot], p.k, mr[t], mu[t], mv[t]);
                    const bool skip = (c & C_SKIP) != 0;
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        f[t][q] = skip ? own[t][q] : f[t][q];
                }
            }

            // stores: levels 1..T-1 into their rings, level T to HBM
#pragma unroll
            for (int t = 1; t < T; ++t) {
                const uint32_t c = cd[t - 1];
                float *dst = lv_row(t, rt[t - 1]);
                const bool wr = act[t - 1] && !(c & C_GHOST_SKIP);
                const bool gh = act[t - 1] && (c & C_GHOST_SRC);
                float *d1 = wr ? dst + i + 1 : dummy + i;
                float *d2 = gh ? dst + i + 2 : dummy + 9 * NX + i;
                const int s1 = wr ? LW : NX;
                const int s2 = gh ? LW : NX;
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    d1[q * s1] = f[t - 1][q];
                if (!fast) {
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        d2[q * s2] = f[t - 1][q];
                }
            }
            {
                const uint32_t c = cd[T - 1];
                const int r = rt[T - 1];
                if (act[T - 1] && !(c & C_SKIP) && colcore && r >= ya && r < yb) {
                    E *fo = reinterpret_cast<E *>(p.f_out) + (long long)r * p.pitch + x;
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        fo[q * p.plane] = St::store(f[T - 1][q], q);
                    if (c & C_GHOST_SRC) {
#pragma unroll
                        for (int q = 0; q < 9; ++q)
                            fo[q * p.plane + 1] = St::store(f[T - 1][q], q);
                    }
                    if (p.ux) {
                        const long long id = (long long)r * p.W + x;
                        p.ux[id] = mu[T - 1];
                        p.uy[id] = mv[T - 1];
                        p.rho[id] = mr[T - 1];
                    }
                }
            }
        }
    };
    main_loop();

    // Abort path: wait (bounded) for copies still in flight before the shared
    // memory is released.
    if (tma && s_abort && i == 0) {
        for (int r = next_wait; r < issued_end; ++r) {
            const int rr = r - row0;
            if (!mbar_wait_bounded(&mbar[rr & (DI - 1)], (uint32_t)((rr / DI) & 1)))
                break;
        }
    }
}

template <class C>
__global__ void __launch_bounds__(C::NX, C::MINB)
    wave_kernel(const __grid_constant__ WaveParams p, const __grid_constant__ CUtensorMap tmf,
                const __grid_constant__ CUtensorMap tmm)
{
    pdl_trigger();
    pdl_wait(); // launched with programmatic dependent launch: the previous step's stores first
    wave_tile<C>(p, &tmf, &tmm, blockIdx.x, blockIdx.y, false);
}

} // namespace lbm
