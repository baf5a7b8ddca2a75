// Temporally blocked BGK with the AA pattern in shared memory: the drop-ins for
// lbm_core_smemaa.cu (VARIANT_SMEMAA) and lbm_core_smemaa_policy.cu /
// lbm_core_smemaa_endfused.cu (VARIANT_POLICY).
//
// The slot semantics are those of the reference, so its boundary behaviour is
// reproduced exactly (the smem AA pattern, lbm_core_smemaa.cu:90-485):
//   A phase  local collide, store reversed:    S[opp q](x) = f*_q(x)
//   B phase  gather S[opp q](x - c_q) (or S[q](x) if x - c_q is solid),
//            collide, scatter S[q](x + c_q) (or S[opp q](x) if x + c_q is
//            solid; populations leaving x = 0 to the left are discarded)
//   outlet   after each A (and, for smemaa, each B) column W-1 := column W-2
// A cell is updated when it is in the domain, 0 < y < H-1, x < W-1 and not
// solid; out-of-domain cells are solid with zero populations, column W-1 is
// fluid (open outlet ghost).
//
// B200 design: one CTA of 512 threads owns a 64 x 40 tile (core (64-2T) x
// (40-2T) plus a T-cell halo; 64 x 32 in the edge band of a split launch),
// fetched by a single TMA box [68 x SY x 9] (plus one for the mask) when the
// layout allows it.  Threads have a fixed 2-D map
// (two warps per tile row, eight rows apart), so phases need no integer
// division.  After the load the solid test runs once per tile cell and per cell
// of a one-cell apron (a byte array), and each cell's neighbour code is read
// off those bytes, so the B phase reads one 16-bit code instead of nine mask
// bytes.  Two CTAs fit per SM.
#pragma once

#include "wave.cuh" // IntC

namespace lbm {

enum : int { VARIANT_SMEMAA = 0, VARIANT_POLICY = 1 };

struct AaParams {
    const float *f_in;
    float *f_out;
    const uint8_t *mask;
    float *ux, *uy, *rho; // VARIANT_SMEMAA only
    int W, H;
    int use_tma;
    int *err;
    Phys k;
    // Edge-only launch (1-D grid): skip the tiles with etx0 <= tx < etx1 and
    // ety0 <= ty < ety1 (computed by another kernel); nx tile columns.
    int edge_only, etx0, etx1, ety0, ety1, nx;
};

// Tile coordinates of 1-D block b of an edge-only launch: the tile rows below
// ety0 in full, then the rows [ety0, ety1) with only their edge columns, then
// the rows from ety1 on in full.
__device__ __forceinline__ void aa_edge_tile(const AaParams &p, int b, int &tx, int &ty)
{
    const int top = p.ety0 * p.nx;
    const int nl = p.etx0, nr = p.nx - p.etx1, mid = (p.ety1 - p.ety0) * (nl + nr);
    if (b < top) {
        tx = b % p.nx;
        ty = b / p.nx;
    } else if (b < top + mid) {
        const int j = b - top, r = j / (nl + nr), c = j % (nl + nr);
        ty = p.ety0 + r;
        tx = c < nl ? c : p.etx1 + (c - nl);
    } else {
        const int j = b - top - mid;
        tx = j % p.nx;
        ty = p.ety1 + j / p.nx;
    }
}

template <int T_, int VAR_, int SX_ = 64, int SY_ = 32, int NT_ = 256, int NB_ = 4, int MINB_ = 2> struct AaCfg {
    static constexpr int T = T_;
    static constexpr int VAR = VAR_;
    static constexpr int SX = SX_, SY = SY_; // tile incl. halo
    static constexpr int CX = SX - 2 * T, CY = SY - 2 * T;
    static constexpr int SW = SX + 4;      // smem row stride: room for the 16-byte TMA alignment offset
    static constexpr int PL = SW * SY;     // floats per population plane
    static constexpr int MW = SX + 16;     // mask row bytes (TMA box, 16-byte aligned origin)
    static constexpr int NT = NT_;
    static constexpr int MINB = MINB_;
    static constexpr int WPR = SX / 32;            // warps per tile row
    static constexpr int RSTEP = NT / SX;          // rows between a thread's cells
    static constexpr int ROWS_PER_THREAD = SY / RSTEP;
    static_assert(SX % 32 == 0 && NT % SX == 0 && SY % RSTEP == 0, "thread map");
    static constexpr int OFF_F = 128;
    static constexpr int OFF_M = OFF_F + 9 * PL * 4;
    static constexpr int OFF_C = OFF_M + round_up(MW * SY, 128);
    static constexpr int OFF_LU = OFF_C + SX * SY * 2;
    static constexpr int SBW = SX + 2;             // solid-flag rows: the tile plus a one-cell apron
    static constexpr int OFF_SB = OFF_LU + round_up(SY * 4, 16);
    static constexpr int SMEM = OFF_SB + round_up(SBW * (SY + 2), 16);
    static constexpr int BATCH = NB_;
    static_assert(ROWS_PER_THREAD % NB_ == 0, "batch");
    static constexpr uint32_t TX = 9 * PL * 4 + MW * SY;
    static_assert(T % 2 == 0 && T >= 2 && CY > 0, "T");
    static_assert(SMEM <= 227 * 1024, "shared memory");
};

// code bits: bit q (1..8) = the cell x - c_q is solid; bit 0 = cell updated.
enum : uint16_t { AA_UPD = 1 };

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) aa_tile_kernel(const __grid_constant__ AaParams p,
                                                           const __grid_constant__ CUtensorMap tmf,
                                                           const __grid_constant__ CUtensorMap tmm)
{
    constexpr int T = C::T, SX = C::SX, SY = C::SY, CX = C::CX, CY = C::CY, SW = C::SW, PL = C::PL, MW = C::MW;
    pdl_trigger();
    pdl_wait(); // launched with programmatic dependent launch: the previous launch's stores first
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    float *S = reinterpret_cast<float *>(smem + C::OFF_F);
    uint8_t *M = smem + C::OFF_M;
    uint16_t *code = reinterpret_cast<uint16_t *>(smem + C::OFF_C);

    const int W = p.W, H = p.H;
    const int tid = threadIdx.x;
    const int col = (tid & 31) + 32 * ((tid >> 5) % C::WPR); // 0..SX-1
    const int rb = (tid >> 5) / C::WPR;                       // 0..RSTEP-1
    constexpr int RS = C::RSTEP;
    int tile_x = blockIdx.x, tile_y = blockIdx.y;
    if (p.edge_only)
        aa_edge_tile(p, blockIdx.x, tile_x, tile_y);
    const int xt = tile_x * CX - T; // global x of tile column 0
    const int yt = tile_y * CY - T;
    const bool tma = p.use_tma != 0;
    const int xf = tma ? floor_div(xt, 4) * 4 : xt; // global x of smem row entry 0
    const int xm = tma ? floor_div(xt, 16) * 16 : xt;
    const int of = xt - xf, om = xt - xm;

    // ---- load the tile: canonical f (zero outside) and the mask ----
    if (tma) {
        if (tid == 0) {
            mbar_init(bar, 1);
            mbar_fence_init();
            mbar_arrive_expect_tx(bar, C::TX);
            tma_load_3d(S, &tmf, bar, xf, yt, 0);
            tma_load_2d(M, &tmm, bar, xm, yt);
        }
        __syncthreads();
        if (!mbar_wait_bounded(bar, 0)) {
            if (p.err)
                atomicOr(p.err, 1);
            return; // every thread waits on the same barrier and gives up together
        }
    } else {
        for (int e = tid; e < SX * SY; e += C::NT) {
            const int c = e % SX, r = e / SX;
            const int x = xt + c, y = yt + r;
            const bool in = x >= 0 && x < W && y >= 0 && y < H;
            const long long id = (long long)y * W + x;
#pragma unroll
            for (int q = 0; q < 9; ++q)
                S[q * PL + r * SW + c + of] = in ? p.f_in[q * (long long)W * H + id] : 0.0f;
            M[r * MW + c + om] = in ? p.mask[id] : (uint8_t)0;
        }
        __syncthreads();
    }

    // ---- per-cell codes (solid test as lbm_core_smemaa.cu:39-70) ----
    auto solid = [&](int c, int r) -> bool { // tile cell, may lie one cell outside the tile
        const int x = xt + c, y = yt + r;
        if (x < 0 || x >= W || y < 0 || y >= H)
            return true;
        if (x == W - 1)
            return false;
        if (c < 0 || c >= SX || r < 0 || r >= SY)
            return true; // outside the tile: only read for cells whose results are discarded
        return M[r * MW + c + om] != 0;
    };
    // solid flags of every tile cell and of a one-cell apron around the tile, once
    constexpr int SBW = C::SBW;
    uint8_t *SB = smem + C::OFF_SB;
    for (int e = tid; e < SBW * (SY + 2); e += C::NT)
        SB[e] = solid(e % SBW - 1, e / SBW - 1) ? 1 : 0;
    // Inlet velocity of each tile row (only the tile holding column 0 uses it).
    float *lu_row = reinterpret_cast<float *>(smem + C::OFF_LU);
    if (tid < SY)
        lu_row[tid] = inlet_u(p.k, yt + tid);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < C::ROWS_PER_THREAD; ++j) {
        const int r = rb + RS * j, c = col;
        const int x = xt + c, y = yt + r;
        const uint8_t *sb = SB + (r + 1) * SBW + (c + 1);
        uint32_t cd = (x >= 0 && x < W - 1 && y > 0 && y < H - 1 && !sb[0]) ? AA_UPD : 0u;
#pragma unroll
        for (int q = 1; q < 9; ++q)
            cd |= (uint32_t)sb[-cx(q) - cy(q) * SBW] << q;
        code[r * SX + c] = (uint16_t)cd;
    }
    __syncthreads();

    auto sl = [&](int q, int c, int r) -> float & { return S[q * PL + r * SW + c + of]; };

    const int cg = (W - 1) - xt; // tile column of the outlet ghost
    const bool has_outlet = cg - 1 >= 0 && cg < SX;
    auto ghost_copy = [&]() {
        for (int e = tid; e < SY * 9; e += C::NT) {
            const int r = e / 9, q = e % 9;
            const int y = yt + r;
            if (y >= 1 && y <= H - 2)
                sl(q, cg, r) = sl(q, cg - 1, r);
        }
    };

    auto bgk_cell = [&](float (&f)[9], int x, int y) {
        float r, u, v;
        collide<PhysBgkRef>(f, x == 0, y, p.k, r, u, v);
    };

    // Cells are processed in batches of C::BATCH rows per thread: all loads,
    // then all collisions, then all stores, so the independent cells overlap.
    // Inactive cells read from a cell inside the margin and write to the sink.
    constexpr int NB = C::BATCH;

    // A phase at margin m: local collide, reversed store.
    auto phase_a = [&](auto zh_tag, int m) {
        constexpr bool ZH = decltype(zh_tag)::value;
#pragma unroll
        for (int b = 0; b < C::ROWS_PER_THREAD; b += NB) {
            float f[NB][9];
            bool act[NB];
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rb + RS * (b + jj), c = col;
                act[jj] = r >= m && r < SY - m && c >= m && c < SX - m && (code[r * SX + c] & AA_UPD);
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    f[jj][q] = sl(q, c, r);
            }
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rb + RS * (b + jj);
                float rr, uu, vv;
                collide_bf<PhysBgkRef, ZH>(f[jj], ZH && (xt + col == 0), ZH ? lu_row[r] : 0.0f, p.k, rr, uu, vv);
            }
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rb + RS * (b + jj), c = col;
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    if (act[jj])
                        sl(opp(q), c, r) = f[jj][q];
            }
        }
    };

    // B phase at margin m >= 1 into shared memory: gather, collide, scatter.
    // A warp whose cells are all interior fluid (or outside the margin) takes the
    // fast body: plain gather and scatter; otherwise bounce-back and the inlet's
    // discard slot are resolved per population.
    auto phase_b = [&](auto zh_tag, int m) {
        constexpr bool ZH = decltype(zh_tag)::value;
#pragma unroll
        for (int b = 0; b < C::ROWS_PER_THREAD; b += NB) {
            float f[NB][9];
            bool act[NB];
            uint16_t cdv[NB];
            int rr_[NB], cc_[NB];
            bool ok = true;
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r0 = rb + RS * (b + jj), c0 = col;
                const bool in = r0 >= m && r0 < SY - m && c0 >= m && c0 < SX - m;
                rr_[jj] = in ? r0 : m;
                cc_[jj] = in ? c0 : m;
                const uint16_t cd = code[rr_[jj] * SX + cc_[jj]];
                act[jj] = in && (cd & AA_UPD);
                cdv[jj] = cd;
                ok = ok && (!in || (cd == AA_UPD && !(ZH && xt + c0 == 0)));
            }
            const bool fast = __all_sync(0xffffffffu, ok);
            if (fast) {
#pragma unroll
                for (int jj = 0; jj < NB; ++jj)
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        f[jj][q] = sl(opp(q), cc_[jj] - cx(q), rr_[jj] - cy(q));
#pragma unroll
                for (int jj = 0; jj < NB; ++jj) {
                    float r_, u_, v_;
                    collide_bf<PhysBgkRef, false>(f[jj], false, 0.0f, p.k, r_, u_, v_);
                }
#pragma unroll
                for (int jj = 0; jj < NB; ++jj) {
                    const int r = rr_[jj], c = cc_[jj];
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        if (act[jj])
                            sl(q, c + cx(q), r + cy(q)) = f[jj][q];
                }
                continue;
            }
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rr_[jj], c = cc_[jj];
                const uint16_t cd = cdv[jj];
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    f[jj][q] = (cd & (1u << q)) ? sl(q, c, r) : sl(opp(q), c - cx(q), r - cy(q));
            }
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rb + RS * (b + jj);
                float r_, u_, v_;
                collide_bf<PhysBgkRef, ZH>(f[jj], ZH && (xt + col == 0), ZH ? lu_row[r] : 0.0f, p.k, r_, u_, v_);
            }
#pragma unroll
            for (int jj = 0; jj < NB; ++jj) {
                const int r = rr_[jj], c = cc_[jj];
                const uint16_t cd = cdv[jj];
                const bool left = xt + c == 0;
#pragma unroll
                for (int q = 0; q < 9; ++q) {
                    float *dst;
                    if (cx(q) < 0 && left)
                        dst = &sl(q, c + cx(q), r + cy(q)); // discard slot left of the inlet
                    else if (q && (cd & (1u << opp(q))))   // x + c_q is solid: bounce back
                        dst = &sl(opp(q), c, r);
                    else
                        dst = &sl(q, c + cx(q), r + cy(q));
                    if (act[jj])
                        *dst = f[jj][q];
                }
            }
        }
    };

    // Policy B-final at margin T-1: gather, collide, scatter straight into f_out
    // (lbm_core_smemaa_policy.cu:338-424).
    auto phase_b_final = [&](int m) {
        const long long N = (long long)W * H;
#pragma unroll
        for (int j = 0; j < C::ROWS_PER_THREAD; ++j) {
            const int r = rb + RS * j, c = col;
            if (r < m || r >= SY - m || c < m || c >= SX - m)
                continue;
            const uint16_t cd = code[r * SX + c];
            if (!(cd & AA_UPD))
                continue;
            const int x = xt + c, y = yt + r;
            float f[9];
#pragma unroll
            for (int q = 0; q < 9; ++q)
                f[q] = (cd & (1u << q)) ? sl(q, c, r) : sl(opp(q), c - cx(q), r - cy(q));
            bgk_cell(f, x, y);
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                if (x == 0 && cx(q) < 0)
                    continue;
                int tx, ty, tq;
                if (q && (cd & (1u << opp(q)))) {
                    tx = x;
                    ty = y;
                    tq = opp(q);
                } else {
                    tx = x + cx(q);
                    ty = y + cy(q);
                    tq = q;
                }
                if (tx == W - 1)
                    continue;
                if (tx < xt + T || tx >= xt + T + CX || ty < yt + T || ty >= yt + T + CY || tx < 0 || tx >= W ||
                    ty < 0 || ty >= H)
                    continue;
                float *dst = p.f_out + tq * N + (long long)ty * W + tx;
                dst[0] = f[q];
                if (tx == W - 2)
                    dst[1] = f[q];
            }
        }
    };

    auto run = [&](auto zh_tag) {
        for (int pr = 0; pr < T / 2; ++pr) {
            phase_a(zh_tag, 2 * pr);
            __syncthreads();
            if (has_outlet) {
                ghost_copy();
                __syncthreads();
            }
            const bool last = pr == T / 2 - 1;
            if (C::VAR == VARIANT_POLICY && last) {
                phase_b_final(2 * pr + 1);
                return;
            }
            phase_b(zh_tag, 2 * pr + 1);
            __syncthreads();
            if (C::VAR == VARIANT_SMEMAA && has_outlet) {
                ghost_copy();
                __syncthreads();
            }
        }
    };
    if (xt <= 0)
        run(IntC<1>{});
    else
        run(IntC<0>{});
    if (C::VAR == VARIANT_POLICY)
        return;

    // ---- smemaa epilogue: canonical core and u, v, rho (lbm_core_smemaa.cu:500-546) ----
    const long long N = (long long)W * H;
#pragma unroll
    for (int j = 0; j < C::ROWS_PER_THREAD; ++j) {
        const int r = rb + RS * j, c = col;
        if (r < T || r >= T + CY || c < T || c >= T + CX)
            continue;
        const int x = xt + c, y = yt + r;
        if (x >= W || y >= H)
            continue;
        const long long id = (long long)y * W + x;
        float f[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            f[q] = sl(q, c, r);
            p.f_out[q * N + id] = f[q];
        }
        if (code[r * SX + c] & AA_UPD) {
            float rr, uu, vv;
            moments_seq(f, rr, uu, vv);
            p.ux[id] = uu;
            p.uy[id] = vv;
            p.rho[id] = rr;
        }
    }
}

} // namespace lbm
