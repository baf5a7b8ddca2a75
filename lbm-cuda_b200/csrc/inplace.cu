// In-place time stepping of the general solver: ONE state buffer, the AA access
// pattern, two kernels per pair of steps.
//
// The buffer holds the general solver's canonical state (post-collision
// populations, plane q = f*_q) at even step counts, exactly as lbm_run's
// buffers.  A pair of steps is:
//   pull-push  cell x pulls f*_q(x - c_q) from plane q of its source (its own
//              plane opp(q) for a bounce-back source, plus the moving-wall term),
//              collides, and pushes f'*_q(x) to plane opp(q) of x + c_q, the
//              cell that pulls it next; a value whose destination is solid (or
//              outside the domain) goes to the cell's own plane q, where the
//              next step reads it as its bounce-back value, and a value whose
//              destination is never updated (the outflow column) is dropped;
//   local      cell x reads its pre-collision populations from its own planes
//              opp(q), collides, and writes f''*_q(x) to its own plane q.
// Within each kernel every location is read and written by one cell only (the
// cell it belongs to in the pull step's source/destination pairing), so the
// steps are race-free in place.  The outflow ghost (column W-1 = column W-2
// after each step) is carried by the W-2 cells: in the pull-push step they also
// make the three pushes the ghost would make towards column W-2 (directions 3,
// 6, 7), in the local step they also write the ghost's planes; a ghost cell
// that is never copied (its row's W-2 cell is solid) keeps its values, which
// the W-2 cells pulling from it pass on to their own local step.  Boundary codes,
// the Zou-He inlet, the moving-wall term and the collision are those of the
// pull kernel (build_code_general, collide_bf), so the state after an even
// number of steps equals lbm_run's.
//
// One thread per cell, 128 x 2 cells per CTA; the 3 x 3 mask neighbourhood is
// read per cell (L1-resident).  Memory traffic: 72 B per update in FP32, like
// the ping-pong streaming kernel, with half the state memory.  The two kernels
// of a pair of steps run back to back: each is launched with programmatic
// dependent launch (its CTAs are scheduled while the previous step drains and
// wait in griddepcontrol.wait until that step's stores are visible), which
// hides the gap between consecutive one-step launches.
#include <type_traits>

#include "dispatch.cuh"
#include "stream.cuh" // Raw4, ld4, ld1, pack4, unpack4

namespace lbm {

struct InplaceParams {
    void *f;
    const uint8_t *mask;
    float *ux, *uy, *rho; // local step only, may be null
    int W, H;
    int bc_left, bc_right, bc_y;
    Phys k;
};

// One cell (x, y) of one step, scalar accesses.
template <class Ph, class St, bool LID, bool LOCAL>
__device__ __forceinline__ void inplace_cell(const InplaceParams &p, int x, int y)
{
    using E = typename St::T;
    const int W = p.W, H = p.H;
    const bool px = p.bc_left == LBM_BC_PERIODIC, py = p.bc_y == LBM_BC_PERIODIC;
    const bool outflow = p.bc_right == LBM_BC_OUTFLOW;
    // neighbour columns and row offsets (one cell away: wrapped where periodic,
    // clamped otherwise; a clamped index is only used where its value is not)
    const int cols[3] = {x > 0 ? x - 1 : (px ? W - 1 : 0), x, x < W - 1 ? x + 1 : (px ? 0 : W - 1)};
    const long long rows[3] = {(long long)(y > 0 ? y - 1 : (py ? H - 1 : 0)) * W, (long long)y * W,
                               (long long)(y < H - 1 ? y + 1 : (py ? 0 : H - 1)) * W};
    Nbhd n;
    uint32_t any = 0;
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx) {
            n.m[dy + 1][dx + 1] = p.mask[rows[dy + 1] + cols[dx + 1]];
            any |= n.m[dy + 1][dx + 1];
        }
    // interior fluid (no solid neighbour, away from every domain edge, not the
    // inlet, the outlet's source or its ghost): code 0 without the builder
    uint32_t code = 0;
    if (any || x < 1 || x > W - 3 || y < 1 || y > H - 2) {
        WaveParams wp; // the fields build_code_general reads
        wp.W = W;
        wp.H = H;
        wp.bc_left = p.bc_left;
        wp.bc_right = p.bc_right;
        wp.bc_y = p.bc_y;
        code = build_code_general(n, x, y, wp);
    }
    if (code & C_SKIP)
        return;
    const long long N = (long long)W * H;
    E *f = reinterpret_cast<E *>(p.f);
    const long long id = rows[1] + x;
    // cell index of the neighbour (x + dx, y + dy), |dx|, |dy| <= 1
    auto at = [&](int dx, int dy) -> long long { return rows[1 + dy] + cols[1 + dx]; };
    float g[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const bool bounce = q && ((code >> q) & 1u);
        float v;
        if (LOCAL || bounce || q == 0)
            v = St::load(f[(q == 0 ? 0 : opp(q)) * N + id], q == 0 ? 0 : opp(q));
        else
            v = St::load(f[q * N + at(-cx(q), -cy(q))], q);
        if (LID && bounce && ((code >> (C_MOVING_SHIFT + q)) & 1u))
            v += 6.0f * wgt(q) * (float)cx(q) * p.k.u_lid;
        g[q] = v;
    }
    // W-2 cells pulling from a ghost cell that is never copied (the W-2 cell of
    // its row is solid): the ghost keeps its value, so the value pulled now is
    // also the one to pull next step; keep it for the local step (below)
    float gq[3];
    if (!LOCAL) {
        gq[0] = g[3];
        gq[1] = g[6];
        gq[2] = g[7];
    }
    const bool zh = p.bc_left == LBM_BC_ZOUHE || p.bc_left == LBM_BC_ZOUHE_RAMP;
    const float lu = (zh && x == 0) ? inlet_u(p.k, y) : 0.0f;
    float r, u, v;
    collide_bf<Ph, true>(g, (code & C_INLET) != 0, lu, p.k, r, u, v);
    if (LOCAL) {
        const bool ghost = (code & C_GHOST_SRC) != 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const E e = St::store(g[q], q);
            f[q * N + id] = e;
            if (ghost)
                f[q * N + id + 1] = e; // column W-1 of the same row
        }
        if (p.ux) {
            p.ux[id] = u;
            p.uy[id] = v;
            p.rho[id] = r;
        }
        return;
    }
    f[id] = St::store(g[0], 0);
#pragma unroll
    for (int q = 1; q < 9; ++q) {
        const E e = St::store(g[q], q);
        if ((code >> opp(q)) & 1u) { // x + c_q is solid: bounce-back, read by this cell next step
            f[q * N + id] = e;
            continue;
        }
        if (outflow && x + cx(q) == W - 1) // the ghost column is not updated: nothing pulls from it
            continue;
        f[opp(q) * N + at(cx(q), cy(q))] = e;
    }
    if (outflow && x == W - 2) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int q = i == 0 ? 3 : (i == 1 ? 6 : 7);
            // a solid source (bounce-back), or a copied ghost (its W-2 cell of row
            // y - c_y pushes the value), needs nothing here
            if (((code >> q) & 1u) || n.m[1 - cy(q)][1] == 0)
                continue;
            f[opp(q) * N + id] = St::store(gq[i], q);
        }
    }
    // the ghost's pushes towards column W-2 (it holds this cell's values), when
    // the ghost cell is not solid and the receiving W-2 cell is updated
    if ((code & C_GHOST_SRC) && !((code >> 3) & 1u)) {
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int q = i == 0 ? 3 : (i == 1 ? 6 : 7);
            const int ry = y + cy(q);
            if (!py && (ry < 0 || ry >= H))
                continue;
            if (n.m[1 + cy(q)][1] != 0) // the receiving cell (W-2, ry) is solid
                continue;
            f[opp(q) * N + at(0, cy(q))] = St::store(g[q], q);
        }
    }
}

// Scalar kernel: one cell per thread, 128 x 2 cells per CTA (any W, any alignment).
template <class Ph, class St, bool LID, bool LOCAL>
__global__ void __launch_bounds__(256) inplace_kernel(const __grid_constant__ InplaceParams p)
{
    pdl_trigger();
    pdl_wait(); // the previous step's kernel has completed: its stores are visible
    const int x = blockIdx.x * 128 + threadIdx.x;
    const int y = blockIdx.y * 2 + threadIdx.y;
    if (x < p.W && y < p.H)
        inplace_cell<Ph, St, LID, LOCAL>(p, x, y);
}

#ifndef LBM_INPLACE_MINB
#define LBM_INPLACE_MINB 3 // CTAs of 256 threads per SM the vector kernel's registers are sized for
#endif

// Vector kernel (W % 4 == 0, 16-byte aligned planes, mask and macro arrays):
// four consecutive cells per thread, a warp covers 128 columns of one row, 256
// columns x 4 rows per CTA.  A warp whose 128 cells are all interior fluid (no
// solid cell in their 3 x 3 neighbourhoods, away from every domain edge) moves
// each plane with 128-bit (FP32) or 64-bit (16-bit storage) accesses: in the
// pull-push step the +-1 column shifts come from the neighbouring lane by warp
// shuffle, and the one element that crosses the warp's edge is loaded or stored
// by lane 0 or lane 31 alone; every aligned vector is loaded and stored by the
// same thread (the pull of plane k from row r and the push into plane k of row
// r belong to the cells of row r + c_y(k)).  Other warps run the per-cell code.
template <class Ph, class St, bool LID, bool LOCAL>
__global__ void __launch_bounds__(256, LBM_INPLACE_MINB) inplace_vec_kernel(const __grid_constant__ InplaceParams p)
{
    using E = typename St::T;
    using V = typename Raw4<E>::type;
    pdl_trigger();
    pdl_wait(); // the previous step's kernel has completed: its stores are visible
    const int W = p.W, H = p.H;
    const int x4 = (blockIdx.x * 64 + threadIdx.x) * 4;
    const int y = blockIdx.y * 4 + threadIdx.y;
    const int lane = threadIdx.x & 31;
    const bool xok = x4 < W && y < H;
    bool interior = xok && x4 >= 1 && x4 + 3 <= W - 3 && y >= 1 && y <= H - 2;
    // The mask loads of the interior test and the population loads of the vector
    // path are issued together, so that one memory latency covers both; a warp
    // that turns out not to be interior drops the populations (its per-cell code
    // loads them again, from cache).  The loads are predicated on the cell and
    // its source row being inside the domain.
    uint32_t any = 0;
    if (interior) {
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy) {
            const uint8_t *m = p.mask + (long long)(y + dy) * W + x4;
            any |= *reinterpret_cast<const uint32_t *>(m) | m[-1] | m[4];
        }
    }
    const long long N = (long long)W * H;
    const long long id = (long long)y * W + x4;
    E *f = reinterpret_cast<E *>(p.f);
    V raw[9];
    float edge[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        edge[q] = 0.0f;
        if (LOCAL) {
            raw[q] = ld4<E>(f + (q == 0 ? 0 : opp(q)) * N + id, xok);
        } else {
            const int sy = y - cy(q);
            const bool rok = xok && sy >= 0 && sy < H;
            const E *src = f + q * N + id - (long long)cy(q) * W;
            raw[q] = ld4<E>(src, rok);
            if (cx(q) > 0) // column x4 - 1, for lane 0
                edge[q] = ld1<St>(src - 1, rok && lane == 0 && x4 >= 1, q);
            else if (cx(q) < 0) // column x4 + 4, for lane 31
                edge[q] = ld1<St>(src + 4, rok && lane == 31 && x4 + 4 < W, q);
        }
    }
    interior = interior && any == 0;
    if (!__all_sync(0xffffffffu, interior)) {
        if (xok) {
#pragma unroll 1
            for (int j = 0; j < 4; ++j)
                inplace_cell<Ph, St, LID, LOCAL>(p, x4 + j, y);
        }
        return;
    }
    float g[4][9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        float o[4];
        if (LOCAL) {
            unpack4<St>(raw[q], q == 0 ? 0 : opp(q), o);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                g[j][q] = o[j];
        } else {
            unpack4<St>(raw[q], q, o);
            if (cx(q) == 0) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    g[j][q] = o[j];
            } else if (cx(q) > 0) { // column x - 1
                float prev = __shfl_up_sync(0xffffffffu, o[3], 1);
                if (lane == 0)
                    prev = edge[q];
                g[0][q] = prev;
                g[1][q] = o[0];
                g[2][q] = o[1];
                g[3][q] = o[2];
            } else { // column x + 1
                float next = __shfl_down_sync(0xffffffffu, o[0], 1);
                if (lane == 31)
                    next = edge[q];
                g[0][q] = o[1];
                g[1][q] = o[2];
                g[2][q] = o[3];
                g[3][q] = next;
            }
        }
    }
    float r[4], u[4], v[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
        collide_bf<Ph, true>(g[j], false, 0.0f, p.k, r[j], u[j], v[j]);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        float o[4] = {g[0][q], g[1][q], g[2][q], g[3][q]};
        if (LOCAL || q == 0) {
            *reinterpret_cast<V *>(f + q * N + id) = pack4<St>(o, q);
            continue;
        }
        E *dst = f + opp(q) * N + id + (long long)cy(q) * W; // row y + c_y, aligned at x4
        if (cx(q) == 0) {
            *reinterpret_cast<V *>(dst) = pack4<St>(o, q);
        } else if (cx(q) > 0) { // destinations x4 + 1 .. x4 + 4
            const float prev = __shfl_up_sync(0xffffffffu, o[3], 1);
            if (lane == 0) {
                dst[1] = St::store(o[0], q);
                dst[2] = St::store(o[1], q);
                dst[3] = St::store(o[2], q);
            } else {
                const float w4[4] = {prev, o[0], o[1], o[2]};
                *reinterpret_cast<V *>(dst) = pack4<St>(w4, q);
            }
            if (lane == 31)
                dst[4] = St::store(o[3], q);
        } else { // destinations x4 - 1 .. x4 + 2
            const float next = __shfl_down_sync(0xffffffffu, o[0], 1);
            if (lane == 31) {
                dst[0] = St::store(o[1], q);
                dst[1] = St::store(o[2], q);
                dst[2] = St::store(o[3], q);
            } else {
                const float w4[4] = {o[1], o[2], o[3], next};
                *reinterpret_cast<V *>(dst) = pack4<St>(w4, q);
            }
            if (lane == 0)
                dst[-1] = St::store(o[0], q);
        }
    }
    if (LOCAL && p.ux) {
        *reinterpret_cast<float4 *>(p.ux + id) = make_float4(u[0], u[1], u[2], u[3]);
        *reinterpret_cast<float4 *>(p.uy + id) = make_float4(v[0], v[1], v[2], v[3]);
        *reinterpret_cast<float4 *>(p.rho + id) = make_float4(r[0], r[1], r[2], r[3]);
    }
}

static bool al16(const void *q)
{
    return (reinterpret_cast<uintptr_t>(q) & 15u) == 0;
}

template <class Ph, class St, bool LID> static int inplace_pair(const InplaceParams &p, bool local, cudaStream_t s)
{
    const bool vec = p.W % 4 == 0 && al16(p.f) && al16(p.mask) && (!p.ux || (al16(p.ux) && al16(p.uy) && al16(p.rho)));
    if (vec) {
        const dim3 block(64, 4), grid((p.W / 4 + 63) / 64, (p.H + 3) / 4);
        return status(local ? launch_pdl(inplace_vec_kernel<Ph, St, LID, true>, grid, block, 0, s, p)
                            : launch_pdl(inplace_vec_kernel<Ph, St, LID, false>, grid, block, 0, s, p));
    }
    const dim3 block(128, 2), grid((p.W + 127) / 128, (p.H + 1) / 2);
    return status(local ? launch_pdl(inplace_kernel<Ph, St, LID, true>, grid, block, 0, s, p)
                        : launch_pdl(inplace_kernel<Ph, St, LID, false>, grid, block, 0, s, p));
}

template <class St> static int inplace_variant(int variant, const InplaceParams &p, bool local, cudaStream_t s)
{
    switch (variant) {
    case VAR_MRT_SMAG_CLAMP:
        return inplace_pair<PhysMrtSmagClamp, St, false>(p, local, s);
    case VAR_MRT_SMAG:
        return inplace_pair<PhysMrtSmag, St, false>(p, local, s);
    case VAR_MRT:
        return inplace_pair<PhysMrt, St, false>(p, local, s);
    default:
        break;
    }
    if constexpr (std::is_same<St, StoreF32>::value) {
        if (variant == VAR_MRT_LID)
            return inplace_pair<PhysMrt, St, true>(p, local, s);
        if (variant == VAR_BGK)
            return inplace_pair<PhysBgk, St, false>(p, local, s);
    }
    return LBM_ERR_UNSUPPORTED;
}

// One step of the in-place scheme (local = false: the pull-push step, true: the
// local step).  Kernels launch on `s`; nothing synchronises.
int inplace_step(int variant, int storage, const InplaceParams &p, bool local, cudaStream_t s)
{
    switch (storage) {
    case LBM_STORE_F32:
        return inplace_variant<StoreF32>(variant, p, local, s);
    case LBM_STORE_F16DEV:
        return inplace_variant<StoreF16Dev>(variant, p, local, s);
    case LBM_STORE_BF16DEV:
        return inplace_variant<StoreBF16Dev>(variant, p, local, s);
    default:
        return LBM_ERR_ARG;
    }
}

} // namespace lbm
