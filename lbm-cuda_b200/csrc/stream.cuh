// Single-step pull kernel (T = 1) with 128-bit coalesced SoA access.
//
// Same state convention and boundary rules as the wavefront kernel (wave.cuh):
// f_out(x) = collide(pull(f_in)) with post-collision storage.  Each thread owns
// four consecutive cells of one row; a warp covers 128 columns.  For each
// population plane the thread loads one aligned 128-bit vector from the source
// row y - c_y; the one-column shift of the populations with c_x = +-1 comes
// from the neighbouring lane through a warp shuffle (edge lanes load the one
// missing value).  The mask is read as one 32-bit word per row.
//
// All global loads are issued up front as predicated loads (no branches), so
// each thread has 9 vector loads plus a few scalars in flight.  A warp whose
// 128 cells are all interior fluid (no solid neighbour, not an inlet, outlet
// or wall row) takes the fast path: plain pull, collide, one vector store per
// plane.  Other warps take the generic path (bounce-back, Zou-He inlet, outlet
// ghost, cells that are not updated).
//
// Requirements: W % 4 == 0 and 16-byte aligned planes (else the wavefront
// kernel's plain-load path runs the step).
#pragma once

#include "wave.cuh"

namespace lbm {

template <class Ph_, class St_, int MODE_, bool LID_ = false> struct StreamCfg {
    using Ph = Ph_;
    using St = St_;
    using E = typename St::T;
    static constexpr int MODE = MODE_;
    static constexpr bool LID = LID_;
};

// ---- predicated global loads (a false predicate issues no memory access) ----
__device__ __forceinline__ float4 ldg_v4f_pred(const void *p, bool pred)
{
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %5, 0;\n\t"
                 "@q ld.global.nc.v4.f32 {%0, %1, %2, %3}, [%4];\n\t}"
                 : "+f"(v.x), "+f"(v.y), "+f"(v.z), "+f"(v.w)
                 : "l"(p), "r"((unsigned)pred));
    return v;
}
__device__ __forceinline__ uint2 ldg_v2u_pred(const void *p, bool pred)
{
    uint2 v = make_uint2(0u, 0u);
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %3, 0;\n\t"
                 "@q ld.global.nc.v2.u32 {%0, %1}, [%2];\n\t}"
                 : "+r"(v.x), "+r"(v.y)
                 : "l"(p), "r"((unsigned)pred));
    return v;
}
__device__ __forceinline__ uint32_t ldg_u32_pred(const void *p, bool pred)
{
    uint32_t v = 0u;
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t"
                 "@q ld.global.nc.u32 %0, [%1];\n\t}"
                 : "+r"(v)
                 : "l"(p), "r"((unsigned)pred));
    return v;
}
__device__ __forceinline__ uint32_t ldg_u16_pred(const void *p, bool pred)
{
    unsigned short v = 0;
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t"
                 "@q ld.global.nc.u16 %0, [%1];\n\t}"
                 : "+h"(v)
                 : "l"(p), "r"((unsigned)pred));
    return v;
}
__device__ __forceinline__ uint32_t ldg_u8_pred(const void *p, bool pred)
{
    unsigned short v = 0;
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %2, 0;\n\t"
                 "@q ld.global.nc.u8 %0, [%1];\n\t}"
                 : "+h"(v)
                 : "l"(p), "r"((unsigned)pred));
    return v;
}

// Four consecutive populations of one plane, raw storage bits.
template <class E> struct Raw4 {
    using type = float4;
};
template <> struct Raw4<__half> {
    using type = uint2;
};
template <> struct Raw4<__nv_bfloat16> {
    using type = uint2;
};

template <class E> __device__ __forceinline__ typename Raw4<E>::type ld4(const E *p, bool pred)
{
    if constexpr (sizeof(E) == 4)
        return ldg_v4f_pred(p, pred);
    else
        return ldg_v2u_pred(p, pred);
}

template <class St> __device__ __forceinline__ float ld1(const typename St::T *p, bool pred, int q)
{
    using E = typename St::T;
    if constexpr (sizeof(E) == 4) {
        return __uint_as_float(ldg_u32_pred(p, pred));
    } else {
        const unsigned short b = (unsigned short)ldg_u16_pred(p, pred);
        return pred ? St::load(*reinterpret_cast<const E *>(&b), q) : 0.0f;
    }
}

template <class St> __device__ __forceinline__ void unpack4(const typename Raw4<typename St::T>::type &v, int q, float (&o)[4])
{
    using E = typename St::T;
    if constexpr (sizeof(E) == 4) {
        o[0] = v.x;
        o[1] = v.y;
        o[2] = v.z;
        o[3] = v.w;
    } else {
        const E *e = reinterpret_cast<const E *>(&v);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            o[j] = St::load(e[j], q);
    }
}

template <class St> __device__ __forceinline__ typename Raw4<typename St::T>::type pack4(const float (&o)[4], int q)
{
    using E = typename St::T;
    typename Raw4<E>::type v;
    if constexpr (sizeof(E) == 4) {
        v.x = o[0];
        v.y = o[1];
        v.z = o[2];
        v.w = o[3];
    } else {
        E *e = reinterpret_cast<E *>(&v);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            e[j] = St::store(o[j], q);
    }
    return v;
}

template <class C> __global__ void __launch_bounds__(128, 4) stream_kernel(const __grid_constant__ WaveParams p)
{
    using St = typename C::St;
    using E = typename C::E;
    using V = typename Raw4<E>::type;
    using Ph = typename C::Ph;
    pdl_trigger();
    pdl_wait(); // launched with programmatic dependent launch: the previous step's stores first
    const int W = p.W, H = p.H;
    const int lane = threadIdx.x;
    const int x4 = 4 * (blockIdx.x * 32 + lane);
    const int y = blockIdx.y * 4 + threadIdx.y;
    const bool pxper = (C::MODE == MODE_GENERAL) && p.bc_left == LBM_BC_PERIODIC;
    const bool pyper = (C::MODE == MODE_GENERAL) && p.bc_y == LBM_BC_PERIODIC;
    const bool xok = x4 < W;
    const bool redge = lane == 31 || x4 + 4 >= W; // right neighbour column not held by the next lane
    const E *fin = reinterpret_cast<const E *>(p.f_in);
    int xl = x4 - 1, xr = x4 + 4;
    if (pxper) {
        xl = wrap(xl, W);
        xr = wrap(xr, W);
    }
    const bool xl_ok = xl >= 0 && xl < W, xr_ok = xr >= 0 && xr < W;

    // ---------------- round 1: every load of the step ----------------
    // Row offsets of rows y-1, y, y+1 (wrapped when periodic), computed once.
    long long roff[3], moff[3];
    bool rok[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        int r = y + d - 1;
        if (pyper)
            r = wrap(r, H);
        rok[d] = r >= 0 && r < H;
        roff[d] = (long long)r * p.pitch;
        moff[d] = (long long)r * p.mask_pitch;
    }
    uint32_t mw[3], ml[3], mr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const uint8_t *mrow = p.mask + moff[d];
        mw[d] = ldg_u32_pred(mrow + x4, rok[d] && xok);
        ml[d] = ldg_u8_pred(mrow + xl, rok[d] && lane == 0 && xl_ok);
        mr[d] = ldg_u8_pred(mrow + xr, rok[d] && redge && xr_ok);
    }
    V v[9];
    float edge[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int d = 1 - cy(q); // source row y - c_y
        const E *rowp = fin + q * p.plane + roff[d];
        v[q] = ld4<E>(rowp + x4, rok[d] && xok);
        if (cx(q) == 1)
            edge[q] = ld1<St>(rowp + xl, rok[d] && lane == 0 && xl_ok, q);
        else if (cx(q) == -1)
            edge[q] = ld1<St>(rowp + xr, rok[d] && redge && xr_ok, q);
        else
            edge[q] = 0.0f;
    }

    // ---------------- pull: x shift through shuffles ----------------
    float f[9][4];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        float c4[4];
        unpack4<St>(v[q], q, c4);
        if (cx(q) == 0) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                f[q][j] = c4[j];
        } else if (cx(q) == 1) { // source column x - 1
            const float left = __shfl_up_sync(0xffffffffu, c4[3], 1);
            f[q][0] = lane == 0 ? edge[q] : left;
            f[q][1] = c4[0];
            f[q][2] = c4[1];
            f[q][3] = c4[2];
        } else { // source column x + 1
            const float right = __shfl_down_sync(0xffffffffu, c4[0], 1);
            f[q][0] = c4[1];
            f[q][1] = c4[2];
            f[q][2] = c4[3];
            f[q][3] = redge ? edge[q] : right;
        }
    }
    // mask bytes of columns x4-1 and x4+4 come from the neighbouring lanes
    uint32_t mlx[3], mrx[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const uint32_t left = __shfl_up_sync(0xffffffffu, mw[d], 1) >> 24;
        const uint32_t right = __shfl_down_sync(0xffffffffu, mw[d], 1) & 0xffu;
        mlx[d] = lane == 0 ? ml[d] : left;
        mrx[d] = redge ? mr[d] : right;
    }

    // Interior cells: rows 1..H-2 (every row when y is periodic: the row loads
    // above already wrapped, so the first and last rows pull like any other and
    // the arithmetic does not depend on the row), columns 1..W-3 (no inlet,
    // outlet source or ghost), no solid cell in the 3x3 neighbourhood of any of
    // the four cells.
    const uint32_t any_solid = mw[0] | mw[1] | mw[2] | mlx[0] | mlx[1] | mlx[2] | mrx[0] | mrx[1] | mrx[2];
    const bool yin = pyper ? (y >= 0 && y < H) : (y >= 1 && y <= H - 2);
    const bool interior = xok && yin && x4 >= 1 && x4 + 3 <= W - 3 && any_solid == 0;
    const bool fast = __all_sync(0xffffffffu, interior);

    float out[9][4], ro[4], uo[4], vo[4];
    bool wr[4];
    if (fast) {
        float g[4][9];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int q = 0; q < 9; ++q)
                g[j][q] = f[q][j];
        if constexpr (Ph::kRefOrder) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                collide_bf<Ph, false>(g[j], false, 0.0f, p.k, ro[j], uo[j], vo[j]);
        } else {
            collide_multi<Ph, 4>(g, p.k, ro, uo, vo);
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int q = 0; q < 9; ++q)
                out[q][j] = g[j][q];
            wr[j] = true;
        }
    } else {
        // ---------------- generic path ----------------
        uint64_t win[3];
#pragma unroll
        for (int d = 0; d < 3; ++d)
            win[d] = (uint64_t)mlx[d] | ((uint64_t)mw[d] << 8) | ((uint64_t)mrx[d] << 40);
        uint32_t code[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            Nbhd n;
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx)
                    n.m[dy + 1][dx + 1] = (uint8_t)((win[dy + 1] >> (8 * (j + dx + 1))) & 0xffu);
            if (C::MODE == MODE_CORE4)
                code[j] = build_code_core4(n, x4 + j, y, W, H);
            else
                code[j] = build_code_general(n, x4 + j, y, p);
        }
        // round 2 (cells next to solids only): the cell's own post-collision
        // value of the opposite direction, for half-way bounce-back
        const uint32_t allc = code[0] | code[1] | code[2] | code[3];
        const bool yok = y >= 0 && y < H;
#pragma unroll
        for (int q = 1; q < 9; ++q) {
            const int qo = opp(q);
            const V ov = ld4<E>(fin + qo * p.plane + (long long)y * p.pitch + x4, yok && xok && (allc & (1u << q)));
            float o4[4];
            unpack4<St>(ov, qo, o4);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float b = o4[j];
                if (C::LID)
                    b += ((code[j] >> (C_MOVING_SHIFT + q)) & 1u) ? 6.0f * wgt(q) * (float)cx(q) * p.k.u_lid : 0.0f;
                f[q][j] = ((code[j] >> q) & 1u) ? b : f[q][j];
            }
        }
        const bool zh = (C::MODE == MODE_CORE4 || p.bc_left == LBM_BC_ZOUHE || p.bc_left == LBM_BC_ZOUHE_RAMP) &&
                        x4 == 0;
        const float lu = zh ? inlet_u(p.k, pyper ? wrap(y, H) : y) : 0.0f;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float g[9];
#pragma unroll
            for (int q = 0; q < 9; ++q)
                g[q] = f[q][j];
            collide_bf<Ph, true>(g, (code[j] & C_INLET) != 0, lu, p.k, ro[j], uo[j], vo[j]);
#pragma unroll
            for (int q = 0; q < 9; ++q)
                out[q][j] = g[q];
            wr[j] = !(code[j] & C_SKIP);
        }
        // W % 4 == 0: column W-1 is element 3 and W-2 element 2 of the last vector.
        if (code[2] & C_GHOST_SRC) {
#pragma unroll
            for (int q = 0; q < 9; ++q)
                out[q][3] = out[q][2];
            wr[3] = true;
        }
    }

    // ---------------- store ----------------
    if (!xok || y < 0 || y >= H)
        return;
    E *fo = reinterpret_cast<E *>(p.f_out) + (long long)y * p.pitch + x4;
    if (wr[0] && wr[1] && wr[2] && wr[3]) {
#pragma unroll
        for (int q = 0; q < 9; ++q)
            *reinterpret_cast<V *>(fo + q * p.plane) = pack4<St>(out[q], q);
    } else {
#pragma unroll
        for (int q = 0; q < 9; ++q)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (wr[j])
                    fo[q * p.plane + j] = St::store(out[q][j], q);
    }
    if (p.ux) {
        const long long id = (long long)y * W + x4;
        // macroscopic values of updated cells only (the ghost column excluded)
        bool mw4[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            mw4[j] = wr[j] && !(j == 3 && x4 + 3 == W - 1 && (C::MODE == MODE_CORE4 || p.bc_right == LBM_BC_OUTFLOW));
        if (mw4[0] && mw4[1] && mw4[2] && mw4[3]) {
            *reinterpret_cast<float4 *>(p.ux + id) = make_float4(uo[0], uo[1], uo[2], uo[3]);
            *reinterpret_cast<float4 *>(p.uy + id) = make_float4(vo[0], vo[1], vo[2], vo[3]);
            *reinterpret_cast<float4 *>(p.rho + id) = make_float4(ro[0], ro[1], ro[2], ro[3]);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (mw4[j]) {
                    p.ux[id + j] = uo[j];
                    p.uy[id + j] = vo[j];
                    p.rho[id + j] = ro[j];
                }
        }
    }
}

} // namespace lbm
