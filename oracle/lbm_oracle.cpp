// CPU oracle for the D2Q9 collide-stream path of Qianyv-Li8262/LBM-CUDA.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is called by tests/,
// by the smoke check in __graft_entry__.py and by the cpu_baseline leg of
// bench.py, never by the product path (lbm-cuda_b200/), which fails loudly when
// its CUDA library is missing.
//
// Every routine restates the arithmetic of one reference kernel on the CPU, in
// plain loops, templated on the scalar type S (float = same precision as the
// reference, double = FP64 oracle).  Each function cites the reference lines it
// follows.  Parity is pinned by tests/golden/*.npz: outputs of the reference's
// own kernels (compiled from its .cu sources by oracle/Makefile into
// oracle/_ref/) on seeded inputs, produced on a B200 by tests/golden/make_golden.py.
//
// Lattice convention (lbm_core4.cu:1-3, lbm_core_smemaa.cu:1-5):
//   c_x = {0,1,0,-1,0,1,-1,-1,1}, c_y = {0,0,1,0,-1,1,1,-1,-1}, opp = {0,3,4,1,2,7,8,5,6}
//   populations are SoA planes f[q*W*H + y*W + x]; the mask is one byte per cell.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int CX[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
constexpr int CY[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
constexpr int OPP[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};

template <class S> inline S wq(int q)
{
    // lbm_core_smemaa.cu:4-5 (written there as 9-digit decimals; here as exact ratios)
    return q == 0 ? S(4) / S(9) : (q < 5 ? S(1) / S(9) : S(1) / S(36));
}

template <class S> inline S clampv(S v, S lo, S hi)
{
    return std::min(hi, std::max(lo, v));
}

// Smoothed Zou-He inlet velocity profile: lbm_core4.cu:46-51 (same in every kernel).
template <class S> inline S ramp_u(S u_in, int y, int H)
{
    S d = std::min(S(y), S(H - 1 - y));
    S sm = S(1);
    if (d < S(50))
        sm = S(0.5) * (S(1) - std::cos(S(3.14159f) * d / S(50)));
    return u_in * sm;
}

// Zou-He reconstruction of f1, f5, f8 at x=0 and the inlet density: lbm_core4.cu:54-57.
template <class S> inline S zou_he(S *f, S lu)
{
    S rho = (f[0] + f[2] + f[4] + S(2) * (f[3] + f[6] + f[7])) / (S(1) - lu);
    f[1] = f[3] + S(0.666666667f) * rho * lu;
    f[5] = f[7] - S(0.5) * (f[2] - f[4]) + S(0.16666666666f) * rho * lu;
    f[8] = f[6] + S(0.5) * (f[2] - f[4]) + S(0.16666666666f) * rho * lu;
    return rho;
}

// MRT relaxation in the Lallemand-Luo basis followed by the inverse transform:
// lbm_core4.cu:69-108 (inlet) and :150-199 (interior).  m0 = rho and m3/m5 are the
// momenta the caller chose (clamped ones in the interior); s_nu relaxes the two
// stress moments, s_e/s_eps/s_q the energy, energy-square and heat-flux moments.
template <class S> inline void mrt_relax(S *f, S rho, S ux, S uy, S s_e, S s_eps, S s_q, S s_nu)
{
    S f14 = f[1] + f[2] + f[3] + f[4];
    S f58 = f[5] + f[6] + f[7] + f[8];
    S m[9];
    m[0] = rho;
    m[1] = S(-4) * f[0] + S(2) * f58 - f14;
    m[2] = S(4) * f[0] + f58 - S(2) * f14;
    m[3] = rho * ux;
    m[4] = S(-2) * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
    m[5] = rho * uy;
    m[6] = S(-2) * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
    m[7] = f[1] - f[2] + f[3] - f[4];
    m[8] = f[5] - f[6] + f[7] - f[8];
    S usq = ux * ux + uy * uy;
    S m1eq = (S(3) * usq - S(2)) * rho;
    S m2eq = (S(1) - S(3) * usq) * rho;
    S m7eq = rho * (ux * ux - uy * uy);
    S m8eq = rho * ux * uy;
    m[1] -= s_e * (m[1] - m1eq);
    m[2] -= s_eps * (m[2] - m2eq);
    m[4] -= s_q * (m[4] + m[3]);
    m[6] -= s_q * (m[6] + m[5]);
    m[7] -= s_nu * (m[7] - m7eq);
    m[8] -= s_nu * (m[8] - m8eq);
    const S inv9 = S(1) / S(9), inv36 = S(1) / S(36);
    S t0 = m[0] - m[1] + m[2];
    S t1 = S(4) * m[0] - m[1] - S(2) * m[2];
    S t2 = S(4) * m[0] + S(2) * m[1] + m[2];
    f[0] = t0 * inv9;
    f[1] = (t1 + S(6) * m[3] - S(6) * m[4] + S(9) * m[7]) * inv36;
    f[2] = (t1 + S(6) * m[5] - S(6) * m[6] - S(9) * m[7]) * inv36;
    f[3] = (t1 - S(6) * m[3] + S(6) * m[4] + S(9) * m[7]) * inv36;
    f[4] = (t1 - S(6) * m[5] + S(6) * m[6] - S(9) * m[7]) * inv36;
    f[5] = (t2 + S(6) * m[3] + S(3) * m[4] + S(6) * m[5] + S(3) * m[6] + S(9) * m[8]) * inv36;
    f[6] = (t2 - S(6) * m[3] - S(3) * m[4] + S(6) * m[5] + S(3) * m[6] - S(9) * m[8]) * inv36;
    f[7] = (t2 - S(6) * m[3] - S(3) * m[4] - S(6) * m[5] - S(3) * m[6] + S(9) * m[8]) * inv36;
    f[8] = (t2 + S(6) * m[3] + S(3) * m[4] - S(6) * m[5] - S(3) * m[6] - S(9) * m[8]) * inv36;
}

// Smagorinsky-corrected stress relaxation rate: lbm_core4.cu:171-177.
template <class S> inline S smag_rate(const S *f, S rho, S ux, S uy, S tau0, S cs)
{
    S m7 = f[1] - f[2] + f[3] - f[4];
    S m8 = f[5] - f[6] + f[7] - f[8];
    S n7 = m7 - rho * (ux * ux - uy * uy);
    S n8 = m8 - rho * ux * uy;
    S Q = std::sqrt(n7 * n7 + n8 * n8 + S(1e-8f));
    S tau_eff = S(0.5) * (tau0 + std::sqrt(tau0 * tau0 + S(18) * cs * cs * Q / rho));
    return S(1) / tau_eff;
}

// Second-order BGK collision: lbm_core_smemaa.cu:206-212.
template <class S> inline void bgk(S *f, S rho, S ux, S uy, S s_nu)
{
    S usq = ux * ux + uy * uy;
    for (int q = 0; q < 9; ++q) {
        S cu = S(CX[q]) * ux + S(CY[q]) * uy;
        S feq = wq<S>(q) * rho * (S(1) + S(3) * cu + S(4.5) * cu * cu - S(1.5) * usq);
        f[q] += s_nu * (feq - f[q]);
    }
}

// Macroscopic density and velocity of one cell (lbm_core_smemaa.cu:194-201).
template <class S> inline void moments(const S *f, S &rho, S &ux, S &uy)
{
    rho = 0;
    ux = 0;
    uy = 0;
    for (int q = 0; q < 9; ++q) {
        rho += f[q];
        ux += f[q] * S(CX[q]);
        uy += f[q] * S(CY[q]);
    }
    ux /= rho;
    uy /= rho;
}

// ---------------------------------------------------------------------------
// lbm_core4.cu fused_lbmkernel: one pull-stream + MRT(+Smagorinsky) step,
// ping-pong f_now -> f_out, writes u, v, rho.  Follows lbm_core4.cu:14-212:
//   * rows 1..H-2, columns 0..W-2 are updated; solid cells (x>0) are skipped;
//   * x=0: pulls from x=-1 read 0, Zou-He with the cosine ramp, MRT with tau_inv
//     and no Smagorinsky (:29-118);
//   * interior: pull with half-way bounce-back from solid sources, clamps on u and
//     rho, Smagorinsky with Cs = cs (0.20 in the reference), s_e = s_eps = s_q = si
//     (1.1 in the reference) (:120-211);
//   * every population is clamped to [0, 10]; the W-2 column is duplicated into
//     the W-1 outlet ghost (:109-117, :200-210).
// ---------------------------------------------------------------------------
template <class S>
void core4_step(const uint8_t *mask, const S *fn, S *fo, S *ux, S *uy, S *rho, int W, int H, S tau_inv, S u_in, S cs,
                S si)
{
    const long N = (long)W * H;
    const S tau0 = S(1) / tau_inv;
#pragma omp parallel for schedule(static)
    for (int y = 1; y < H - 1; ++y) {
        for (int x = 0; x < W - 1; ++x) {
            const long pid = (long)y * W + x;
            S f[9];
            S r, u, v, s_nu;
            if (x == 0) {
                for (int q = 0; q < 9; ++q) {
                    int sx = -CX[q], sy = y - CY[q];
                    if (sx < 0) {
                        f[q] = 0;
                    } else {
                        long sid = (long)sy * W + sx;
                        f[q] = mask[sid] ? fn[OPP[q] * N + pid] : fn[q * N + sid];
                    }
                }
                S lu = ramp_u(u_in, y, H);
                r = zou_he(f, lu);
                u = lu;
                v = 0;
                s_nu = tau_inv;
            } else {
                if (mask[pid])
                    continue;
                for (int q = 0; q < 9; ++q) {
                    int sx = x - CX[q], sy = y - CY[q];
                    long sid = (long)sy * W + sx;
                    f[q] = mask[sid] ? fn[OPP[q] * N + pid] : fn[q * N + sid];
                }
                moments(f, r, u, v);
                u = clampv(u, S(-0.4), S(0.4));
                v = clampv(v, S(-0.4), S(0.4));
                r = clampv(r, S(0), S(1.5));
                s_nu = smag_rate(f, r, u, v, tau0, cs);
            }
            ux[pid] = u;
            uy[pid] = v;
            rho[pid] = r;
            mrt_relax(f, r, u, v, si, si, si, s_nu);
            for (int q = 0; q < 9; ++q) {
                S o = clampv(f[q], S(0), S(10));
                fo[q * N + pid] = o;
                if (x == W - 2)
                    fo[q * N + pid + 1] = o;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Shared-memory AA pattern of the smemaa / policy / endfused kernels, restated
// on the whole domain.  The slot array has a one-cell frame of out-of-domain
// cells around the domain.  smask follows lbm_core_smemaa.cu:39-70 /
// lbm_core_smemaa_policy.cu:106-118: out-of-domain = solid, column W-1 = fluid
// (open outlet ghost, corners included), else the user mask.  A cell is
// "updated" when it is in the domain, 0 < y < H-1, x < W-1 and not solid.
// ---------------------------------------------------------------------------
template <class S> struct AaDomain {
    int W, H, WP, HP; // WP/HP include the frame
    std::vector<S> slot; // [9][HP][WP]
    std::vector<uint8_t> smask; // [HP][WP]
    long plane() const
    {
        return (long)WP * HP;
    }
    long at(int x, int y) const
    {
        return (long)(y + 1) * WP + (x + 1);
    }
    S &s(int q, int x, int y)
    {
        return slot[q * plane() + at(x, y)];
    }
    bool solid(int x, int y) const
    {
        return smask[at(x, y)] != 0;
    }
    bool updated(int x, int y) const
    {
        return x >= 0 && x < W - 1 && y > 0 && y < H - 1 && !solid(x, y);
    }

    // Tile load of lbm_core_smemaa.cu:34-71: canonical f and mask; frame = 0 / solid.
    void load(const uint8_t *mask, const S *f)
    {
        WP = W + 2;
        HP = H + 2;
        slot.assign(9 * plane(), S(0));
        smask.assign(plane(), 1);
        const long N = (long)W * H;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                long id = (long)y * W + x;
                smask[at(x, y)] = (x == W - 1) ? 0 : (mask[id] ? 1 : 0);
                for (int q = 0; q < 9; ++q)
                    s(q, x, y) = f[q * N + id];
            }
    }

    // Zou-He (x = 0) or moment evaluation, then BGK: lbm_core_smemaa.cu:159-212.
    void collide(S *f, int x, int y, S tau_inv, S u_in) const
    {
        S r, u, v;
        if (x == 0) {
            S lu = ramp_u(u_in, y, H);
            r = zou_he(f, lu);
            u = lu;
            v = 0;
        } else {
            moments(f, r, u, v);
        }
        bgk(f, r, u, v, tau_inv);
    }

    // A phase, lbm_core_smemaa.cu:107-223: local collide, reversed store.
    void phase_a(S tau_inv, S u_in)
    {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                if (!updated(x, y))
                    continue;
                S f[9];
                for (int q = 0; q < 9; ++q)
                    f[q] = s(q, x, y);
                collide(f, x, y, tau_inv, u_in);
                for (int q = 0; q < 9; ++q)
                    s(OPP[q], x, y) = clampv(f[q], S(0), S(10));
            }
    }

    // B phase, lbm_core_smemaa.cu:293-445: gather s[opp q][x-c_q] (or s[q][x] if the
    // source is solid), collide, scatter to s[q][x+c_q] (or s[opp q][x] if the target
    // is solid; x=0 populations leaving to the left go to the discard frame).  Each
    // cell reads exactly the slots it writes, so cells are independent.
    void phase_b(S tau_inv, S u_in)
    {
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                if (!updated(x, y))
                    continue;
                S f[9];
                for (int q = 0; q < 9; ++q) {
                    int sx = x - CX[q], sy = y - CY[q];
                    f[q] = solid(sx, sy) ? s(q, x, y) : s(OPP[q], sx, sy);
                }
                collide(f, x, y, tau_inv, u_in);
                for (int q = 0; q < 9; ++q) {
                    int dx = x + CX[q], dy = y + CY[q];
                    S o = clampv(f[q], S(0), S(10));
                    if (x == 0 && CX[q] < 0)
                        s(q, dx, dy) = o;
                    else if (solid(dx, dy))
                        s(OPP[q], x, y) = o;
                    else
                        s(q, dx, dy) = o;
                }
            }
    }

    // Outlet ghost copy W-2 -> W-1 on rows 1..H-2: lbm_core_smemaa.cu:237-266 / :461-479.
    void ghost_copy()
    {
        if (W < 2)
            return;
        for (int y = 1; y < H - 1; ++y)
            for (int q = 0; q < 9; ++q)
                s(q, W - 1, y) = s(q, W - 2, y);
    }
};

// lbm_core_smemaa.cu fused_lbmkernel (BGK, T steps per launch, T even): tile load,
// T/2 A/B pairs with the outlet copy after each phase, store of canonical f for
// every in-domain cell and u, v, rho of updated cells (:500-546).
template <class S>
void smemaa_launch(const uint8_t *mask, const S *fn, S *fo, S *ux, S *uy, S *rho, int W, int H, S tau_inv, S u_in,
                   int T)
{
    AaDomain<S> d;
    d.W = W;
    d.H = H;
    d.load(mask, fn);
    for (int p = 0; p < T / 2; ++p) {
        d.phase_a(tau_inv, u_in);
        d.ghost_copy();
        d.phase_b(tau_inv, u_in);
        d.ghost_copy();
    }
    const long N = (long)W * H;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            long id = (long)y * W + x;
            for (int q = 0; q < 9; ++q)
                fo[q * N + id] = d.s(q, x, y);
            if (!d.solid(x, y) && x < W - 1 && y > 0 && y < H - 1) {
                S f[9], r, u, v;
                for (int q = 0; q < 9; ++q)
                    f[q] = d.s(q, x, y);
                moments(f, r, u, v);
                ux[id] = u;
                uy[id] = v;
                rho[id] = r;
            }
        }
}

// lbm_core_smemaa_policy.cu / lbm_core_smemaa_endfused.cu fused_lbmkernel (BGK,
// T steps, T even >= 2).  A0 reads canonical f from f_now (:103-163), the outlet
// copy follows every A phase only (:169-179, :312-326), and B-final scatters
// straight into f_out (:338-424): populations leaving x=0 to the left are dropped,
// targets in column W-1 are skipped, targets in column W-2 are duplicated into
// W-1, and f_out entries no scatter reaches keep their previous contents.
// The reference leaves the slots of cells A0 does not update uninitialised; the
// only such slots it can read are those of the fluid outlet corners (W-1,0) and
// (W-1,H-1).  Here every slot starts from f_now (as in lbm_core_smemaa.cu), so a
// parity comparison with the reference is meaningful only for masks in which
// (W-2,1) and (W-2,H-2) are solid.
template <class S>
void policy_launch(const uint8_t *mask, const S *fn, S *fo, int W, int H, S tau_inv, S u_in, int T)
{
    AaDomain<S> d;
    d.W = W;
    d.H = H;
    d.load(mask, fn);
    d.phase_a(tau_inv, u_in);
    d.ghost_copy();
    for (int stage = 1; stage < T - 1; ++stage) {
        if (stage & 1) {
            d.phase_b(tau_inv, u_in);
        } else {
            d.phase_a(tau_inv, u_in);
            d.ghost_copy();
        }
    }
    // B-final
    const long N = (long)W * H;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            if (!d.updated(x, y))
                continue;
            S f[9];
            for (int q = 0; q < 9; ++q) {
                int sx = x - CX[q], sy = y - CY[q];
                f[q] = d.solid(sx, sy) ? d.s(q, x, y) : d.s(OPP[q], sx, sy);
            }
            d.collide(f, x, y, tau_inv, u_in);
            for (int q = 0; q < 9; ++q) {
                if (x == 0 && CX[q] < 0)
                    continue;
                int tx, ty, tq;
                if (d.solid(x + CX[q], y + CY[q])) {
                    tx = x;
                    ty = y;
                    tq = OPP[q];
                } else {
                    tx = x + CX[q];
                    ty = y + CY[q];
                    tq = q;
                }
                if (tx == W - 1 || tx < 0 || tx >= W || ty < 0 || ty >= H)
                    continue;
                S o = clampv(f[q], S(0), S(10));
                fo[tq * N + (long)ty * W + tx] = o;
                if (tx == W - 2)
                    fo[tq * N + (long)ty * W + (W - 1)] = o;
            }
        }
}

// lbm_core_smemaa_policy.cu macro_kernel (:431-476): u, v, rho of updated columns
// 0..W-2, rows 1..H-2, non-solid; Zou-He at x = 0 before the moments.
template <class S>
void macro(const S *f, S *ux, S *uy, S *rho, const uint8_t *mask, int W, int H, S u_in)
{
    const long N = (long)W * H;
    for (int y = 1; y < H - 1; ++y)
        for (int x = 0; x < W - 1; ++x) {
            long pid = (long)y * W + x;
            if (mask[pid])
                continue;
            S fl[9], r, u, v;
            for (int q = 0; q < 9; ++q)
                fl[q] = f[q * N + pid];
            if (x == 0) {
                S lu = ramp_u(u_in, y, H);
                r = zou_he(fl, lu);
                u = lu;
                v = 0;
            } else {
                moments(fl, r, u, v);
            }
            ux[pid] = u;
            uy[pid] = v;
            rho[pid] = r;
        }
}

// visualizekernel (lbm_core4.cu:214-255): central-difference vorticity to RGBA.
void visualize(const float *ux, const float *uy, uint8_t *img, const uint8_t *mask, int W, int H, float vort_scale)
{
    for (int y = 1; y < H - 1; ++y)
        for (int x = 1; x < W - 1; ++x) {
            long pid = (long)y * W + x;
            img[pid * 4 + 3] = 255;
            if (mask[pid]) {
                img[pid * 4 + 0] = 0;
                img[pid * 4 + 1] = 0;
                img[pid * 4 + 2] = 0;
                continue;
            }
            float vort = ((uy[pid + 1] - uy[pid - 1]) - (ux[pid + W] - ux[pid - W])) * vort_scale;
            float r = std::min(std::max(1.0f + vort, 0.0f), 1.0f);
            float g = std::min(std::max(1.0f - std::fabs(vort), 0.0f), 1.0f);
            float b = std::min(std::max(1.0f - vort, 0.0f), 1.0f);
            img[pid * 4 + 0] = (uint8_t)(r * 255);
            img[pid * 4 + 1] = (uint8_t)(g * 255);
            img[pid * 4 + 2] = (uint8_t)(b * 255);
        }
}


// ---------------------------------------------------------------------------
// General solver step (lbm_params semantics; no reference counterpart beyond
// the physics above).  Pull step on post-collision populations, ping-pong:
//   * out-of-domain sources are stationary walls unless the side is periodic;
//   * mask 0 = fluid, 2 = wall moving with (u_lid, 0) (Ladd: the bounced
//     population gains 6 w_q rho_w c_q.u_w, rho_w = 1), other nonzero = solid;
//   * bc_left Zou-He (flat or the reference's ramp) on the fluid cells of x = 0;
//   * bc_right outflow: column W-1 is a ghost receiving the post-collision
//     populations of x = W-2 (lbm_core4.cu:114-116);
//   * cells that are not updated keep f_out's previous contents.
// iparams = {W, H, collision(0 BGK, 1 MRT), closure(0 none, 1 Smagorinsky, 2 ReLU MLP, 3 SiLU MLP),
//            bc_left, bc_right, bc_y, ref_clamps}
// dparams = {s_nu, s_e, s_eps, s_q, cs, u_in, u_lid}
// BC codes: 0 wall, 1 periodic, 2 Zou-He, 3 Zou-He with ramp, 4 outflow.
// ---------------------------------------------------------------------------
// Learned closure (closure code 2: ReLU network, 3: SiLU network): nu_t =
// out_scale softplus(MLP(in_scale x)), MLP 5 -> 32 -> 32 -> 1, in double
// precision, silu(a) = a / (1 + exp(-a)); x = (n7, n8, ne,
// |(n7, n8)|, rho - 1) of the pre-collision populations.  Parameters: W1[32][5],
// b1[32], W2[32][32], b2[32], w3[32], b3 (set by orc_set_mlp).
struct MlpParams {
    double p[32 * 5 + 32 + 32 * 32 + 32 + 32 + 1];
    double in_scale[5];
    double out_scale;
    bool set;
};
static MlpParams g_mlp = {{0}, {0}, 1.0, false};


inline double mlp_act(double a, bool silu)
{
    return silu ? a / (1.0 + std::exp(-a)) : std::max(a, 0.0);
}

template <class S> inline S mlp_rate(const S *f, S r, S u, S v, S tau0, bool silu)
{
    const double n7 = double((f[1] - f[2] + f[3] - f[4]) - r * (u * u - v * v));
    const double n8 = double((f[5] - f[6] + f[7] - f[8]) - r * u * v);
    const double m1 = double(-S(4) * f[0] - (f[1] + f[2] + f[3] + f[4]) + S(2) * (f[5] + f[6] + f[7] + f[8]));
    const double ne = m1 - double(r) * (3.0 * double(u * u + v * v) - 2.0);
    const double x[5] = {n7, n8, ne, std::sqrt(n7 * n7 + n8 * n8), double(r) - 1.0};
    const double *P = g_mlp.p;
    double h1[32], h2[32];
    for (int i = 0; i < 32; ++i) {
        double a = P[160 + i];
        for (int k = 0; k < 5; ++k)
            a += P[i * 5 + k] * x[k] * g_mlp.in_scale[k];
        h1[i] = mlp_act(a, silu);
    }
    for (int i = 0; i < 32; ++i) {
        double a = P[192 + 1024 + i];
        for (int k = 0; k < 32; ++k)
            a += P[192 + i * 32 + k] * h1[k];
        h2[i] = mlp_act(a, silu);
    }
    double z = P[192 + 1024 + 32 + 32];
    for (int k = 0; k < 32; ++k)
        z += P[192 + 1024 + 32 + k] * h2[k];
    const double sp = z > 30.0 ? z : std::log1p(std::exp(z));
    return S(1) / (tau0 + S(3.0 * g_mlp.out_scale * sp));
}

template <class S>
void general_step(const int *ip, const double *dp, const uint8_t *mask, const S *fn, S *fo, S *ux, S *uy, S *rho)
{
    const int W = ip[0], H = ip[1], coll = ip[2], clos = ip[3], bl = ip[4], br = ip[5], by = ip[6], clamps = ip[7];
    const S s_nu = S(dp[0]), s_e = S(dp[1]), s_eps = S(dp[2]), s_q = S(dp[3]), cs = S(dp[4]), u_in = S(dp[5]),
            u_lid = S(dp[6]);
    const bool px = bl == 1, py = by == 1, outflow = br == 4, zh = bl == 2 || bl == 3, ramp = bl == 3;
    const long N = (long)W * H;
    const S tau0 = S(1) / s_nu;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y) {
        for (int x = 0; x < W; ++x) {
            const long pid = (long)y * W + x;
            if (mask[pid] != 0 || (outflow && x == W - 1))
                continue;
            S f[9];
            for (int q = 0; q < 9; ++q) {
                int sx = x - CX[q], sy = y - CY[q];
                bool out = false;
                if (px)
                    sx = (sx + W) % W;
                else if (sx < 0 || sx >= W)
                    out = true;
                if (py)
                    sy = (sy + H) % H;
                else if (sy < 0 || sy >= H)
                    out = true;
                int mv = out ? 1 : mask[(long)sy * W + sx];
                if (mv) {
                    S b = fn[OPP[q] * N + pid];
                    if (mv == 2)
                        b += S(6) * wq<S>(q) * S(CX[q]) * u_lid;
                    f[q] = b;
                } else {
                    f[q] = fn[q * N + (long)sy * W + sx];
                }
            }
            S r, u, v, s = s_nu;
            const bool inlet = zh && x == 0;
            if (inlet) {
                S lu = ramp ? ramp_u(u_in, y, H) : u_in;
                r = zou_he(f, lu);
                u = lu;
                v = 0;
            } else {
                moments(f, r, u, v);
                if (clamps) {
                    u = clampv(u, S(-0.4), S(0.4));
                    v = clampv(v, S(-0.4), S(0.4));
                    r = clampv(r, S(0), S(1.5));
                }
                if (clos == 1)
                    s = smag_rate(f, r, u, v, tau0, cs);
                else if (clos == 2 || clos == 3)
                    s = mlp_rate(f, r, u, v, tau0, clos == 3);
            }
            ux[pid] = u;
            uy[pid] = v;
            rho[pid] = r;
            if (coll == 1)
                mrt_relax(f, r, u, v, s_e, s_eps, s_q, s);
            else
                bgk(f, r, u, v, s);
            for (int q = 0; q < 9; ++q) {
                S o = clamps ? clampv(f[q], S(0), S(10)) : f[q];
                fo[q * N + pid] = o;
                if (outflow && x == W - 2)
                    fo[q * N + pid + 1] = o;
            }
        }
    }
}

} // namespace

extern "C" {

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_mlp(const float *params, const float *in_scale, double out_scale)
{
    for (int i = 0; i < 32 * 5 + 32 + 32 * 32 + 32 + 32 + 1; ++i)
        g_mlp.p[i] = params[i];
    for (int k = 0; k < 5; ++k)
        g_mlp.in_scale[k] = in_scale[k];
    g_mlp.out_scale = out_scale;
    g_mlp.set = true;
}

void orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0)
        omp_set_num_threads(n);
#else
    (void)n;
#endif
}

void orc_core4_step_f32(const uint8_t *mask, const float *fn, float *fo, float *ux, float *uy, float *rho, int W, int H,
                        float tau_inv, float u_in, float cs, float si)
{
    core4_step<float>(mask, fn, fo, ux, uy, rho, W, H, tau_inv, u_in, cs, si);
}

void orc_core4_step_f64(const uint8_t *mask, const double *fn, double *fo, double *ux, double *uy, double *rho, int W,
                        int H, double tau_inv, double u_in, double cs, double si)
{
    core4_step<double>(mask, fn, fo, ux, uy, rho, W, H, tau_inv, u_in, cs, si);
}

void orc_smemaa_launch_f32(const uint8_t *mask, const float *fn, float *fo, float *ux, float *uy, float *rho, int W,
                           int H, float tau_inv, float u_in, int T)
{
    smemaa_launch<float>(mask, fn, fo, ux, uy, rho, W, H, tau_inv, u_in, T);
}

void orc_smemaa_launch_f64(const uint8_t *mask, const double *fn, double *fo, double *ux, double *uy, double *rho,
                           int W, int H, double tau_inv, double u_in, int T)
{
    smemaa_launch<double>(mask, fn, fo, ux, uy, rho, W, H, tau_inv, u_in, T);
}

void orc_policy_launch_f32(const uint8_t *mask, const float *fn, float *fo, int W, int H, float tau_inv, float u_in,
                           int T)
{
    policy_launch<float>(mask, fn, fo, W, H, tau_inv, u_in, T);
}

void orc_policy_launch_f64(const uint8_t *mask, const double *fn, double *fo, int W, int H, double tau_inv,
                           double u_in, int T)
{
    policy_launch<double>(mask, fn, fo, W, H, tau_inv, u_in, T);
}

void orc_macro_f32(const float *f, float *ux, float *uy, float *rho, const uint8_t *mask, int W, int H, float u_in)
{
    macro<float>(f, ux, uy, rho, mask, W, H, u_in);
}

void orc_general_step_f32(const int *ip, const double *dp, const uint8_t *mask, const float *fn, float *fo, float *ux,
                          float *uy, float *rho)
{
    general_step<float>(ip, dp, mask, fn, fo, ux, uy, rho);
}

void orc_general_step_f64(const int *ip, const double *dp, const uint8_t *mask, const double *fn, double *fo,
                          double *ux, double *uy, double *rho)
{
    general_step<double>(ip, dp, mask, fn, fo, ux, uy, rho);
}

void orc_visualize(const float *ux, const float *uy, uint8_t *img, const uint8_t *mask, int W, int H,
                   float vort_scale)
{
    visualize(ux, uy, img, mask, W, H, vort_scale);
}

} // extern "C"
