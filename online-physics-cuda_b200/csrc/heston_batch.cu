// Batched Heston ADI: many European options, each on its own (uneven) grid, priced in one persistent launch.
//
// The PDE and its discretisation are the law's (tests/laws/heston_douglas.law and heston_hv.law; the reference's
// bench/laws/heston_adi.law): x = ln S along x on [ln K - 3, ln K + 3] (h = 6 / nx), the variance along y (var_j =
// sigma (j + 1/2) h), put payoff, time to maturity in `steps` steps. F = A0 + A1 + A2 with A0 = rho var V_xy
// (gx(gy(V)), explicit), A1 the x operator and A2 the y operator (three-point, flux form in y with exact face
// variances, forward drift on the first row), each carrying half of -r V. Schemes, in increments:
//   Douglas (th = 1/2):  (I - th dt A1) D1 = dt F(U);  (I - th dt A2) D2 = D1;  U' = U + D2
//   HV (th = 1/2 + sqrt3/6): the above, then (I - th dt A1) E1 = dt F(U) - D2 + dt/2 F(D2); (I - th dt A2) E2 = E1;
//                            U' = U + D2 + E2
// Per cell the coefficients and F are the law's fp32 arithmetic (the cross-derivative's divisions by h and by the
// span are multiplications by the reciprocal here).
//
// Schedule (B200): the state of an option never leaves the chip between its first and its last step. A persistent
// grid of 8-CTA clusters (one CTA an SM, 512 threads, ~210 KB of shared memory each) takes tasks from a work counter,
// largest first. An option of up to 16K cells lives in one CTA's shared memory; a larger one is split by rows over C =
// 2, 4 or 8 CTAs of the cluster (512 x 256: 32 rows each), so a task is 8 / C options of the same C. A time step is
//   X: a warp segment of nx / MX lanes per row forms dt F for its MX cells from a sliding 3 x 3 window (the rows above
//      and below a CTA's block are read from the neighbour CTA's shared memory over DSMEM) and solves the x line by
//      the partition method (tridiag.cuh: in-lane sweeps, PCR across the segment's lanes);
//   Y: a thread per (column, row block) sweeps its block in place (the partition method again, its multipliers shared
//      by all columns because the y coefficients depend on the row only), the blocks' two boundary equations of every
//      column go to a small exchange array, and after a cluster barrier each thread solves its column's reduced system
//      (2 unknowns a block, blocks of all the option's CTAs read over DSMEM) by two precomputed rows of its inverse,
//      then back-substitutes its rows and updates U.
// Douglas takes 2 cluster barriers a step, HV 4. HBM traffic is the payoff load and the final store: 8 bytes a cell
// for the whole run. Each option's arithmetic is fixed by its own shape and the split (MX, row blocks), not by which
// cluster or CTA runs it, so its result does not depend on the schedule.
#include "../../include/fe.h"

#include "api_common.hpp"
#include "cuda_ctx.hpp"
#include "fe_device.cuh"
#include "tridiag.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace cg = cooperative_groups;

namespace fe {
namespace {

constexpr int kMaxThreads = 512;
constexpr int kCluster = 8;
constexpr int kCapCells = 16384;   // cells a CTA holds
constexpr int kMaxRows = 128;      // rows a CTA holds
constexpr int kMaxBlocks = 16;     // row blocks of one column over all the option's CTAs (2 unknowns each)
constexpr int kMaxNy = 256;
constexpr int kMaxNx = 512;
constexpr int kXch = kMaxThreads > kMaxNx ? kMaxThreads : kMaxNx;   // columns x row blocks of one CTA's y solves
constexpr int kXTab = 768;         // float4s of x-sweep tables a CTA holds: (MX + 2) a row

// Cells a lane holds in the x solves for an option of nx columns and R rows a CTA, at most `cap`: the largest of 16, 8,
// 4 whose row tables fit and whose lines take at most 32 lanes (0: none).
__host__ __device__ constexpr int lane_cells(int nx, int R, int cap)
{
    for (int m = 16; m >= 4; m /= 2) {
        if (m <= cap && R * (m + 2) <= kXTab && nx / m <= 32) return m;
    }
    return 0;
}
// Shared arrays are stored with one pad float after every 32, so lanes reading a row with a stride of MX cells, or
// rows of one column, hit distinct banks.
constexpr int kArr = kCapCells + kCapCells / 32;

__host__ __device__ constexpr int padded(int i) { return i + (i >> 5); }

struct OptionDev {
    int nx, ny;
    int C;          // CTAs the option is split over (by rows)
    int pad;
    float h, dt, th;
    float kappa, theta, sigma, rho, r;
    float x0;       // ln K - 3 + h/2: the centre of cell 0
    long long at;   // offset of the option's grid in the batch buffer
};

// A cluster's unit of work: 8 / C options that are each split over C CTAs (-1: that group of CTAs idles).
struct TaskDev {
    int C;
    int opt[kCluster];
};

struct ClusterArgs {
    const OptionDev* opts;
    const TaskDev* tasks;
    int ntasks;
    int steps;
    int sy;             // most row blocks a CTA splits a column into for the y solves
    int mx;             // most cells a lane holds in the x solves
    float* V;
    unsigned* next;     // work counter
};

// One row's coefficients, in the law's fp32 order (heston_douglas.law's lets).
struct RowCoef {
    float wxm, wxp, wym, wyp, rv;        // explicit operator: x/y neighbour weights, rho var
    float ax, bx, cx, ay, by, cy;        // implicit halves: (I - th dt A) rows
};

__device__ __forceinline__ RowCoef row_coef(const OptionDev& o, int j)
{
    RowCoef c;
    const float h = o.h;
    const float var = static_cast<float>(static_cast<double>(o.sigma) * (j + 0.5) * static_cast<double>(h));
    const float first = (o.sigma * h - var) > 0.f ? 1.f : 0.f;
    const float drift = o.kappa * (o.theta - var) / o.sigma - 0.5f * o.sigma;
    const float hh = h * h;
    const float h2 = 2.f * h;
    c.wxm = 0.5f * var / hh - (o.r - 0.5f * var) / h2;
    c.wxp = 0.5f * var / hh + (o.r - 0.5f * var) / h2;
    c.wym = 0.5f * (var - 0.5f * o.sigma * h) / hh - (1.f - first) * drift / h2;
    c.wyp = 0.5f * (var + 0.5f * o.sigma * h) / hh + (1.f + first) * drift / h2;
    const float cxd = 0.f - c.wxm - c.wxp - 0.5f * o.r;
    const float cyd = 0.f - c.wym - c.wyp - 0.5f * o.r;
    c.rv = o.rho * var;
    const float tdt = o.th * o.dt;
    c.ax = 0.f - tdt * c.wxm;
    c.bx = 1.f - tdt * cxd;
    c.cx = 0.f - tdt * c.wxp;
    c.ay = 0.f - tdt * c.wym;
    c.by = 1.f - tdt * cyd;
    c.cy = 0.f - tdt * c.wyp;
    return c;
}

// The y line's row j with the edge repeat folded in (b + a in row 0, b + c in row ny-1).
__device__ __forceinline__ void y_row(const OptionDev& o, int j, float& a, float& b, float& c)
{
    const RowCoef rc = row_coef(o, j);
    a = j == 0 ? 0.f : rc.ay;
    b = rc.by;
    if (j == 0) b = b + rc.ay;
    if (j == o.ny - 1) b = b + rc.cy;
    c = j == o.ny - 1 ? 0.f : rc.cy;
}

// The X phase's per-row data: F's weights, the x line's coefficients, 1 / (h * the y span of the cross derivative).
struct RowX {
    float wxm, wxp, wym, wyp, rv, ax, bx, cx, ihy;
};

// The Y phase's per-row data within the row's block: the down-sweep multiplier f, the up-sweep multiplier g, the
// row's coupling a, 1 / B and C of the up-swept row (x r-1, x r, x last).
struct RowY {
    float a, f, g, ib, C;
};

struct Smem {
    float U[kArr];
    float D[kArr];
    float E[kArr];
    RowX rx[kMaxRows];
    RowY ry[kMaxRows];
    float4 xt[kXTab];                          // x-sweep tables: per row {f, g, C, 1/B} for each of MX rows, then
                                               // {al, be, be at the last lane, B0}, {B0 at the first lane, -, -, -}
    float xch[2 * kXch];                       // [block][first, last][column]
    float red[kMaxBlocks][6];                  // this CTA's blocks' reduced equations: a0 B0 C0 | a1 B1 C1
    float minv[kMaxBlocks][2][2 * kMaxBlocks]; // rows (first, last) of the reduced inverse for this CTA's blocks
    float sysA[2 * kMaxBlocks], sysB[2 * kMaxBlocks], sysC[2 * kMaxBlocks];
    int task;
};

static_assert(sizeof(Smem) <= 232448, "the batch kernel's shared memory must fit one CTA of an SM (227 KB)");

struct Geometry {
    int nx, ny, C, c, g, R, r0, S, Rb, P, stride, mx;
};

// The x line's right-hand side for MX consecutive cells i0 .. i0 + MX - 1 of a row, from sliding 3 x 3 windows over
// the rows above (u*), at (c*) and below (d*): TWO = false: dt F(U); TWO = true: dt F(U) - D + dt/2 F(D).
template <int MX, bool TWO>
__device__ __forceinline__ void rhs_row(const float* uu, const float* cu, const float* du, const float* ud, const float* cd,
    const float* dd, int i0, int nx, const RowX& w, float ihx_in, float ihx_edge, float r, float dt, float (&out)[MX])
{
    auto F = [&](float uL, float uC, float uR, float cL, float cC, float cR, float dL, float dC, float dR, float ihx) {
        const float gy_p = (dR - uR) * w.ihy;
        const float gy_m = (dL - uL) * w.ihy;
        const float gxy = (gy_p - gy_m) * ihx;
        float f = w.rv * gxy;
        f = f + w.wxm * (cL - cC);
        f = f + w.wxp * (cR - cC);
        f = f + w.wym * (uC - cC);
        f = f + w.wyp * (dC - cC);
        return f - r * cC;
    };
    const int il = max(i0 - 1, 0);
    float uL = uu[padded(il)], cL = cu[padded(il)], dL = du[padded(il)];
    float uC = uu[padded(i0)], cC = cu[padded(i0)], dC = du[padded(i0)];
    float vL = 0.f, eL = 0.f, fL = 0.f, vC = 0.f, eC = 0.f, fC = 0.f;
    if (TWO) {
        vL = ud[padded(il)], eL = cd[padded(il)], fL = dd[padded(il)];
        vC = ud[padded(i0)], eC = cd[padded(i0)], fC = dd[padded(i0)];
    }
#pragma unroll
    for (int m = 0; m < MX; ++m) {
        const int i = i0 + m;
        const int ip = min(i + 1, nx - 1);
        const float ihx = (i == 0 || i == nx - 1) ? ihx_edge : ihx_in;
        const float uR = uu[padded(ip)], cR = cu[padded(ip)], dR = du[padded(ip)];
        float v = dt * F(uL, uC, uR, cL, cC, cR, dL, dC, dR, ihx);
        uL = uC; cL = cC; dL = dC;
        uC = uR; cC = cR; dC = dR;
        if (TWO) {
            const float vR = ud[padded(ip)], eR = cd[padded(ip)], fR = dd[padded(ip)];
            v = (v - eC) + (0.5f * dt) * F(vL, vC, vR, eL, eC, eR, fL, fC, fR, ihx);
            vL = vC; eL = eC; fL = fC;
            vC = vR; eC = eR; fC = fR;
        }
        out[m] = v;
    }
}

// The address of global row j of array `base` (U, D or E) of this option: this CTA's or a neighbour's over DSMEM.
__device__ __forceinline__ const float* row_ptr(cg::cluster_group& cl, float* base, const Geometry& G, int j)
{
    const int owner = j / G.R;
    const int local = j - owner * G.R;
    float* p = base + local * G.stride;
    if (owner == G.c) return p;
    return cl.map_shared_rank(p, static_cast<unsigned>(G.g * G.C + owner));
}

// Per task, one thread a row: the in-lane sweeps of an interior lane of the row's x lines (M rows of (a, b, c), no
// edge repeat), which every step reuses: down-sweep multipliers f, up-sweep multipliers g, C and 1 / B of the up-swept
// rows, and the reduced equations' coefficients (the first lane's row 0 and the last lane's row M-1 carry the fold).
template <int M>
__device__ __forceinline__ void x_table(float4* tb, float a, float b, float c)
{
    float al = a, be = b;
    tb[0].x = 0.f;
    tb[1].x = 0.f;
    for (int r = 2; r < M; ++r) {
        const float f = a / be;
        tb[r].x = f;
        al = -f * al;
        be = b - f * c;
    }
    float Bn = b, Cn = c;
    tb[M - 1].y = 0.f;
    tb[M - 1].z = 0.f;
    tb[M - 1].w = 0.f;
    tb[M - 2].y = 0.f;
    tb[M - 2].z = Cn;
    tb[M - 2].w = 1.f / Bn;
    for (int r = M - 3; r >= 0; --r) {
        const float g = c / Bn;
        Bn = b - g * a;
        Cn = -g * Cn;
        tb[r].y = g;
        tb[r].z = Cn;
        tb[r].w = 1.f / Bn;
    }
    tb[M] = make_float4(al, be, be + c, Bn);
    tb[M + 1] = make_float4(Bn + a, 0.f, 0.f, 0.f);
}

// One x line of a row by the segment's K lanes with the row's sweep table: the in-lane sweeps are two FMAs a cell, the
// lanes' reduced system is solved by PCR (tridiag.cuh), then each lane back-substitutes its cells.
template <int M>
__device__ __forceinline__ void solve_row(const float4* tb, float a, float c, float (&d)[M], int k, int K)
{
    const bool lo = k == 0, hi = k == K - 1;
    float de = d[1];
#pragma unroll
    for (int r = 2; r < M; ++r) de = d[r] - tb[r].x * de;
#pragma unroll
    for (int r = M - 3; r >= 0; --r) d[r] = d[r] - tb[r].y * d[r + 1];
    const float4 sp = tb[M];
    const float b0 = lo ? tb[M + 1].x : sp.w;
    float first, last;
    fe_pcr_pairs(lo ? 0.f : a, b0, tb[0].z, d[0], sp.x, hi ? sp.z : sp.y, hi ? 0.f : c, de, k, K, first, last);
    float prev = first;
    d[0] = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        const float4 t = tb[r];
        prev = (d[r] - a * prev - t.z * last) * t.w;
        d[r] = prev;
    }
    d[M - 1] = last;
}

// X phase: for each of this CTA's rows, the right-hand side (kind 0: dt F(U); kind 1: dt F(U) - D + dt/2 F(D)) and the
// x line's solve, written to `out`.
template <int MX>
__device__ __forceinline__ void x_phase(cg::cluster_group& cl, Smem& sm, const OptionDev& o, const Geometry& G, int kind,
    float* out)
{
    const int nx = G.nx;
    const int K = nx > MX ? nx / MX : 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = lane / K, k = lane % K;
    const int per_warp = 32 / K;
    const float ihx_in = 1.f / (o.h * 2.f), ihx_edge = 1.f / o.h;
    for (int base = warp * per_warp; base < G.R; base += static_cast<int>(blockDim.x / 32) * per_warp) {
        const int rl = min(base + seg, G.R - 1);
        const int j = G.r0 + rl;
        const RowX w = sm.rx[rl];
        const int jm = max(j - 1, 0), jp = min(j + 1, G.ny - 1);
        float d[MX];
        if (kind == 0) {
            rhs_row<MX, false>(row_ptr(cl, sm.U, G, jm), sm.U + rl * G.stride, row_ptr(cl, sm.U, G, jp), nullptr, nullptr,
                nullptr, k * MX, nx, w, ihx_in, ihx_edge, o.r, o.dt, d);
        } else {
            rhs_row<MX, true>(row_ptr(cl, sm.U, G, jm), sm.U + rl * G.stride, row_ptr(cl, sm.U, G, jp), row_ptr(cl, sm.D, G, jm),
                sm.D + rl * G.stride, row_ptr(cl, sm.D, G, jp), k * MX, nx, w, ihx_in, ihx_edge, o.r, o.dt, d);
        }
        if (K == 1) fe_thomas_row<MX>(w.ax, w.bx, w.cx, d, nx);
        else solve_row<MX>(sm.xt + rl * (MX + 2), w.ax, w.cx, d, k, K);
        if (base + seg < G.R) {
            float* orow = out + rl * G.stride;
#pragma unroll
            for (int m = 0; m < MX; ++m) {
                if (K > 1 || m < nx) orow[padded(k * MX + m)] = d[m];
            }
        }
    }
}

// Y phase, first half: each (column, block) thread sweeps its block of W in place and leaves its two boundary
// equations' right-hand sides in xch.
__device__ __forceinline__ void y_sweep(Smem& sm, const Geometry& G, float* W)
{
    for (int t = threadIdx.x; t < G.S * G.nx; t += blockDim.x) {
        const int i = t % G.nx, s = t / G.nx;
        const int b0 = s * G.Rb;
        float* col = W + padded(i);
        const int st = G.stride;
        float de = col[(b0 + 1) * st];
        for (int r = 2; r < G.Rb; ++r) de = col[(b0 + r) * st] - sm.ry[b0 + r].f * de;
        float Dn = col[(b0 + G.Rb - 2) * st];
        for (int r = G.Rb - 3; r >= 0; --r) {
            Dn = col[(b0 + r) * st] - sm.ry[b0 + r].g * Dn;
            col[(b0 + r) * st] = Dn;
        }
        sm.xch[(2 * s) * G.nx + i] = Dn;
        sm.xch[(2 * s + 1) * G.nx + i] = de;
    }
}

// Y phase, second half: the column's reduced system by this block's two rows of its inverse, then the block's rows.
// mode 0: W = x; mode 1: U += x; mode 2: U += D + x.
__device__ __forceinline__ void y_solve(cg::cluster_group& cl, Smem& sm, const Geometry& G, float* W, int mode)
{
    for (int t = threadIdx.x; t < G.S * G.nx; t += blockDim.x) {
        const int i = t % G.nx, s = t / G.nx;
        const float* mf = sm.minv[s][0];
        const float* ml = sm.minv[s][1];
        float xf = 0.f, xl = 0.f;
        for (int cc = 0; cc < G.C; ++cc) {
            const float* x = sm.xch;
            if (cc != G.c) x = cl.map_shared_rank(sm.xch, static_cast<unsigned>(G.g * G.C + cc));
            for (int sb = 0; sb < G.S; ++sb) {
                const int q = 2 * (cc * G.S + sb);
                const float v0 = x[(2 * sb) * G.nx + i], v1 = x[(2 * sb + 1) * G.nx + i];
                xf = xf + mf[q] * v0;
                xf = xf + mf[q + 1] * v1;
                xl = xl + ml[q] * v0;
                xl = xl + ml[q + 1] * v1;
            }
        }
        const int b0 = s * G.Rb;
        const int st = G.stride;
        float* col = W + padded(i);
        float* ucol = sm.U + padded(i);
        const float* dcol = sm.D + padded(i);
        auto put = [&](int r, float x) {
            if (mode == 0) col[r * st] = x;
            else if (mode == 1) ucol[r * st] = ucol[r * st] + x;
            else ucol[r * st] = ucol[r * st] + (dcol[r * st] + x);
        };
        float prev = xf;
        for (int r = 1; r < G.Rb - 1; ++r) {
            const RowY y = sm.ry[b0 + r];
            const float x = (col[(b0 + r) * st] - y.a * prev - y.C * xl) * y.ib;
            put(b0 + r - 1, prev);
            prev = x;
        }
        put(b0 + G.Rb - 2, prev);
        put(b0 + G.Rb - 1, xl);
    }
}

// Per task: the y sweeps' multipliers for this CTA's blocks and their reduced equations (one thread a block).
__device__ __forceinline__ void y_setup(Smem& sm, const OptionDev& o, const Geometry& G)
{
    const int s = threadIdx.x;
    if (s >= G.S) return;
    const int b0 = s * G.Rb, jb = G.r0 + b0, Rb = G.Rb;
    float a, b, c;
    // Down: rows 1 .. Rb-1 in terms of (x first, x r, x r+1).
    y_row(o, jb + 1, a, b, c);
    float al = a, be = b, cprev = c;
    sm.ry[b0].f = 0.f;
    sm.ry[b0 + 1].f = 0.f;
    for (int r = 2; r < Rb; ++r) {
        y_row(o, jb + r, a, b, c);
        const float f = a / be;
        sm.ry[b0 + r].f = f;
        al = -f * al;
        be = b - f * cprev;
        cprev = c;
    }
    const float c_last = cprev;
    // Up: rows Rb-2 .. 0 in terms of (x r-1, x r, x last).
    float an, bn, cn;
    y_row(o, jb + Rb - 2, an, bn, cn);
    float Bn = bn, Cn = cn;
    sm.ry[b0 + Rb - 2].g = 0.f;
    sm.ry[b0 + Rb - 1].g = 0.f;
    sm.ry[b0 + Rb - 2].ib = 1.f / Bn;
    sm.ry[b0 + Rb - 2].C = Cn;
    sm.ry[b0 + Rb - 2].a = an;
    float a_up = an;
    for (int r = Rb - 3; r >= 0; --r) {
        y_row(o, jb + r, a, b, c);
        const float g = c / Bn;
        Bn = b - g * a_up;
        Cn = -g * Cn;
        sm.ry[b0 + r].g = g;
        sm.ry[b0 + r].ib = 1.f / Bn;
        sm.ry[b0 + r].C = Cn;
        sm.ry[b0 + r].a = a;
        a_up = a;
    }
    float* e = sm.red[s];
    e[0] = a_up;   // row 0's coupling to the block above
    e[1] = Bn;
    e[2] = Cn;
    e[3] = al;
    e[4] = be;
    e[5] = c_last;
}

// Per task, after every CTA's y_setup: the option's reduced system (2 P unknowns) and, for this CTA's blocks, the two
// rows of its inverse (solutions of the transposed system with unit right-hand sides).
__device__ __forceinline__ void reduced_setup(cg::cluster_group& cl, Smem& sm, const Geometry& G)
{
    const int n = 2 * G.P;
    const int t = threadIdx.x;
    if (t < G.P) {
        const int cc = t / G.S, sb = t % G.S;
        const float* e = sm.red[sb];
        if (cc != G.c) e = cl.map_shared_rank(sm.red[sb], static_cast<unsigned>(G.g * G.C + cc));
        sm.sysA[2 * t] = e[0];
        sm.sysB[2 * t] = e[1];
        sm.sysC[2 * t] = e[2];
        sm.sysA[2 * t + 1] = e[3];
        sm.sysB[2 * t + 1] = e[4];
        sm.sysC[2 * t + 1] = e[5];
    }
    __syncthreads();
    if (t < 2 * G.S) {
        const int s = t / 2, which = t % 2;
        const int m = 2 * (G.c * G.S + s) + which;
        // Transposed system: row q: C[q-1] y[q-1] + B[q] y[q] + A[q+1] y[q+1] = (q == m).
        float cp[2 * kMaxBlocks], dp[2 * kMaxBlocks];
        float cprev = 0.f, dprev = 0.f;
        for (int q = 0; q < n; ++q) {
            const float lo = q == 0 ? 0.f : sm.sysC[q - 1];
            const float up = q + 1 == n ? 0.f : sm.sysA[q + 1];
            const float den = sm.sysB[q] - lo * cprev;
            dprev = ((q == m ? 1.f : 0.f) - lo * dprev) / den;
            cprev = up / den;
            cp[q] = cprev;
            dp[q] = dprev;
        }
        float next = 0.f;
        for (int q = n - 1; q >= 0; --q) {
            next = dp[q] - cp[q] * next;
            sm.minv[s][which][q] = next;
        }
    }
}

template <bool HV>
__device__ __forceinline__ void x_any(cg::cluster_group& cl, Smem& sm, const OptionDev& o, const Geometry& G, int kind, float* out)
{
    if (G.mx == 16) x_phase<16>(cl, sm, o, G, kind, out);
    else if (G.mx == 8) x_phase<8>(cl, sm, o, G, kind, out);
    else x_phase<4>(cl, sm, o, G, kind, out);
}

template <bool HV, int NT>
__global__ void __launch_bounds__(NT, 1) heston_cluster(const ClusterArgs args)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& sm = *reinterpret_cast<Smem*>(smem_raw);
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) sm.task = static_cast<int>(atomicAdd(args.next, 1u));
        cl.sync();
        const int t = *cl.map_shared_rank(&sm.task, 0u);
        cl.sync();
        if (t >= args.ntasks) break;
        const TaskDev task = args.tasks[t];
        Geometry G{};
        G.C = task.C;
        G.g = static_cast<int>(rank) / G.C;
        G.c = static_cast<int>(rank) % G.C;
        const int oi = task.opt[G.g];
        const bool active = oi >= 0;
        OptionDev o{};
        if (active) {
            o = args.opts[oi];
            G.nx = o.nx;
            G.ny = o.ny;
            G.R = o.ny / G.C;
            G.r0 = G.c * G.R;
            G.stride = padded(o.nx);
            // Row blocks: a power of two (so they divide the rows), at most sy, NT / nx, R / 2 and 16 / C.
            const int s_cap = min(min(args.sy, max(1, NT / o.nx)), min(G.R / 2, kMaxBlocks / G.C));
            G.S = 1;
            while (2 * G.S <= s_cap) G.S *= 2;
            G.Rb = G.R / G.S;
            G.P = G.C * G.S;
            const float* src = args.V + o.at + static_cast<long long>(G.r0) * o.nx;
            for (int e = threadIdx.x; e < G.R * o.nx; e += NT) {
                const int r = e / o.nx, i = e - r * o.nx;
                sm.U[r * G.stride + padded(i)] = src[e];
            }
            G.mx = lane_cells(o.nx, G.R, args.mx);
            for (int r = threadIdx.x; r < G.R; r += NT) {
                const int j = G.r0 + r;
                const RowCoef c = row_coef(o, j);
                const int span = min(j + 1, o.ny - 1) - max(j - 1, 0);
                sm.rx[r] = RowX{c.wxm, c.wxp, c.wym, c.wyp, c.rv, c.ax, c.bx, c.cx, 1.f / (o.h * static_cast<float>(span))};
                float4* tb = sm.xt + r * (G.mx + 2);
                if (G.mx == 16) x_table<16>(tb, c.ax, c.bx, c.cx);
                else if (G.mx == 8) x_table<8>(tb, c.ax, c.bx, c.cx);
                else x_table<4>(tb, c.ax, c.bx, c.cx);
            }
            y_setup(sm, o, G);
        }
        cl.sync();
        if (active) reduced_setup(cl, sm, G);
        for (int step = 0; step < args.steps; ++step) {
            cl.sync();
            if (active) {
                x_any<HV>(cl, sm, o, G, 0, sm.D);
                __syncthreads();
                y_sweep(sm, G, sm.D);
            }
            cl.sync();
            if (active) y_solve(cl, sm, G, sm.D, HV ? 0 : 1);
            if (HV) {
                cl.sync();
                if (active) {
                    x_any<HV>(cl, sm, o, G, 1, sm.E);
                    __syncthreads();
                    y_sweep(sm, G, sm.E);
                }
                cl.sync();
                if (active) y_solve(cl, sm, G, sm.E, 2);
            }
        }
        cl.sync();
        if (active) {
            float* dst = args.V + o.at + static_cast<long long>(G.r0) * o.nx;
            for (int e = threadIdx.x; e < G.R * o.nx; e += NT) {
                const int r = e / o.nx, i = e - r * o.nx;
                dst[e] = sm.U[r * G.stride + padded(i)];
            }
        }
    }
}

using ClusterKernel = void (*)(const ClusterArgs);

constexpr int kMs[3] = {4, 8, 16};
constexpr int kNTs[3] = {256, 384, 512};

// The kernel for the scheme and nt threads a CTA (nullptr: not built).
ClusterKernel cluster_kernel(bool hv, int nt)
{
    static const ClusterKernel table[3][2] = {
        {heston_cluster<false, 256>, heston_cluster<true, 256>},
        {heston_cluster<false, 384>, heston_cluster<true, 384>},
        {heston_cluster<false, 512>, heston_cluster<true, 512>},
    };
    const int t = nt == 256 ? 0 : (nt == 384 ? 1 : (nt == 512 ? 2 : -1));
    return t < 0 ? nullptr : table[t][hv ? 1 : 0];
}

// The put payoff averaged over each cell: (1/h) int max(K - e^x, 0) dx over [x - h/2, x + h/2].
__global__ void heston_init(const OptionDev* opts, const float* strikes, int n, float* V)
{
    const int o = blockIdx.y;
    if (o >= n) return;
    const OptionDev op = opts[o];
    const double K = strikes[o];
    const double lk = std::log(K);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < op.nx * op.ny; c += gridDim.x * blockDim.x) {
        const int i = c % op.nx;
        const double h = op.h;
        const double x = lk - 3.0 + (i + 0.5) * h;
        const double lo = x - 0.5 * h, hi = std::fmin(x + 0.5 * h, lk);
        double v = 0.0;
        if (hi > lo) v = (K * (hi - lo) - (std::exp(hi) - std::exp(lo))) / h;
        V[op.at + c] = static_cast<float>(v);
    }
}

// Weights of the cubic through four consecutive cell centres (at -1, 0, 1, 2 from the second), at offset t from the
// second: Lagrange interpolation, extrapolating smoothly for t < 0 at the lattice's edge.
__device__ void cubic_weights(double t, double w[4])
{
    w[0] = -t * (t - 1.0) * (t - 2.0) / 6.0;
    w[1] = (t + 1.0) * (t - 1.0) * (t - 2.0) / 2.0;
    w[2] = -(t + 1.0) * t * (t - 2.0) / 2.0;
    w[3] = (t + 1.0) * t * (t - 1.0) / 6.0;
}

// The first of the four centres along an axis of n cells for a point at fractional centre index f, and the point's
// offset from the second. f below the first centre (v0 under the first variance row) extrapolates from the edge.
__device__ int cubic_start(double f, int n, double& t)
{
    const int s = max(0, min(n - 4, static_cast<int>(std::floor(f)) - 1));
    t = f - (s + 1);
    return s;
}

// Price at (ln S0, v0): bicubic through the 4 x 4 cell centres around it (local Lagrange, O(h^4) for smooth prices),
// the way the reference reads its batch (a bicubic spline at (ln 100, v0), bench/finance.py:280-286).
__global__ void heston_price(const OptionDev* opts, const float* spot, const float* v0, int n, const float* V, float* out)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const OptionDev op = opts[o];
    const float* U = V + op.at;
    const double fx = (std::log(static_cast<double>(spot[o])) - (op.x0)) / op.h;
    const double fy = static_cast<double>(v0[o]) / (static_cast<double>(op.sigma) * op.h) - 0.5;
    double tx = 0.0, ty = 0.0, wx[4], wy[4];
    const int i0 = cubic_start(fx, op.nx, tx);
    const int j0 = cubic_start(fy, op.ny, ty);
    cubic_weights(tx, wx);
    cubic_weights(ty, wy);
    double p = 0.0;
    for (int b = 0; b < 4; ++b) {
        double row = 0.0;
        for (int a = 0; a < 4; ++a) row += wx[a] * static_cast<double>(U[(j0 + b) * op.nx + i0 + a]);
        p += wy[b] * row;
    }
    out[o] = static_cast<float>(p);
}

} // namespace
} // namespace fe

struct fe_heston_batch {
    int n = 0;
    int steps = 0;
    int scheme = 0;
    int mx = 16;            // cells a lane holds along x
    int sy = 4;             // most row blocks a CTA splits a column into
    int threads = 384;      // threads a CTA
    int clusters_by_nt[3] = {0, 0, 0};   // clusters of the persistent grid for 256, 384, 512 threads a CTA
    int clusters = 0;
    int ntasks = 0;
    std::vector<fe::OptionDev> host;
    fe::OptionDev* opts = nullptr;
    fe::TaskDev* tasks = nullptr;
    float* V = nullptr;
    unsigned* next = nullptr;
    float* strikes = nullptr;
    float* spots = nullptr;
    float* v0s = nullptr;
    float* prices = nullptr;
    long long total = 0;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
};

namespace {

bool pow2_between(int v, int lo, int hi)
{
    return v >= lo && v <= hi && (v & (v - 1)) == 0;
}

int nt_index(int nt)
{
    return nt == 256 ? 0 : (nt == 384 ? 1 : (nt == 512 ? 2 : -1));
}

bool split_fits(const fe_heston_batch* b, int mx, int sy, int nt)
{
    if (fe::cluster_kernel(false, nt) == nullptr || !pow2_between(sy, 1, fe::kMaxBlocks) || !pow2_between(mx, 4, 16)) return false;
    if (b->clusters_by_nt[nt_index(nt)] <= 0) return false;
    for (const fe::OptionDev& o : b->host) {
        if (fe::lane_cells(o.nx, o.ny / o.C, mx) == 0) return false;
    }
    return true;
}

void release(fe_heston_batch* b)
{
    if (b == nullptr) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (void* p : {static_cast<void*>(b->opts), static_cast<void*>(b->tasks), static_cast<void*>(b->V), static_cast<void*>(b->next),
             static_cast<void*>(b->strikes), static_cast<void*>(b->spots), static_cast<void*>(b->v0s), static_cast<void*>(b->prices)}) {
        if (p) cudaFree(p);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

cudaLaunchConfig_t cluster_config(int clusters, int nt, cudaStream_t stream, cudaLaunchAttribute* attr)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(clusters * fe::kCluster);
    cfg.blockDim = dim3(nt);
    cfg.dynamicSmemBytes = sizeof(fe::Smem);
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = fe::kCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cfg;
}

int launch_run(fe_heston_batch* b, std::string& why, int steps_limit = 0)
{
    fe::ClusterArgs a{};
    a.opts = b->opts;
    a.tasks = b->tasks;
    a.ntasks = b->ntasks;
    a.steps = steps_limit > 0 ? std::min(b->steps, steps_limit) : b->steps;
    a.sy = b->sy;
    a.V = b->V;
    a.next = b->next;
    a.mx = b->mx;
    const fe::ClusterKernel kernel = fe::cluster_kernel(b->scheme == FE_ADI_HV, b->threads);
    if (kernel == nullptr) {
        why = "no kernel for that split";
        return FE_EINVAL;
    }
    if (!fe::cuda_ok(cudaMemsetAsync(b->next, 0, sizeof(unsigned), b->stream), "reset queue", why)) return FE_ECUDA;
    fe::heston_init<<<dim3(64, b->n), 256, 0, b->stream>>>(b->opts, b->strikes, b->n, b->V);
    cudaLaunchAttribute attr[1];
    const cudaLaunchConfig_t cfg = cluster_config(b->clusters, b->threads, b->stream, attr);
    if (!fe::cuda_ok(cudaLaunchKernelEx(&cfg, kernel, a), "heston cluster launch", why)) return FE_ECUDA;
    fe::heston_price<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->opts, b->spots, b->v0s, b->n, b->V, b->prices);
    if (!fe::cuda_ok(cudaGetLastError(), "heston launch", why)) return FE_ECUDA;
    return FE_OK;
}

// CTAs an option is split over: its cells at 16K a CTA, and at most 128 rows a CTA.
int ctas_for(int nx, int ny)
{
    int C = 1;
    while (static_cast<long long>(nx) * ny > static_cast<long long>(C) * fe::kCapCells || ny / C > fe::kMaxRows) C *= 2;
    return C;
}

} // namespace

extern "C" {

int fe_heston_batch_create(const fe_heston_option* options, int n, int steps, int scheme, fe_heston_batch** out)
{
    using namespace fe;
    if (options == nullptr || out == nullptr || n <= 0 || n > 65535 || steps <= 0 || (scheme != FE_ADI_DOUGLAS && scheme != FE_ADI_HV)) {
        return fail(FE_EINVAL, "fe_heston_batch_create: bad arguments");
    }
    *out = nullptr;
    for (int i = 0; i < n; ++i) {
        const fe_heston_option& s = options[i];
        if (!pow2_between(s.nx, 4, kMaxNx) || !pow2_between(s.ny, 4, kMaxNy) || !(s.strike > 0) || !(s.maturity > 0) || !(s.sigma > 0) ||
            !(s.spot > 0) || !(s.v0 >= 0)) {
            return fail(FE_EINVAL, "option " + std::to_string(i) + ": nx a power of two in [4, 512], ny in [4, 256], positive strike, "
                "maturity, sigma and spot, v0 >= 0");
        }
    }
    std::string why;
    if (!device_ready(why)) return fail(FE_ENODEV, why);
    auto* b = new fe_heston_batch();
    b->n = n;
    b->steps = steps;
    b->scheme = scheme;
    long long at = 0;
    std::vector<float> strikes(n), spots(n), v0s(n);
    for (int i = 0; i < n; ++i) {
        const fe_heston_option& s = options[i];
        OptionDev o{};
        o.nx = s.nx;
        o.ny = s.ny;
        o.C = ctas_for(s.nx, s.ny);
        o.h = static_cast<float>(6.0 / s.nx);
        o.dt = static_cast<float>(static_cast<double>(s.maturity) / steps);
        o.th = scheme == FE_ADI_DOUGLAS ? 0.5f : static_cast<float>(0.5 + std::sqrt(3.0) / 6.0);
        o.kappa = s.kappa;
        o.theta = s.theta;
        o.sigma = s.sigma;
        o.rho = s.rho;
        o.r = s.r;
        o.x0 = static_cast<float>(std::log(static_cast<double>(s.strike)) - 3.0 + 0.5 * o.h);
        o.at = at;
        at += static_cast<long long>(s.nx) * s.ny;
        b->host.push_back(o);
        strikes[i] = s.strike;
        spots[i] = s.spot;
        v0s[i] = s.v0;
    }
    b->total = at;
    // Tasks: options of the same split, 8 / C at a time, widest splits and largest options first.
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
        const OptionDev &a = b->host[p], &c = b->host[q];
        if (a.C != c.C) return a.C > c.C;
        return static_cast<long long>(a.nx) * a.ny > static_cast<long long>(c.nx) * c.ny;
    });
    std::vector<TaskDev> tasks;
    for (size_t i = 0; i < order.size();) {
        TaskDev t{};
        t.C = b->host[order[i]].C;
        const int per = kCluster / t.C;
        for (int g = 0; g < kCluster; ++g) t.opt[g] = -1;
        for (int g = 0; g < per && i < order.size() && b->host[order[i]].C == t.C; ++g, ++i) t.opt[g] = order[i];
        tasks.push_back(t);
    }
    b->ntasks = static_cast<int>(tasks.size());
    bool ok = true;
    for (int t = 0; t < 3 && ok; ++t) {
        for (const bool hv : {false, true}) {
            ok = ok && cuda_ok(cudaFuncSetAttribute(cluster_kernel(hv, kNTs[t]), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(sizeof(Smem))), "shared memory size", why);
        }
        if (!ok) break;
        cudaLaunchAttribute attr[1];
        const cudaLaunchConfig_t cfg = cluster_config(32, kNTs[t], nullptr, attr);
        int clusters = 0;
        ok = cuda_ok(cudaOccupancyMaxActiveClusters(&clusters, cluster_kernel(true, kNTs[t]), &cfg), "cluster occupancy", why);
        b->clusters_by_nt[t] = clusters;
    }
    if (ok && b->clusters_by_nt[nt_index(b->threads)] <= 0) {
        ok = false;
        why = "no 8-CTA cluster of the batch kernel fits the device";
    }
    b->clusters = ok ? b->clusters_by_nt[nt_index(b->threads)] : 0;
    ok = ok && cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream", why) &&
        cuda_ok(cudaMalloc(&b->opts, sizeof(OptionDev) * n), "opts", why) &&
        cuda_ok(cudaMalloc(&b->tasks, sizeof(TaskDev) * tasks.size()), "tasks", why) &&
        cuda_ok(cudaMalloc(&b->V, sizeof(float) * static_cast<size_t>(at)), "grids", why) &&
        cuda_ok(cudaMalloc(&b->next, sizeof(unsigned)), "queue", why) && cuda_ok(cudaMalloc(&b->strikes, sizeof(float) * n), "strikes", why) &&
        cuda_ok(cudaMalloc(&b->spots, sizeof(float) * n), "spots", why) && cuda_ok(cudaMalloc(&b->v0s, sizeof(float) * n), "v0", why) &&
        cuda_ok(cudaMalloc(&b->prices, sizeof(float) * n), "prices", why);
    ok = ok && cuda_ok(cudaMemcpy(b->opts, b->host.data(), sizeof(OptionDev) * n, cudaMemcpyHostToDevice), "opts", why) &&
        cuda_ok(cudaMemcpy(b->tasks, tasks.data(), sizeof(TaskDev) * tasks.size(), cudaMemcpyHostToDevice), "tasks", why) &&
        cuda_ok(cudaMemcpy(b->strikes, strikes.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "strikes", why) &&
        cuda_ok(cudaMemcpy(b->spots, spots.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "spots", why) &&
        cuda_ok(cudaMemcpy(b->v0s, v0s.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "v0", why);
    if (!ok) {
        release(b);
        return fail(FE_ECUDA, why);
    }
    if (!split_fits(b, b->mx, b->sy, b->threads)) b->mx = 16;
    *out = b;
    return fe::ok();
}

void fe_heston_batch_destroy(fe_heston_batch* batch)
{
    if (batch) cudaStreamSynchronize(batch->stream);
    release(batch);
}

int fe_heston_batch_set_split(fe_heston_batch* b, int mx, int sy, int threads)
{
    if (b == nullptr || !split_fits(b, mx, sy, threads)) {
        return fe::fail(FE_EINVAL, "split: mx 4, 8 or 16, enough for every option's lines to take at most 32 lanes; sy a power "
            "of two in [1, 16]; threads 256, 384 or 512");
    }
    b->mx = mx;
    b->sy = sy;
    b->threads = threads;
    b->clusters = b->clusters_by_nt[nt_index(threads)];
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    return fe::ok();
}

int fe_heston_batch_run(fe_heston_batch* b, int use_graph)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null batch");
    std::string why;
    if (!use_graph) {
        const int s = launch_run(b, why);
        return s == FE_OK ? fe::ok() : fe::fail(s, why);
    }
    if (b->graph == nullptr) {
        if (!fe::cuda_ok(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture", why)) return fe::fail(FE_ECUDA, why);
        const int s = launch_run(b, why);
        cudaGraph_t captured = nullptr;
        const cudaError_t e = cudaStreamEndCapture(b->stream, &captured);
        if (s != FE_OK || e != cudaSuccess) {
            if (captured) cudaGraphDestroy(captured);
            return fe::fail(FE_ECUDA, s != FE_OK ? why : std::string("capture: ") + cudaGetErrorString(e));
        }
        const cudaError_t ie = cudaGraphInstantiate(&b->graph, captured, 0);
        cudaGraphDestroy(captured);
        if (ie != cudaSuccess) return fe::fail(FE_ECUDA, std::string("instantiate: ") + cudaGetErrorString(ie));
    }
    if (!fe::cuda_ok(cudaGraphLaunch(b->graph, b->stream), "graph launch", why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_heston_batch_prices(fe_heston_batch* b, float* host_prices)
{
    if (b == nullptr || host_prices == nullptr) return fe::fail(FE_EINVAL, "null argument");
    std::string why;
    if (!fe::cuda_ok(cudaMemcpyAsync(host_prices, b->prices, sizeof(float) * b->n, cudaMemcpyDeviceToHost, b->stream), "prices", why) ||
        !fe::cuda_ok(cudaStreamSynchronize(b->stream), "prices", why)) {
        return fe::fail(FE_ECUDA, why);
    }
    return fe::ok();
}

int fe_heston_batch_grid(fe_heston_batch* b, int option, float* host_grid)
{
    if (b == nullptr || host_grid == nullptr || option < 0 || option >= b->n) return fe::fail(FE_EINVAL, "bad argument");
    const fe::OptionDev& o = b->host[static_cast<size_t>(option)];
    std::string why;
    if (!fe::cuda_ok(cudaMemcpyAsync(host_grid, b->V + o.at, sizeof(float) * o.nx * o.ny, cudaMemcpyDeviceToHost, b->stream), "grid", why) ||
        !fe::cuda_ok(cudaStreamSynchronize(b->stream), "grid", why)) {
        return fe::fail(FE_ECUDA, why);
    }
    return fe::ok();
}

int fe_heston_batch_time(fe_heston_batch* b, int use_graph, float* ms)
{
    if (b == nullptr || ms == nullptr) return fe::fail(FE_EINVAL, "null argument");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, b->stream);
    const int s = fe_heston_batch_run(b, use_graph);
    cudaEventRecord(e1, b->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

int fe_heston_batch_layout(const fe_heston_batch* b, int* clusters, int* tasks)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null batch");
    if (clusters) *clusters = b->clusters;
    if (tasks) *tasks = b->ntasks;
    return fe::ok();
}

int fe_heston_batch_autotune(fe_heston_batch* b, int* mx_out, int* sy_out, int* threads_out)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null batch");
    // Each candidate runs the whole batch for a few steps (the next real run sets the grids up again).
    float best = 1e30f;
    int bx = b->mx, by = b->sy, bt = b->threads;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (const int nt : fe::kNTs) {
        for (const int mx : fe::kMs) {
            for (int sy = 1; sy <= fe::kMaxBlocks; sy *= 2) {
                if (!split_fits(b, mx, sy, nt)) continue;
                b->mx = mx;
                b->sy = sy;
                b->threads = nt;
                b->clusters = b->clusters_by_nt[nt_index(nt)];
                std::string why;
                cudaEventRecord(e0, b->stream);
                const int s = launch_run(b, why, 8);
                cudaEventRecord(e1, b->stream);
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (s == FE_OK && ms < best) {
                    best = ms;
                    bx = mx;
                    by = sy;
                    bt = nt;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int s = fe_heston_batch_set_split(b, bx, by, bt);
    if (mx_out) *mx_out = bx;
    if (sy_out) *sy_out = by;
    if (threads_out) *threads_out = bt;
    return s;
}

} // extern "C"
