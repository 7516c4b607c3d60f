// The hand-written 7-point explicit heat step, d T = diffuse(k, T) with one k everywhere, on sm_100a.
//
// It is the bit-identity reference for the step the law compiler generates for the same law (the reference's own check
// of its engine against a hand-written kernel is bench/stencil_bench.cpp:46-65 and :291-294), so it does the law's
// arithmetic in the law's order (the reference's generated diffuse body, cuda/CudaCodegen.cpp:193-206, and its
// ping-pong store, :593-601):
//
//   acc = 0; acc += T(x-1) - c; acc += T(x+1) - c; acc += T(y-1) - c; acc += T(y+1) - c; acc += T(z-1) - c; acc += T(z+1) - c
//         (a face past the lattice's edge is left out: zero flux, the edge cell repeating)
//   r = (max(k, 0) * acc) / (h * h);   d = r * dt;   next = c + d          (fp32, no FMA contraction)
//
// Memory schedule (B200): a CTA owns a 128 x TY column of the lattice and marches along z through a chunk of planes.
// Each plane of its tile plus a one-cell halo (x widened to 4 cells each side, so every TMA box starts on a 16-byte
// boundary) comes into a ring of shared-memory stages by one TMA load, NST - 3 planes ahead of the plane being computed.
// A warp computes 4 consecutive cells a lane (one float4) on R rows; the x neighbours come from the next lanes by
// shuffle. T is read from HBM once and the next state written once: 8 bytes a cell.
//
// The conserved-total, range/NaN, bounds and change-flag contracts are fused into the same pass (fe_device.cuh): FP64
// partial sums per block in a fixed order, integer atomics for the order-free parts.
#include "heat7.hpp"

namespace fe {

constexpr int kHeatTX = 128; // cells along x a CTA covers: 32 lanes x 4
constexpr int kHeatPadX = 4; // halo columns each side (16 bytes, the TMA alignment)


template <int W, int R>
struct HeatTile {
    static constexpr int TY = W * R;
    static constexpr int PX = kHeatTX + 2 * kHeatPadX;  // 136 floats
    static constexpr int PY = TY + 2;
    static constexpr int PLANE = ((PX * PY + 31) / 32) * 32; // floats a stage, 128-byte multiple
    static constexpr unsigned BOX_BYTES = PX * PY * 4u;
};

template <int W, int R, int NST, bool DIV>
__global__ void __launch_bounds__(W * 32) heat7_tma(const __grid_constant__ FeTensorMap tin, const HeatArgs a)
{
    using Tile = HeatTile<W, R>;
    extern __shared__ __align__(128) float sm[];
    __shared__ __align__(8) fe_u64 bar[NST];
    __shared__ double scratch[4 * W];
    __shared__ int failed;

    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int x0 = blockIdx.x * kHeatTX;
    const int y0 = blockIdx.y * Tile::TY;
    const int zb = blockIdx.z * a.zchunk;
    const int ze = min(nz, zb + a.zchunk);
    const int zlo = max(zb - 1, 0);
    const int zhi = min(ze, nz - 1);
    const int nplanes = zhi - zlo + 1;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;

    static_assert(NST >= 4, "the ring holds z-1, z, z+1 and the plane being fetched");
    int issued = 0; // planes [0, issued) have been asked for (thread 0's count; the only thread that issues)
    if (threadIdx.x == 0) {
        failed = 0;
        fe_prefetch_tensormap(&tin);
        for (int s = 0; s < NST; ++s) {
            fe_mbar_init(&bar[s], 1);
        }
        fe_fence_mbar_init();
        issued = min(NST, nplanes);
        for (int j = 0; j < issued; ++j) {
            fe_mbar_expect_tx(&bar[j], Tile::BOX_BYTES);
            fe_tma_load_3d(sm + j * Tile::PLANE, &tin, &bar[j], x0 - kHeatPadX, y0 - 1, zlo + j);
        }
    }
    __syncthreads();

    const float kk = fmaxf(a.k, 0.f);
    const float hh = a.h * a.h;
    const bool check = a.rec != nullptr;
    FeAcc acc;
    fe_acc_init(acc);

    // Every thread waits (bounded) for the planes a z needs; one barrier a plane makes the outcome uniform and frees
    // the stage of the plane no longer needed.
    int waited = 0; // planes [0, waited) have landed
    auto wait_upto = [&](int j) {
        while (waited <= j) {
            const unsigned parity = static_cast<unsigned>((waited / NST) & 1);
            if (!fe_mbar_wait(&bar[waited % NST], parity, 1u << 20)) {
                failed = 1;
            }
            ++waited;
        }
    };
    if (zb < ze) {
        wait_upto(min(zb + 1, nz - 1) - zlo);
    }
    __syncthreads();
    const int px = kHeatPadX + 4 * lane;
    const int x = x0 + 4 * lane;
    const bool xin = x < nx;
    const bool xm_ok = x > 0;       // this lane's first cell has a -x face
    const bool xp_ok = x + 4 < nx;  // its last cell has a +x face (nx is a multiple of 4)
    const bool before = a.totals_before != 0;
    const bool after = a.totals_after != 0;
    for (int z = zb; z < ze && !failed; ++z) {
        // A face past the lattice's edge reads the cell itself, so it adds (c - c) = +0, which leaves the sum as it is:
        // the sum starts at +0 and a round-to-nearest sum of nonzero terms is never -0, so this and skipping the face
        // agree to the bit. Along z the edge plane stands in for the missing one; along y, the row itself.
        const int jm = max(z - 1, 0) - zlo;
        const int jc = z - zlo;
        const int jp = min(z + 1, nz - 1) - zlo;
        const float* pm = sm + (jm % NST) * Tile::PLANE;
        const float* pc = sm + (jc % NST) * Tile::PLANE;
        const float* pp = sm + (jp % NST) * Tile::PLANE;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int ty = warp * R + r;
            const int y = y0 + ty;
            const int row = (ty + 1) * Tile::PX;
            const float4 c = *reinterpret_cast<const float4*>(pc + row + px);
            float left = __shfl_up_sync(0xffffffffu, c.w, 1);
            float right = __shfl_down_sync(0xffffffffu, c.x, 1);
            if (lane == 0) left = pc[row + kHeatPadX - 1];
            if (lane == 31) right = pc[row + kHeatPadX + kHeatTX];
            if (!xin || y >= ny) {
                continue;
            }
            left = xm_ok ? left : c.x;
            right = xp_ok ? right : c.w;
            const int row_up = y > 0 ? row - Tile::PX : row;
            const int row_dn = y + 1 < ny ? row + Tile::PX : row;
            const float4 up = *reinterpret_cast<const float4*>(pc + row_up + px);
            const float4 dn = *reinterpret_cast<const float4*>(pc + row_dn + px);
            const float4 zm = *reinterpret_cast<const float4*>(pm + row + px);
            const float4 zp = *reinterpret_cast<const float4*>(pp + row + px);
            const float cv[4] = {c.x, c.y, c.z, c.w};
            const float xl[4] = {left, c.x, c.y, c.z};
            const float xr[4] = {c.y, c.z, c.w, right};
            const float yl[4] = {up.x, up.y, up.z, up.w};
            const float yr[4] = {dn.x, dn.y, dn.z, dn.w};
            const float zl[4] = {zm.x, zm.y, zm.z, zm.w};
            const float zr[4] = {zp.x, zp.y, zp.z, zp.w};
            float o[4];
            bool moved = false;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float cc = cv[q];
                float s = 0.f;
                s = __fadd_rn(s, __fsub_rn(xl[q], cc));
                s = __fadd_rn(s, __fsub_rn(xr[q], cc));
                s = __fadd_rn(s, __fsub_rn(yl[q], cc));
                s = __fadd_rn(s, __fsub_rn(yr[q], cc));
                s = __fadd_rn(s, __fsub_rn(zl[q], cc));
                s = __fadd_rn(s, __fsub_rn(zr[q], cc));
                const float ks = __fmul_rn(kk, s);
                // (k s) / h^2: when h^2 is a power of two its exact reciprocal multiplies instead, to the bit.
                const float rate = DIV ? __fdiv_rn(ks, hh) : __fmul_rn(ks, a.inv_hh);
                const float d = __fmul_rn(rate, a.dt);
                o[q] = d != 0.f ? __fadd_rn(cc, d) : cc;
                moved = moved || d != 0.f;
            }
            const size_t at = static_cast<size_t>(x) + static_cast<size_t>(nx) * (static_cast<size_t>(y) + static_cast<size_t>(ny) * z);
            if (check) {
                // The change flag as the reference's gather sets it: an increment that is not zero (CudaCodegen.cpp:598).
                fe_acc_row4<false>(acc, cv, o, a.lo, a.hi, static_cast<unsigned>(at), before, after);
                acc.changed |= moved ? 1u : 0u;
            }
            *reinterpret_cast<float4*>(a.out + at) = make_float4(o[0], o[1], o[2], o[3]);
        }
        fe_acc_flush(acc);
        if (z + 1 < ze) {
            wait_upto(min(z + 2, nz - 1) - zlo);
        }
        // Everyone is done with plane z - 1: its stage takes the plane NST further on.
        __syncthreads();
        const int release = z - 1 - zlo;
        if (threadIdx.x == 0 && !failed && release >= 0 && release + NST < nplanes) {
            const int j = release + NST;
            fe_fence_proxy_async();
            fe_mbar_expect_tx(&bar[j % NST], Tile::BOX_BYTES);
            fe_tma_load_3d(sm + (j % NST) * Tile::PLANE, &tin, &bar[j % NST], x0 - kHeatPadX, y0 - 1, zlo + j);
            issued = j + 1;
        }
    }
    if (failed) {
        // Let every load this block issued land (bounded) before its shared memory goes away; then report.
        if (threadIdx.x == 0) {
            atomicOr(a.err, FE_ERR_MBAR_TIMEOUT);
            for (int j = 0; j < issued; ++j) {
                fe_mbar_wait(&bar[j % NST], static_cast<unsigned>((j / NST) & 1), 1u << 16);
            }
        }
        return;
    }
    if (check) {
        const int block = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        const int blocks = gridDim.x * gridDim.y * gridDim.z;
        fe_acc_block(acc, scratch, a.partials + 4 * block, a.rec);
        fe_acc_finish(a.partials, blocks, a.count, scratch, a.rec, a.totals_before != 0, a.totals_after != 0);
    }
}

// A plain device-to-device copy: the bandwidth roof the stencil is measured against, timed in the same run. Two 16-byte
// loads in flight a thread, streamed past the caches (each byte is touched once), 4 CTAs an SM: measured on a B200 at
// 512 MiB, 6.40 TB/s against 5.81 for one load a thread at 8 CTAs an SM (cudaMemcpyAsync: 6.31).
__global__ void __launch_bounds__(256) copy_f4(const float4* __restrict__ a, float4* __restrict__ b, size_t n4)
{
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x;
    for (; i + stride < n4; i += 2 * stride) {
        const float4 v0 = __ldcs(a + i);
        const float4 v1 = __ldcs(a + i + stride);
        __stcs(b + i, v0);
        __stcs(b + i + stride, v1);
    }
    for (; i < n4; i += stride) b[i] = a[i];
}

// The same step as heat7_tma with plain loads and no shared memory, thread per (x, y) column marching z. Used for
// lattices whose x extent is not a multiple of 4 (TMA needs 16-byte row pitches), and as a second witness of the
// arithmetic.
__global__ void __launch_bounds__(256) heat7_plain(const float* __restrict__ T, const HeatArgs a)
{
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const bool live = x < nx && y < ny;
    const float kk = fmaxf(a.k, 0.f);
    const float hh = a.h * a.h;
    const bool check = a.rec != nullptr;
    FeAcc acc;
    fe_acc_init(acc);
    const size_t plane = static_cast<size_t>(nx) * ny;
    const int zb = blockIdx.z * a.zchunk;
    const int ze = min(nz, zb + a.zchunk);
    for (int z = zb; live && z < ze; ++z) {
        const size_t i = static_cast<size_t>(x) + static_cast<size_t>(nx) * y + plane * z;
        const float c = T[i];
        float s = 0.f;
        if (x > 0) s += __fsub_rn(T[i - 1], c);
        if (x + 1 < nx) s += __fsub_rn(T[i + 1], c);
        if (y > 0) s += __fsub_rn(T[i - nx], c);
        if (y + 1 < ny) s += __fsub_rn(T[i + nx], c);
        if (z > 0) s += __fsub_rn(T[i - plane], c);
        if (z + 1 < nz) s += __fsub_rn(T[i + plane], c);
        const float ks = __fmul_rn(kk, s);
        const float rate = a.inv_hh != 0.f ? __fmul_rn(ks, a.inv_hh) : __fdiv_rn(ks, hh);
        const float d = __fmul_rn(rate, a.dt);
        const float o = d != 0.f ? __fadd_rn(c, d) : c;
        a.out[i] = o;
        if (check) {
            fe_acc_cell(acc, c, o, a.lo, a.hi, static_cast<unsigned>(i), a.totals_before != 0, a.totals_after != 0);
        }
    }
    if (check) {
        __shared__ double scratch[4 * 8];
        const int block = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
        const int blocks = gridDim.x * gridDim.y * gridDim.z;
        fe_acc_block(acc, scratch, a.partials + 4 * block, a.rec);
        fe_acc_finish(a.partials, blocks, a.count, scratch, a.rec, a.totals_before != 0, a.totals_after != 0);
    }
}

// Every cell of a buffer to one value (a field's `init`).
__global__ void __launch_bounds__(256) fill_f32(float* __restrict__ p, size_t n, float v)
{
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        p[i] = v;
    }
}

cudaError_t launch_fill(float* p, size_t n, float v, int sms, cudaStream_t stream)
{
    fill_f32<<<sms * 4, 256, 0, stream>>>(p, n, v);
    return cudaGetLastError();
}

// ---- host side: launches (called from the C-ABI in api.cpp) ---------------------------------------------------------

struct HeatShape {
    int W, R, NST, zchunk;
};

template <int W, int R, int NST, bool DIV>
cudaError_t launch_heat7_tma_d(const FeTensorMap& map, const HeatArgs& a, cudaStream_t stream)
{
    using Tile = HeatTile<W, R>;
    const size_t smem = static_cast<size_t>(NST) * Tile::PLANE * sizeof(float);
    static bool configured = false;
    if (!configured) {
        const cudaError_t e = cudaFuncSetAttribute(heat7_tma<W, R, NST, DIV>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) {
            return e;
        }
        configured = true;
    }
    const dim3 grid((a.nx + kHeatTX - 1) / kHeatTX, (a.ny + Tile::TY - 1) / Tile::TY, (a.nz + a.zchunk - 1) / a.zchunk);
    heat7_tma<W, R, NST, DIV><<<grid, W * 32, smem, stream>>>(map, a);
    return cudaGetLastError();
}

template <int W, int R, int NST>
cudaError_t launch_heat7_tma_t(const FeTensorMap& map, const HeatArgs& a, cudaStream_t stream)
{
    return a.inv_hh != 0.f ? launch_heat7_tma_d<W, R, NST, false>(map, a, stream) : launch_heat7_tma_d<W, R, NST, true>(map, a, stream);
}

// Tile rows (W warps x R rows) and ring depth: the shapes the autotuner may pick from.
cudaError_t launch_heat7_tma(int variant, const FeTensorMap& map, const HeatArgs& a, cudaStream_t stream)
{
    switch (variant) {
    case 0: return launch_heat7_tma_t<8, 2, 6>(map, a, stream);   // 128 x 16 tile
    case 1: return launch_heat7_tma_t<8, 4, 5>(map, a, stream);   // 128 x 32 tile
    case 2: return launch_heat7_tma_t<4, 4, 6>(map, a, stream);   // 128 x 16 tile, 128 threads
    case 3: return launch_heat7_tma_t<8, 1, 8>(map, a, stream);   // 128 x 8 tile, deep ring
    default: return cudaErrorInvalidValue;
    }
}

int heat7_tma_rows(int variant)
{
    switch (variant) {
    case 0: return 16;
    case 1: return 32;
    case 2: return 16;
    case 3: return 8;
    default: return 0;
    }
}

int heat7_tma_blocks(int variant, int nx, int ny, int nz, int zchunk)
{
    const int ty = heat7_tma_rows(variant);
    if (ty == 0) {
        return 0;
    }
    return ((nx + kHeatTX - 1) / kHeatTX) * ((ny + ty - 1) / ty) * ((nz + zchunk - 1) / zchunk);
}

cudaError_t launch_heat7_plain(const float* T, const HeatArgs& a, cudaStream_t stream)
{
    const dim3 grid((a.nx + 31) / 32, (a.ny + 7) / 8, (a.nz + a.zchunk - 1) / a.zchunk);
    heat7_plain<<<grid, 256, 0, stream>>>(T, a);
    return cudaGetLastError();
}

int heat7_plain_blocks(int nx, int ny, int nz, int zchunk)
{
    return ((nx + 31) / 32) * ((ny + 7) / 8) * ((nz + zchunk - 1) / zchunk);
}

cudaError_t launch_copy(const float* a, float* b, size_t n, int sms, cudaStream_t stream)
{
    const size_t n4 = n / 4;
    copy_f4<<<sms * 4, 256, 0, stream>>>(reinterpret_cast<const float4*>(a), reinterpret_cast<float4*>(b), n4);
    return cudaGetLastError();
}

} // namespace fe
