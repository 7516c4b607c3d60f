// The totals of one field (sum and sum of |v|, FP64) into a contract record's before slots, for a term whose
// conservation contract needs them when no earlier pass left them (the first step, a step after the host edited the
// field, a step after an unchecked one). The reference takes these totals with separate row and plane passes before
// every term (cuda/CudaCodegen.cpp:196-219, cuda/CudaSolver.cpp:501-508); here the generated passes carry them from
// one step to the next and this kernel only starts the chain.
//
// Deterministic: a fixed grid, each block a fixed contiguous slice, FP64 sums in a fixed tree, the blocks folded in
// block order by whichever block finishes last.
#include "heat7.hpp"

namespace fe {

__global__ void __launch_bounds__(256) totals_f32(const float* __restrict__ v, size_t n, FeCheck* rec, double* partials, unsigned* count)
{
    __shared__ double scratch[4 * 8];
    // `v` may start inside a 16-byte word (a slab's owned planes start at plane * z0 cells): the cells up to the first
    // 16-byte boundary are block 0's head, the rest is read as float4s from an aligned pointer.
    const size_t head = min(n, static_cast<size_t>(((16u - (reinterpret_cast<size_t>(v) & 15u)) & 15u) / 4u));
    const float* w = v + head;
    const size_t m = n - head;
    // Block b sums cells [b0, b1) of w: a whole number of float4s, the last non-empty block the tail.
    const size_t per = ((m + gridDim.x - 1) / gridDim.x + 3) / 4 * 4;
    const size_t b0 = min(m, per * blockIdx.x);
    const size_t b1 = min(m, b0 + per);
    const float4* w4 = reinterpret_cast<const float4*>(w);
    FeAcc acc;
    fe_acc_init(acc);
    if (blockIdx.x == 0 && threadIdx.x < head) {
        const double x = static_cast<double>(v[threadIdx.x]);
        fe_kahan_add(acc.before, acc.before_c, x);
        acc.before_abs += fabs(x);
    }
#pragma unroll 4
    for (size_t i = b0 / 4 + threadIdx.x; i < b1 / 4; i += blockDim.x) {
        const float4 x = __ldg(w4 + i);
        // Four floats summed in FP64 are exact unless their exponents span more than 29 bits; the group then goes
        // into the compensated total.
        fe_kahan_add(acc.before, acc.before_c, (static_cast<double>(x.x) + static_cast<double>(x.y)) + (static_cast<double>(x.z) + static_cast<double>(x.w)));
        acc.before_abs += fabs(static_cast<double>(x.x));
        acc.before_abs += fabs(static_cast<double>(x.y));
        acc.before_abs += fabs(static_cast<double>(x.z));
        acc.before_abs += fabs(static_cast<double>(x.w));
    }
    // The tail past the last float4 belongs to the block whose slice holds it (empty slices at the end hold nothing).
    for (size_t i = max(b0, b1 / 4 * 4) + threadIdx.x; i < b1; i += blockDim.x) {
        const double x = static_cast<double>(w[i]);
        fe_kahan_add(acc.before, acc.before_c, x);
        acc.before_abs += fabs(x);
    }
    fe_acc_block(acc, scratch, partials + 4 * static_cast<size_t>(blockIdx.x), rec);
    fe_acc_finish(partials, static_cast<int>(gridDim.x), count, scratch, rec, true, false);
}

// The least and largest value of n cells (NaN left out, infinities kept) into rec->lo_inv / hi_key as ordered keys,
// the contract record's convention (rec must start all zero). Min and max are exact and integer atomics land in any
// order, so the answer does not depend on the schedule. For what an upload brings: the idle-term test needs the
// bounds of every field it reads, and the uploaded cells are already on the card.
__global__ void __launch_bounds__(256) bounds_f32(const float* __restrict__ v, size_t n, FeCheck* rec)
{
    const size_t head = min(n, static_cast<size_t>(((16u - (reinterpret_cast<size_t>(v) & 15u)) & 15u) / 4u));
    const float* w = v + head;
    const size_t m4 = (n - head) / 4;
    const float4* w4 = reinterpret_cast<const float4*>(w);
    float lo = __int_as_float(0x7f800000), hi = __int_as_float(0xff800000);
    const size_t tid = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    if (tid < head) {
        lo = fminf(lo, v[tid]);
        hi = fmaxf(hi, v[tid]);
    }
#pragma unroll 4
    for (size_t i = tid; i < m4; i += stride) {
        const float4 x = __ldg(w4 + i);
        lo = fminf(fminf(lo, x.x), fminf(x.y, fminf(x.z, x.w)));
        hi = fmaxf(fmaxf(hi, x.x), fmaxf(x.y, fmaxf(x.z, x.w)));
    }
    for (size_t i = 4 * m4 + tid; i < n - head; i += stride) {
        lo = fminf(lo, w[i]);
        hi = fmaxf(hi, w[i]);
    }
    // fminf/fmaxf return the other operand for a NaN, so a thread that saw only NaNs keeps lo > hi: nothing seen.
    const unsigned klo = fe_warp_min(lo <= hi ? fe_order_key(lo) : 0xffffffffu);
    const unsigned khi = fe_warp_max(lo <= hi ? fe_order_key(hi) : 0u);
    if ((threadIdx.x & 31) == 0) {
        if (klo != 0xffffffffu) atomicMax(&rec->lo_inv, ~klo);
        if (khi != 0u) atomicMax(&rec->hi_key, khi);
    }
}

cudaError_t launch_bounds(const float* v, size_t n, FeCheck* rec, int sms, cudaStream_t stream)
{
    bounds_f32<<<4 * sms, 256, 0, stream>>>(v, n, rec);
    return cudaGetLastError();
}

// dst(x, y, z) = src((x + dx) mod nx, (y + dy) mod ny, (z + dz) mod nz): a lattice whose window moved by (dx, dy, dz)
// cells, every cell's value carried to where it now is and the cells that left wrapped round to the side that arrives
// (what a ring-addressed lattice reads there after its origin moves). 0 <= dx < nx, 0 <= dy < ny, 0 <= dz < nz.
__global__ void __launch_bounds__(256) rotate_f32(const float* __restrict__ src, float* __restrict__ dst, int nx, int ny, int nz, int dx,
    int dy, int dz)
{
    const size_t n = static_cast<size_t>(nx) * ny * nz;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const int x = static_cast<int>(i % nx);
        const size_t row = i / nx;
        const int y = static_cast<int>(row % ny);
        const int z = static_cast<int>(row / ny);
        const int sx = x + dx >= nx ? x + dx - nx : x + dx;
        const int sy = y + dy >= ny ? y + dy - ny : y + dy;
        const int sz = z + dz >= nz ? z + dz - nz : z + dz;
        dst[i] = src[(static_cast<size_t>(sz) * ny + sy) * nx + sx];
    }
}

cudaError_t launch_rotate(const float* src, float* dst, int nx, int ny, int nz, int dx, int dy, int dz, int sms, cudaStream_t stream)
{
    rotate_f32<<<8 * sms, 256, 0, stream>>>(src, dst, nx, ny, nz, dx, dy, dz);
    return cudaGetLastError();
}

cudaError_t launch_totals(const float* v, size_t n, FeCheck* rec, double* partials, unsigned* count, cudaStream_t stream)
{
    totals_f32<<<kTotalsBlocks, 256, 0, stream>>>(v, n, rec, partials, count);
    return cudaGetLastError();
}

} // namespace fe
