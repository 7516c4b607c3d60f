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
    // Block b sums cells [b0, b1): a whole number of float4s (the buffer is 256-byte aligned), the last block the tail.
    const size_t per = ((n + gridDim.x - 1) / gridDim.x + 3) / 4 * 4;
    const size_t b0 = min(n, per * blockIdx.x);
    const size_t b1 = min(n, b0 + per);
    const float4* v4 = reinterpret_cast<const float4*>(v);
    FeAcc acc;
    fe_acc_init(acc);
#pragma unroll 4
    for (size_t i = b0 / 4 + threadIdx.x; i < b1 / 4; i += blockDim.x) {
        const float4 x = __ldg(v4 + i);
        acc.before += static_cast<double>(x.x);
        acc.before += static_cast<double>(x.y);
        acc.before += static_cast<double>(x.z);
        acc.before += static_cast<double>(x.w);
        acc.before_abs += fabs(static_cast<double>(x.x));
        acc.before_abs += fabs(static_cast<double>(x.y));
        acc.before_abs += fabs(static_cast<double>(x.z));
        acc.before_abs += fabs(static_cast<double>(x.w));
    }
    for (size_t i = b1 / 4 * 4 + threadIdx.x; i < b1; i += blockDim.x) {
        const double x = static_cast<double>(v[i]);
        acc.before += x;
        acc.before_abs += fabs(x);
    }
    fe_acc_block(acc, scratch, partials + 4 * static_cast<size_t>(blockIdx.x), rec);
    fe_acc_finish(partials, static_cast<int>(gridDim.x), count, scratch, rec, true, false);
}

cudaError_t launch_totals(const float* v, size_t n, FeCheck* rec, double* partials, unsigned* count, cudaStream_t stream)
{
    totals_f32<<<kTotalsBlocks, 256, 0, stream>>>(v, n, rec, partials, count);
    return cudaGetLastError();
}

} // namespace fe
