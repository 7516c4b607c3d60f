// Host-side interface of the hand-written kernels in heat7.cu, totals.cu and field_solves.cu.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>

#include "fe_device.cuh"

namespace fe {

struct HeatArgs {
    float* out;
    int nx, ny, nz;
    int zchunk;
    float k, h, dt;
    float inv_hh;       // 1 / (h*h) when h*h is a power of two (exact), else 0: divide
    float lo, hi;       // the field's declared range (range contract)
    int totals_before;  // this pass starts the term: record the totals before it
    int totals_after;   // this pass ends the term: record the totals after it
    FeCheck* rec;       // null: no contracts in this pass
    double* partials;   // 4 doubles a block
    unsigned* count;    // blocks finished (reset by the last)
    unsigned* err;      // error word (bounded waits)
};

// 1/v when v is a power of two whose reciprocal is a normal float (then x / v == x * (1/v) to the bit), else 0.
inline float exact_reciprocal(float v)
{
    int e = 0;
    const float m = std::frexp(v, &e);
    if (!(v > 0.0f) || m != 0.5f) return 0.0f;
    const float r = 1.0f / v;
    return std::isnormal(r) ? r : 0.0f;
}

cudaError_t launch_heat7_tma(int variant, const FeTensorMap& map, const HeatArgs& a, cudaStream_t stream);
cudaError_t launch_heat7_plain(const float* T, const HeatArgs& a, cudaStream_t stream);
cudaError_t launch_fill(float* p, size_t n, float v, int sms, cudaStream_t stream);
// Sum and sum of |v| of n cells (a 16-byte aligned buffer) into rec->before / before_abs (totals.cu): kTotalsBlocks blocks,
// 4 partial doubles each.
constexpr int kTotalsBlocks = 1184;
cudaError_t launch_totals(const float* v, size_t n, FeCheck* rec, double* partials, unsigned* count, cudaStream_t stream);
// The least and largest non-NaN value of n cells into rec->lo_inv / hi_key (ordered keys; rec all zero before).
cudaError_t launch_bounds(const float* v, size_t n, FeCheck* rec, int sms, cudaStream_t stream);
// dst = src with its window moved by (dx, dy, dz), 0 <= d < n on each axis, wrapping (totals.cu rotate_f32).
cudaError_t launch_rotate(const float* src, float* dst, int nx, int ny, int nz, int dx, int dy, int dz, int sms, cudaStream_t stream);
cudaError_t launch_copy(const float* a, float* b, size_t n, int sms, cudaStream_t stream);
// The solves of distance and poisson (field_solves.cu), after their seed pass; each kernel returns at once unless *flag.
// distance slots: 0 the answer, 1 seeds inside, 2 seeds outside, 3 and 4 scratch, 5 and 6 squared distances. Launches:
// 7 for distance, `iterations` (+1 when odd) for poisson.
cudaError_t launch_distance_solve(float* const slots[7], int nx, int ny, int nz, float h, const unsigned* flag, int sms, cudaStream_t stream);
cudaError_t launch_poisson_solve(float* answer, float* other, const float* source, int iterations, int nx, int ny, int nz, float h,
    const unsigned* flag, int sms, cudaStream_t stream);
int heat7_tma_rows(int variant);
int heat7_tma_blocks(int variant, int nx, int ny, int nz, int zchunk);
int heat7_plain_blocks(int nx, int ny, int nz, int zchunk);

} // namespace fe
