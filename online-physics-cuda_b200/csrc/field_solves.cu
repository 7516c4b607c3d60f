// The fixed kernels of the law's two whole-lattice ops, run after their seed pass (generated, fe_seed_pass) and only
// when it raised the op's change flag (the reference recomputes them only when their input changed: CudaSolver.cpp
// 394-434, Law.cpp:1042-1181).
//
//   distance(a): signed distance in metres to the surface of the solid set {a >= 0.5}: exact squared distances to the
//     nearest solid and the nearest open cell by three separable passes (x, y, z), each cell looking outward along the
//     axis until no farther cell can do better; then the surface half a cell from the last solid cell's centre, and
//     beyond the lattice open (a solid cell is never farther from open than the lattice border).
//   poisson(s, n): n Jacobi sweeps of lap(phi) = s with phi = 0 outside the lattice, warm-started from the last answer.
//
// fp32 like the reference's CUDA path (its CPU path rounds the same sums from double: the two agree to float rounding).
#include "heat7.hpp"

#include <algorithm>
#include <utility>

namespace fe {

namespace {

constexpr float kFar = 1e30f;

__device__ __forceinline__ void cell_of(size_t i, int nx, int ny, int& x, int& y, int& z)
{
    x = static_cast<int>(i % static_cast<size_t>(nx));
    y = static_cast<int>((i / static_cast<size_t>(nx)) % static_cast<size_t>(ny));
    z = static_cast<int>(i / (static_cast<size_t>(nx) * ny));
}

__global__ void __launch_bounds__(256) dist_scan(const float* __restrict__ from, float* __restrict__ to, int nx, int ny, int nz, int axis,
    const unsigned* flag)
{
    if (*flag == 0u) return;
    const size_t cells = static_cast<size_t>(nx) * ny * nz;
    const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
    const size_t step = axis == 0 ? 1 : (axis == 1 ? static_cast<size_t>(nx) : static_cast<size_t>(nx) * ny);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        cell_of(i, nx, ny, x, y, z);
        const int q = axis == 0 ? x : (axis == 1 ? y : z);
        float best = kFar;
        for (int r = 0; r < n; ++r) {
            const float rr = static_cast<float>(r) * static_cast<float>(r);
            if (rr >= best || (q - r < 0 && q + r >= n)) break;
            if (q - r >= 0) best = fminf(best, from[i - static_cast<size_t>(r) * step] + rr);
            if (q + r < n) best = fminf(best, from[i + static_cast<size_t>(r) * step] + rr);
        }
        to[i] = best;
    }
}

__global__ void __launch_bounds__(256) dist_signed(const float* __restrict__ to_in, const float* __restrict__ to_out,
    const float* __restrict__ seed_in, float* __restrict__ result, int nx, int ny, int nz, float h, const unsigned* flag)
{
    if (*flag == 0u) return;
    const size_t cells = static_cast<size_t>(nx) * ny * nz;
    const float far_m = static_cast<float>(nx + ny + nz) * h;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        cell_of(i, nx, ny, x, y, z);
        float d;
        if (seed_in[i] == 0.f) {
            // Solid: to the nearest open cell, or across the nearest lattice border (an axis one cell thick has none).
            float border = 1e30f;
            if (nx > 1) border = fminf(border, static_cast<float>(min(x + 1, nx - x)));
            if (ny > 1) border = fminf(border, static_cast<float>(min(y + 1, ny - y)));
            if (nz > 1) border = fminf(border, static_cast<float>(min(z + 1, nz - z)));
            const float o = to_out[i];
            d = -(fminf(o < 1e29f ? sqrtf(o) : far_m / h, border) - 0.5f) * h;
        } else {
            const float o = to_in[i];
            d = o < 1e29f ? (sqrtf(o) - 0.5f) * h : far_m;
        }
        result[i] = d;
    }
}

__global__ void __launch_bounds__(256) poisson_jacobi(const float* __restrict__ from, float* __restrict__ to, const float* __restrict__ src,
    int nx, int ny, int nz, float h, const unsigned* flag)
{
    if (*flag == 0u) return;
    const size_t cells = static_cast<size_t>(nx) * ny * nz;
    const size_t sy = static_cast<size_t>(nx), sz = static_cast<size_t>(nx) * ny;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        int x, y, z;
        cell_of(i, nx, ny, x, y, z);
        float sum = 0.f;
        int axes = 0;
        if (nx > 1) {
            ++axes;
            if (x > 0) sum += from[i - 1];
            if (x + 1 < nx) sum += from[i + 1];
        }
        if (ny > 1) {
            ++axes;
            if (y > 0) sum += from[i - sy];
            if (y + 1 < ny) sum += from[i + sy];
        }
        if (nz > 1) {
            ++axes;
            if (z > 0) sum += from[i - sz];
            if (z + 1 < nz) sum += from[i + sz];
        }
        to[i] = (sum - h * h * src[i]) / (2.f * static_cast<float>(max(axes, 1)));
    }
}

__global__ void __launch_bounds__(256) copy_flagged(const float* __restrict__ from, float* __restrict__ to, size_t n, const unsigned* flag)
{
    if (*flag == 0u) return;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        to[i] = from[i];
    }
}

unsigned blocks_for(size_t cells, int sms)
{
    return static_cast<unsigned>(std::min<size_t>((cells + 255) / 256, static_cast<size_t>(sms) * 8));
}

} // namespace

cudaError_t launch_distance_solve(float* const slots[7], int nx, int ny, int nz, float h, const unsigned* flag, int sms, cudaStream_t stream)
{
    // slots: 0 the answer, 1 seeds inside, 2 seeds outside, 3 and 4 scratch, 5 squared distance to inside, 6 to outside.
    const size_t cells = static_cast<size_t>(nx) * ny * nz;
    const unsigned g = blocks_for(cells, sms);
    for (const int k : {0, 1}) {
        const float* seed = slots[1 + k];
        float* to = slots[5 + k];
        dist_scan<<<g, 256, 0, stream>>>(seed, slots[3], nx, ny, nz, 0, flag);
        dist_scan<<<g, 256, 0, stream>>>(slots[3], slots[4], nx, ny, nz, 1, flag);
        dist_scan<<<g, 256, 0, stream>>>(slots[4], to, nx, ny, nz, 2, flag);
    }
    dist_signed<<<g, 256, 0, stream>>>(slots[5], slots[6], slots[1], slots[0], nx, ny, nz, h, flag);
    return cudaGetLastError();
}

cudaError_t launch_poisson_solve(float* answer, float* other, const float* source, int iterations, int nx, int ny, int nz, float h,
    const unsigned* flag, int sms, cudaStream_t stream)
{
    const size_t cells = static_cast<size_t>(nx) * ny * nz;
    const unsigned g = blocks_for(cells, sms);
    float* from = answer;
    float* to = other;
    for (int it = 0; it < iterations; ++it) {
        poisson_jacobi<<<g, 256, 0, stream>>>(from, to, source, nx, ny, nz, h, flag);
        std::swap(from, to);
    }
    if (from != answer) copy_flagged<<<g, 256, 0, stream>>>(from, answer, cells, flag);
    return cudaGetLastError();
}

} // namespace fe
