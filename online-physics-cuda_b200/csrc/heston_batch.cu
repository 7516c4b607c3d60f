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
// Per cell, every coefficient and F are the law's fp32 arithmetic in the law's order.
//
// Schedule (B200): a persistent grid (a few CTAs an SM) takes options from a work counter, largest first; one CTA
// steps one option through all its time steps with the option's arrays in L2-resident scratch (the CTA's own). Rows'
// coefficients depend only on the row (the variance), so they sit in shared memory. The explicit operator is a pass
// of all 256 threads over the cells; each implicit half is a batch of tridiagonal solves by warp segments of K = n / M
// lanes, M cells a lane (tridiag.cuh: a PCR/Thomas hybrid, K = 1 being Thomas), M chosen per axis by the autotuner. Each option's result is
// the same whichever CTA takes it, so the prices do not depend on the schedule.
#include "../../include/fe.h"

#include "api_common.hpp"
#include "cuda_ctx.hpp"
#include "fe_device.cuh"
#include "tridiag.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace fe {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxNy = 256;
constexpr int kMaxNx = 512;

struct OptionDev {
    int nx, ny;
    int steps;
    int pad;
    float h, dt, th;
    float kappa, theta, sigma, rho, r;
    float x0;       // ln K - 3 + h/2: the centre of cell 0
    long long at;   // offset of the option's grid in the batch buffer
};

struct BatchArgs {
    const OptionDev* opts;
    const int* order;   // options by descending size: the work queue
    int n;
    int scheme;         // 0 Douglas, 1 HV
    float* V;
    float* scratch;     // per CTA: 4 arrays of kMaxNx * kMaxNy
    unsigned* next;     // work counter
    int steps_limit;    // > 0: at most this many steps an option (the autotuner's short runs)
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

// F(W) at (i, j): rho var gx(gy(W)) + the four neighbour differences - r W, as the law writes it (clamped reads; gx and
// gy divide by the span they cover, one cell at an edge).
__device__ __forceinline__ float op_F(const float* W, int nx, int ny, int i, int j, float h, float r, const RowCoef& c)
{
    const int im = max(i - 1, 0), ip = min(i + 1, nx - 1);
    const int jm = max(j - 1, 0), jp = min(j + 1, ny - 1);
    const float w = W[j * nx + i];
    const float sy = static_cast<float>(jp - jm);
    const float sx = static_cast<float>(ip - im);
    const float gy_p = jp - jm > 0 ? (W[jp * nx + ip] - W[jm * nx + ip]) / (h * sy) : 0.f;
    const float gy_m = jp - jm > 0 ? (W[jp * nx + im] - W[jm * nx + im]) / (h * sy) : 0.f;
    const float gxy = ip - im > 0 ? (gy_p - gy_m) / (h * sx) : 0.f;
    float f = c.rv * gxy;
    f = f + c.wxm * (W[j * nx + im] - w);
    f = f + c.wxp * (W[j * nx + ip] - w);
    f = f + c.wym * (W[jm * nx + i] - w);
    f = f + c.wyp * (W[jp * nx + i] - w);
    return f - r * w;
}

// The x lines of one option: rows j, M cells a lane, K = nx / M lanes a line (K = 1: the line is one lane's, Thomas).
// `in` holds the right-hand sides, `out` gets the answers (may be `in`).
template <int M>
__device__ __forceinline__ void solve_x(const float* in, float* out, int nx, int ny, const RowCoef* rc)
{
    const int K = nx > M ? nx / M : 1;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / K;
    const int k = lane % K;
    const int per_warp = 32 / K;
    const int nwarps = blockDim.x >> 5;
    for (int base = warp * per_warp; base < ny; base += nwarps * per_warp) {
        const int j = base + seg;
        const bool live = j < ny;
        const int jj = live ? j : ny - 1;
        const RowCoef c = rc[jj];
        float a[M], b[M], cc[M], d[M];
#pragma unroll
        for (int r = 0; r < M; ++r) {
            const int i = min(k * M + r, nx - 1);
            a[r] = i == 0 ? 0.f : c.ax;
            cc[r] = i == nx - 1 ? 0.f : c.cx;
            b[r] = c.bx;
            if (i == 0) b[r] += c.ax;
            if (i == nx - 1) b[r] += c.cx;
            d[r] = in[jj * nx + i];
        }
        if (K == 1) fe_thomas_n<M>(a, b, cc, d, nx);
        else fe_tri_segment_k<M>(a, b, cc, d, k, K);
        if (live) {
#pragma unroll
            for (int r = 0; r < M; ++r) {
                if (k * M + r < nx) out[j * nx + k * M + r] = d[r];
            }
        }
    }
}

// The y lines: columns i, M cells a lane, K = ny / M lanes a line; mode 0 writes the answer to `out`, mode 1 adds it
// to `out` (U += D2), mode 2 adds it and `add` (U += D2 + E2).
template <int M>
__device__ __forceinline__ void solve_y(const float* in, float* out, const float* add, int mode, int nx, int ny, const RowCoef* rc)
{
    const int K = ny > M ? ny / M : 1;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int seg = lane / K;
    const int k = lane % K;
    const int per_warp = 32 / K;
    const int nwarps = blockDim.x >> 5;
    for (int base = warp * per_warp; base < nx; base += nwarps * per_warp) {
        const int i = base + seg;
        const bool live = i < nx;
        const int ii = live ? i : nx - 1;
        float a[M], b[M], cc[M], d[M];
#pragma unroll
        for (int r = 0; r < M; ++r) {
            const int j = min(k * M + r, ny - 1);
            const RowCoef& c = rc[j];
            a[r] = j == 0 ? 0.f : c.ay;
            cc[r] = j == ny - 1 ? 0.f : c.cy;
            b[r] = c.by;
            if (j == 0) b[r] += c.ay;
            if (j == ny - 1) b[r] += c.cy;
            d[r] = in[j * nx + ii];
        }
        if (K == 1) fe_thomas_n<M>(a, b, cc, d, ny);
        else fe_tri_segment_k<M>(a, b, cc, d, k, K);
        if (live) {
#pragma unroll
            for (int r = 0; r < M; ++r) {
                const int j = k * M + r;
                if (j >= ny) continue;
                const int at = j * nx + i;
                if (mode == 0) out[at] = d[r];
                else if (mode == 1) out[at] = out[at] + d[r];
                else out[at] = out[at] + (d[r] + add[at]);
            }
        }
    }
}

// MX, MY: cells a lane holds along x and y (the autotuner's choice); a line takes n / M lanes (at most 32).
template <int MX, int MY>
__global__ void __launch_bounds__(kThreads) heston_adi_batch(const BatchArgs args)
{
    __shared__ RowCoef rc[kMaxNy];
    __shared__ int task;
    const size_t plane = static_cast<size_t>(kMaxNx) * kMaxNy;
    float* F0 = args.scratch + blockIdx.x * 4 * plane; // dt F(U)
    float* D = F0 + plane;                             // D1, then D2
    float* E = D + plane;                              // HV: E1, then E2
    for (;;) {
        if (threadIdx.x == 0) task = static_cast<int>(atomicAdd(args.next, 1u));
        __syncthreads();
        const int t = task;
        __syncthreads();
        if (t >= args.n) break;
        const OptionDev o = args.opts[args.order[t]];
        const int nx = o.nx, ny = o.ny, cells = nx * ny;
        float* U = args.V + o.at;
        for (int j = threadIdx.x; j < ny; j += blockDim.x) rc[j] = row_coef(o, j);
        __syncthreads();
        const int steps = args.steps_limit > 0 ? min(o.steps, args.steps_limit) : o.steps;
        for (int s = 0; s < steps; ++s) {
            for (int c = threadIdx.x; c < cells; c += blockDim.x) {
                const int i = c % nx, j = c / nx;
                F0[c] = o.dt * op_F(U, nx, ny, i, j, o.h, o.r, rc[j]);
            }
            __syncthreads();
            solve_x<MX>(F0, D, nx, ny, rc);
            __syncthreads();
            if (args.scheme == 0) {
                solve_y<MY>(D, U, nullptr, 1, nx, ny, rc);
                __syncthreads();
                continue;
            }
            solve_y<MY>(D, D, nullptr, 0, nx, ny, rc);
            __syncthreads();
            for (int c = threadIdx.x; c < cells; c += blockDim.x) {
                const int i = c % nx, j = c / nx;
                E[c] = F0[c] - D[c] + 0.5f * o.dt * op_F(D, nx, ny, i, j, o.h, o.r, rc[j]);
            }
            __syncthreads();
            solve_x<MX>(E, E, nx, ny, rc);
            __syncthreads();
            solve_y<MY>(E, U, D, 2, nx, ny, rc);
            __syncthreads();
        }
    }
}

using BatchKernel = void (*)(const BatchArgs);

// The (MX, MY) pairs built: cells a lane along x and along y.
constexpr int kMs[3] = {4, 8, 16};

BatchKernel batch_kernel(int mx, int my)
{
    static const BatchKernel table[3][3] = {
        {heston_adi_batch<4, 4>, heston_adi_batch<4, 8>, heston_adi_batch<4, 16>},
        {heston_adi_batch<8, 4>, heston_adi_batch<8, 8>, heston_adi_batch<8, 16>},
        {heston_adi_batch<16, 4>, heston_adi_batch<16, 8>, heston_adi_batch<16, 16>},
    };
    auto at = [](int m) { return m == 4 ? 0 : (m == 8 ? 1 : (m == 16 ? 2 : -1)); };
    const int x = at(mx), y = at(my);
    return x < 0 || y < 0 ? nullptr : table[x][y];
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

// Price at (ln S0, v0): bilinear between the four cell centres around it.
__global__ void heston_price(const OptionDev* opts, const float* spot, const float* v0, int n, const float* V, float* out)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    const OptionDev op = opts[o];
    const float* U = V + op.at;
    const double fx = (std::log(static_cast<double>(spot[o])) - (op.x0)) / op.h;
    const double fy = static_cast<double>(v0[o]) / (static_cast<double>(op.sigma) * op.h) - 0.5;
    const int i0 = max(0, min(op.nx - 2, static_cast<int>(std::floor(fx))));
    const int j0 = max(0, min(op.ny - 2, static_cast<int>(std::floor(fy))));
    const double tx = fmin(fmax(fx - i0, 0.0), 1.0), ty = fmin(fmax(fy - j0, 0.0), 1.0);
    const double a = U[j0 * op.nx + i0], b = U[j0 * op.nx + i0 + 1], c = U[(j0 + 1) * op.nx + i0], d = U[(j0 + 1) * op.nx + i0 + 1];
    out[o] = static_cast<float>((1 - ty) * ((1 - tx) * a + tx * b) + ty * ((1 - tx) * c + tx * d));
}

} // namespace
} // namespace fe

struct fe_heston_batch {
    int n = 0;
    int steps = 0;
    int scheme = 0;
    int mx = 16, my = 8;   // cells a lane holds along x and along y
    int ctas = 0;
    std::vector<fe::OptionDev> host;
    fe::OptionDev* opts = nullptr;
    int* order = nullptr;
    float* V = nullptr;
    float* scratch = nullptr;
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

// Whether every option's lines fit M cells a lane in at most 32 lanes.
bool split_fits(const fe_heston_batch* b, int mx, int my)
{
    if (fe::batch_kernel(mx, my) == nullptr) return false;
    for (const fe::OptionDev& o : b->host) {
        if (o.nx / mx > 32 || o.ny / my > 32) return false;
    }
    return true;
}

void release(fe_heston_batch* b)
{
    if (b == nullptr) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (void* p : {static_cast<void*>(b->opts), static_cast<void*>(b->order), static_cast<void*>(b->V), static_cast<void*>(b->scratch),
             static_cast<void*>(b->next), static_cast<void*>(b->strikes), static_cast<void*>(b->spots), static_cast<void*>(b->v0s),
             static_cast<void*>(b->prices)}) {
        if (p) cudaFree(p);
    }
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

int launch_run(fe_heston_batch* b, std::string& why, int steps_limit = 0)
{
    fe::BatchArgs a{};
    a.steps_limit = steps_limit;
    a.opts = b->opts;
    a.order = b->order;
    a.n = b->n;
    a.scheme = b->scheme;
    a.V = b->V;
    a.scratch = b->scratch;
    a.next = b->next;
    const fe::BatchKernel kernel = fe::batch_kernel(b->mx, b->my);
    if (kernel == nullptr) {
        why = "no kernel for that split";
        return FE_EINVAL;
    }
    if (!fe::cuda_ok(cudaMemsetAsync(b->next, 0, sizeof(unsigned), b->stream), "reset queue", why)) return FE_ECUDA;
    fe::heston_init<<<dim3(64, b->n), 256, 0, b->stream>>>(b->opts, b->strikes, b->n, b->V);
    kernel<<<b->ctas, fe::kThreads, 0, b->stream>>>(a);
    fe::heston_price<<<(b->n + 127) / 128, 128, 0, b->stream>>>(b->opts, b->spots, b->v0s, b->n, b->V, b->prices);
    if (!fe::cuda_ok(cudaGetLastError(), "heston launch", why)) return FE_ECUDA;
    return FE_OK;
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
        o.steps = steps;
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
    // The work queue: largest grids first, so the last CTAs to finish are on small ones.
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
        return static_cast<long long>(b->host[p].nx) * b->host[p].ny > static_cast<long long>(b->host[q].nx) * b->host[q].ny;
    });
    if (!split_fits(b, b->mx, b->my)) {
        b->mx = 16;
        b->my = 16;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel(16, 16), kThreads, 0);
    b->ctas = std::max(1, std::min(n, sm_count() * std::max(1, per_sm)));
    const size_t plane = static_cast<size_t>(kMaxNx) * kMaxNy;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream", why) &&
        cuda_ok(cudaMalloc(&b->opts, sizeof(OptionDev) * n), "opts", why) && cuda_ok(cudaMalloc(&b->order, sizeof(int) * n), "order", why) &&
        cuda_ok(cudaMalloc(&b->V, sizeof(float) * static_cast<size_t>(at)), "grids", why) &&
        cuda_ok(cudaMalloc(&b->scratch, sizeof(float) * 4 * plane * b->ctas), "scratch", why) &&
        cuda_ok(cudaMalloc(&b->next, sizeof(unsigned)), "queue", why) && cuda_ok(cudaMalloc(&b->strikes, sizeof(float) * n), "strikes", why) &&
        cuda_ok(cudaMalloc(&b->spots, sizeof(float) * n), "spots", why) && cuda_ok(cudaMalloc(&b->v0s, sizeof(float) * n), "v0", why) &&
        cuda_ok(cudaMalloc(&b->prices, sizeof(float) * n), "prices", why);
    ok = ok && cuda_ok(cudaMemcpy(b->opts, b->host.data(), sizeof(OptionDev) * n, cudaMemcpyHostToDevice), "opts", why) &&
        cuda_ok(cudaMemcpy(b->order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "order", why) &&
        cuda_ok(cudaMemcpy(b->strikes, strikes.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "strikes", why) &&
        cuda_ok(cudaMemcpy(b->spots, spots.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "spots", why) &&
        cuda_ok(cudaMemcpy(b->v0s, v0s.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "v0", why);
    if (!ok) {
        release(b);
        return fail(FE_ECUDA, why);
    }
    *out = b;
    return fe::ok();
}

void fe_heston_batch_destroy(fe_heston_batch* batch)
{
    if (batch) cudaStreamSynchronize(batch->stream);
    release(batch);
}

int fe_heston_batch_set_split(fe_heston_batch* b, int mx, int my)
{
    if (b == nullptr || !split_fits(b, mx, my)) {
        return fe::fail(FE_EINVAL, "cells a lane: 4, 8 or 16 each way, and no line may take more than 32 lanes");
    }
    b->mx = mx;
    b->my = my;
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

int fe_heston_batch_autotune(fe_heston_batch* b, int* mx_out, int* my_out)
{
    if (b == nullptr) return fe::fail(FE_EINVAL, "null batch");
    // Each candidate runs the whole batch for a few steps (the next real run sets the grids up again).
    float best = 1e30f;
    int bx = b->mx, by = b->my;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (const int mx : fe::kMs) {
        for (const int my : fe::kMs) {
            if (!split_fits(b, mx, my)) continue;
            b->mx = mx;
            b->my = my;
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
                by = my;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const int s = fe_heston_batch_set_split(b, bx, by);
    if (mx_out) *mx_out = bx;
    if (my_out) *my_out = by;
    return s;
}

} // extern "C"
