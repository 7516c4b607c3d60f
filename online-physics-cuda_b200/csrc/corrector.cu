// The learned coarse-lattice correction on the tensor cores: tcgen05 MMAs with BF16 operands in shared memory and FP32
// accumulators in tensor memory, inference and training (forward and backward) in one hand-written kernel.
//
// The network, per cell of a coarse 2-D lattice (every z-plane a sample): the 3 x 3 neighbourhood of (u, v) with the
// edge cell repeating (18 numbers) and the time since the start of the solve -> 64 (ReLU) -> 64 (ReLU) -> 2, the
// correction added to the state the plain coarse step left: a 3x3 convolution with 2 input and 64 output channels (and
// the time), then two pointwise (1x1) layers. Biases are rows of the weight matrices fed by a constant-1 input feature
// (input 18 of layer 1, feature 64 of the hidden layers), so each layer is one GEMM over 128-cell tiles: Z1 = X0 W1
// (K 32), Z2 = H1 W2 (K 80), Y = H2 W3 (K 80, N 16 of which 2 used).
//
// Layout: every operand is a 128-row (cells) or in-feature-row matrix of BF16 in the canonical no-swizzle core-matrix
// layout (8 rows x 16 bytes a core matrix, element (r, c) at ((c/8) (R/8) + r/8) 128 + (r%8) 16 + (c%8) 2 bytes). The
// same buffer is read K-major or MN-major by the descriptors, so each weight matrix is stored once (rows = inputs) and
// serves the forward (as MN-major B) and the backward (W^T, as K-major B), and the activation tiles X0 | H1 | H2 are
// stored back to back so that one M = 128 MMA over them, MN-major, gives a weight gradient H^T dZ (its first rows;
// the rest of the 128 is ignored). Backward of loss = 1/2 sum (u* + y - target)^2:
//   dY = u* + y - target; dH2 = dY W3^T; dZ2 = dH2 (Z2 > 0); dH1 = dZ2 W2^T; dZ1 = dH1 (Z1 > 0);
//   dW3 += H2^T dY; dW2 += H1^T dZ2; dW1 += X0^T dZ1   (all on the tensor cores; per CTA in tensor memory)
// then a fixed-order sum over CTAs and an Adam step on FP32 master weights (deterministic).
//
// One CTA of 128 threads an SM (thread t owns cell t of a tile and TMEM lane t), persistent over tiles; one elected
// thread issues the MMAs and commits them to an mbarrier the others wait on with a bounded wait (a wait that gives up
// sets an error word and the kernel returns through its normal exit, tensor memory freed).
#include "../../include/fe.h"

#include "api_common.hpp"
#include "cuda_ctx.hpp"
#include "fe_device.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace fe {
namespace {

constexpr int kTile = 128;
constexpr int kThreadsC = 128;
// Weights: W1 32 x 64, W2 80 x 64, W3 80 x 16 (rows = inputs with the bias row, cols = outputs).
constexpr int kW1 = 32 * 64, kW2 = 80 * 64, kW3 = 80 * 16;
constexpr int kWeights = kW1 + kW2 + kW3;
// Shared memory (bytes): the activation stack X0 (4 feature groups of 8) | H1 (10) | H2 (10) | spare (6), each group
// 128 cells x 16 bytes; then the weights, dY (2 groups), dZ2 and dZ1 (8 each).
constexpr unsigned kGroup = kTile * 16;
constexpr unsigned kX0 = 0, kH1 = 4 * kGroup, kH2 = 14 * kGroup, kStack = 30 * kGroup;
// Tensor memory columns (FP32): Z1 | Z2 | Y | dH2 | dH1 | dW1 | dW2 | dW3.
constexpr unsigned kTZ1 = 0, kTZ2 = 64, kTDH2 = 144, kTDH1 = 224, kTDW1 = 304, kTDW2 = 368, kTDW3 = 432;

// The two layouts. Training keeps the spare groups after H2 (the weight-gradient MMAs read 128 feature rows from X0, H1
// or H2), dY, dZ2, dZ1 and 512 tensor-memory columns: one CTA an SM. Inference needs X0 | H1 and the weights (45 KB;
// H2 is written over H1 once the MMA that read H1 has completed) and 128 columns (Y reuses Z1's, consumed by then):
// four CTAs an SM, the tensor memory's 512 columns (the size is padded so a fifth never waits for columns).
template <bool TRAIN>
struct Layout {
    static constexpr unsigned H2 = TRAIN ? kH2 : kH1;
    static constexpr unsigned WB1 = TRAIN ? kStack : 14 * kGroup;
    static constexpr unsigned WB2 = WB1 + kW1 * 2, WB3 = WB2 + kW2 * 2, WEnd = WB3 + kW3 * 2;
    static constexpr unsigned DY = WEnd, DZ2 = DY + 2 * kGroup, DZ1 = DZ2 + 8 * kGroup;
    static constexpr unsigned BAR = TRAIN ? DZ1 + 8 * kGroup : WEnd;
    static constexpr unsigned SMEM = TRAIN ? BAR + 64 : 46592u;
    static constexpr unsigned TY = TRAIN ? 128u : 0u;
    static constexpr unsigned TCOLS = TRAIN ? 512u : 128u;
    static constexpr int PER_SM = TRAIN ? 1 : 4;
    static_assert(TRAIN || (BAR + 64 <= SMEM && 5 * SMEM > 232448u), "inference: four CTAs an SM, never five");
};
constexpr unsigned kWaitLimit = 1u << 22;

struct CorrArgs {
    const float* u;      // the state after the plain coarse step
    const float* v;
    const float* tu;     // targets (training)
    const float* tv;
    float* ou;           // corrected state (inference)
    float* ov;
    const unsigned short* w;   // BF16 weights, W1 | W2 | W3 each in its core layout
    float* gpart;        // training: per CTA dW1 | dW2 | dW3, FP32, row-major
    double* lpart;       // training: per CTA 1/2 sum of squared errors
    unsigned* err;       // [0] waits that gave up, [1] corrected cells out of range or not finite
    int nx, ny, nz;
    long long cells;
    float lo, hi;
    float time;          // the time since the start of the solve: input 19 of every cell
};

__host__ __device__ constexpr unsigned core_off(int r, int c, int R)
{
    return static_cast<unsigned>(((c >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

#if defined(__CUDACC__)

__device__ __forceinline__ unsigned long long sdesc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    unsigned long long d = static_cast<unsigned long long>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<unsigned long long>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<unsigned long long>((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;   // descriptor version 1 (sm_100); base offset 0, swizzle none
    return d;
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, M x N, A/B K-major (false) or MN-major (true).
__host__ __device__ constexpr unsigned idesc(int M, int N, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (a_mn ? 1u << 15 : 0u) | (b_mn ? 1u << 16 : 0u) |
        (static_cast<unsigned>(N >> 3) << 17) | (static_cast<unsigned>(M >> 4) << 24);
}

__device__ __forceinline__ void mma(unsigned dtmem, unsigned long long a, unsigned long long b, unsigned id, unsigned accumulate)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 ::"r"(dtmem), "l"(a), "l"(b), "r"(id), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void mma_commit(fe_u64* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(fe_smem(bar)) : "memory");
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void tld16(unsigned taddr, float (&r)[16])
{
    unsigned x[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7]), "=r"(x[8]),
                   "=r"(x[9]), "=r"(x[10]), "=r"(x[11]), "=r"(x[12]), "=r"(x[13]), "=r"(x[14]), "=r"(x[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(x[i]);
}

__device__ __forceinline__ unsigned pack2(float a, float b)
{
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const unsigned*>(&p);
}

// Eight consecutive columns c0 .. c0 + 7 of row r (R rows) as one 16-byte store.
__device__ __forceinline__ void put8(unsigned char* base, int r, int c0, int R, const float* x)
{
    const uint4 q = make_uint4(pack2(x[0], x[1]), pack2(x[2], x[3]), pack2(x[4], x[5]), pack2(x[6], x[7]));
    *reinterpret_cast<uint4*>(base + core_off(r, c0, R)) = q;
}

// A tile's MMAs done: every thread waits for the commit (bounded), then may read tensor memory. The verdict is the
// block's (all threads agree), so a wait that gave up ends the tile loop for every thread together.
__device__ __forceinline__ bool mma_wait(fe_u64* bar, unsigned& phase, unsigned* err)
{
    const bool mine = fe_mbar_wait(bar, phase, kWaitLimit);
    const bool ok = __syncthreads_and(mine) != 0;
    if (ok) phase ^= 1u;
    else if (threadIdx.x == 0) atomicAdd(err, 1u);
    tc_after();
    return ok;
}

// Operands written by threads (generic proxy) and tensor-memory reads done, before the elected thread's next MMAs.
__device__ __forceinline__ void hand_over()
{
    fe_fence_proxy_async();
    tld_wait();
    tc_before();
    __syncthreads();
}

// Hidden layer out of tensor memory: ReLU(Z) as BF16 into the activation stack (64 values, the constant 1, zeros).
__device__ __forceinline__ void hidden_out(unsigned tz, unsigned char* sm, unsigned at, int t)
{
    for (int c = 0; c < 64; c += 16) {
        float z[16];
        tld16(tz + c, z);
        tld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) z[i] = fmaxf(z[i], 0.f);
        put8(sm + at, t, c, kTile, z);
        put8(sm + at, t, c + 8, kTile, z + 8);
    }
    float tail[16] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    put8(sm + at, t, 64, kTile, tail);
    put8(sm + at, t, 72, kTile, tail + 8);
}

// dZ = dH (Z > 0), 64 columns, as BF16 into `at`.
__device__ __forceinline__ void relu_back(unsigned tdh, unsigned tz, unsigned char* sm, unsigned at, int t, bool valid)
{
    for (int c = 0; c < 64; c += 16) {
        float g[16], z[16];
        tld16(tdh + c, g);
        tld16(tz + c, z);
        tld_wait();
#pragma unroll
        for (int i = 0; i < 16; ++i) g[i] = (valid && z[i] > 0.f) ? g[i] : 0.f;
        put8(sm + at, t, c, kTile, g);
        put8(sm + at, t, c + 8, kTile, g + 8);
    }
}

template <bool TRAIN>
__global__ void __launch_bounds__(kThreadsC, Layout<TRAIN>::PER_SM) corr_kernel(const CorrArgs a)
{
    using L = Layout<TRAIN>;
    extern __shared__ __align__(1024) unsigned char sm[];
    fe_u64* bar = reinterpret_cast<fe_u64*>(sm + L::BAR);
    unsigned* tslot = reinterpret_cast<unsigned*>(sm + L::BAR + 16);
    const int t = threadIdx.x;
    const int warp = t >> 5;
    // Weights into shared memory (already in their core layouts), the mbarrier, tensor memory.
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.w);
        uint4* dst = reinterpret_cast<uint4*>(sm + L::WB1);
        for (int i = t; i < kWeights * 2 / 16; i += kThreadsC) dst[i] = src[i];
    }
    if (t == 0) {
        fe_mbar_init(bar, 1);
        fe_fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(fe_smem(tslot)), "r"(L::TCOLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fe_fence_proxy_async();
    tc_before();
    __syncthreads();
    tc_after();
    const unsigned tbase = *tslot;
    const unsigned lane_base = tbase + (static_cast<unsigned>(warp * 32) << 16);
    const unsigned s0 = fe_smem(sm);
    unsigned phase = 0;
    bool ok = true;
    double loss = 0.0;
    int done = 0;
    const long long tiles = (a.cells + kTile - 1) / kTile;
    const long long plane = static_cast<long long>(a.nx) * a.ny;

    for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x, ++done) {
        const long long cell = tile * kTile + t;
        const bool valid = cell < a.cells;
        const long long cz = valid ? cell / plane : 0;
        const int rem = valid ? static_cast<int>(cell - cz * plane) : 0;
        const int cy = rem / a.nx, cx = rem - (rem / a.nx) * a.nx;
        // 1. X0: the 3 x 3 neighbourhood of (u, v), the constant 1, zeros.
        float x0[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) x0[i] = 0.f;
        float uc = 0.f, vc = 0.f;
        if (valid) {
            const float* up = a.u + cz * plane;
            const float* vp = a.v + cz * plane;
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
                for (int dx = -1; dx <= 1; ++dx) {
                    const int yy = min(max(cy + dy, 0), a.ny - 1), xx = min(max(cx + dx, 0), a.nx - 1);
                    const int k = 2 * (3 * (dy + 1) + (dx + 1));
                    x0[k] = up[yy * a.nx + xx];
                    x0[k + 1] = vp[yy * a.nx + xx];
                }
            }
            x0[18] = 1.f;
            x0[19] = a.time;
            uc = x0[8];
            vc = x0[9];
        }
#pragma unroll
        for (int c = 0; c < 32; c += 8) put8(sm + kX0, t, c, kTile, x0 + c);
        hand_over();
        if (t == 0) {
            tc_after();
            for (int k = 0; k < 2; ++k) {
                mma(tbase + kTZ1, sdesc(s0 + kX0 + k * 2 * kGroup, kGroup, 128), sdesc(s0 + L::WB1 + k * 2 * 128, 128, (32 / 8) * 128),
                    idesc(128, 64, false, true), k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        // 2. H1 = ReLU(Z1); Z2 = H1 W2.
        hidden_out(lane_base + kTZ1, sm, kH1, t);
        hand_over();
        if (t == 0) {
            tc_after();
            for (int k = 0; k < 5; ++k) {
                mma(tbase + kTZ2, sdesc(s0 + kH1 + k * 2 * kGroup, kGroup, 128), sdesc(s0 + L::WB2 + k * 2 * 128, 128, (80 / 8) * 128),
                    idesc(128, 64, false, true), k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        // 3. H2 = ReLU(Z2); Y = H2 W3.
        hidden_out(lane_base + kTZ2, sm, L::H2, t);
        hand_over();
        if (t == 0) {
            tc_after();
            for (int k = 0; k < 5; ++k) {
                mma(tbase + L::TY, sdesc(s0 + L::H2 + k * 2 * kGroup, kGroup, 128), sdesc(s0 + L::WB3 + k * 2 * 128, 128, (80 / 8) * 128),
                    idesc(128, 16, false, true), k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        float y[16];
        tld16(lane_base + L::TY, y);
        tld_wait();
        if constexpr (!TRAIN) {
            if (valid) {
                const float nu = uc + y[0], nv = vc + y[1];
                const bool in = nu == nu && nv == nv && nu >= a.lo && nu <= a.hi && nv >= a.lo && nv <= a.hi;
                if (!in) atomicAdd(a.err + 1, 1u);
                a.ou[cell] = nu;
                a.ov[cell] = nv;
            }
            tc_before();
            __syncthreads();
            continue;
        } else {
        // 4. Backward: dY, then dH2 = dY W3^T and dW3 += H2^T dY.
        float dy[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) dy[i] = 0.f;
        if (valid) {
            dy[0] = uc + y[0] - a.tu[cell];
            dy[1] = vc + y[1] - a.tv[cell];
            loss += 0.5 * (static_cast<double>(dy[0]) * dy[0] + static_cast<double>(dy[1]) * dy[1]);
        }
        put8(sm + L::DY, t, 0, kTile, dy);
        put8(sm + L::DY, t, 8, kTile, dy + 8);
        hand_over();
        if (t == 0) {
            tc_after();
            mma(tbase + kTDH2, sdesc(s0 + L::DY, kGroup, 128), sdesc(s0 + L::WB3, (80 / 8) * 128, 128), idesc(128, 80, false, false), 0);
            for (int k = 0; k < 8; ++k) {
                mma(tbase + kTDW3, sdesc(s0 + kH2 + k * 256, 128, kGroup), sdesc(s0 + L::DY + k * 256, 128, kGroup), idesc(128, 16, true, true),
                    done > 0 || k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        // 5. dZ2 = dH2 (Z2 > 0); dH1 = dZ2 W2^T and dW2 += H1^T dZ2.
        relu_back(lane_base + kTDH2, lane_base + kTZ2, sm, L::DZ2, t, valid);
        hand_over();
        if (t == 0) {
            tc_after();
            for (int k = 0; k < 4; ++k) {
                mma(tbase + kTDH1, sdesc(s0 + L::DZ2 + k * 2 * kGroup, kGroup, 128), sdesc(s0 + L::WB2 + k * 2 * (80 / 8) * 128, (80 / 8) * 128, 128),
                    idesc(128, 80, false, false), k > 0);
            }
            for (int k = 0; k < 8; ++k) {
                mma(tbase + kTDW2, sdesc(s0 + kH1 + k * 256, 128, kGroup), sdesc(s0 + L::DZ2 + k * 256, 128, kGroup), idesc(128, 64, true, true),
                    done > 0 || k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        // 6. dZ1 = dH1 (Z1 > 0); dW1 += X0^T dZ1.
        relu_back(lane_base + kTDH1, lane_base + kTZ1, sm, L::DZ1, t, valid);
        hand_over();
        if (t == 0) {
            tc_after();
            for (int k = 0; k < 8; ++k) {
                mma(tbase + kTDW1, sdesc(s0 + kX0 + k * 256, 128, kGroup), sdesc(s0 + L::DZ1 + k * 256, 128, kGroup), idesc(128, 64, true, true),
                    done > 0 || k > 0);
            }
            mma_commit(bar);
        }
        if (!(ok = mma_wait(bar, phase, a.err))) break;
        tc_before();
        __syncthreads();
        }
    }

    if constexpr (TRAIN) {
        // This CTA's weight gradients out of tensor memory (rows = TMEM lanes), and its share of the loss.
        float* g = a.gpart + static_cast<long long>(blockIdx.x) * kWeights;
        const int row = t;
        auto out = [&](unsigned tcol, int rows, int cols, int offset) {
            for (int c = 0; c < cols; c += 16) {
                float r[16];
                tld16(lane_base + tcol + c, r);
                tld_wait();
                if (row < rows) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) g[offset + row * cols + c + i] = (done > 0 && ok) ? r[i] : 0.f;
                }
            }
        };
        out(kTDW1, 32, 64, 0);
        out(kTDW2, 80, 64, kW1);
        out(kTDW3, 80, 16, kW1 + kW2);
        __shared__ double part[kThreadsC];
        part[t] = loss;
        __syncthreads();
        if (t == 0) {
            double s = 0.0;
            for (int i = 0; i < kThreadsC; ++i) s += part[i];
            a.lpart[blockIdx.x] = s;
        }
    }
    if (!ok) {
        // The MMAs of the tile whose wait gave up may still be running: give them one more bounded wait before the
        // tensor memory they write is freed.
        fe_mbar_wait(bar, phase, kWaitLimit);
    }
    tld_wait();
    tc_before();
    __syncthreads();
    if (warp == 0) {
        tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(L::TCOLS) : "memory");
    }
}

// The corrected state replaces the plain step's only when no cell left the range and no wait gave up (decided on the
// card: the on-card contract of the guarded learned step). flag[0] = 1 when the step was reverted.
__global__ void corr_commit(const float* ou, const float* ov, float* u, float* v, long long cells, const unsigned* err, unsigned* flag)
{
    const bool keep = err[0] == 0u && err[1] == 0u;
    if (blockIdx.x == 0 && threadIdx.x == 0) flag[0] = keep ? 0u : 1u;
    if (!keep) return;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < cells; i += static_cast<long long>(gridDim.x) * blockDim.x) {
        u[i] = ou[i];
        v[i] = ov[i];
    }
}

// Fixed-order sum of the CTAs' gradients, then Adam on the FP32 masters; the BF16 copy is rewritten in its core layout.
// Padding rows and columns (inputs 20..31 of W1, 65..79 of W2 and W3, outputs 2..15 of W3) stay zero.
__global__ void corr_adam(float* w, float* m, float* v2, unsigned short* wb, const float* gpart, int parts, float scale, float lr,
    float b1t, float b2t, float* grad_out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kWeights) return;
    int rows, cols, off, r, c;
    if (i < kW1) { rows = 32; cols = 64; off = 0; }
    else if (i < kW1 + kW2) { rows = 80; cols = 64; off = kW1; }
    else { rows = 80; cols = 16; off = kW1 + kW2; }
    r = (i - off) / cols;
    c = (i - off) - r * cols;
    const bool pad = (off == 0 && r > 19) || (off != 0 && r > 64) || (off == kW1 + kW2 && c > 1);
    double g = 0.0;
    for (int p = 0; p < parts; ++p) g += gpart[static_cast<long long>(p) * kWeights + i];
    const float gs = pad ? 0.f : static_cast<float>(g) * scale;
    if (grad_out) grad_out[i] = gs;
    if (lr > 0.f && !pad) {
        const float mi = 0.9f * m[i] + 0.1f * gs;
        const float vi = 0.999f * v2[i] + 0.001f * gs * gs;
        m[i] = mi;
        v2[i] = vi;
        w[i] -= lr * (mi / b1t) / (sqrtf(vi / b2t) + 1e-8f);
    }
    const float wv = pad ? 0.f : w[i];
    const __nv_bfloat16 hb = __float2bfloat16_rn(wv);
    wb[off + core_off(r, c, rows) / 2] = *reinterpret_cast<const unsigned short*>(&hb);
}

#endif // __CUDACC__

} // namespace
} // namespace fe

struct fe_corrector {
    float* w = nullptr;            // FP32 masters
    float* m = nullptr;
    float* v = nullptr;
    unsigned short* wb = nullptr;  // BF16 core-layout copy
    float* gpart = nullptr;
    double* lpart = nullptr;
    unsigned* err = nullptr;       // [0] waits, [1] range, [2] reverted flag
    float* grad = nullptr;         // the last gradient (FP32)
    float* ou = nullptr;
    float* ov = nullptr;
    long long scratch_cells = 0;
    int ctas = 0;
    long long adam_t = 0;
};

namespace {

bool ensure_scratch(fe_corrector* c, long long cells, std::string& why)
{
    if (cells <= c->scratch_cells) return true;
    if (c->ou) cudaFree(c->ou);
    if (c->ov) cudaFree(c->ov);
    c->ou = c->ov = nullptr;
    c->scratch_cells = 0;
    if (!fe::cuda_ok(cudaMalloc(&c->ou, sizeof(float) * cells), "scratch", why) || !fe::cuda_ok(cudaMalloc(&c->ov, sizeof(float) * cells), "scratch", why)) {
        return false;
    }
    c->scratch_cells = cells;
    return true;
}

fe::CorrArgs base_args(fe_corrector* c, int nx, int ny, int nz)
{
    fe::CorrArgs a{};
    a.w = c->wb;
    a.gpart = c->gpart;
    a.lpart = c->lpart;
    a.err = c->err;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.cells = static_cast<long long>(nx) * ny * nz;
    return a;
}

int run_grads(fe_corrector* c, const float* u, const float* v, const float* tu, const float* tv, int nx, int ny, int nz, float time,
    cudaStream_t s, float lr, double* host_loss, float* host_grads)
{
    std::string why;
    if (!c || !u || !v || !tu || !tv || nx < 1 || ny < 1 || nz < 1) return fe::fail(FE_EINVAL, "corrector: bad arguments");
    fe::CorrArgs a = base_args(c, nx, ny, nz);
    a.u = u;
    a.v = v;
    a.tu = tu;
    a.tv = tv;
    a.time = time;
    const long long tiles = (a.cells + fe::kTile - 1) / fe::kTile;
    const int grid = static_cast<int>(std::min<long long>(tiles, static_cast<long long>(c->ctas) * fe::Layout<true>::PER_SM));
    if (!fe::cuda_ok(cudaMemsetAsync(c->err, 0, 4 * sizeof(unsigned), s), "reset", why)) return fe::fail(FE_ECUDA, why);
    fe::corr_kernel<true><<<grid, fe::kThreadsC, fe::Layout<true>::SMEM, s>>>(a);
    ++c->adam_t;
    const float b1t = lr > 0.f ? 1.f - std::pow(0.9f, static_cast<float>(c->adam_t)) : 1.f;
    const float b2t = lr > 0.f ? 1.f - std::pow(0.999f, static_cast<float>(c->adam_t)) : 1.f;
    if (lr <= 0.f) --c->adam_t;
    fe::corr_adam<<<(fe::kWeights + 255) / 256, 256, 0, s>>>(c->w, c->m, c->v, c->wb, c->gpart, grid, 1.f / static_cast<float>(a.cells), lr,
        b1t, b2t, c->grad);
    if (!fe::cuda_ok(cudaGetLastError(), "corrector launch", why)) return fe::fail(FE_ECUDA, why);
    if (host_loss || host_grads) {
        std::vector<double> parts(static_cast<size_t>(grid));
        unsigned err[2] = {0, 0};
        if (!fe::cuda_ok(cudaMemcpyAsync(parts.data(), c->lpart, sizeof(double) * grid, cudaMemcpyDeviceToHost, s), "loss", why) ||
            !fe::cuda_ok(cudaMemcpyAsync(err, c->err, sizeof(err), cudaMemcpyDeviceToHost, s), "err", why) ||
            (host_grads && !fe::cuda_ok(cudaMemcpyAsync(host_grads, c->grad, sizeof(float) * fe::kWeights, cudaMemcpyDeviceToHost, s), "grads", why)) ||
            !fe::cuda_ok(cudaStreamSynchronize(s), "sync", why)) {
            return fe::fail(FE_ECUDA, why);
        }
        if (err[0] != 0u) return fe::fail(FE_EKERNEL, "corrector: a tensor-core wait gave up");
        if (host_loss) {
            double sum = 0.0;
            for (const double p : parts) sum += p;
            *host_loss = sum / static_cast<double>(a.cells);
        }
    }
    return fe::ok();
}

} // namespace

extern "C" {

int fe_corr_create(fe_corrector** out)
{
    if (out == nullptr) return fe::fail(FE_EINVAL, "null out");
    *out = nullptr;
    std::string why;
    if (!fe::device_ready(why)) return fe::fail(FE_ENODEV, why);
    auto* c = new fe_corrector();
    c->ctas = fe::sm_count();
    bool ok = fe::cuda_ok(cudaFuncSetAttribute(fe::corr_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              static_cast<int>(fe::Layout<true>::SMEM)), "smem", why) &&
        fe::cuda_ok(cudaFuncSetAttribute(fe::corr_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                        static_cast<int>(fe::Layout<false>::SMEM)), "smem", why) &&
        fe::cuda_ok(cudaMalloc(&c->w, sizeof(float) * fe::kWeights), "w", why) && fe::cuda_ok(cudaMalloc(&c->m, sizeof(float) * fe::kWeights), "m", why) &&
        fe::cuda_ok(cudaMalloc(&c->v, sizeof(float) * fe::kWeights), "v", why) &&
        fe::cuda_ok(cudaMalloc(&c->wb, sizeof(unsigned short) * fe::kWeights), "wb", why) &&
        fe::cuda_ok(cudaMalloc(&c->gpart, sizeof(float) * fe::kWeights * c->ctas), "gpart", why) &&
        fe::cuda_ok(cudaMalloc(&c->lpart, sizeof(double) * c->ctas), "lpart", why) &&
        fe::cuda_ok(cudaMalloc(&c->err, sizeof(unsigned) * 4), "err", why) && fe::cuda_ok(cudaMalloc(&c->grad, sizeof(float) * fe::kWeights), "grad", why);
    ok = ok && fe::cuda_ok(cudaMemset(c->w, 0, sizeof(float) * fe::kWeights), "w", why) &&
        fe::cuda_ok(cudaMemset(c->m, 0, sizeof(float) * fe::kWeights), "m", why) && fe::cuda_ok(cudaMemset(c->v, 0, sizeof(float) * fe::kWeights), "v", why) &&
        fe::cuda_ok(cudaMemset(c->wb, 0, sizeof(unsigned short) * fe::kWeights), "wb", why) &&
        fe::cuda_ok(cudaMemset(c->err, 0, sizeof(unsigned) * 4), "err", why);
    if (!ok) {
        fe_corr_destroy(c);
        return fe::fail(FE_ECUDA, why);
    }
    *out = c;
    return fe::ok();
}

void fe_corr_destroy(fe_corrector* c)
{
    if (!c) return;
    cudaDeviceSynchronize();
    for (void* p : {static_cast<void*>(c->w), static_cast<void*>(c->m), static_cast<void*>(c->v), static_cast<void*>(c->wb), static_cast<void*>(c->gpart),
             static_cast<void*>(c->lpart), static_cast<void*>(c->err), static_cast<void*>(c->grad), static_cast<void*>(c->ou), static_cast<void*>(c->ov)}) {
        if (p) cudaFree(p);
    }
    delete c;
}

int fe_corr_weight_count(void) { return fe::kWeights; }

int fe_corr_set_weights(fe_corrector* c, const float* host_w)
{
    if (!c || !host_w) return fe::fail(FE_EINVAL, "null argument");
    std::string why;
    if (!fe::cuda_ok(cudaMemcpy(c->w, host_w, sizeof(float) * fe::kWeights, cudaMemcpyHostToDevice), "weights", why) ||
        !fe::cuda_ok(cudaMemset(c->m, 0, sizeof(float) * fe::kWeights), "m", why) || !fe::cuda_ok(cudaMemset(c->v, 0, sizeof(float) * fe::kWeights), "v", why)) {
        return fe::fail(FE_ECUDA, why);
    }
    c->adam_t = 0;
    // The BF16 copy: an Adam call with no step rewrites it from the masters (and its gradient is not used).
    fe::corr_adam<<<(fe::kWeights + 255) / 256, 256>>>(c->w, c->m, c->v, c->wb, c->gpart, 0, 0.f, 0.f, 1.f, 1.f, nullptr);
    if (!fe::cuda_ok(cudaDeviceSynchronize(), "weights", why)) return fe::fail(FE_ECUDA, why);
    return fe::ok();
}

int fe_corr_get_weights(fe_corrector* c, float* host_w)
{
    if (!c || !host_w) return fe::fail(FE_EINVAL, "null argument");
    std::string why;
    if (!fe::cuda_ok(cudaDeviceSynchronize(), "sync", why) ||
        !fe::cuda_ok(cudaMemcpy(host_w, c->w, sizeof(float) * fe::kWeights, cudaMemcpyDeviceToHost), "weights", why)) {
        return fe::fail(FE_ECUDA, why);
    }
    return fe::ok();
}

int fe_corr_grads(fe_corrector* c, const float* u, const float* v, const float* tu, const float* tv, int nx, int ny, int nz, float time,
    void* stream, double* host_loss, float* host_grads)
{
    return run_grads(c, u, v, tu, tv, nx, ny, nz, time, static_cast<cudaStream_t>(stream), 0.f, host_loss, host_grads);
}

int fe_corr_train_step(fe_corrector* c, const float* u, const float* v, const float* tu, const float* tv, int nx, int ny, int nz, float time,
    void* stream, float lr, double* host_loss)
{
    if (!(lr > 0.f)) return fe::fail(FE_EINVAL, "learning rate must be positive");
    return run_grads(c, u, v, tu, tv, nx, ny, nz, time, static_cast<cudaStream_t>(stream), lr, host_loss, nullptr);
}

int fe_corr_apply(fe_corrector* c, float* u, float* v, int nx, int ny, int nz, float time, float lo, float hi, void* stream, int* reverted)
{
    std::string why;
    if (!c || !u || !v || nx < 1 || ny < 1 || nz < 1) return fe::fail(FE_EINVAL, "corrector: bad arguments");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    fe::CorrArgs a = base_args(c, nx, ny, nz);
    if (!ensure_scratch(c, a.cells, why)) return fe::fail(FE_ECUDA, why);
    a.u = u;
    a.v = v;
    a.ou = c->ou;
    a.ov = c->ov;
    a.lo = lo;
    a.hi = hi;
    a.time = time;
    const long long tiles = (a.cells + fe::kTile - 1) / fe::kTile;
    const int grid = static_cast<int>(std::min<long long>(tiles, static_cast<long long>(c->ctas) * fe::Layout<false>::PER_SM));
    if (!fe::cuda_ok(cudaMemsetAsync(c->err, 0, 4 * sizeof(unsigned), s), "reset", why)) return fe::fail(FE_ECUDA, why);
    fe::corr_kernel<false><<<grid, fe::kThreadsC, fe::Layout<false>::SMEM, s>>>(a);
    fe::corr_commit<<<std::max(1, std::min(1024, static_cast<int>((a.cells + 255) / 256))), 256, 0, s>>>(c->ou, c->ov, u, v, a.cells, c->err,
        c->err + 2);
    if (!fe::cuda_ok(cudaGetLastError(), "corrector launch", why)) return fe::fail(FE_ECUDA, why);
    if (reverted) {
        unsigned flag[3] = {0, 0, 0};
        if (!fe::cuda_ok(cudaMemcpyAsync(flag, c->err, sizeof(flag), cudaMemcpyDeviceToHost, s), "flag", why) ||
            !fe::cuda_ok(cudaStreamSynchronize(s), "sync", why)) {
            return fe::fail(FE_ECUDA, why);
        }
        if (flag[0] != 0u) return fe::fail(FE_EKERNEL, "corrector: a tensor-core wait gave up");
        *reverted = static_cast<int>(flag[2]);
    }
    return fe::ok();
}

} // extern "C"
