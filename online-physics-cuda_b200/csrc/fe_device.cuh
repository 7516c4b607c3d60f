// Device primitives for sm_100a shared by the hand-written kernels (compiled by nvcc) and by the kernels the law
// compiler generates at run time (this file is embedded, verbatim, at the top of every generated translation unit and
// compiled by NVRTC). It includes no header, so it compiles the same way under both.
//
// What is here: mbarrier waits with an iteration limit, TMA tiled loads (cp.async.bulk.tensor, never multicast), the
// ordered-integer keys used for order-free min/max, and the contract record every gather pass fills.
#ifndef FE_DEVICE_CUH
#define FE_DEVICE_CUH

typedef unsigned long long fe_u64;

// A CUtensorMap, opaque: 128 bytes, 64-byte aligned (the driver writes it, the TMA unit reads it).
struct alignas(64) FeTensorMap {
    fe_u64 words[16];
};

// What one fused gather pass records for the contracts of the term it runs, per checked field (see FeCheckSlot):
// totals in FP64 (fixed order, so two runs agree to the bit), bounds as ordered-integer keys (the empty record is all zero bytes), range/NaN counts and the
// first bad cell. Filled by the kernels, read and judged by the host.
struct FeCheck {
    double before;       // sum of the field at the start of the term (first substep's pre-state)
    double before_abs;   // sum of |field| at the start of the term
    double after;        // sum after the term's last substep
    double after_abs;
    unsigned out_of_range;
    unsigned not_finite;
    unsigned first_bad;  // ~(linear index) of the first bad cell: the least index wins under atomicMax
    unsigned lo_inv;     // ~order_key(least value) (atomicMax of the inverted key): all-zero bytes are the empty record
    unsigned hi_key;     // order_key(largest value) (atomicMax)
    unsigned changed;    // any cell moved
    unsigned pad[2];
};

// Error words a kernel raises instead of hanging or trapping (bounded waits).
#define FE_ERR_MBAR_TIMEOUT 1u

// Everything below is device code (nvcc's device pass or NVRTC); host translation units see only the types above.
#if defined(__CUDACC__) || defined(__CUDACC_RTC__)

__device__ __forceinline__ unsigned fe_smem(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void fe_mbar_init(fe_u64* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(fe_smem(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fe_fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Generic-proxy reads of a stage are ordered before the async-proxy (TMA) write that refills it.
__device__ __forceinline__ void fe_fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fe_mbar_expect_tx(fe_u64* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fe_smem(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool fe_mbar_try_wait(fe_u64* bar, unsigned parity)
{
    unsigned ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(fe_smem(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits for a phase of an mbarrier, at most `limit` polls (each try_wait itself suspends for a while). Returns false
// when it gave up: the caller records an error and returns, and the kernel never hangs the GPU.
__device__ __forceinline__ bool fe_mbar_wait(fe_u64* bar, unsigned parity, unsigned limit)
{
    for (unsigned i = 0; i < limit; ++i) {
        if (fe_mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

// One tiled 3-D TMA load of a box into shared memory, completion counted on `bar` in bytes. The innermost coordinate
// times 4 bytes must be a multiple of 16 (x a multiple of 4 for fp32); the other coordinates may be negative or past
// the end (the box is filled with zeros there, and no kernel reads those cells).
__device__ __forceinline__ void fe_tma_load_3d(void* dst, const FeTensorMap* map, fe_u64* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(fe_smem(dst)), "l"(reinterpret_cast<fe_u64>(map)), "r"(fe_smem(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void fe_prefetch_tensormap(const FeTensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<fe_u64>(map)) : "memory");
}

// Floats as unsigned keys with the same order, so min and max are integer atomics whose result does not depend on
// the order they land in.
__device__ __forceinline__ unsigned fe_order_key(float v)
{
    const unsigned b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__device__ __forceinline__ bool fe_not_finite(float v)
{
    return (__float_as_uint(v) & 0x7f800000u) == 0x7f800000u;
}

// Sum of a double over a warp in a fixed tree (16, 8, 4, 2, 1): the bits do not depend on timing.
__device__ __forceinline__ double fe_warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

__device__ __forceinline__ unsigned fe_warp_min(unsigned v)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

__device__ __forceinline__ unsigned fe_warp_max(unsigned v)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Per-thread contract accumulators of one checked field in a gather pass.
struct FeAcc {
    double before, before_abs, after, after_abs;
    unsigned lo, hi, bad, nan, first, changed;
};

__device__ __forceinline__ void fe_acc_init(FeAcc& a)
{
    a.before = 0.0; a.before_abs = 0.0; a.after = 0.0; a.after_abs = 0.0;
    a.lo = 0xffffffffu; a.hi = 0u; a.bad = 0u; a.nan = 0u; a.first = 0u; a.changed = 0u;
}

// One cell: its value before the pass and after it. lo/hi are the field's declared range (range contract).
__device__ __forceinline__ void fe_acc_cell(FeAcc& a, float before, float after, float lo, float hi, unsigned index,
    bool totals_before, bool totals_after)
{
    if (totals_before) {
        a.before += static_cast<double>(before);
        a.before_abs += fabs(static_cast<double>(before));
    }
    if (totals_after) {
        a.after += static_cast<double>(after);
        a.after_abs += fabs(static_cast<double>(after));
    }
    const bool nan = fe_not_finite(after);
    if (!nan) {
        const unsigned k = fe_order_key(after);
        a.lo = k < a.lo ? k : a.lo;
        a.hi = k > a.hi ? k : a.hi;
    }
    if (nan || after < lo || after > hi) {
        if (nan) ++a.nan; else ++a.bad;
        const unsigned f = ~index;
        a.first = f > a.first ? f : a.first;
    }
    a.changed |= (__float_as_uint(before) != __float_as_uint(after)) ? 1u : 0u;
}

// The block's contract accumulators into its partial slot (fixed-order sums), plus the order-free integer parts
// straight into the record. `scratch` holds 4 doubles per warp. Every thread of the block calls it.
__device__ __forceinline__ void fe_acc_block(FeAcc& a, double* scratch, double* partial, FeCheck* rec)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    const double s0 = fe_warp_sum(a.before);
    const double s1 = fe_warp_sum(a.before_abs);
    const double s2 = fe_warp_sum(a.after);
    const double s3 = fe_warp_sum(a.after_abs);
    const unsigned lo = fe_warp_min(a.lo);
    const unsigned hi = fe_warp_max(a.hi);
    const unsigned changed = __any_sync(0xffffffffu, a.changed != 0u) ? 1u : 0u;
    const unsigned bad = __reduce_add_sync(0xffffffffu, a.bad);
    const unsigned nan = __reduce_add_sync(0xffffffffu, a.nan);
    const unsigned first = __reduce_max_sync(0xffffffffu, a.first);
    if (lane == 0) {
        scratch[4 * warp + 0] = s0;
        scratch[4 * warp + 1] = s1;
        scratch[4 * warp + 2] = s2;
        scratch[4 * warp + 3] = s3;
        if (lo != 0xffffffffu) atomicMax(&rec->lo_inv, ~lo);
        if (hi != 0u) atomicMax(&rec->hi_key, hi);
        if (changed && rec->changed == 0u) rec->changed = 1u;
        if (bad) atomicAdd(&rec->out_of_range, bad);
        if (nan) atomicAdd(&rec->not_finite, nan);
        if (first) atomicMax(&rec->first_bad, first);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        for (int w = 0; w < warps; ++w) {
            t0 += scratch[4 * w + 0];
            t1 += scratch[4 * w + 1];
            t2 += scratch[4 * w + 2];
            t3 += scratch[4 * w + 3];
        }
        partial[0] = t0;
        partial[1] = t1;
        partial[2] = t2;
        partial[3] = t3;
    }
}

// The last block of a pass to finish folds every block's partial into the record, in block order: which block is last
// changes, the order of the sum does not. `count` is reset for the next pass. Every thread of the block calls it;
// `scratch` holds 4 doubles per warp.
__device__ __forceinline__ void fe_acc_finish(const double* partials, int blocks, unsigned* count, double* scratch,
    FeCheck* rec, bool totals_before, bool totals_after)
{
    __shared__ unsigned last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned done = atomicAdd(count, 1u);
        last = (done + 1u == static_cast<unsigned>(blocks)) ? 1u : 0u;
    }
    __syncthreads();
    if (!last) {
        return;
    }
    __threadfence();
    // Thread t sums blocks t, t + T, t + 2T, ... in order; then a fixed tree over the threads.
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) {
        const volatile double* p = partials + 4 * b;
        t0 += p[0];
        t1 += p[1];
        t2 += p[2];
        t3 += p[3];
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    t0 = fe_warp_sum(t0);
    t1 = fe_warp_sum(t1);
    t2 = fe_warp_sum(t2);
    t3 = fe_warp_sum(t3);
    __syncthreads();
    if (lane == 0) {
        scratch[4 * warp + 0] = t0;
        scratch[4 * warp + 1] = t1;
        scratch[4 * warp + 2] = t2;
        scratch[4 * warp + 3] = t3;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int w = 0; w < warps; ++w) {
            s0 += scratch[4 * w + 0];
            s1 += scratch[4 * w + 1];
            s2 += scratch[4 * w + 2];
            s3 += scratch[4 * w + 3];
        }
        if (totals_before) {
            rec->before = s0;
            rec->before_abs = s1;
        }
        if (totals_after) {
            rec->after = s2;
            rec->after_abs = s3;
        }
        *count = 0u;
    }
}

#endif // device code

#endif // FE_DEVICE_CUH
