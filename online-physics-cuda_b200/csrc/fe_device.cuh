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

// The one parameter block of every generated pass kernel (a fused gather, or a group of stored stages): the host fills
// it, the kernel reads it as a __grid_constant__. Sources are the buffers the pass reads (a field's current buffer or a
// stage's slot), each with its TMA map in a slab pass; outputs are the buffers it writes, each optionally with a
// contract record.
#define FE_MAX_MAP 12   // sources a TMA slab pass stages through shared memory
#define FE_MAX_SRC 32   // sources a plain pass reads
#define FE_MAX_OUT 8
struct FePassArgs {
    FeTensorMap map[FE_MAX_MAP];
    const float* src[FE_MAX_SRC];
    float* out[FE_MAX_OUT];
    FeCheck* rec[FE_MAX_OUT];  // null: this output is not checked in this pass
    // The record of the pass that last wrote this output's field, whose totals after it are the totals before this
    // pass: copied into rec's before/before_abs when the pass ends (null: they are already there, or not needed).
    const FeCheck* carry[FE_MAX_OUT];
    float lo[FE_MAX_OUT];      // declared range of a checked output's field
    float hi[FE_MAX_OUT];
    double* partials;          // [FE_MAX_OUT][blocks][4]
    unsigned* count;           // [FE_MAX_OUT] blocks finished
    unsigned* flag;            // a distance's or poisson's change flag (its seed pass sets it)
    unsigned* err;
    float dt;
    int flags;                 // FE_PASS_AFTER | FE_PASS_RANGE
    int zchunk;
    int blocks;
    int own_z0, own_z1;        // contracts cover planes [own_z0, own_z1) (the rest: halo planes another rank owns)
};
#define FE_PASS_AFTER 2   // record the totals after the pass (the term's last substep)
#define FE_PASS_RANGE 4   // record range/NaN counts and bounds of what the pass writes (the term's last substep)

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

// Neumaier's compensated summation: c collects what adding x to s rounds away (the larger magnitude's error term), so
// s + c is the sum to about one rounding whatever the order of magnitudes. Used in a fixed order everywhere, so two
// runs still agree to the bit.
__device__ __forceinline__ void fe_kahan_add(double& s, double& c, double x)
{
    const double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
}

// A compensated sum (s, c) over a warp in the fixed tree (16, 8, 4, 2, 1), folded to one double.
__device__ __forceinline__ double fe_warp_sum_c(double s, double c)
{
    for (int o = 16; o > 0; o >>= 1) {
        const double ps = __shfl_down_sync(0xffffffffu, s, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
        fe_kahan_add(s, c, ps);
    }
    return s + c;
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

// Per-thread contract accumulators of one checked field in a gather pass. Totals are FP64; each group of 4 cells a lane
// owns is first summed in fp32 ((c0 + c1) + (c2 + c3)), whose rounding (a few 1e-8 of the group) is far below the
// conservation tolerance (1e-5 of the total of |field|). From there on the totals compared for conservation are
// compensated (Neumaier, fe_kahan_add) at every level: a lane's planes, the warp tree, the block's warps, the blocks. Bounds are float min/max (NaN ignored), turned into ordered
// keys once per block.
struct FeAcc {
    double before, before_abs, after, after_abs;
    double before_c, after_c;  // compensation of before and after (fe_kahan_add)
    float pb, pba, pa;  // this plane's fp32 partials of before, |before| and after (fe_acc_flush moves them to FP64)
    float lo, hi;
    unsigned bad, nan, first, changed;
};

__device__ __forceinline__ void fe_acc_init(FeAcc& a)
{
    a.before = 0.0; a.before_abs = 0.0; a.after = 0.0; a.after_abs = 0.0;
    a.before_c = 0.0; a.after_c = 0.0;
    a.pb = 0.f; a.pba = 0.f; a.pa = 0.f;
    a.lo = __int_as_float(0x7f800000); a.hi = __int_as_float(0xff800000);
    a.bad = 0u; a.nan = 0u; a.first = 0u; a.changed = 0u;
}

// The lane's fp32 partials of one plane (its R rows of 4 cells: a few cells, rounded a few 1e-8 of their sum) into
// the FP64 totals. Called once a plane, in a fixed order.
__device__ __forceinline__ void fe_acc_flush(FeAcc& a)
{
    fe_kahan_add(a.before, a.before_c, static_cast<double>(a.pb));
    a.before_abs += static_cast<double>(a.pba);
    fe_kahan_add(a.after, a.after_c, static_cast<double>(a.pa));
    a.pb = 0.f; a.pba = 0.f; a.pa = 0.f;
}

__device__ __forceinline__ void fe_acc_bad(FeAcc& a, float after, unsigned index)
{
    if (fe_not_finite(after)) ++a.nan; else ++a.bad;
    const unsigned f = ~index;
    a.first = f > a.first ? f : a.first;
}

// Four consecutive cells (index0 .. index0 + 3): their values before the pass and after it; lo/hi the declared range.
// The sum of |after| is not kept (the judge scales its tolerance by the sum of |before|, Solver.cpp:439-453). With
// BITS the change flag compares the cells' bits; without it the caller sets a.changed itself (from its increments).
template <bool BITS = true>
__device__ __forceinline__ void fe_acc_row4(FeAcc& a, const float* before, const float* after, float lo, float hi,
    unsigned index0, bool totals_before, bool totals_after, bool range = true)
{
    if (totals_before) {
        a.pb += (before[0] + before[1]) + (before[2] + before[3]);
        a.pba += (fabsf(before[0]) + fabsf(before[1])) + (fabsf(before[2]) + fabsf(before[3]));
    }
    const float s4 = (after[0] + after[1]) + (after[2] + after[3]);
    if (totals_after) {
        a.pa += s4;
    }
    if (range) {
        // The group's least and most (NaN ignored) give the bounds and the range test at once; a NaN or an infinity
        // anywhere makes the group's sum non-finite. Only a group that fails is looked at cell by cell.
        const float mn = fminf(fminf(after[0], after[1]), fminf(after[2], after[3]));
        const float mx = fmaxf(fmaxf(after[0], after[1]), fmaxf(after[2], after[3]));
        a.lo = fminf(a.lo, mn);
        a.hi = fmaxf(a.hi, mx);
        if (!(mn >= lo && mx <= hi && fabsf(s4) <= 3.0e38f)) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (!(after[q] >= lo && after[q] <= hi)) fe_acc_bad(a, after[q], index0 + q);
            }
        }
    }
    if (BITS) {
        a.changed |= ((__float_as_uint(before[0]) ^ __float_as_uint(after[0])) | (__float_as_uint(before[1]) ^ __float_as_uint(after[1])) |
                         (__float_as_uint(before[2]) ^ __float_as_uint(after[2])) | (__float_as_uint(before[3]) ^ __float_as_uint(after[3]))) != 0u
            ? 1u : 0u;
    }
}

// One cell (the plain passes).
__device__ __forceinline__ void fe_acc_cell(FeAcc& a, float before, float after, float lo, float hi, unsigned index,
    bool totals_before, bool totals_after, bool range = true)
{
    if (totals_before) {
        fe_kahan_add(a.before, a.before_c, static_cast<double>(before));
        a.before_abs += static_cast<double>(fabsf(before));
    }
    if (totals_after) {
        fe_kahan_add(a.after, a.after_c, static_cast<double>(after));
    }
    if (range) {
        a.lo = fminf(a.lo, after);
        a.hi = fmaxf(a.hi, after);
        if (!(after >= lo && after <= hi)) fe_acc_bad(a, after, index);
    }
    a.changed |= (__float_as_uint(before) != __float_as_uint(after)) ? 1u : 0u;
}

// Per-thread contract accumulators of one checked output of a generated pass. The pass keeps the totals of what it
// writes (sum and sum of |v|: FP64, from fp32 partials of the lane's cells of one plane), the bounds and the change
// flag. The totals before the term are not summed here: they are the totals after the pass that last wrote the field
// (FePassArgs::carry), or fe::launch_totals sums them first. The range/NaN test runs once a plane, on the bounds so far
// and the plane's sum (a NaN or an infinity makes it non-finite); a plane that fails it is read back cell by cell, and
// its bad cells are counted in the block's shared `fails` (out of range, not finite, ~index of the first).
struct FeOutAcc {
    double after, after_abs;
    double after_c;  // compensation of after (fe_kahan_add)
    float pa, paa;  // this plane's fp32 partials of after and |after|
    float lo, hi;   // least and most value so far (NaN ignored)
    unsigned changed;
    unsigned diff;  // this plane's cells' before ^ after, OR-ed (fe_out_plane folds it into changed)
};

__device__ __forceinline__ void fe_out_init(FeOutAcc& a)
{
    a.after = 0.0; a.after_abs = 0.0; a.after_c = 0.0;
    a.pa = 0.f; a.paa = 0.f;
    a.lo = __int_as_float(0x7f800000); a.hi = __int_as_float(0xff800000);
    a.changed = 0u;
    a.diff = 0u;
}

// Four consecutive cells: their values before the pass (for the change flag) and after it. A halo plane's sums and
// change bits are dropped at the plane's end.
__device__ __forceinline__ void fe_out_row4(FeOutAcc& a, const float* before, const float* after, bool range)
{
    a.pa += (after[0] + after[1]) + (after[2] + after[3]);
    a.paa += (fabsf(after[0]) + fabsf(after[1])) + (fabsf(after[2]) + fabsf(after[3]));
    if (range) {
        a.lo = fminf(a.lo, fminf(fminf(after[0], after[1]), fminf(after[2], after[3])));
        a.hi = fmaxf(a.hi, fmaxf(fmaxf(after[0], after[1]), fmaxf(after[2], after[3])));
    }
    // One three-input logic op a cell ((b ^ a) | diff); the test against zero waits for the plane's end.
#pragma unroll
    for (int q = 0; q < 4; ++q) a.diff |= __float_as_uint(before[q]) ^ __float_as_uint(after[q]);
}

// Ends a plane: its partials into the FP64 totals. True when the plane may hold a bad cell (a bound past the declared
// range, or a non-finite sum): the caller reads the plane's cells back. Once a cell is bad the bounds stay past the
// range, so every later plane of the pass is read back too, and each bad cell is counted once, in its own plane.
__device__ __forceinline__ bool fe_out_plane(FeOutAcc& a, float lo, float hi, bool range)
{
    a.changed |= a.diff != 0u ? 1u : 0u;
    a.diff = 0u;
    const bool suspect = range && !(a.lo >= lo && a.hi <= hi && fabsf(a.pa) <= 3.0e38f);
    fe_kahan_add(a.after, a.after_c, static_cast<double>(a.pa));
    a.after_abs += static_cast<double>(a.paa);
    a.pa = 0.f;
    a.paa = 0.f;
    return suspect;
}

__device__ __forceinline__ void fe_out_bad(unsigned* fails, float v, unsigned index)
{
    atomicAdd(&fails[fe_not_finite(v) ? 1 : 0], 1u);
    atomicMax(&fails[2], ~index);
}

// One cell (the plain passes): FP64 totals straight away, the range test per cell.
__device__ __forceinline__ void fe_out_cell(FeOutAcc& a, float before, float after, float lo, float hi, unsigned index, bool range,
    unsigned* fails)
{
    fe_kahan_add(a.after, a.after_c, static_cast<double>(after));
    a.after_abs += static_cast<double>(fabsf(after));
    if (range) {
        a.lo = fminf(a.lo, after);
        a.hi = fmaxf(a.hi, after);
        if (!(after >= lo && after <= hi)) fe_out_bad(fails, after, index);
    }
    a.changed |= (__float_as_uint(before) != __float_as_uint(after)) ? 1u : 0u;
}

// The block's output accumulators into its partial slot (fixed-order sums; the before slots stay zero), the order-free
// parts into the record. Every thread of the block calls it; `fails` is the block's shared tally.
__device__ __forceinline__ void fe_out_block(FeOutAcc& a, double* scratch, double* partial, FeCheck* rec, const unsigned* fails)
{
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    const double s2 = fe_warp_sum_c(a.after, a.after_c);
    const double s3 = fe_warp_sum(a.after_abs);
    const unsigned lo = fe_warp_min(a.lo <= a.hi ? fe_order_key(a.lo) : 0xffffffffu);
    const unsigned hi = fe_warp_max(a.lo <= a.hi ? fe_order_key(a.hi) : 0u);
    const unsigned changed = __any_sync(0xffffffffu, a.changed != 0u) ? 1u : 0u;
    if (lane == 0) {
        scratch[4 * warp + 2] = s2;
        scratch[4 * warp + 3] = s3;
        if (lo != 0xffffffffu) atomicMax(&rec->lo_inv, ~lo);
        if (hi != 0u) atomicMax(&rec->hi_key, hi);
        if (changed && rec->changed == 0u) rec->changed = 1u;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t2 = 0.0, t3 = 0.0, c2 = 0.0;
        for (int w = 0; w < warps; ++w) {
            fe_kahan_add(t2, c2, scratch[4 * w + 2]);
            t3 += scratch[4 * w + 3];
        }
        t2 += c2;
        partial[0] = 0.0;
        partial[1] = 0.0;
        partial[2] = t2;
        partial[3] = t3;
        if (fails[0]) atomicAdd(&rec->out_of_range, fails[0]);
        if (fails[1]) atomicAdd(&rec->not_finite, fails[1]);
        if (fails[2]) atomicMax(&rec->first_bad, fails[2]);
    }
}

// The block's contract accumulators into its partial slot (fixed-order sums), plus the order-free integer parts
// straight into the record. `scratch` holds 4 doubles per warp. Every thread of the block calls it.
__device__ __forceinline__ void fe_acc_block(FeAcc& a, double* scratch, double* partial, FeCheck* rec)
{
    fe_acc_flush(a);
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    const double s0 = fe_warp_sum_c(a.before, a.before_c);
    const double s1 = fe_warp_sum(a.before_abs);
    const double s2 = fe_warp_sum_c(a.after, a.after_c);
    const double s3 = fe_warp_sum(a.after_abs);
    // Float bounds to ordered keys (no finite-or-infinite value seen: the empty keys).
    const unsigned lo = fe_warp_min(a.lo <= a.hi ? fe_order_key(a.lo) : 0xffffffffu);
    const unsigned hi = fe_warp_max(a.lo <= a.hi ? fe_order_key(a.hi) : 0u);
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
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0, c0 = 0.0, c2 = 0.0;
        for (int w = 0; w < warps; ++w) {
            fe_kahan_add(t0, c0, scratch[4 * w + 0]);
            t1 += scratch[4 * w + 1];
            fe_kahan_add(t2, c2, scratch[4 * w + 2]);
            t3 += scratch[4 * w + 3];
        }
        t0 += c0;
        t2 += c2;
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
    FeCheck* rec, bool totals_before, bool totals_after, const FeCheck* carry = nullptr)
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
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0, c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) {
        const volatile double* p = partials + 4 * b;
        fe_kahan_add(t0, c0, p[0]);
        fe_kahan_add(t1, c1, p[1]);
        fe_kahan_add(t2, c2, p[2]);
        fe_kahan_add(t3, c3, p[3]);
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = (blockDim.x + 31) >> 5;
    t0 = fe_warp_sum_c(t0, c0);
    t1 = fe_warp_sum_c(t1, c1);
    t2 = fe_warp_sum_c(t2, c2);
    t3 = fe_warp_sum_c(t3, c3);
    __syncthreads();
    if (lane == 0) {
        scratch[4 * warp + 0] = t0;
        scratch[4 * warp + 1] = t1;
        scratch[4 * warp + 2] = t2;
        scratch[4 * warp + 3] = t3;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0, k0 = 0.0, k1 = 0.0, k2 = 0.0, k3 = 0.0;
        for (int w = 0; w < warps; ++w) {
            fe_kahan_add(s0, k0, scratch[4 * w + 0]);
            fe_kahan_add(s1, k1, scratch[4 * w + 1]);
            fe_kahan_add(s2, k2, scratch[4 * w + 2]);
            fe_kahan_add(s3, k3, scratch[4 * w + 3]);
        }
        s0 += k0;
        s1 += k1;
        s2 += k2;
        s3 += k3;
        if (carry != nullptr) {
            // The totals after the pass that last wrote the field are the totals before this one.
            rec->before = carry->after;
            rec->before_abs = carry->after_abs;
        } else if (totals_before) {
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

// ---- the generated passes' skeletons -------------------------------------------------------------------------------
// A pass traits struct P (generated per pass) gives the lattice (NX, NY, NZ), the tile (W warps x R rows, 128 cells
// wide), the sources' halos (ax(k) a multiple of 4, ry(k), one RZ), the ring depth NST, the smem layout (base, pl, px),
// which outputs carry contracts (checked(j)), and `cell(ctx, x, y, z, out, before)`, which evaluates every output of the
// pass at one cell.

// A compile-time flag passed by value, for the generic lambdas of the pass skeletons.
template <bool B>
struct FeFlag {
    static constexpr bool value = B;
};

// Shared-memory reads of the staged sources: ld<k>(X, Y, Z) is source k at lattice cell (X, Y, Z), which the pass's
// halos guarantee lies in the staged box.
//
// Plane carry (P::ZCARRY, passes with RZ = 1 whose every read below the cell's plane is the cell's own column, one
// plane down): a source with such reads (P::cslot(k) >= 0) keeps the lane's own cells of plane z - 1 (R rows of 4) in
// registers, captured while plane z - 1 was computed. The ring then holds planes z and z + 1 only, and a plane's stage
// is handed back as soon as the plane is computed.
template <class P>
struct FeSlabCtx {
    const float* sm;
    int slots[2 * P::RZ + 1]; // the ring stage of plane z + d at slots[d + RZ]
    int x0, y0, z;
    int xl, yl;               // the lane's first column and the warp's first row
    float dt;
    float carry[P::NCARRY > 0 ? P::NCARRY : 1][P::R][4];
    // The stage of plane Z (|Z - z| <= RZ): a chain of selects, so the table stays in registers whatever Z is.
    __device__ __forceinline__ int stage(int Z) const
    {
        const int d = Z - z + P::RZ;
        int s = slots[0];
#pragma unroll
        for (int i = 1; i < 2 * P::RZ + 1; ++i) s = d == i ? slots[i] : s;
        return s;
    }
    // A carried cell by its row and column within the lane's: constants in the clamp-free code, a chain of selects
    // (no indexed register array) where clamps leave them to run time.
    __device__ __forceinline__ float pick(const float (&cr)[P::R][4], int dr, int dq) const
    {
        float v = cr[0][0];
#pragma unroll
        for (int r = 0; r < P::R; ++r) {
#pragma unroll
            for (int q = 0; q < 4; ++q) v = (dr == r && dq == q) ? cr[r][q] : v;
        }
        return v;
    }
    template <int k>
    __device__ __forceinline__ float ld(int X, int Y, int Z) const
    {
        if constexpr (P::ZCARRY && P::cslot(k) >= 0) {
            if (Z < z) return pick(carry[P::cslot(k)], Y - yl, X - xl);
        }
        return sm[P::base(k) + stage(Z) * P::pl(k) + (Y - y0 + P::ry(k)) * P::px(k) + (X - x0 + P::ax(k))];
    }
};

// For passes whose x edge the halo can carry (P::XFILL): after a plane lands in ring stage `stage`, the staged columns
// past the lattice's x
// edge get the edge cell's value, what a clamped read returns there. Only the CTAs at an x edge do anything; one row a
// thread.
template <class P>
__device__ __forceinline__ void fe_fill_x_edges(float* sm, int stage, int x0)
{
    if (!P::XFILL) return;
    const bool left = x0 == 0;
    const int inside = P::NX - x0; // columns of this tile inside the lattice
    const bool right = x0 + 128 >= P::NX;
    if (!left && !right) return;
#pragma unroll
    for (int k = 0; k < P::NSRC; ++k) {
        const int ax = P::ax(k);
        if (ax == 0) continue;
        const int rows = P::W * P::R + 2 * P::ry(k);
        const int px = P::px(k);
        float* plane = sm + P::base(k) + stage * P::pl(k);
        for (int row = threadIdx.x; row < rows; row += blockDim.x) {
            float* r = plane + row * px;
            if (left) {
                const float edge = r[ax];
                for (int c = 0; c < ax; ++c) r[c] = edge;
            }
            if (right) {
                const int first_out = ax + min(inside, 128);
                const float edge = r[first_out - 1];
                for (int c = first_out; c < px; ++c) r[c] = edge;
            }
        }
    }
}

// Global-memory reads (through the read-only path), for passes the TMA cannot stage (an x extent not a multiple of 4).
template <class P>
struct FePlainCtx {
    const float* const* src;
    float dt;
    template <int k>
    __device__ __forceinline__ float ld(int X, int Y, int Z) const
    {
        return __ldg(src[k] + (static_cast<fe_u64>(Z) * P::NY + static_cast<fe_u64>(Y)) * P::NX + static_cast<fe_u64>(X));
    }
};

template <class P>
__device__ __forceinline__ void fe_pass_contracts(FeOutAcc* acc, double* scratch, unsigned (*fails)[3], const FePassArgs& a)
{
    const int block = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const int blocks = gridDim.x * gridDim.y * gridDim.z;
#pragma unroll
    for (int j = 0; j < P::NOUT; ++j) {
        if (P::checked(j) && a.rec[j] != nullptr) {
            fe_out_block(acc[j], scratch, a.partials + 4 * (static_cast<fe_u64>(j) * blocks + block), a.rec[j], fails[j]);
            fe_acc_finish(a.partials + 4 * static_cast<fe_u64>(j) * blocks, blocks, a.count + j, scratch, a.rec[j], false,
                (a.flags & FE_PASS_AFTER) != 0, a.carry[j]);
        }
    }
}

// The carried sources' cells of row r of plane z (the lane's 4 columns), into the plane carry (P::ZCARRY).
template <class P, int K = 0>
__device__ __forceinline__ void fe_carry_row(FeSlabCtx<P>& c, int r, int x, int y, int z)
{
    if constexpr (K < P::NSRC) {
        if constexpr (P::cslot(K) >= 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q) c.carry[P::cslot(K)][r][q] = c.template ld<K>(x + q, y, z);
        }
        fe_carry_row<P, K + 1>(c, r, x, y, z);
    }
}

// The TMA z-marching pass: a CTA owns a 128 x TY column and marches a chunk of z-planes; every source's plane (with its
// halo) comes into a ring of NST stages by one TMA load each, NST - 2 RZ - 1 planes ahead (NST - RZ - 1 with the plane
// carry); one mbarrier a stage counts the bytes of all sources. A lane computes 4 consecutive cells on R rows and stores
// them as float4. HALO: the handle holds halo planes another rank owns (a lattice split in z-slabs), left out of the
// contracts.
template <class P, bool HALO = false>
__device__ __forceinline__ void fe_slab_pass(const FePassArgs& a)
{
    extern __shared__ __align__(128) float fe_sm[];
    __shared__ __align__(8) fe_u64 bar[P::NST];
    __shared__ double scratch[4 * P::W];
    __shared__ unsigned fails[P::NOUT][3];
    static_assert(P::NST >= (P::ZCARRY ? P::RZ + 2 : 2 * P::RZ + 2),
        "the ring holds the planes a z reads from shared memory and the one being fetched");
    static_assert(!P::ZCARRY || P::RZ == 1, "the plane carry holds one plane");
    const int x0 = blockIdx.x * 128;
    const int y0 = blockIdx.y * (P::W * P::R);
    const int zb = blockIdx.z * a.zchunk;
    const int ze = min(P::NZ, zb + a.zchunk);
    const int zlo = max(zb - P::RZ, 0);
    const int zhi = min(ze - 1 + P::RZ, P::NZ - 1);
    const int nplanes = zhi - zlo + 1;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    // Plane j of the chunk (lattice plane zlo + j) lands in ring stage j % NST, in phase (j / NST) & 1 of its barrier.
    auto issue = [&](int j) {
        const int st = j % P::NST;
        fe_mbar_expect_tx(&bar[st], P::BYTES);
#pragma unroll
        for (int k = 0; k < P::NSRC; ++k) {
            fe_tma_load_3d(fe_sm + P::base(k) + st * P::pl(k), &a.map[k], &bar[st], x0 - P::ax(k), y0 - P::ry(k), zlo + j);
        }
    };
    int issued = 0;
    if (threadIdx.x == 0) {
        for (int j = 0; j < P::NOUT; ++j) fails[j][0] = fails[j][1] = fails[j][2] = 0u;
        for (int s = 0; s < P::NST; ++s) fe_mbar_init(&bar[s], 1);
        fe_fence_mbar_init();
        issued = min(P::NST, nplanes);
        for (int j = 0; j < issued; ++j) issue(j);
    }
    __syncthreads();
    FeOutAcc acc[P::NOUT];
#pragma unroll
    for (int j = 0; j < P::NOUT; ++j) fe_out_init(acc[j]);
    // Every thread waits (bounded) for the planes a z needs, and evens the x edge of each plane that landed (XFILL);
    // the barrier that follows makes both visible and, OR-ing the outcomes, the decision to go on uniform. The next
    // plane to wait for is tracked by its stage and phase, stepped rather than divided.
    int waited = 0;
    int wst = 0;
    unsigned wpar = 0u;
    bool ok = true;
    const bool edge = P::XFILL && (x0 == 0 || x0 + 128 >= P::NX);
    auto wait_upto = [&](int j) {
        while (waited <= j) {
            if (!fe_mbar_wait(&bar[wst], wpar, 1u << 20)) ok = false;
            else if (edge) fe_fill_x_edges<P>(fe_sm, wst, x0);
            ++waited;
            if (++wst == P::NST) {
                wst = 0;
                wpar ^= 1u;
            }
        }
    };
    if (zb < ze) wait_upto(min(zb + P::RZ, P::NZ - 1) - zlo);
    const int x = x0 + 4 * lane;
    FeSlabCtx<P> c;
    c.sm = fe_sm;
    c.x0 = x0;
    c.y0 = y0;
    c.xl = x;
    c.yl = y0 + warp * P::R;
    c.dt = a.dt;
    // With the plane carry, a chunk that starts above the lattice's first plane takes plane zb - 1 (ring stage 0, which
    // this thread waited for) into it; the stage goes back to the ring after the barrier.
    const bool carry_in = P::ZCARRY && zb > zlo;
    if (carry_in && ok) {
        c.z = zlo;
#pragma unroll
        for (int d = 0; d < 2 * P::RZ + 1; ++d) c.slots[d] = 0;
#pragma unroll
        for (int r = 0; r < P::R; ++r) fe_carry_row<P>(c, r, x, y0 + warp * P::R + r, zlo);
    }
    bool failed = __syncthreads_or(ok ? 0 : 1) != 0;
    int released = 0; // thread 0's next plane to hand back to the ring
    if (carry_in && threadIdx.x == 0 && !failed) {
        if (P::NST < nplanes) {
            if (edge) fe_fence_proxy_async();
            issue(P::NST);
            issued = P::NST + 1;
        }
        released = 1;
    }
    // With the x edge carried by the halo, whether a row's cells are interior depends only on the row and the plane, so
    // a warp takes one path. Which of this warp's rows lie in the lattice, and which have their whole y reach inside
    // it, are fixed for the pass.
    const bool xin = P::XFILL || (x - P::RXT >= 0 && x + 3 + P::RXT < P::NX);
    constexpr bool ragged = (P::NY % (P::W * P::R)) != 0 || (P::NX % 128) != 0;
    unsigned live = 0u;
    unsigned yin = 0u;
#pragma unroll
    for (int r = 0; r < P::R; ++r) {
        const int y = y0 + warp * P::R + r;
        if (y < P::NY && x < P::NX) live |= 1u << r;
        if (y - P::RYT >= 0 && y + P::RYT < P::NY) yin |= 1u << r;
    }
    constexpr unsigned all_rows = (1u << P::R) - 1u;
    const bool range = (a.flags & FE_PASS_RANGE) != 0;
    const fe_u64 row0 = static_cast<fe_u64>(P::NX) * static_cast<fe_u64>(y0 + warp * P::R) + static_cast<fe_u64>(x);
    // The ring stage of plane z, stepped with z; planes whose z reach stays in the lattice take their neighbours'
    // stages from it, the clamped ones at the lattice's z ends recompute them.
    int sz = zb - zlo;
    for (int z = zb; z < ze && !failed; ++z) {
        // Halo planes (another rank's) are computed like the rest; their contributions to the contracts are dropped.
        const bool own = !HALO || (z >= a.own_z0 && z < a.own_z1);
        const bool range_here = range && own;
        c.z = z;
        if (z - P::RZ >= 0 && z + P::RZ < P::NZ) {
#pragma unroll
            for (int d = -P::RZ; d <= P::RZ; ++d) {
                int st = sz + d;
                if (d < 0 && st < 0) st += P::NST;
                if (d > 0 && st >= P::NST) st -= P::NST;
                c.slots[d + P::RZ] = st;
            }
        } else {
#pragma unroll
            for (int d = -P::RZ; d <= P::RZ; ++d) c.slots[d + P::RZ] = (min(max(z + d, 0), P::NZ - 1) - zlo) % P::NST;
        }
        const bool plane_in = xin && z - P::RZT >= 0 && z + P::RZT < P::NZ;
        const fe_u64 plane0 = static_cast<fe_u64>(P::NX) * static_cast<fe_u64>(P::NY) * static_cast<fe_u64>(z) + row0;
        // One row of four cells, clamp-free (IN) or clamped. The stores name the global space, so the compiler may
        // move the next row's shared-memory loads above them. A checked output's sums, bounds and change bits are taken
        // whether or not the launch asked for them (no branch a row): a launch without a record never reads them, and
        // one without the range test has its bounds emptied before they are folded (a halo plane's stay out by test).
        auto row = [&](int r, auto in) {
            constexpr bool IN = decltype(in)::value;
            const int y = y0 + warp * P::R + r;
            float o[4][P::NOUT];
            float b[4][P::NOUT];
#pragma unroll
            for (int q = 0; q < 4; ++q) P::template cell<IN>(c, x + q, y, z, o[q], b[q]);
            // The row's cells of plane z replace those of plane z - 1 in the carry (read above, by this row only).
            if constexpr (P::ZCARRY) fe_carry_row<P>(c, r, x, y, z);
            const fe_u64 at = plane0 + static_cast<fe_u64>(r) * P::NX;
#pragma unroll
            for (int j = 0; j < P::NOUT; ++j) {
                __stwb(reinterpret_cast<float4*>(a.out[j] + at), make_float4(o[0][j], o[1][j], o[2][j], o[3][j]));
                if (P::checked(j)) {
                    const float bb[4] = {b[0][j], b[1][j], b[2][j], b[3][j]};
                    const float oo[4] = {o[0][j], o[1][j], o[2][j], o[3][j]};
                    fe_out_row4(acc[j], bb, oo, HALO ? range_here : true);
                }
            }
        };
        if (plane_in && yin == all_rows && (!ragged || live == all_rows)) {
            // The tile's whole plane is inside the lattice with its reach: its R rows are one branch-free block.
#pragma unroll
            for (int r = 0; r < P::R; ++r) row(r, FeFlag<true>{});
        } else {
#pragma unroll
            for (int r = 0; r < P::R; ++r) {
                if (ragged && !((live >> r) & 1u)) continue;
                // Four cells whose whole reach is inside the lattice take the clamp-free code; the rest the clamped one.
                if (plane_in && ((yin >> r) & 1u)) row(r, FeFlag<true>{});
                else row(r, FeFlag<false>{});
            }
        }
#pragma unroll
        for (int j = 0; j < P::NOUT; ++j) {
            if (!own) {
                acc[j].pa = 0.f;
                acc[j].paa = 0.f;
                acc[j].diff = 0u;
            } else if (P::checked(j) && a.rec[j] != nullptr && fe_out_plane(acc[j], a.lo[j], a.hi[j], range)) {
                // Read this lane's cells of the plane back (its own stores, through L2) and tally the bad ones.
#pragma unroll
                for (int r = 0; r < P::R; ++r) {
                    if (ragged && !((live >> r) & 1u)) continue;
                    const fe_u64 at = plane0 + static_cast<fe_u64>(r) * P::NX;
                    const float4 v4 = __ldcg(reinterpret_cast<const float4*>(a.out[j] + at));
                    const float v[4] = {v4.x, v4.y, v4.z, v4.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        if (!(v[q] >= a.lo[j] && v[q] <= a.hi[j])) fe_out_bad(fails[j], v[q], static_cast<unsigned>(at) + q);
                    }
                }
            }
        }
        if (z + 1 < ze) wait_upto(min(z + 1 + P::RZ, P::NZ - 1) - zlo);
        failed = __syncthreads_or(ok ? 0 : 1) != 0;
        // The planes no later z reads from shared memory go back to the ring: plane z - RZ, or plane z itself with the
        // carry. Their last readers passed the barrier above; only the x-edge fill wrote them through the generic proxy,
        // and those writes must be ordered before the TMA overwrites them.
        if (threadIdx.x == 0 && !failed) {
            const int upto = z - (P::ZCARRY ? 0 : P::RZ) - zlo;
            if (released <= upto && released + P::NST < nplanes && edge) fe_fence_proxy_async();
            while (released <= upto && released + P::NST < nplanes) {
                issue(released + P::NST);
                issued = released + P::NST + 1;
                ++released;
            }
        }
        if (++sz == P::NST) sz = 0;
    }
    if (failed) {
        if (threadIdx.x == 0) {
            atomicOr(a.err, FE_ERR_MBAR_TIMEOUT);
            for (int j = 0; j < issued; ++j) fe_mbar_wait(&bar[j % P::NST], static_cast<unsigned>((j / P::NST) & 1), 1u << 16);
        }
        return;
    }
    if (!range) {
#pragma unroll
        for (int j = 0; j < P::NOUT; ++j) {
            acc[j].lo = __int_as_float(0x7f800000);
            acc[j].hi = __int_as_float(0xff800000);
        }
    }
    fe_pass_contracts<P>(acc, scratch, fails, a);
}

// The plain pass: a thread a (x, y) column marching a chunk of z-planes, reads through the read-only path.
template <class P, bool HALO = false>
__device__ __forceinline__ void fe_plain_pass(const FePassArgs& a)
{
    __shared__ double scratch[4 * 8];
    __shared__ unsigned fails[P::NOUT][3];
    const int x = blockIdx.x * 32 + (threadIdx.x & 31);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 5);
    const bool live = x < P::NX && y < P::NY;
    const int zb = blockIdx.z * a.zchunk;
    const int ze = min(P::NZ, zb + a.zchunk);
    if (threadIdx.x < 3 * P::NOUT) fails[threadIdx.x / 3][threadIdx.x % 3] = 0u;
    __syncthreads();
    const bool range = (a.flags & FE_PASS_RANGE) != 0;
    FeOutAcc acc[P::NOUT];
#pragma unroll
    for (int j = 0; j < P::NOUT; ++j) fe_out_init(acc[j]);
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    for (int z = zb; live && z < ze; ++z) {
        float o[P::NOUT];
        float b[P::NOUT];
        P::template cell<false>(c, x, y, z, o, b);
        const fe_u64 at = static_cast<fe_u64>(x) + static_cast<fe_u64>(P::NX) * (static_cast<fe_u64>(y) + static_cast<fe_u64>(P::NY) * z);
#pragma unroll
        for (int j = 0; j < P::NOUT; ++j) {
            a.out[j][at] = o[j];
            if (P::checked(j) && a.rec[j] != nullptr && (!HALO || (z >= a.own_z0 && z < a.own_z1))) {
                fe_out_cell(acc[j], b[j], o[j], a.lo[j], a.hi[j], static_cast<unsigned>(at), range, fails[j]);
            }
        }
    }
    fe_pass_contracts<P>(acc, scratch, fails, a);
}

// The seed pass of a distance (DIST) or poisson op: its argument at every cell against what was last solved, kept in
// out[0]; when any cell differs, the flag is raised and the solve kernels after it run. distance: the seed is 0 where the
// argument is at least 0.5 (solid) and 1e30 elsewhere, out[1] the complement; poisson: out[0] the source itself.
template <class P, int DIST>
__device__ __forceinline__ void fe_seed_pass(const FePassArgs& a)
{
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    const fe_u64 cells = static_cast<fe_u64>(P::NX) * P::NY * P::NZ;
    const fe_u64 stride = static_cast<fe_u64>(gridDim.x) * blockDim.x;
    bool changed = false;
    for (fe_u64 i = blockIdx.x * static_cast<fe_u64>(blockDim.x) + threadIdx.x; i < cells; i += stride) {
        const int x = static_cast<int>(i % P::NX);
        const int y = static_cast<int>((i / P::NX) % P::NY);
        const int z = static_cast<int>(i / (static_cast<fe_u64>(P::NX) * P::NY));
        const float v = P::value(c, x, y, z);
        const float seed = DIST ? (v >= 0.5f ? 0.f : 1e30f) : v;
        if (__float_as_uint(a.out[0][i]) != __float_as_uint(seed)) {
            a.out[0][i] = seed;
            if (DIST) a.out[1][i] = seed == 0.f ? 1e30f : 0.f;
            changed = true;
        }
    }
    if (__any_sync(0xffffffffu, changed) && (threadIdx.x & 31) == 0) atomicOr(a.flag, 1u);
}

// A deterministic reduction of one expression over the lattice (maxof / minof / sumof): a fixed assignment of cells to
// threads, FP64 sums, a fixed tree, then the last block folds the blocks in order. The result lands in *out.
template <class P>
__device__ __forceinline__ void fe_reduce_pass(const FePassArgs& a, float* out)
{
    __shared__ double scratch[4 * 8];
    __shared__ unsigned last;
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    const fe_u64 cells = static_cast<fe_u64>(P::NX) * P::NY * P::NZ;
    double sum = 0.0;
    float lo = 3.0e38f, hi = -3.0e38f;
    const fe_u64 stride = static_cast<fe_u64>(gridDim.x) * blockDim.x;
    for (fe_u64 i = blockIdx.x * static_cast<fe_u64>(blockDim.x) + threadIdx.x; i < cells; i += stride) {
        const int x = static_cast<int>(i % P::NX);
        const int y = static_cast<int>((i / P::NX) % P::NY);
        const int z = static_cast<int>(i / (static_cast<fe_u64>(P::NX) * P::NY));
        const float v = P::value(c, x, y, z);
        sum += static_cast<double>(v);
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    sum = fe_warp_sum(sum);
    for (int o = 16; o > 0; o >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
        scratch[4 * warp] = sum;
        scratch[4 * warp + 1] = lo;
        scratch[4 * warp + 2] = hi;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        float l = 3.0e38f, h = -3.0e38f;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            s += scratch[4 * w];
            l = fminf(l, static_cast<float>(scratch[4 * w + 1]));
            h = fmaxf(h, static_cast<float>(scratch[4 * w + 2]));
        }
        a.partials[4 * blockIdx.x] = s;
        a.partials[4 * blockIdx.x + 1] = l;
        a.partials[4 * blockIdx.x + 2] = h;
        __threadfence();
        const unsigned done = atomicAdd(a.count, 1u);
        last = done + 1u == gridDim.x ? 1u : 0u;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double s = 0.0;
        float l = 3.0e38f, h = -3.0e38f;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            const volatile double* p = a.partials + 4 * b;
            s += p[0];
            l = fminf(l, static_cast<float>(p[1]));
            h = fmaxf(h, static_cast<float>(p[2]));
        }
        *out = P::KIND == 0 ? static_cast<float>(s) : (P::KIND == 1 ? h : l);
        *a.count = 0u;
    }
}

// ---- tridiagonal solves: the partition method (per-lane Thomas sweeps, PCR across lanes) -----------------------------

// 1 / x by the hardware approximation (rcp.approx, about 1 ulp), for solves checked to a tolerance.
__device__ __forceinline__ float fe_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The reduced system of a segment of K lanes (a power of two, 2..32): lane k holds two equations, row 2k
// (a0 x[2k-1] + b0 x[2k] + c0 x[2k+1] = d0) and row 2k+1 (a1 x[2k] + b1 x[2k+1] + c1 x[2k+2] = d1), solved by parallel
// cyclic reduction over log2(2K) rounds of shuffles. Returns x[2k] in `first` and x[2k+1] in `last`. Every lane of the
// warp must call it.
template <bool RN = false>
__device__ __forceinline__ void fe_pcr_pairs(float a0, float b0, float c0, float d0, float a1, float b1, float c1, float d1,
    int k, int K, float& first, float& last)
{
    auto rcp = [](float x) { return RN ? __frcp_rn(x) : fe_rcp(x); };
    const unsigned mask = 0xffffffffu;
    for (int s = 1; s < 2 * K; s *= 2) {
        const int q = s == 1 ? 1 : s / 2;
        const bool has_lo = k - q >= 0, has_hi = k + q < K;
        const float p0a = __shfl_up_sync(mask, s == 1 ? a1 : a0, q, K), p0b = __shfl_up_sync(mask, s == 1 ? b1 : b0, q, K);
        const float p0c = __shfl_up_sync(mask, s == 1 ? c1 : c0, q, K), p0d = __shfl_up_sync(mask, s == 1 ? d1 : d0, q, K);
        const float q1a = __shfl_down_sync(mask, s == 1 ? a0 : a1, q, K), q1b = __shfl_down_sync(mask, s == 1 ? b0 : b1, q, K);
        const float q1c = __shfl_down_sync(mask, s == 1 ? c0 : c1, q, K), q1d = __shfl_down_sync(mask, s == 1 ? d0 : d1, q, K);
        float q0a, q0b, q0c, q0d, p1a, p1b, p1c, p1d;
        if (s == 1) {
            q0a = a1; q0b = b1; q0c = c1; q0d = d1;
            p1a = a0; p1b = b0; p1c = c0; p1d = d0;
        } else {
            q0a = __shfl_down_sync(mask, a0, q, K); q0b = __shfl_down_sync(mask, b0, q, K);
            q0c = __shfl_down_sync(mask, c0, q, K); q0d = __shfl_down_sync(mask, d0, q, K);
            p1a = __shfl_up_sync(mask, a1, q, K); p1b = __shfl_up_sync(mask, b1, q, K);
            p1c = __shfl_up_sync(mask, c1, q, K); p1d = __shfl_up_sync(mask, d1, q, K);
        }
        // Missing neighbours are identity rows.
        const bool lo0 = has_lo, hi0 = s == 1 ? true : has_hi, lo1 = s == 1 ? true : has_lo, hi1 = has_hi;
        const float la0 = lo0 ? p0a : 0.f, lb0 = lo0 ? p0b : 1.f, lc0 = lo0 ? p0c : 0.f, ld0 = lo0 ? p0d : 0.f;
        const float ua0 = hi0 ? q0a : 0.f, ub0 = hi0 ? q0b : 1.f, uc0 = hi0 ? q0c : 0.f, ud0 = hi0 ? q0d : 0.f;
        const float la1 = lo1 ? p1a : 0.f, lb1 = lo1 ? p1b : 1.f, lc1 = lo1 ? p1c : 0.f, ld1 = lo1 ? p1d : 0.f;
        const float ua1 = hi1 ? q1a : 0.f, ub1 = hi1 ? q1b : 1.f, uc1 = hi1 ? q1c : 0.f, ud1 = hi1 ? q1d : 0.f;
        const float k10 = a0 * rcp(lb0), k20 = c0 * rcp(ub0), k11 = a1 * rcp(lb1), k21 = c1 * rcp(ub1);
        const float na0 = -k10 * la0, nc0 = -k20 * uc0, nb0 = b0 - k10 * lc0 - k20 * ua0, nd0 = d0 - k10 * ld0 - k20 * ud0;
        const float na1 = -k11 * la1, nc1 = -k21 * uc1, nb1 = b1 - k11 * lc1 - k21 * ua1, nd1 = d1 - k11 * ld1 - k21 * ud1;
        a0 = na0; b0 = nb0; c0 = nc0; d0 = nd0;
        a1 = na1; b1 = nb1; c1 = nc1; d1 = nd1;
    }
    first = d0 * rcp(b0);
    last = d1 * rcp(b1);
}

// One line of n <= 32 M rows (a power-of-two K = 32 lanes, M rows a lane: lane k rows k M .. k M + M - 1) with its own
// coefficients in every row: a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i], the edge repeat already folded (a = 0 in
// the line's first row, c = 0 in its last) and rows past the line's end the identity (a = c = d = 0, b = 1).
// 1. Each lane eliminates inside its rows: a sweep down leaves its last row in terms of its first and the next lane's
//    first unknown; a sweep up leaves every row in terms of the previous row, itself and the lane's last unknown.
// 2. The lanes' first and last unknowns (a tridiagonal system of 64) by parallel cyclic reduction over shuffles.
// 3. Each lane's interior rows by back-substitution. On return d holds the solution. Every lane of the warp calls it.
// Reciprocals are correctly rounded (the law's own solves are held to the reference's CPU solver to a tolerance).
// With M = 1 a lane would hold one row: M >= 2.
template <int M>
__device__ __forceinline__ void fe_tri_line(float (&a)[M], float (&b)[M], float (&c)[M], float (&d)[M], int k)
{
    static_assert(M >= 2, "two rows a lane at least");
    float al = a[1], be = b[1], de = d[1];
#pragma unroll
    for (int r = 2; r < M; ++r) {
        const float f = a[r] * __frcp_rn(be);
        al = -f * al;
        be = b[r] - f * c[r - 1];
        de = d[r] - f * de;
    }
    // Up, in place: b[r] becomes 1 / (row r's diagonal), c[r] the coefficient of the lane's last unknown.
    float diag0 = b[M - 2];
    b[M - 2] = __frcp_rn(diag0);
#pragma unroll
    for (int r = M - 3; r >= 0; --r) {
        const float g = c[r] * b[r + 1];
        diag0 = b[r] - g * a[r + 1];
        c[r] = -g * c[r + 1];
        d[r] = d[r] - g * d[r + 1];
        b[r] = __frcp_rn(diag0);
    }
    float first, last;
    fe_pcr_pairs<true>(a[0], diag0, c[0], d[0], al, be, c[M - 1], de, k, 32, first, last);
    float prev = first;
    d[0] = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        prev = (d[r] - a[r] * prev - c[r] * last) * b[r];
        d[r] = prev;
    }
    d[M - 1] = last;
}

// Tridiagonal solves along x, a warp a line (the partition method, fe_tri_line; M = ceil(NX / 32) rows a lane): the
// warp forms the line's coefficients 32 consecutive cells at a time (coalesced reads), stages them in its shared
// memory (padded one word in 32 so a lane's M consecutive rows fall in different banks), each lane takes its M rows,
// the warp solves, and the answer goes back out through the same staging, coalesced. Lines: NY * NZ, WARPS a block.
template <class P, int M, int WARPS>
__device__ __forceinline__ void fe_tridiag_x_warp(const FePassArgs& a)
{
    constexpr int S = 32 * M + M; // a staged row of 32 M cells, padded
    extern __shared__ __align__(128) float fe_sm[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float* sa = fe_sm + warp * 4 * S;
    float* sb = sa + S;
    float* sc = sb + S;
    float* sd = sc + S;
    const fe_u64 line = static_cast<fe_u64>(blockIdx.x) * WARPS + warp;
    if (line >= static_cast<fe_u64>(P::NY) * P::NZ) return; // a whole warp leaves together
    const int y = static_cast<int>(line % P::NY);
    const int z = static_cast<int>(line / P::NY);
    FePlainCtx<P> ctx;
    ctx.src = a.src;
    ctx.dt = a.dt;
    auto pad = [](int i) { return i + (i >> 5); };
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const int x = i * 32 + lane;
        float lo = 0.f, di = 1.f, up = 0.f, rhs = 0.f;
        if (x < P::NX) {
            P::coef(ctx, x, y, z, lo, di, up, rhs);
            if (x == 0) { di += lo; lo = 0.f; }
            if (x + 1 == P::NX) { di += up; up = 0.f; }
        }
        sa[pad(x)] = lo;
        sb[pad(x)] = di;
        sc[pad(x)] = up;
        sd[pad(x)] = rhs;
    }
    __syncwarp();
    float ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int i = pad(lane * M + r);
        ra[r] = sa[i];
        rb[r] = sb[i];
        rc[r] = sc[i];
        rd[r] = sd[i];
    }
    fe_tri_line<M>(ra, rb, rc, rd, lane);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < M; ++r) sd[pad(lane * M + r)] = rd[r];
    __syncwarp();
    float* out = a.out[0] + (static_cast<fe_u64>(z) * P::NY + y) * P::NX;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const int x = i * 32 + lane;
        if (x < P::NX) out[x] = sd[pad(x)];
    }
}

// Tridiagonal solves along x, 32 lines a block (32 consecutive y at one z): coefficient tiles come in coalesced through
// shared memory, each thread runs Thomas' recurrence on its line (in the reference's order: the edge cell repeating, its
// missing neighbour's coefficient landing on the diagonal), keeping c' and d' for the whole line in shared memory, so
// global memory sees the coefficients read once and the answer written once. NXS: the x extent kept (>= NX).
template <class P>
__device__ __forceinline__ void fe_tridiag_x_pass(const FePassArgs& a)
{
    extern __shared__ __align__(128) float fe_sm[];
    float* cs = fe_sm;                 // [NX][33]: c' of line tx at x
    float* ds = fe_sm + P::NX * 33;    // [NX][33]: d', then the answer
    __shared__ float ta[32][33], tb[32][33], tu[32][33], td[32][33];
    const int tx = threadIdx.x;
    const int y0 = blockIdx.x * 32;
    const int z = blockIdx.y;
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    float cp = 0.f, dp = 0.f;
    for (int x0 = 0; x0 < P::NX; x0 += 32) {
        const int x = x0 + tx;
        for (int j = 0; j < 32; ++j) {
            const int y = y0 + j;
            float lo = 0.f, di = 1.f, up = 0.f, rhs = 0.f;
            if (x < P::NX && y < P::NY) {
                P::coef(c, x, y, z, lo, di, up, rhs);
                if (x == 0) di += lo;
                if (x + 1 == P::NX) di += up;
            }
            ta[j][tx] = lo;
            tb[j][tx] = di;
            tu[j][tx] = up;
            td[j][tx] = rhs;
        }
        __syncthreads();
        const int m = min(32, P::NX - x0);
        for (int i = 0; i < m; ++i) {
            const float lo = ta[tx][i];
            const float den = tb[tx][i] - lo * cp;
            dp = (td[tx][i] - lo * dp) / den;
            cp = x0 + i + 1 == P::NX ? 0.f : tu[tx][i] / den;
            cs[(x0 + i) * 33 + tx] = cp;
            ds[(x0 + i) * 33 + tx] = dp;
        }
        __syncthreads();
    }
    float next = 0.f;
    for (int i = P::NX - 1; i >= 0; --i) {
        next = ds[i * 33 + tx] - cs[i * 33 + tx] * next;
        ds[i * 33 + tx] = next;
    }
    __syncthreads();
    for (int j = 0; j < 32; ++j) {
        const int y = y0 + j;
        if (y >= P::NY) break;
        for (int x = tx; x < P::NX; x += 32) {
            a.out[0][(static_cast<fe_u64>(z) * P::NY + y) * P::NX + x] = ds[x * 33 + j];
        }
    }
}

// Tridiagonal solves along y or z by the partition method, 32 lines a block (32 consecutive x at one z, or one y), each
// line cut into K segments of M rows: thread (k, line) = threadIdx.x = 32 k + line holds rows k M .. k M + M - 1, so
// every load and store of a warp touches 32 consecutive x (coalesced). Each thread eliminates inside its rows (the
// sweeps of fe_tri_line), leaving two rows that couple its first and last unknowns to the neighbouring segments'; those
// 2 K rows a line go to shared memory, one thread a line solves them (Thomas), and every thread back-substitutes its
// interior rows. Lines: NX x NZ (y) or NX x NY (z); the edge repeat folded at each line's ends, rows past the end the
// identity. Reciprocals correctly rounded.
template <class P, int AXIS, int M, int K>
__device__ __forceinline__ void fe_tridiag_yz_seg(const FePassArgs& a)
{
    static_assert(M >= 2 && K >= 1 && K <= 16, "2 rows a segment at least, at most 16 segments");
    __shared__ float red[32][8 * K + 1]; // per line: its 2 K reduced rows, (a, b, c, d) each
    __shared__ float sol[32][2 * K + 1]; // per line: the segments' first and last unknowns
    const int line = threadIdx.x & 31;
    const int k = threadIdx.x >> 5;
    const int n = AXIS == 1 ? P::NY : P::NZ;
    const int x = blockIdx.x * 32 + line;
    const int other = blockIdx.y; // the z of a y line, the y of a z line
    const bool live = x < P::NX;
    FePlainCtx<P> ctx;
    ctx.src = a.src;
    ctx.dt = a.dt;
    float ra[M], rb[M], rc[M], rd[M];
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int i = k * M + r;
        float lo = 0.f, di = 1.f, up = 0.f, rhs = 0.f;
        if (live && i < n) {
            if (AXIS == 1) P::coef(ctx, x, i, other, lo, di, up, rhs);
            else P::coef(ctx, x, other, i, lo, di, up, rhs);
            if (i == 0) { di += lo; lo = 0.f; }
            if (i + 1 == n) { di += up; up = 0.f; }
        }
        ra[r] = lo;
        rb[r] = di;
        rc[r] = up;
        rd[r] = rhs;
    }
    // Down: the segment's last row in terms of its first unknown, itself and the next segment's first.
    float al = ra[1], be = rb[1], de = rd[1];
#pragma unroll
    for (int r = 2; r < M; ++r) {
        const float f = ra[r] * __frcp_rn(be);
        al = -f * al;
        be = rb[r] - f * rc[r - 1];
        de = rd[r] - f * de;
    }
    // Up, in place: rb[r] becomes 1 / (row r's diagonal), rc[r] the coefficient of the segment's last unknown.
    float diag0 = rb[M - 2];
    rb[M - 2] = __frcp_rn(diag0);
#pragma unroll
    for (int r = M - 3; r >= 0; --r) {
        const float g = rc[r] * rb[r + 1];
        diag0 = rb[r] - g * ra[r + 1];
        rc[r] = -g * rc[r + 1];
        rd[r] = rd[r] - g * rd[r + 1];
        rb[r] = __frcp_rn(diag0);
    }
    float* mine = &red[line][8 * k];
    mine[0] = ra[0]; mine[1] = diag0; mine[2] = rc[0]; mine[3] = rd[0];
    mine[4] = al; mine[5] = be; mine[6] = rc[M - 1]; mine[7] = de;
    __syncthreads();
    if (k == 0) {
        // The line's 2 K reduced rows by Thomas, c' kept in place of the rows' c.
        float* row = &red[line][0];
        float cp = 0.f, dp = 0.f;
        for (int j = 0; j < 2 * K; ++j) {
            const float aj = row[4 * j], bj = row[4 * j + 1], cj = row[4 * j + 2], dj = row[4 * j + 3];
            const float inv = __frcp_rn(bj - aj * cp);
            cp = cj * inv;
            dp = (dj - aj * dp) * inv;
            row[4 * j + 2] = cp;
            row[4 * j + 3] = dp;
        }
        float next = 0.f;
        for (int j = 2 * K - 1; j >= 0; --j) {
            next = row[4 * j + 3] - row[4 * j + 2] * next;
            sol[line][j] = next;
        }
    }
    __syncthreads();
    const float first = sol[line][2 * k], last = sol[line][2 * k + 1];
    float prev = first;
    rd[0] = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        prev = (rd[r] - ra[r] * prev - rc[r] * last) * rb[r];
        rd[r] = prev;
    }
    rd[M - 1] = last;
    if (!live) return;
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int i = k * M + r;
        if (i >= n) break;
        const fe_u64 at = AXIS == 1 ? (static_cast<fe_u64>(other) * P::NY + i) * P::NX + x : (static_cast<fe_u64>(i) * P::NY + other) * P::NX + x;
        a.out[0][at] = rd[r];
    }
}

// Tridiagonal solves along y or z, a thread a line; consecutive threads take consecutive x, so every step of the
// recurrence reads and writes whole rows (coalesced). c' goes to out[1] (scratch), d' and then the answer to out[0].
template <class P, int AXIS>
__device__ __forceinline__ void fe_tridiag_yz_pass(const FePassArgs& a)
{
    const fe_u64 k = blockIdx.x * static_cast<fe_u64>(blockDim.x) + threadIdx.x;
    const int n = AXIS == 1 ? P::NY : P::NZ;
    const fe_u64 lines = AXIS == 1 ? static_cast<fe_u64>(P::NX) * P::NZ : static_cast<fe_u64>(P::NX) * P::NY;
    if (k >= lines) return;
    const int x = static_cast<int>(k % P::NX);
    const int other = static_cast<int>(k / P::NX); // z for y-lines, y for z-lines
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    float* ans = a.out[0];
    float* cps = a.out[1];
    auto at = [&](int i) -> fe_u64 {
        const int y = AXIS == 1 ? i : other;
        const int z = AXIS == 1 ? other : i;
        return (static_cast<fe_u64>(z) * P::NY + y) * P::NX + x;
    };
    float cp = 0.f, dp = 0.f;
    for (int i = 0; i < n; ++i) {
        const int y = AXIS == 1 ? i : other;
        const int z = AXIS == 1 ? other : i;
        float lo, di, up, rhs;
        P::coef(c, x, y, z, lo, di, up, rhs);
        if (i == 0) di += lo;
        if (i + 1 == n) di += up;
        const float den = di - lo * cp;
        dp = (rhs - lo * dp) / den;
        cp = i + 1 == n ? 0.f : up / den;
        ans[at(i)] = dp;
        cps[at(i)] = cp;
    }
    float next = 0.f;
    for (int i = n - 1; i >= 0; --i) {
        next = ans[at(i)] - cps[at(i)] * next;
        ans[at(i)] = next;
    }
}

// ---- tcgen05 (the fifth-generation tensor cores), for the law's `half` nets ----------------------------------------
// Operands are BF16 matrices in shared memory in the canonical no-swizzle core-matrix layout: a core matrix is 8 rows
// of 16 bytes, element (r, c) of an R-row matrix at ((c / 8) (R / 8) + r / 8) 128 + (r % 8) 16 + (c % 8) 2 bytes.
// Accumulators are FP32 in tensor memory, one lane a row. One thread issues the MMAs and commits them to an mbarrier
// that every thread waits on with a bounded wait.
__device__ __forceinline__ unsigned fe_tc_core(int r, int c, int R)
{
    return static_cast<unsigned>(((c >> 3) * (R >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets (16-byte units), sm_100 version 1, no swizzle.
__device__ __forceinline__ fe_u64 fe_tc_sdesc(unsigned saddr, unsigned lbo, unsigned sbo)
{
    fe_u64 d = static_cast<fe_u64>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<fe_u64>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<fe_u64>((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;
    return d;
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A (K-major) and B (MN-major), M x N.
__device__ __forceinline__ unsigned fe_tc_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | (static_cast<unsigned>(N >> 3) << 17) | (static_cast<unsigned>(M >> 4) << 24);
}

__device__ __forceinline__ void fe_tc_mma(unsigned dtmem, fe_u64 a, fe_u64 b, unsigned id, unsigned accumulate)
{
    asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
                 ::"r"(dtmem), "l"(a), "l"(b), "r"(id), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void fe_tc_commit(fe_u64* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(fe_smem(bar)) : "memory");
}

__device__ __forceinline__ void fe_tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fe_tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fe_tc_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's tensor-memory lane.
__device__ __forceinline__ void fe_tc_ld16(unsigned taddr, float* r)
{
    unsigned x[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7]), "=r"(x[8]),
                   "=r"(x[9]), "=r"(x[10]), "=r"(x[11]), "=r"(x[12]), "=r"(x[13]), "=r"(x[14]), "=r"(x[15])
                 : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; ++i) r[i] = __uint_as_float(x[i]);
}

// Two floats as BF16 (round to nearest even), the first in the low half.
__device__ __forceinline__ unsigned fe_tc_bf16x2(float lo, float hi)
{
    unsigned r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// Row r's columns c0 .. c0 + 7 of a 128-row operand tile, one 16-byte store.
__device__ __forceinline__ void fe_tc_put8(unsigned char* tile, int r, int c0, const float* v)
{
    const uint4 q = make_uint4(fe_tc_bf16x2(v[0], v[1]), fe_tc_bf16x2(v[2], v[3]), fe_tc_bf16x2(v[4], v[5]), fe_tc_bf16x2(v[6], v[7]));
    *reinterpret_cast<uint4*>(tile + fe_tc_core(r, c0, 128)) = q;
}

// A net op whose net is declared `half` (the reference's tensor-core nets, CudaNet.cpp:175-277), as one stage kernel:
// 128 threads, thread t owns cell t of a 128-cell tile and row / tensor-memory lane t, persistent over tiles. A cell
// needs P::E evaluations of the net (mlp 1; flux and ldiffuse 12: six faces, both ways round); P::EC of them at a time
// (whole faces) are 128-row tiles in shared memory, and each layer is P::EC M = 128 MMAs (K = 16 a step) into their
// own accumulator columns. Between layers every thread reads its row back, adds the bias, applies the activation and
// writes the next layer's BF16 operand over the last one (whose MMAs have completed). P::prepare gathers what a cell's
// evaluations read once (its arguments, or each face's two sides or window); P::take folds a face's two evaluations
// (or mlp's one) into the cell's value, in FP32, as soon as they are out. `wblob`: every half net's weights, BF16,
// each layer's K x N matrix in the core layout (rows = inputs). A wait that gives up sets a.err and the rest of the
// tile's MMAs are skipped; the kernel leaves through its normal exit (tensor memory freed).
template <class P>
__device__ __forceinline__ void fe_net_pass(const FePassArgs& a, const unsigned short* wblob)
{
    extern __shared__ __align__(128) float fe_sm[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(fe_sm);
    unsigned char* weights = sm + P::EC * P::A_BYTES;
    fe_u64* bar = reinterpret_cast<fe_u64*>(weights + P::W_BYTES);
    unsigned* tslot = reinterpret_cast<unsigned*>(bar + 1);
    const int t = threadIdx.x;
    const int warp = t >> 5;
    {
        const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const unsigned char*>(wblob) + P::WOFF);
        uint4* dst = reinterpret_cast<uint4*>(weights);
        for (int i = t; i < static_cast<int>(P::W_BYTES / 16); i += 128) dst[i] = src[i];
    }
    if (t == 0) {
        fe_mbar_init(bar, 1);
        fe_fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(fe_smem(tslot)), "r"(P::TCOLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fe_fence_proxy_async();
    fe_tc_before();
    __syncthreads();
    fe_tc_after();
    const unsigned tbase = *tslot;
    const unsigned lane = tbase + (static_cast<unsigned>(warp * 32) << 16);
    const unsigned s0 = fe_smem(sm);
    const unsigned w0 = fe_smem(weights);
    FePlainCtx<P> c;
    c.src = a.src;
    c.dt = a.dt;
    const fe_u64 cells = static_cast<fe_u64>(P::NX) * P::NY * P::NZ;
    const fe_u64 tiles = (cells + 127) / 128;
    unsigned phase = 0;
    bool ok = true;
    for (fe_u64 tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const fe_u64 cell = tile * 128 + static_cast<fe_u64>(t);
        const bool valid = cell < cells;
        const fe_u64 at = valid ? cell : cells - 1;
        const int x = static_cast<int>(at % P::NX);
        const int y = static_cast<int>((at / P::NX) % P::NY);
        const int z = static_cast<int>(at / (static_cast<fe_u64>(P::NX) * P::NY));
        typename P::Keep keep;
        P::prepare(c, x, y, z, keep);
        float o = 0.f;
        // One chunk of a cell's evaluations through every layer. A deep net's chunks stay one copy of the code (the
        // unrolled form outgrows the instruction cache: ldiffuse 5-8-8-4, 0.27 -> 0.23 ms a step at 1M cells); a
        // shallow one's are unrolled, which lets the gathered inputs stay in registers.
        auto chunk = [&](int ch) {
            // Layer 0's operands: the inputs, shifted and scaled (FP32), then BF16; zeros past the net's inputs.
#pragma unroll
            for (int ee = 0; ee < P::EC; ++ee) {
                float xin[P::KP0];
#pragma unroll
                for (int i = 0; i < P::KP0; ++i) xin[i] = 0.f;
                P::input(keep, ch + ee, xin);
#pragma unroll
                for (int i = 0; i < P::NIN; ++i) xin[i] = (xin[i] - P::shift(i)) * P::scale(i);
#pragma unroll
                for (int c0 = 0; c0 < P::KP0; c0 += 8) fe_tc_put8(sm + ee * P::A_BYTES, t, c0, xin + c0);
            }
            float yout[P::EC][P::NOUT];
#pragma unroll
            for (int l = 0; l < P::L; ++l) {
                if (ok) {
                    fe_fence_proxy_async();
                    fe_tc_ld_wait();
                    fe_tc_before();
                    __syncthreads();
                    if (t == 0) {
                        fe_tc_after();
                        for (int ee = 0; ee < P::EC; ++ee) {
                            for (int ks = 0; ks < P::kp(l) / 16; ++ks) {
                                fe_tc_mma(tbase + static_cast<unsigned>(ee * P::NMAX),
                                    fe_tc_sdesc(s0 + ee * P::A_BYTES + ks * 2 * 2048, 2048, 128),
                                    fe_tc_sdesc(w0 + P::wb(l) + ks * 2 * 128, 128, (P::kp(l) / 8) * 128), fe_tc_idesc(128, P::np(l)), ks > 0);
                            }
                        }
                        fe_tc_commit(bar);
                    }
                    const bool mine = fe_mbar_wait(bar, phase, 1u << 22);
                    ok = __syncthreads_and(mine) != 0;
                    fe_tc_after();
                    if (ok) phase ^= 1u;
                    else if (t == 0) atomicOr(a.err, FE_ERR_MBAR_TIMEOUT);
                }
#pragma unroll
                for (int ee = 0; ee < P::EC && ok; ++ee) {
#pragma unroll
                    for (int c0 = 0; c0 < P::np(l); c0 += 16) {
                        float v[16];
                        fe_tc_ld16(lane + static_cast<unsigned>(ee * P::NMAX + c0), v);
                        fe_tc_ld_wait();
                        if (l + 1 < P::L) {
#pragma unroll
                            for (int i = 0; i < 16; ++i) v[i] = c0 + i < P::no(l) ? P::act(v[i] + P::bias(l, c0 + i)) : 0.f;
                            fe_tc_put8(sm + ee * P::A_BYTES, t, c0, v);
                            fe_tc_put8(sm + ee * P::A_BYTES, t, c0 + 8, v + 8);
                        } else {
#pragma unroll
                            for (int i = 0; i < 16; ++i) {
                                if (c0 + i < P::NOUT) yout[ee][c0 + i] = (v[i] + P::bias(l, c0 + i)) * P::OSCALE;
                            }
                        }
                    }
                }
            }
#pragma unroll
            for (int ee = 0; ee < P::EC; ee += P::PAIR) P::take(keep, ch + ee, yout[ee], yout[ee + P::PAIR - 1], o);
        };
        if constexpr (P::ROLL) {
#pragma unroll 1
            for (int ch = 0; ch < P::E; ch += P::EC) chunk(ch);
        } else {
#pragma unroll
            for (int ch = 0; ch < P::E; ch += P::EC) chunk(ch);
        }
        if (ok && valid) a.out[0][cell] = P::result(o);
    }
    if (!ok) {
        // The MMAs whose wait gave up may still run: one more bounded wait before their tensor memory is freed.
        fe_mbar_wait(bar, phase, 1u << 22);
    }
    fe_tc_ld_wait();
    fe_tc_before();
    __syncthreads();
    if (warp == 0) {
        fe_tc_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(P::TCOLS) : "memory");
    }
}

// Activations of the tensor-core nets, whose layers are BF16 (8 significant bits): the hardware's approximate tanh
// and exponential are well inside that.
__device__ __forceinline__ float fe_tanh_approx(float v)
{
    float r;
    asm("tanh.approx.f32 %0, %1;" : "=f"(r) : "f"(v));
    return r;
}
__device__ __forceinline__ float fe_silu_approx(float v) { return __fdividef(v, 1.f + __expf(-v)); }

#endif // device code

#endif // FE_DEVICE_CUH
