// Tridiagonal solves by a segment of K lanes of a warp: a PCR/Thomas hybrid (the partition method).
//
// A line of n = K * M rows is held M rows a lane by the K lanes of a segment (lane k: rows k M .. k M + M - 1). Row i is
//   a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i],   with a[0] = c[n-1] = 0 (an edge repeat is folded into b first).
// 1. Each lane eliminates inside its own rows (Thomas-like sweeps down and up), leaving two equations that couple only
//    its first and last unknowns to the neighbouring lanes' last and first: a tridiagonal system of 2K unknowns.
// 2. That reduced system is solved by parallel cyclic reduction across the segment's lanes (log2(2K) rounds of
//    shuffles).
// 3. Each lane back-substitutes its interior rows from its first and last unknowns.
// With K = 1 it is Thomas' algorithm in the reference's order (src/field/Law.cpp:1098-1138; the GPU's
// cuda/CudaCodegen.cpp:402-412), so a one-lane solve gives the engine's tridiag bits.
//
// No pivoting, like the reference: the systems the law's implicit schemes build are diagonally dominant.
#ifndef FE_TRIDIAG_CUH
#define FE_TRIDIAG_CUH

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)

// Thomas over M rows held by one thread (a[0] and c[M-1] are ignored as couplings).
template <int M>
__device__ __forceinline__ void fe_thomas(const float (&a)[M], const float (&b)[M], const float (&c)[M], float (&d)[M])
{
    float cp[M];
    float cprev = 0.f, dprev = 0.f;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const float lo = i == 0 ? 0.f : a[i];
        const float den = b[i] - lo * cprev;
        dprev = (d[i] - lo * dprev) / den;
        cprev = i + 1 == M ? 0.f : c[i] / den;
        cp[i] = cprev;
        d[i] = dprev;
    }
    float next = 0.f;
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        next = d[i] - cp[i] * next;
        d[i] = next;
    }
}

// The segment solve: K lanes (a power of two, 2..32, aligned within the warp), M >= 2 rows a lane. `k` is this lane's
// index in its segment. Every lane of the warp must call it (the shuffles are warp-wide).
template <int K, int M>
__device__ __forceinline__ void fe_tri_segment(const float (&a)[M], const float (&b)[M], const float (&c)[M], float (&d)[M], int k)
{
    static_assert(M >= 2, "two rows a lane at least");
    // Down: rows 1 .. M-1 in terms of (x first, x r, x r+1); row M-1 keeps its coupling to the next lane.
    float al = a[1], be = b[1], de = d[1];
#pragma unroll
    for (int r = 2; r < M; ++r) {
        const float f = a[r] / be;
        al = -f * al;
        be = b[r] - f * c[r - 1];
        de = d[r] - f * de;
    }
    // Up: rows M-2 .. 0 in terms of (x r-1, x r, x last); row 0 keeps its coupling to the previous lane.
    float B[M - 1], C[M - 1], D[M - 1];
    B[M - 2] = b[M - 2];
    C[M - 2] = c[M - 2];
    D[M - 2] = d[M - 2];
#pragma unroll
    for (int r = M - 3; r >= 0; --r) {
        const float g = c[r] / B[r + 1];
        B[r] = b[r] - g * a[r + 1];
        C[r] = -g * C[r + 1];
        D[r] = d[r] - g * D[r + 1];
    }
    // The reduced system: unknown 2k (this lane's first) and 2k+1 (its last).
    float ra[2] = {a[0], al}, rb[2] = {B[0], be}, rc[2] = {C[0], c[M - 1]}, rd[2] = {D[0], de};
    const unsigned mask = 0xffffffffu;
#pragma unroll
    for (int s = 1; s < 2 * K; s *= 2) {
        float na[2], nb[2], nc[2], nd[2];
        // The equations s below and s above each of this lane's two: for s = 1, one is this lane's other equation.
        float la[2], lb[2], lc[2], ld[2], ua[2], ub[2], uc[2], ud[2];
        if (s == 1) {
            // Below 2k is 2k-1 (lane k-1, second); above 2k+1 is 2k+2 (lane k+1, first).
            const float pa = __shfl_up_sync(mask, ra[1], 1, K), pb = __shfl_up_sync(mask, rb[1], 1, K);
            const float pc = __shfl_up_sync(mask, rc[1], 1, K), pd = __shfl_up_sync(mask, rd[1], 1, K);
            const float qa = __shfl_down_sync(mask, ra[0], 1, K), qb = __shfl_down_sync(mask, rb[0], 1, K);
            const float qc = __shfl_down_sync(mask, rc[0], 1, K), qd = __shfl_down_sync(mask, rd[0], 1, K);
            const bool has_lo = k > 0, has_hi = k + 1 < K;
            la[0] = has_lo ? pa : 0.f; lb[0] = has_lo ? pb : 1.f; lc[0] = has_lo ? pc : 0.f; ld[0] = has_lo ? pd : 0.f;
            ua[0] = ra[1]; ub[0] = rb[1]; uc[0] = rc[1]; ud[0] = rd[1];
            la[1] = ra[0]; lb[1] = rb[0]; lc[1] = rc[0]; ld[1] = rd[0];
            ua[1] = has_hi ? qa : 0.f; ub[1] = has_hi ? qb : 1.f; uc[1] = has_hi ? qc : 0.f; ud[1] = has_hi ? qd : 0.f;
        } else {
            const int q = s / 2;
            const bool has_lo = k - q >= 0, has_hi = k + q < K;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const float pa = __shfl_up_sync(mask, ra[t], q, K), pb = __shfl_up_sync(mask, rb[t], q, K);
                const float pc = __shfl_up_sync(mask, rc[t], q, K), pd = __shfl_up_sync(mask, rd[t], q, K);
                const float qa = __shfl_down_sync(mask, ra[t], q, K), qb = __shfl_down_sync(mask, rb[t], q, K);
                const float qc = __shfl_down_sync(mask, rc[t], q, K), qd = __shfl_down_sync(mask, rd[t], q, K);
                la[t] = has_lo ? pa : 0.f; lb[t] = has_lo ? pb : 1.f; lc[t] = has_lo ? pc : 0.f; ld[t] = has_lo ? pd : 0.f;
                ua[t] = has_hi ? qa : 0.f; ub[t] = has_hi ? qb : 1.f; uc[t] = has_hi ? qc : 0.f; ud[t] = has_hi ? qd : 0.f;
            }
        }
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            const float k1 = ra[t] / lb[t];
            const float k2 = rc[t] / ub[t];
            na[t] = -k1 * la[t];
            nc[t] = -k2 * uc[t];
            nb[t] = rb[t] - k1 * lc[t] - k2 * ua[t];
            nd[t] = rd[t] - k1 * ld[t] - k2 * ud[t];
        }
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            ra[t] = na[t];
            rb[t] = nb[t];
            rc[t] = nc[t];
            rd[t] = nd[t];
        }
    }
    const float first = rd[0] / rb[0];
    const float last = rd[1] / rb[1];
    // Back: the interior rows from the lane's first and last unknowns.
    d[0] = first;
    float prev = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        prev = (D[r] - a[r] * prev - C[r] * last) / B[r];
        d[r] = prev;
    }
    d[M - 1] = last;
}

// Thomas over the first n <= M rows held by one thread (runtime length).
template <int M>
__device__ __forceinline__ void fe_thomas_n(const float (&a)[M], const float (&b)[M], const float (&c)[M], float (&d)[M], int n)
{
    float cp[M];
    float cprev = 0.f, dprev = 0.f;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i < n) {
            const float lo = i == 0 ? 0.f : a[i];
            const float den = b[i] - lo * cprev;
            dprev = (d[i] - lo * dprev) / den;
            cprev = i + 1 == n ? 0.f : c[i] / den;
            cp[i] = cprev;
            d[i] = dprev;
        }
    }
    float next = 0.f;
#pragma unroll
    for (int i = M - 1; i >= 0; --i) {
        if (i < n) {
            next = d[i] - cp[i] * next;
            d[i] = next;
        }
    }
}

// The segment solve with the segment's width K a run-time value (a power of two, 2..32): the same algorithm as
// fe_tri_segment, one instantiation for every K.
template <int M>
__device__ __forceinline__ void fe_tri_segment_k(const float (&a)[M], const float (&b)[M], const float (&c)[M], float (&d)[M], int k,
    int K)
{
    static_assert(M >= 2, "two rows a lane at least");
    float al = a[1], be = b[1], de = d[1];
#pragma unroll
    for (int r = 2; r < M; ++r) {
        const float f = a[r] / be;
        al = -f * al;
        be = b[r] - f * c[r - 1];
        de = d[r] - f * de;
    }
    float B[M - 1], C[M - 1], D[M - 1];
    B[M - 2] = b[M - 2];
    C[M - 2] = c[M - 2];
    D[M - 2] = d[M - 2];
#pragma unroll
    for (int r = M - 3; r >= 0; --r) {
        const float g = c[r] / B[r + 1];
        B[r] = b[r] - g * a[r + 1];
        C[r] = -g * C[r + 1];
        D[r] = d[r] - g * D[r + 1];
    }
    float a0 = a[0], b0 = B[0], c0 = C[0], d0 = D[0];
    float a1 = al, b1 = be, c1 = c[M - 1], d1 = de;
    const unsigned mask = 0xffffffffu;
    for (int s = 1; s < 2 * K; s *= 2) {
        const int q = s == 1 ? 1 : s / 2;
        const bool has_lo = k - q >= 0, has_hi = k + q < K;
        // Below and above each equation: for s = 1 one of them is this lane's other equation.
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
        const float k10 = a0 / lb0, k20 = c0 / ub0, k11 = a1 / lb1, k21 = c1 / ub1;
        const float na0 = -k10 * la0, nc0 = -k20 * uc0, nb0 = b0 - k10 * lc0 - k20 * ua0, nd0 = d0 - k10 * ld0 - k20 * ud0;
        const float na1 = -k11 * la1, nc1 = -k21 * uc1, nb1 = b1 - k11 * lc1 - k21 * ua1, nd1 = d1 - k11 * ld1 - k21 * ud1;
        a0 = na0; b0 = nb0; c0 = nc0; d0 = nd0;
        a1 = na1; b1 = nb1; c1 = nc1; d1 = nd1;
    }
    const float first = d0 / b0;
    const float last = d1 / b1;
    d[0] = first;
    float prev = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        prev = (D[r] - a[r] * prev - C[r] * last) / B[r];
        d[r] = prev;
    }
    d[M - 1] = last;
}

#endif // device code

#endif // FE_TRIDIAG_CUH
