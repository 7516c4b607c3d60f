// Tridiagonal solves by a segment of K lanes of a warp: a PCR/Thomas hybrid (the partition method).
//
// A line of n = K * M rows is held M rows a lane by the K lanes of a segment (lane k: rows k M .. k M + M - 1). Row i is
//   a[i] x[i-1] + b[i] x[i] + c[i] x[i+1] = d[i],   with a[0] = c[n-1] = 0 (an edge repeat is folded into b first).
// 1. Each lane eliminates inside its own rows (Thomas-like sweeps down and up), leaving two equations that couple only
//    its first and last unknowns to the neighbouring lanes' last and first: a tridiagonal system of 2K unknowns.
// 2. That reduced system is solved by parallel cyclic reduction across the segment's lanes (log2(2K) rounds of
//    shuffles).
// 3. Each lane back-substitutes its interior rows from its first and last unknowns.
// With K = 1 it is Thomas' algorithm (src/field/Law.cpp:1098-1138). Divisions are by approximate reciprocals, so the
// solves agree with the reference's to a tolerance, not bit for bit.
//
// No pivoting, like the reference: the systems the law's implicit schemes build are diagonally dominant.
#ifndef FE_TRIDIAG_CUH
#define FE_TRIDIAG_CUH

#if defined(__CUDACC__) || defined(__CUDACC_RTC__)

// 1 / x by the hardware approximation (rcp.approx, about 1 ulp), for solves checked to a tolerance.
__device__ __forceinline__ float fe_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Thomas over the first n <= M rows held by one thread, the same (a, b, c) in every row and the edge repeat folded at
// the line's two ends (b + a in row 0 with no a; b + c in row n-1 with no c).
template <int M>
__device__ __forceinline__ void fe_thomas_row(float a, float b, float c, float (&d)[M], int n)
{
    float cp[M];
    float cprev = 0.f, dprev = 0.f;
#pragma unroll
    for (int i = 0; i < M; ++i) {
        if (i < n) {
            const bool last = i + 1 == n;
            const float ai = i == 0 ? 0.f : a;
            float bi = b;
            if (i == 0) bi = bi + a;
            if (last) bi = bi + c;
            const float iden = fe_rcp(bi - ai * cprev);
            dprev = (d[i] - ai * dprev) * iden;
            cprev = last ? 0.f : c * iden;
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

// The reduced system of a segment of K lanes (a power of two, 2..32): lane k holds two equations, row 2k
// (a0 x[2k-1] + b0 x[2k] + c0 x[2k+1] = d0) and row 2k+1 (a1 x[2k] + b1 x[2k+1] + c1 x[2k+2] = d1), solved by parallel
// cyclic reduction over log2(2K) rounds of shuffles. Returns x[2k] in `first` and x[2k+1] in `last`. Every lane of the
// warp must call it.
__device__ __forceinline__ void fe_pcr_pairs(float a0, float b0, float c0, float d0, float a1, float b1, float c1, float d1,
    int k, int K, float& first, float& last)
{
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
        const float k10 = a0 * fe_rcp(lb0), k20 = c0 * fe_rcp(ub0), k11 = a1 * fe_rcp(lb1), k21 = c1 * fe_rcp(ub1);
        const float na0 = -k10 * la0, nc0 = -k20 * uc0, nb0 = b0 - k10 * lc0 - k20 * ua0, nd0 = d0 - k10 * ld0 - k20 * ud0;
        const float na1 = -k11 * la1, nc1 = -k21 * uc1, nb1 = b1 - k11 * lc1 - k21 * ua1, nd1 = d1 - k11 * ld1 - k21 * ud1;
        a0 = na0; b0 = nb0; c0 = nc0; d0 = nd0;
        a1 = na1; b1 = nb1; c1 = nc1; d1 = nd1;
    }
    first = d0 * fe_rcp(b0);
    last = d1 * fe_rcp(b1);
}

// A line with the same (a, b, c) in every row, the edge repeat folded at its two ends: the x lines of a row of a law
// whose coefficients vary only across rows. Lane k of K holds rows k M .. k M + M - 1 (K = 1: the first n <= M rows,
// Thomas). The rows' coefficients are formed inside the unrolled loops, so a lane keeps its right-hand sides and the
// up-sweep's two arrays. On return d holds the solution.
template <int M>
__device__ __forceinline__ void fe_tri_row(float a, float b, float c, float (&d)[M], int k, int K, int n)
{
    static_assert(M >= 2, "two rows a lane at least");
    if (K == 1) {
        fe_thomas_row<M>(a, b, c, d, n);
        return;
    }
    const bool lo = k == 0, hi = k == K - 1;
    auto A = [&](int r) { return r == 0 && lo ? 0.f : a; };
    auto Bc = [&](int r) {
        float v = b;
        if (r == 0 && lo) v = v + a;
        if (r == M - 1 && hi) v = v + c;
        return v;
    };
    auto Cc = [&](int r) { return r == M - 1 && hi ? 0.f : c; };
    // Down: rows 1 .. M-1 in terms of (x first, x r, x r+1).
    float al = A(1), be = Bc(1), de = d[1];
#pragma unroll
    for (int r = 2; r < M; ++r) {
        const float f = A(r) * fe_rcp(be);
        al = -f * al;
        be = Bc(r) - f * Cc(r - 1);
        de = d[r] - f * de;
    }
    // Up, in place in d: rows M-2 .. 0 in terms of (x r-1, x r, x last).
    float iB[M - 1], C[M - 1];
    float Bn = Bc(M - 2);
    C[M - 2] = Cc(M - 2);
    iB[M - 2] = fe_rcp(Bn);
#pragma unroll
    for (int r = M - 3; r >= 0; --r) {
        const float g = Cc(r) * iB[r + 1];
        Bn = Bc(r) - g * A(r + 1);
        C[r] = -g * C[r + 1];
        d[r] = d[r] - g * d[r + 1];
        iB[r] = fe_rcp(Bn);
    }
    float first, last;
    fe_pcr_pairs(A(0), Bn, C[0], d[0], al, be, Cc(M - 1), de, k, K, first, last);
    float prev = first;
    d[0] = first;
#pragma unroll
    for (int r = 1; r < M - 1; ++r) {
        prev = (d[r] - A(r) * prev - C[r] * last) * iB[r];
        d[r] = prev;
    }
    d[M - 1] = last;
}

#endif // device code

#endif // FE_TRIDIAG_CUH
