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

// fe_rcp and fe_pcr_pairs (the reduced system's parallel cyclic reduction) live in fe_device.cuh, which the law's
// generated passes share; this file adds the constant-coefficient row solves of the batched Heston kernel.

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
