// ordered_sum.cuh — a left-to-right floating-point sum, bit for bit, by one
// thread block in parallel.
//
// The reference forms its AMR thresholds from sums like
//     do (every leaf in traversal order); S = S + x; end do
// (src/solution.F90:430-457), and each addition rounds, so the result is a
// chain of roundings that no reassociation reproduces.  It can still be
// formed in parallel when the addends are not negative, which holds for the
// squares summed here:
//
//  - While the running sum s stays in one binade [2^E, 2^(E+1)), every
//    partial sum is a multiple of u = 2^(E-52), and RN(s + x) = s + r*u with
//    r = x/u rounded to the nearest integer (x/u is exact: u is a power of
//    two), unless x/u lies exactly halfway between two integers (then the
//    result depends on the parity of s/u + floor(x/u)) or reaches 2^52.
//  - So a run of additions that never leaves the binade and meets no
//    halfway case is an integer sum, s_k = (s/u + r_1 + ... + r_k) * u,
//    which a thread block forms with a prefix sum.  The run stops before the first
//    addition whose integer total reaches 2^53 (the sum would reach the next
//    binade, where the spacing doubles) or which is a halfway case, NaN,
//    infinite or negative; that one addition is made as the reference makes
//    it, s = s + x, and the next run starts from the new s.
//  - A sum that is still zero stays +0 over zero addends; a sum below
//    2^-970 (whose u would be subnormal) is added one element at a time.
//
// s only grows, so it crosses a binade boundary about log2(S/x_1) times in
// all: the rest is block-wide prefix sums of integers.
#pragma once
#include <cstdint>

namespace fdm {

constexpr int OSUM_NT = 1024;   // threads of the summing block
constexpr int OSUM_EPT = 4;     // consecutive elements per thread and run

// x/u rounded to the nearest integer, for 0 <= t = x/u < 2^52: t + 2^52
// rounds t to an integer (the spacing there is 1) and the integer is the
// low mantissa bits; *half: t lies halfway between two integers
__device__ __forceinline__ long long osum_round(double t, bool *half) {
    const double y = t + 0x1p52;
    *half = fabs(t - (y - 0x1p52)) == 0.5;   // exact: both terms lie within one unit of t
    return __double_as_longlong(y) - 0x4330000000000000ll;
}

struct OSumShared {
    long long wtot[32];          // per-warp totals of the block scan
    unsigned long long first;    // block minimum (first failing thread / first non-zero element)
    long long R;                 // accepted integer total of a run
    long long A;                 // element that stopped the run
};

// Inclusive prefix sum of v over the block (NT threads, a multiple of 32).
template <int NT>
__device__ __forceinline__ long long osum_block_scan(long long v, OSumShared &sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long w = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += w;
    }
    if (lane == 31) sh.wtot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        long long w = lane < NT / 32 ? sh.wtot[lane] : 0ll;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        sh.wtot[lane] = w;
    }
    __syncthreads();
    return v + (warp > 0 ? sh.wtot[warp - 1] : 0ll);
}

// Minimum of v over the block (every thread gets it).
__device__ __forceinline__ unsigned long long osum_block_min(unsigned long long v, OSumShared &sh) {
    if (threadIdx.x == 0) sh.first = ~0ull;
    __syncthreads();
    if (v != ~0ull) atomicMin(&sh.first, v);
    __syncthreads();
    const unsigned long long r = sh.first;
    __syncthreads();
    return r;
}

// (...((0 + x(0)) + x(1)) + ...) + x(n-1), x(i) = get(i), by one block of NT
// threads, EPT consecutive elements per thread and run; every thread returns
// the sum.  A subsequence is summed in order by giving +0 for the elements
// left out (s + 0 = s for every s the sum can hold).
template <int NT, int EPT, class Get>
__device__ double ordered_sum_block(const Get &get, int64_t n, OSumShared &sh) {
    const long long TOP = 1ll << 53;
    const int t = threadIdx.x;
    double s = 0.0;
    int64_t start = 0;
    while (start < n) {
        const int64_t end = start + (int64_t)NT * EPT < n ? start + (int64_t)NT * EPT : n;
        const int64_t e0 = start + (int64_t)t * EPT;
        double xv[EPT];
#pragma unroll
        for (int j = 0; j < EPT; ++j) xv[j] = e0 + j < end ? get(e0 + j) : 0.0;
        const unsigned hi = (unsigned)__double2hiint(s);
        const int fld = (int)((hi >> 20) & 0x7ffu);
        if (s == 0.0) {
            // +0 + (+-0) = +0: skip to the first element that is not a zero
            unsigned long long f = ~0ull;
#pragma unroll
            for (int j = EPT - 1; j >= 0; --j)
                if (e0 + j < end && !(xv[j] == 0.0)) f = (unsigned long long)(e0 + j);
            f = osum_block_min(f, sh);
            if (f == ~0ull) {
                start = end;
            } else {
                s = s + get((int64_t)f);
                start = (int64_t)f + 1;
            }
            continue;
        }
        if (fld < 53 || fld == 0x7ff || (hi >> 31)) {   // tiny, not finite or negative: one at a time
            s = s + get(start);
            ++start;
            continue;
        }
        const double uinv = __hiloint2double((2098 - fld) << 20, 0);   // 2^(52-E), E = fld - 1023
        const double u = __hiloint2double((fld - 52) << 20, 0);         // 2^(E-52)
        const long long M = (long long)(s * uinv);                       // s / u, in [2^52, 2^53)
        // this thread's run: the integer increments before its first element
        // that cannot be added as an integer
        int bad = EPT;
        long long T = 0;
#pragma unroll
        for (int j = EPT - 1; j >= 0; --j) {
            const double tt = xv[j] * uinv;
            bool half;
            (void)osum_round(tt, &half);
            if (!(xv[j] >= 0.0) || !(tt < 0x1p52) || half) bad = j;
        }
#pragma unroll
        for (int j = 0; j < EPT; ++j) {
            bool half;
            const long long r = osum_round(xv[j] * uinv, &half);
            T += j < bad ? r : 0ll;
        }
        const long long inc = osum_block_scan<NT>(T, sh);
        const bool failed = bad < EPT || M + inc >= TOP;
        const unsigned long long lim = osum_block_min(failed ? (unsigned long long)t : ~0ull, sh);
        if (lim == ~0ull) {
            if (t == NT - 1) sh.R = inc;
        } else if ((unsigned long long)t == lim) {
            // the element of this thread that stops the run
            long long P = M + (inc - T);
            int stop = bad;
#pragma unroll
            for (int j = 0; j < EPT; ++j) {
                if (j >= stop) break;
                bool half;
                const long long r = osum_round(xv[j] * uinv, &half);
                if (P + r >= TOP) { stop = j; break; }
                P += r;
            }
            sh.R = P - M;
            sh.A = e0 + stop;
        }
        __syncthreads();
        const long long R = sh.R;
        const int64_t A = lim == ~0ull ? end : (int64_t)sh.A;
        __syncthreads();
        s = (double)(M + R) * u;   // exact: an integer below 2^53 times a power of two
        start = A;
        if (A < end) {
            s = s + get(A);
            start = A + 1;
        }
    }
    return s;
}

}  // namespace fdm
