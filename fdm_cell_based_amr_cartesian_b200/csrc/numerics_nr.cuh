// numerics_nr.cuh — correctly rounded FP64 division without branches, for
// the face flux of the exact build.
//
// The compiler's division is correctly rounded, but each one ends in a
// range test with a branch to a slow path, and the branches split the face
// flux into short straight-line pieces: the scheduler cannot interleave the
// independent reconstructions of a face across them, and the kernel waits on
// dependent FP64 chains.  DivNR forms the same quotients, bit for bit, from
// published methods in straight-line code:
//
//  - Reciprocal: the hardware approximation (PTX rcp.approx.ftz.f64) refined
//    by two Newton-Raphson steps, e = 1 - b*y, y = y + y*e (each step squares
//    the relative error), which leaves y within about one ulp of 1/b.
//  - Quotient from such a y: q = a*y, then one correction q = q + (a - b*q)*y
//    with the remainder formed by an FMA; q is then a faithful rounding of
//    a/b (within one ulp).
//  - Rounding decision (exact remainder test): for a faithful q the
//    remainder r = a - b*q is exactly representable and a/b = q + r/b, so
//    RN(a/b) is q or its neighbour towards r/b, and the neighbour is taken
//    exactly when |r| > |b| * (half the gap to it), a comparison of exact
//    values (the half gap is a power of two).  A quotient of two 53-bit
//    numbers is never a midpoint of two doubles, so there are no ties.
//  - Shared denominators: y = RN(1/b) by the same test (a = 1), then for
//    every numerator Markstein's two corrections, q = RN(a*y),
//    q = q + (a - b*q)*y twice: with y within half an ulp of 1/b and the
//    first correction faithful, the second gives RN(a/b) (P. Markstein,
//    "Computation of elementary functions on the IBM RISC System/6000
//    processor", IBM J. Res. Dev. 34(1), 1990).
//
// The steps are exact only away from underflow and overflow, so every
// operand is checked to lie in [2^-450, 2^450] (or to be zero, whose sign
// is taken from a*y): then quotients, remainders and half gaps stay normal.
// Smaller numerators are scaled into that range by a power of two and the
// quotient scaled back (both exact while the quotient is normal).  An
// operand outside clears `ok`, and the caller computes the face again with
// the compiler's division.
#pragma once
#include "numerics.cuh"

namespace fdm {

struct DivNR {
    Den gm1, d2;     // constant denominators, y = RN(1/b) from the host
    bool ok = true;

    __device__ __forceinline__ DivNR(Den g1, Den dd) : gm1(g1), d2(dd) {}

    // |x| in [2^-450, 2^450): biased exponent in [573, 1473)
    __device__ __forceinline__ static bool in_range(double x) {
        const unsigned e = ((unsigned)__double2hiint(x) >> 20) & 0x7ffu;
        return e - 573u < 900u;
    }
    __device__ __forceinline__ static double rcp_newton(double b) {
        double y;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(b));
        double e = __fma_rn(-b, y, 1.0);
        y = __fma_rn(y, e, y);
        e = __fma_rn(-b, y, 1.0);
        return __fma_rn(y, e, y);
    }
    // RN(a/b) from a faithful q (exact remainder test); a, b, q in range
    __device__ __forceinline__ static double round_quotient(double a, double b, double q) {
        const double r = __fma_rn(-b, q, a);                 // exact
        const int qhi = __double2hiint(q), qlo = __double2loint(q);
        const unsigned eq = ((unsigned)qhi >> 20) & 0x7ffu;
        // the step moves |q| up when r/b has the sign of q
        const bool up = (((unsigned)__double2hiint(r) ^ (unsigned)__double2hiint(b)) >> 31) == ((unsigned)qhi >> 31);
        const bool pow2 = ((qhi & 0x000fffff) | qlo) == 0;   // gap below |q| is half the gap above
        const unsigned sh = (!up && pow2) ? 54u : 53u;
        const double half_gap = __hiloint2double((int)((eq - sh) << 20), 0);
        const bool move = fabs(r) > fabs(b) * half_gap;
        const long long qb = __double_as_longlong(q);
        return __longlong_as_double(qb + (move ? (up ? 1ll : -1ll) : 0ll));
    }
    // a denominator with its correctly rounded reciprocal
    __device__ __forceinline__ Den den(double b) {
        ok = ok && in_range(b);
        const double y = rcp_newton(b);
        return Den{b, round_quotient(1.0, b, y)};
    }
    // A numerator below 2^-450 (the characteristic differences of a nearly
    // constant region square down to such values) is scaled by 2^600, which
    // is exact, and the quotient scaled back by 2^-600, which is exact while
    // the quotient stays normal (|q| >= 2^-1022, checked with a margin).
    __device__ __forceinline__ static bool tiny(double a) {
        return (((unsigned)__double2hiint(a) >> 20) & 0x7ffu) < 573u;
    }
    __device__ __forceinline__ bool unscale_ok(double qs) {
        return (((unsigned)__double2hiint(qs) >> 20) & 0x7ffu) >= 603u;
    }
    // a / d.b with y = RN(1/d.b): Markstein's two corrections
    __device__ __forceinline__ double q(double a, const Den &d) {
        const bool t = tiny(a);
        const double as = t ? a * 0x1p600 : a;
        const double q0 = as * d.y;
        const double q1 = __fma_rn(__fma_rn(-d.b, q0, as), d.y, q0);
        const double q2 = __fma_rn(__fma_rn(-d.b, q1, as), d.y, q1);
        const double qs = as == 0.0 ? q0 : q2;
        ok = ok && (as == 0.0 || (in_range(as) && (!t || unscale_ok(qs))));
        return t ? qs * 0x1p-600 : qs;
    }
    // a / b, b used once
    __device__ __forceinline__ double q(double a, double b) {
        const bool t = tiny(a);
        const double as = t ? a * 0x1p600 : a;
        const double y = rcp_newton(b);
        const double q0 = as * y;
        const double q1 = __fma_rn(__fma_rn(-b, q0, as), y, q0);   // faithful
        const double qs = as == 0.0 ? q0 : round_quotient(as, b, q1);
        ok = ok && in_range(b) && (as == 0.0 || (in_range(as) && (!t || unscale_ok(qs))));
        return t ? qs * 0x1p-600 : qs;
    }
};

// Division by the two constant denominators (gama - 1 and d2 of WCNS_Z3)
// with one correction, every other division as the compiler forms it.
// With y = RN(1/c) from the host, q0 = RN(a*y) is already within one ulp of
// a/c for every a when |y*c - 1| < 2^-54 (the error of a*y is then below
// 0.86 ulp of a/c); y*c - 1 is -2^-72 for gama - 1 and -2^-54.46 for d2, so
// one correction q0 + (a - c*q0)*y gives RN(a/c) by Markstein's theorem.
// Numerators below 2^-450 are scaled as in DivNR; any other operand outside
// the range clears ok (the caller computes the face again).
struct DenC {
    double b, y;
};
struct DivConst {
    DenC gm1, d2;
    bool ok = true;
    __device__ __forceinline__ DivConst(DenC g1, DenC dd) : gm1(g1), d2(dd) {}
    __device__ __forceinline__ Den den(double b) const { return Den{b, 0.0}; }
    __device__ __forceinline__ double q(double a, const Den &d) const { return a / d.b; }
    __device__ __forceinline__ double q(double a, double b) const { return a / b; }
    __device__ __forceinline__ double q(double a, const DenC &d) {
        const bool t = DivNR::tiny(a);
        const double as = t ? a * 0x1p600 : a;
        const double q0 = as * d.y;
        const double q1 = __fma_rn(__fma_rn(-d.b, q0, as), d.y, q0);
        const double qs = as == 0.0 ? q0 : q1;
        ok = ok && (as == 0.0 || (DivNR::in_range(as) && (!t || (((unsigned)__double2hiint(qs) >> 20) & 0x7ffu) >= 603u)));
        return t ? qs * 0x1p-600 : qs;
    }
};

}  // namespace fdm
