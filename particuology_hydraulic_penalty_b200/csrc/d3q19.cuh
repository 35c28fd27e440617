// D3Q19 lattice tables and exactly-rounded FP64 helpers shared by every kernel.
//
// Index order, vectors, weights and opposites are those of the reference
// (src/lbm_dem/psc3d.py:17-43): rest, +x, -x, +y, -y, +z, -z, then the twelve
// diagonals in (+,-) pairs.  Keeping the order lets populations be compared
// element-wise with the reference.
#pragma once

#include <stdint.h>

#include <cmath>

#if defined(__CUDACC__)
#define PSC_HD __host__ __device__ __forceinline__
#else
#define PSC_HD inline
#endif

namespace psc {

constexpr int Q = 19;

// Components as constexpr functions (usable in device code with
// --expt-relaxed-constexpr and folded to constants in unrolled loops).
PSC_HD constexpr int cxv(int i) {
    return (i == 1 || i == 7 || i == 9 || i == 11 || i == 13) ? 1
           : (i == 2 || i == 8 || i == 10 || i == 12 || i == 14) ? -1 : 0;
}
PSC_HD constexpr int cyv(int i) {
    return (i == 3 || i == 7 || i == 10 || i == 15 || i == 17) ? 1
           : (i == 4 || i == 8 || i == 9 || i == 16 || i == 18) ? -1 : 0;
}
PSC_HD constexpr int czv(int i) {
    return (i == 5 || i == 11 || i == 14 || i == 15 || i == 18) ? 1
           : (i == 6 || i == 12 || i == 13 || i == 16 || i == 17) ? -1 : 0;
}
// Runtime lookups (one lane per direction): table reads instead of branch chains.
PSC_HD int cxv_rt(int i) {
    const int8_t t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[i];
}
PSC_HD int cyv_rt(int i) {
    const int8_t t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[i];
}
PSC_HD constexpr int cv(int axis, int i) { return axis == 0 ? cxv(i) : (axis == 1 ? cyv(i) : czv(i)); }
PSC_HD constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

// Weights as Python evaluates 1/3, 1/18, 1/36 (correctly rounded doubles).
constexpr double W0 = 1.0 / 3.0;
constexpr double W1 = 1.0 / 18.0;
constexpr double W2 = 1.0 / 36.0;
PSC_HD constexpr double wgt(int i) { return i == 0 ? W0 : (i < 7 ? W1 : W2); }

// c_s^2 = 1/3 and (c_s^2)^2 as the reference computes them (psc3d.py:43, :102).
constexpr double CS2 = 1.0 / 3.0;
constexpr double CS2SQ = CS2 * CS2;
// Their correctly rounded reciprocals (compile-time IEEE divisions), for xdiv_r.
constexpr double RCS2 = 1.0 / CS2;
constexpr double RCS2SQ = 1.0 / CS2SQ;

// The nine directions 2k+1 (k = 0..8) each have their opposite at 2k+2.

// ---------------------------------------------------------------------------
// IEEE round-to-nearest FP64 operations that the compiler may never contract
// into FMAs or reassociate.  They reproduce NumPy's element-wise arithmetic
// exactly (NumPy evaluates one rounded operation per ufunc call).
// ---------------------------------------------------------------------------
#if defined(__CUDA_ARCH__)
PSC_HD double xadd(double a, double b) { return __dadd_rn(a, b); }
PSC_HD double xsub(double a, double b) { return __dsub_rn(a, b); }
PSC_HD double xmul(double a, double b) { return __dmul_rn(a, b); }
PSC_HD double xdiv(double a, double b) { return __ddiv_rn(a, b); }
#else
// Host builds compile with -ffp-contract=off; SSE2 double is IEEE binary64.
PSC_HD double xadd(double a, double b) { return a + b; }
PSC_HD double xsub(double a, double b) { return a - b; }
PSC_HD double xmul(double a, double b) { return a * b; }
PSC_HD double xdiv(double a, double b) { return a / b; }
#endif

#if defined(__CUDA_ARCH__)
PSC_HD double xfma(double a, double b, double c) { return __fma_rn(a, b, c); }
#else
PSC_HD double xfma(double a, double b, double c) { return std::fma(a, b, c); }  // correctly rounded (C99 fma)
#endif

// ---------------------------------------------------------------------------
// Correctly rounded x / y from r = RN(1/y), for a divisor known in advance.
//
// Markstein's theorem (P. Markstein, "Computation of elementary functions on
// the IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990;
// "IA-64 and Elementary Functions", 2000): if r = RN(1/y) and q is a faithful
// approximation of x/y, the remainder e = x - q y is exactly representable (an
// FMA computes it exactly) and RN(q + e r) = RN(x/y).
//   q0 = RN(x r) is within 1.5 ulp of x/y (|x r - x/y| <= u |x/y| <= ulp, plus
//        half an ulp of rounding), not necessarily faithful;
//   q1 = RN(q0 + RN(x - q0 y) r) has error 1/2 ulp + O(u) ulp: faithful;
//   q2 = RN(q1 + (x - q1 y) r) = RN(x/y) by the theorem.
// Range: 2^-8 <= |y| <= 2^8 (checked by the caller: c_s^2, c_s^4, tau and rho
// here) and 2^-900 <= |x| <= 2^900, so that no remainder is subnormal and no
// quotient overflows.  x = +-0 gives x r (the signed zero of x / y); any other
// x outside the range (subnormal, huge, inf, NaN) takes the IEEE division.
// ---------------------------------------------------------------------------
PSC_HD bool div_r_divisor_ok(double y) {
    const double a = y < 0.0 ? -y : y;
    return a >= 0x1p-8 && a <= 0x1p8;
}

PSC_HD double xdiv_r(double x, double y, double r) {
    const double q0 = xmul(x, r);
    const double q1 = xfma(xfma(-q0, y, x), r, q0);
    const double q2 = xfma(xfma(-q1, y, x), r, q1);
    const double ax = x < 0.0 ? -x : x;
    if (ax >= 0x1p-900 && ax <= 0x1p900) return q2;
    return x == 0.0 ? q0 : xdiv(x, y);
}

// A divisor with its reciprocal RN(1/y): x / y by xdiv_r when y is in range,
// else by the IEEE division.
struct Divisor {
    double y, r;
    bool ok;
};
PSC_HD Divisor make_divisor(double y) {
    Divisor d;
    d.y = y;
    d.ok = div_r_divisor_ok(y);
    d.r = d.ok ? xdiv(1.0, y) : 0.0;
    return d;
}
PSC_HD double xdiv_d(double x, const Divisor& d) { return d.ok ? xdiv_r(x, d.y, d.r) : xdiv(x, d.y); }

// c * x for a lattice component c in {-1, 0, 1}.  A zero product is returned
// as +0; it only ever feeds an addition with a non-zero partner or an exact
// zero result, so the sign of zero never reaches a non-zero value.
template <int C>
PSC_HD double cmul(double x) {
    return C == 0 ? 0.0 : (C > 0 ? x : -x);
}

// Sequential sum over populations weighted by one velocity component, in
// index order from +0 (NumPy's axis-0 reduction, psc3d.py:211-214).
template <int AXIS, typename T>
PSC_HD double seq_moment_exact(const T* f) {
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < Q; ++i) {
        const int c = cv(AXIS, i);
        if (c == 1) acc = xadd(acc, f[i]);
        else if (c == -1) acc = xsub(acc, f[i]);
    }
    return acc;
}

// c_i . v for direction i, evaluated as (cx*vx + cy*vy) + cz*vz.
template <int I>
PSC_HD double cdot_exact(double vx, double vy, double vz) {
    return xadd(xadd(cmul<cxv(I)>(vx), cmul<cyv(I)>(vy)), cmul<czv(I)>(vz));
}

}  // namespace psc
