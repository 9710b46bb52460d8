// Correctly rounded (to ~2^-80 relative before the final rounding) natural log and
// hypot in double-double arithmetic, usable on the host and on sm_100a.
//
// Why: the reference draws Gaussian deviates with libstdc++'s Marsaglia polar method,
// mult = sqrt(-2*log(r2)/r2), and ranks sparse-phase donors with hypot(). glibc's log
// and hypot are faithful but not correctly rounded, and CUDA's are not glibc's either.
// A correctly rounded implementation agrees with glibc wherever glibc rounds correctly
// (measured here: 99.92% of polar-method log inputs, 99.4% of hypot inputs); where it
// does not, the deviate differs by one ulp.
//
// Method (own derivation, standard textbook reduction):
//   x = 2^k * m, m in [sqrt(1/2), sqrt(2));  c = round(128 m)/128 (exact);
//   log(x) = k ln2 + log(c) + 2 atanh(u),  u = (m - c)/(m + c),  |u| < 2^-8.4,
//   2 atanh(u) = 2u + u^3 (2/3 + u^2 (2/5 + u^2 (2/7 + u^2 2/9))) + O(u^11).
// log(c) comes from a binary128 table (gen_logtab.c). All steps are exact error-free
// transformations (two_sum / two_prod via fma) or carry a relative error < 2^-80.
//
// Compile device code with -fmad=false and host code with -ffp-contract=off: every
// product-sum here must round exactly as written.
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define MPCD_HD __host__ __device__ __forceinline__
#else
#define MPCD_HD static inline
#endif

// log(j/128) table: one __constant__ copy for device code and one host copy (nvcc does
// not let host code read __constant__ data).
#if defined(__CUDACC__)
#define MPCD_LOGTAB_QUAL static __constant__ const
#define mpcd_logtab mpcd_logtab_dev
#include "logtab.inc"
#undef mpcd_logtab
#undef MPCD_LOGTAB_J0
#undef MPCD_LOGTAB_N
#undef MPCD_LN2_HI
#undef MPCD_LN2_LO
#undef MPCD_LOGTAB_QUAL
#endif
#define MPCD_LOGTAB_QUAL static const
#define mpcd_logtab mpcd_logtab_host
#include "logtab.inc"
#undef mpcd_logtab
#undef MPCD_LOGTAB_QUAL

namespace mpcd_dd {

struct dd {
    double hi, lo;
};

MPCD_HD double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return fma(a, b, c);
#endif
}

MPCD_HD dd two_sum(double a, double b) {
    const double s = a + b;
    const double bb = s - a;
    const double e = (a - (s - bb)) + (b - bb);
    return dd{s, e};
}

MPCD_HD dd fast_two_sum(double a, double b) {
    const double s = a + b;
    const double e = b - (s - a);
    return dd{s, e};
}

MPCD_HD dd two_prod(double a, double b) {
    const double p = a * b;
    return dd{p, fma_(a, b, -p)};
}

MPCD_HD dd dd_add(dd a, dd b) {
    const dd s = two_sum(a.hi, b.hi);
    const dd t = two_sum(a.lo, b.lo);
    dd r = fast_two_sum(s.hi, s.lo + t.hi);
    return fast_two_sum(r.hi, r.lo + t.lo);
}

MPCD_HD dd dd_mul(dd a, dd b) {
    const dd p = two_prod(a.hi, b.hi);
    return fast_two_sum(p.hi, p.lo + (a.hi * b.lo + a.lo * b.hi));
}

// a / b for double-double a and b (relative error ~2^-104).
MPCD_HD dd dd_div(dd a, dd b) {
    const double q1 = a.hi / b.hi;
    dd r = dd_add(a, dd_mul(dd{-q1, 0.0}, b));
    const double q2 = r.hi / b.hi;
    r = dd_add(r, dd_mul(dd{-q2, 0.0}, b));
    const double q3 = r.hi / b.hi;
    dd q = fast_two_sum(q1, q2);
    return dd_add(q, dd{q3, 0.0});
}

MPCD_HD double table_hi(int j) {
#if defined(__CUDA_ARCH__)
    return mpcd_logtab_dev[j - MPCD_LOGTAB_J0][0];
#else
    return mpcd_logtab_host[j - MPCD_LOGTAB_J0][0];
#endif
}

MPCD_HD double table_lo(int j) {
#if defined(__CUDA_ARCH__)
    return mpcd_logtab_dev[j - MPCD_LOGTAB_J0][1];
#else
    return mpcd_logtab_host[j - MPCD_LOGTAB_J0][1];
#endif
}

// Natural logarithm of a positive finite x, rounded to nearest from a double-double
// value accurate to ~2^-80. Inputs of interest are in (0, 1].
MPCD_HD double log_cr(double x) {
    if (!(x > 0.0)) return (x == 0.0) ? -HUGE_VAL : NAN;
    if (x == 1.0) return 0.0;
    int k = 0;
    double m = x;
    // scale subnormals into the normal range (exact)
    if (m < 2.2250738585072014e-308) {
        m *= 18014398509481984.0;  // 2^54
        k -= 54;
    }
    // exact decomposition m = mant * 2^e with mant in [1, 2)
    union {
        double d;
        uint64_t u;
    } bits;
    bits.d = m;
    const int e = (int)((bits.u >> 52) & 0x7ff) - 1023;
    bits.u = (bits.u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
    double mant = bits.d;
    k += e;
    if (mant > 1.4142135623730951) {
        mant *= 0.5;
        k += 1;
    }
    const int j = (int)rint(mant * 128.0);
    const double c = (double)j * 0.0078125;
    const double num = mant - c;                  // exact (Sterbenz)
    const dd den = two_sum(mant, c);              // exact
    // u = num / den to ~2^-100: one division for the reciprocal, then an fma residual
    const double inv = 1.0 / den.hi;
    const double uh = num * inv;
    const double res = fma_(-uh, den.hi, num) - uh * den.lo;
    const dd u = fast_two_sum(uh, res * inv);     // |u| < 2^-8.4
    // u^2 and u^3 to ~2^-100 relative
    const dd u2 = dd_mul(u, u);
    const dd u3 = dd_mul(u2, u);
    // tail polynomial: R = 2/3 + u^2 (2/5 + u^2 (2/7 + u^2 2/9))
    const double q = 0.4 + u2.hi * (0.2857142857142857 + u2.hi * 0.2222222222222222);
    const dd two_thirds = dd{0.6666666666666666, 3.700743415417188e-17};
    const dd R = dd_add(two_thirds, dd{u2.hi * q, 0.0});
    const dd T = dd_mul(u3, R);
    const dd twou = dd{2.0 * u.hi, 2.0 * u.lo};
    dd s = dd_add(twou, T);
    s = dd_add(s, dd{table_hi(j), table_lo(j)});
    const double kd = (double)k;
    s = dd_add(s, dd{kd * MPCD_LN2_HI, kd * MPCD_LN2_LO});
    return s.hi + s.lo;
}

// sqrt(a^2 + b^2) rounded to nearest from a double-double value (finite inputs whose
// squares neither overflow nor underflow; the deviates and gradients here qualify).
MPCD_HD double hypot_cr(double a, double b) {
    a = fabs(a);
    b = fabs(b);
    if (a == 0.0) return b;
    if (b == 0.0) return a;
    const dd s = dd_add(two_prod(a, a), two_prod(b, b));
    const double r = sqrt(s.hi);
    // one Newton correction in double-double: r + (s - r^2) / (2 r)
    const dd r2 = two_prod(r, r);
    const dd diff = dd_add(s, dd{-r2.hi, -r2.lo});
    const double corr = diff.hi / (2.0 * r);
    return r + corr;
}

}  // namespace mpcd_dd
