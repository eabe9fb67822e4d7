/*
 * ln_dd.h -- a natural logarithm for (0, 1] evaluated in double-double
 * arithmetic and rounded once.  The same C source compiles for the host
 * (C or C++) and the device (CUDA) and gives the same bits on both: every
 * operation is an IEEE-754 round-to-nearest +, -, *, / or an fma whose
 * result is exact, written out explicitly so that no compiler may contract
 * or reorder it (on the device through the __d*_rn intrinsics, on the host
 * as plain operators in a translation unit built with -ffp-contract=off).
 * It serves the exponential event-time sampler (`-ln(U(0,1]) / lambda`),
 * whose event times must agree bit for bit between the GPU and its checker.
 *
 * Method: x = m * 2^k with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s) with
 * s = (m - 1) / (m + 1), |s| <= 0.1716, t = s^2 <= 0.02944, summed as
 * 2 s (1 + t/3 + t^2/5 + ... + t^21/43) in double-double arithmetic (Dekker
 * 1971; Knuth's TwoSum; the exact product error fma(a, b, -a*b)); the
 * truncation error t^22/45 is below 2^-117.  Then ln x = k ln 2 + ln m with
 * ln 2 as a double-double constant.  The coefficients 1/(2j+1) and ln 2 are
 * the double-double roundings of the exact values.  The intermediate
 * relative error is ~2^-100, so the final rounding gives the correctly
 * rounded logarithm except for inputs within ~2^-47 ulp of a rounding
 * boundary (none met in tests).
 */
#ifndef NECSIM_LN_DD_H
#define NECSIM_LN_DD_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NECSIM_DD_FN static __host__ __device__ __forceinline__
#else
#define NECSIM_DD_FN static inline
#endif

#if defined(__CUDA_ARCH__)
#define NECSIM_DD_ADD(a, b) __dadd_rn((a), (b))
#define NECSIM_DD_SUB(a, b) __dsub_rn((a), (b))
#define NECSIM_DD_MUL(a, b) __dmul_rn((a), (b))
#define NECSIM_DD_DIV(a, b) __ddiv_rn((a), (b))
#define NECSIM_DD_FMA(a, b, c) __fma_rn((a), (b), (c))
#else
#define NECSIM_DD_ADD(a, b) ((a) + (b))
#define NECSIM_DD_SUB(a, b) ((a) - (b))
#define NECSIM_DD_MUL(a, b) ((a) * (b))
#define NECSIM_DD_DIV(a, b) ((a) / (b))
#define NECSIM_DD_FMA(a, b, c) fma((a), (b), (c))
#endif

typedef struct necsim_dd {
    double hi, lo;
} necsim_dd;

NECSIM_DD_FN necsim_dd necsim_dd_make(double hi, double lo) {
    necsim_dd r;
    r.hi = hi;
    r.lo = lo;
    return r;
}

/* a + b = s + e exactly (Knuth) */
NECSIM_DD_FN necsim_dd necsim_dd_two_sum(double a, double b) {
    const double s = NECSIM_DD_ADD(a, b);
    const double bb = NECSIM_DD_SUB(s, a);
    return necsim_dd_make(s, NECSIM_DD_ADD(NECSIM_DD_SUB(a, NECSIM_DD_SUB(s, bb)), NECSIM_DD_SUB(b, bb)));
}

/* a + b = s + e exactly when |a| >= |b| (Dekker) */
NECSIM_DD_FN necsim_dd necsim_dd_quick_two_sum(double a, double b) {
    const double s = NECSIM_DD_ADD(a, b);
    return necsim_dd_make(s, NECSIM_DD_SUB(b, NECSIM_DD_SUB(s, a)));
}

/* a * b = p + e exactly; the fma computes the exact residual */
NECSIM_DD_FN necsim_dd necsim_dd_two_prod(double a, double b) {
    const double p = NECSIM_DD_MUL(a, b);
    return necsim_dd_make(p, NECSIM_DD_FMA(a, b, -p));
}

NECSIM_DD_FN necsim_dd necsim_dd_add(necsim_dd a, necsim_dd b) {
    necsim_dd s = necsim_dd_two_sum(a.hi, b.hi);
    const necsim_dd t = necsim_dd_two_sum(a.lo, b.lo);
    s = necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, t.hi));
    return necsim_dd_quick_two_sum(s.hi, NECSIM_DD_ADD(s.lo, t.lo));
}

NECSIM_DD_FN necsim_dd necsim_dd_mul(necsim_dd a, necsim_dd b) {
    const necsim_dd p = necsim_dd_two_prod(a.hi, b.hi);
    const double cross = NECSIM_DD_ADD(NECSIM_DD_MUL(a.hi, b.lo), NECSIM_DD_MUL(a.lo, b.hi));
    return necsim_dd_quick_two_sum(p.hi, NECSIM_DD_ADD(p.lo, cross));
}

/* three-quotient long division a / b */
NECSIM_DD_FN necsim_dd necsim_dd_div(necsim_dd a, necsim_dd b) {
    const double q1 = NECSIM_DD_DIV(a.hi, b.hi);
    necsim_dd r = necsim_dd_add(a, necsim_dd_mul(b, necsim_dd_make(-q1, 0.0)));
    const double q2 = NECSIM_DD_DIV(r.hi, b.hi);
    r = necsim_dd_add(r, necsim_dd_mul(b, necsim_dd_make(-q2, 0.0)));
    const double q3 = NECSIM_DD_DIV(r.hi, b.hi);
    return necsim_dd_add(necsim_dd_quick_two_sum(q1, q2), necsim_dd_make(q3, 0.0));
}

/* ln(x) for normal doubles 0 < x <= 1, one rounding of a double-double */
NECSIM_DD_FN double necsim_ln(double x) {
    /* 1/(2j+1), j = 0..21, as double-double roundings of the exact ratios */
    const double c_hi[22] = {
        0x1.0000000000000p+0, 0x1.5555555555555p-2, 0x1.999999999999ap-3, 0x1.2492492492492p-3,
        0x1.c71c71c71c71cp-4, 0x1.745d1745d1746p-4, 0x1.3b13b13b13b14p-4, 0x1.1111111111111p-4,
        0x1.e1e1e1e1e1e1ep-5, 0x1.af286bca1af28p-5, 0x1.8618618618618p-5, 0x1.642c8590b2164p-5,
        0x1.47ae147ae147bp-5, 0x1.2f684bda12f68p-5, 0x1.1a7b9611a7b96p-5, 0x1.0842108421084p-5,
        0x1.f07c1f07c1f08p-6, 0x1.d41d41d41d41dp-6, 0x1.bacf914c1bad0p-6, 0x1.a41a41a41a41ap-6,
        0x1.8f9c18f9c18fap-6, 0x1.7d05f417d05f4p-6};
    const double c_lo[22] = {
        0.0, 0x1.5555555555555p-56, -0x1.999999999999ap-57, 0x1.2492492492492p-57,
        0x1.c71c71c71c71cp-58, -0x1.745d1745d1746p-59, -0x1.3b13b13b13b14p-58, 0x1.1111111111111p-60,
        0x1.e1e1e1e1e1e1ep-61, 0x1.af286bca1af28p-59, 0x1.8618618618618p-59, 0x1.642c8590b2164p-60,
        -0x1.eb851eb851eb8p-61, 0x1.2f684bda12f68p-59, 0x1.1a7b9611a7b96p-61, 0x1.0842108421084p-60,
        -0x1.f07c1f07c1f08p-61, 0x1.0750750750750p-60, -0x1.bacf914c1bad0p-60, 0x1.0690690690690p-60,
        -0x1.f3831f3831f38p-61, 0x1.7d05f417d05f4p-62};
    uint64_t bits;
    double m;
    int k, j;
    necsim_dd s, t, p, r;
    if (x == 1.0) return 0.0;
    memcpy(&bits, &x, 8);
    k = (int)((bits >> 52) & 0x7ff) - 1022; /* x = m * 2^k, m in [0.5, 1) */
    bits = (bits & 0x000fffffffffffffULL) | 0x3fe0000000000000ULL;
    memcpy(&m, &bits, 8);
    if (m < 0.70710678118654752) { /* into [sqrt(1/2), sqrt(2)), exactly */
        m = NECSIM_DD_MUL(m, 2.0);
        k -= 1;
    }
    /* m - 1 is exact (Sterbenz); m + 1 is carried exactly as a pair */
    s = necsim_dd_div(necsim_dd_make(NECSIM_DD_SUB(m, 1.0), 0.0), necsim_dd_two_sum(m, 1.0));
    t = necsim_dd_mul(s, s);
    p = necsim_dd_make(c_hi[21], c_lo[21]);
#if defined(__CUDACC__)
#pragma unroll
#endif
    for (j = 20; j >= 0; --j) p = necsim_dd_add(necsim_dd_make(c_hi[j], c_lo[j]), necsim_dd_mul(t, p));
    p = necsim_dd_mul(s, p);
    p.hi = NECSIM_DD_MUL(p.hi, 2.0); /* exact */
    p.lo = NECSIM_DD_MUL(p.lo, 2.0);
    r = necsim_dd_add(necsim_dd_mul(necsim_dd_make(0x1.62e42fefa39efp-1, 0x1.abc9e3b39803fp-56),
                                    necsim_dd_make((double)k, 0.0)),
                      p);
    return NECSIM_DD_ADD(r.hi, r.lo);
}

#endif /* NECSIM_LN_DD_H */
