/*
 * swehr_math.h -- deterministic elementary functions shared, unchanged, by
 * the CUDA kernels (nvcc, device code) and the CPU restatement (gcc).
 *
 * The reference calls glibc's libm (pow, exp, cos, sin, atan; SWEHR.c:354-374,
 * 728-765, 1243-1280, 1293-1307, 1331-1386, 1477-1483, 1556-1587).  libm
 * results differ between libraries in the last bit, and the SWEHR step
 * amplifies last-bit differences, so a GPU result can only be bit-identical to
 * a CPU result when both use the same function bodies.  These are those
 * bodies.  They use only IEEE-754 double +, -, *, /, sqrt and explicit fma,
 * each correctly rounded on both x86-64 and sm_100a, so a build with FP
 * contraction disabled (gcc -ffp-contract=off, nvcc --fmad=false) gives the
 * same bits on both.
 *
 * Methods (all from the open literature; constants are generated from the
 * mathematics by gen_math_tables.py):
 *   exp:   P.T.P. Tang, "Table-driven implementation of the exponential
 *          function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989:
 *          x = (64m + j) ln2/64 + r, exp(x) = 2^m 2^(j/64) e^r, 64-entry
 *          double-double table, e^r - 1 by its Taylor series to r^6
 *          (|r| <= ln2/128, truncation < 2^-63).
 *   log:   argument reduction to m in [1,2), c = 1 + i/32 nearest m,
 *          log m = log c + 2 atanh((m-c)/(m+c)) (|s| <= 1/128, odd series to
 *          s^11), evaluated in double-double (Dekker / Knuth two-sum,
 *          fma two-product).
 *   pow:   exp(y * log x) with y*log x carried as a double-double, so the
 *          result is within a hair of correct rounding; C99 Annex F special
 *          cases.  pow(x,0.5) is the correctly rounded sqrt (with pow's +0
 *          for -0), pow(x,1) = x, pow(x,2) = x*x (what gcc folds pow(x,2.0) to).
 *   cos(atan x) = 1/sqrt(1+x^2) and sin(atan x) = x/sqrt(1+x^2), exact
 *          identities, evaluated with one double-double Newton correction of
 *          the reciprocal square root.
 * Accuracy (checked by tests/test_math_shim.py against 80-digit decimal
 * references): within 0.52 ulp, i.e. correctly rounded except in rare
 * near-halfway cases.
 */
#ifndef SWEHR_MATH_H
#define SWEHR_MATH_H

#ifdef __CUDACC__
#define SW_HD static __device__ __forceinline__
#define SW_TABLE static __device__
#else
#include <math.h>
#include <stdint.h>
#include <string.h>
#define SW_HD static inline
#define SW_TABLE static
#endif

#include "swehr_math_tables.h"

#define SW_SHIFT 0x1.8p52
#define SW_INF (1.0 / 0.0)

SW_HD long long sw_bits(double x)
{
#ifdef __CUDACC__
    return __double_as_longlong(x);
#else
    long long b;
    memcpy(&b, &x, sizeof b);
    return b;
#endif
}

SW_HD double sw_from_bits(long long b)
{
#ifdef __CUDACC__
    return __longlong_as_double(b);
#else
    double x;
    memcpy(&x, &b, sizeof x);
    return x;
#endif
}

/* e^(x + xlo) for finite x in [-746, 710], |xlo| << ulp(x) allowed. */
SW_HD double sw_exp_core(double x, double xlo)
{
    double kd = fma(x, SW_INVLN2N, SW_SHIFT);
    kd = kd - SW_SHIFT;                       /* nearest integer to x*64/ln2 */
    long long k = (long long)kd;
    int j = (int)(k & 63);
    long long m = (k - j) / 64;
    double r = fma(-kd, SW_LN2N_HI, x);
    r = fma(-kd, SW_LN2N_LO, r);
    r = r + xlo;
    /* e^r - 1 = r + r^2 (1/2 + r/6 + r^2/24 + r^3/120 + r^4/720) */
    double q = fma(r, SW_INVFACT6, SW_INVFACT5);
    q = fma(r, q, SW_INVFACT4);
    q = fma(r, q, SW_INVFACT3);
    q = fma(r, q, SW_INVFACT2);
    double r2 = r * r;
    double p = fma(r2, q, r);
    double th = sw_exp2_hi[j];
    double y = th + fma(th, p, sw_exp2_lo[j]);
    /* y in [0.99, 2): scale by 2^m */
    if (m > -1020 && m < 1020)
        return sw_from_bits(sw_bits(y) + (m << 52));
    if (m >= 1020) {
        y = sw_from_bits(sw_bits(y) + ((m - 10) << 52));
        return y * 0x1p10;                    /* may overflow to +inf */
    }
    y = sw_from_bits(sw_bits(y) + ((m + 1000) << 52));
    return y * 0x1p-1000;                     /* gradual underflow, one rounding */
}

SW_HD double sw_exp(double x)
{
    if (x != x) return x;
    if (x > 709.782712893384) return SW_INF;
    if (x < -745.2) return 0.0;
    if (x > -0x1p-60 && x < 0x1p-60) return 1.0 + x;
    return sw_exp_core(x, 0.0);
}

/* log(x) as a double-double (hi + lo), x finite and > 0. */
SW_HD void sw_log_dd(double x, double *hi, double *lo)
{
    int e = 0;
    if (x < 0x1p-1022) {                      /* subnormal: scale into the normal range */
        x *= 0x1p54;
        e = -54;
    }
    long long b = sw_bits(x);
    e += (int)((b >> 52) & 0x7ff) - 1023;
    double m = sw_from_bits((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL); /* [1,2) */
    int i = (int)((m - 1.0) * 32.0 + 0.5);    /* nearest c = 1 + i/32 */
    double c = 1.0 + (double)i * 0.03125;
    double num = m - c;                       /* exact (Sterbenz) */
    double dh = m + c;                        /* two-sum */
    double bb = dh - m;
    double dl = (m - (dh - bb)) + (c - bb);
    double sh = num / dh;
    double rem = fma(-sh, dh, num);
    rem = fma(-sh, dl, rem);
    double sl = rem / dh;
    double s2 = sh * sh;
    double tq = fma(s2, SW_ATANH_C11, SW_ATANH_C9);
    tq = fma(s2, tq, SW_ATANH_C7);
    tq = fma(s2, tq, SW_ATANH_C5);
    tq = fma(s2, tq, SW_ATANH_C3);
    double tail = (sh * s2) * tq;
    double l1h = 2.0 * sh;
    double l1l = fma(2.0, sl, tail);
    double ed = (double)e;
    double ah = ed * SW_LN2_HI;
    double al = fma(ed, SW_LN2_HI, -ah);
    al = fma(ed, SW_LN2_LO, al);
    /* (ah + logc_hi) + l1h with error terms */
    double s1 = ah + sw_logc_hi[i];
    double t1 = s1 - ah;
    double e1 = (ah - (s1 - t1)) + (sw_logc_hi[i] - t1);
    double s3 = s1 + l1h;
    double t3 = s3 - s1;
    double e3 = (s1 - (s3 - t3)) + (l1h - t3);
    double low = ((al + sw_logc_lo[i]) + l1l) + (e1 + e3);
    double h = s3 + low;
    *lo = low - (h - s3);
    *hi = h;
}

SW_HD double sw_sqrt_pow(double x)
{
    /* pow(x, 0.5): correctly rounded sqrt, +0 for -0, +inf for -inf */
    if (x == -SW_INF) return SW_INF;
    double r = sqrt(x);
    return (r == 0.0) ? 0.0 : r;
}

SW_HD int sw_is_int(double y)
{
    if (y > 0x1p53 || y < -0x1p53) return 1;
    return y == (double)(long long)y;
}

SW_HD int sw_is_odd_int(double y)
{
    if (y > 0x1p53 || y < -0x1p53) return 0;
    long long k = (long long)y;
    return (y == (double)k) && (k & 1);
}

/* x^4 as the square of x^2, both squares carried as double-doubles: the
 * error before the final rounding is about 2^-104 relative, so the result is
 * the correctly rounded x^4 unless x^4 lies that close to a rounding
 * boundary.  Finite x with x^4 in the normal range. */
SW_HD double sw_pow4(double x)
{
    double p = x * x;
    double e = fma(x, x, -p);                 /* x^2 = p + e exactly */
    double P = p * p;
    double lo = fma(p, p, -P);                /* p^2 = P + lo exactly */
    lo = fma(2.0 * p, e, lo);                 /* + 2 p e; e^2 is below 2^-104 P */
    return P + lo;
}

SW_HD double sw_pow(double x, double y)
{
    if (y == 0.5) return sw_sqrt_pow(x);
    if (y == 1.0) return x;
    if (y == 2.0) return x * x;
    if (y == 4.0) {
        double ax4 = x < 0 ? -x : x;
        if (ax4 >= 0x1p-250 && ax4 <= 0x1p250) return sw_pow4(x);
    }
    if (y == 0.0 || x == 1.0) return 1.0;
    if (x != x || y != y) return x + y;
    double ax = x < 0 ? -x : x;
    double sign = 1.0;
    if (x < 0) {
        if (!sw_is_int(y)) return (x - x) / (x - x);   /* NaN */
        if (sw_is_odd_int(y)) sign = -1.0;
    }
    if (ax == 0.0) {
        if (y > 0) return sw_is_odd_int(y) ? x : 0.0;
        return sw_is_odd_int(y) ? 1.0 / x : SW_INF;
    }
    if (ax == SW_INF) {
        if (y > 0) return sign * (SW_INF);
        return sign * 0.0;
    }
    if (y == SW_INF || y == -SW_INF) {
        if (ax == 1.0) return 1.0;
        if ((ax > 1.0) == (y > 0)) return SW_INF;
        return 0.0;
    }
    double lh, ll;
    sw_log_dd(ax, &lh, &ll);
    double th = y * lh;
    double tl = fma(y, lh, -th);
    tl = fma(y, ll, tl);
    if (th > 709.79) return sign * (SW_INF);
    if (th < -745.2) return sign * 0.0;
    return sign * sw_exp_core(th, tl);
}

/* cos(atan(x)) = 1/sqrt(1+x^2) */
SW_HD double sw_cos_atan(double x)
{
    double ax = x < 0 ? -x : x;
    if (ax != ax) return x;
    if (ax > 1e150) return 1.0 / ax;
    double p = ax * ax;
    double pe = fma(ax, ax, -p);
    double sh = 1.0 + p;                      /* two-sum(1, p) */
    double bb = sh - 1.0;
    double sl = ((1.0 - (sh - bb)) + (p - bb)) + pe;
    double r0 = 1.0 / sqrt(sh);
    double q = r0 * r0;
    double qe = fma(r0, r0, -q);
    double e = fma(-sh, q, 1.0);              /* 1 - s r0^2, error terms below */
    e = fma(-sh, qe, e);
    e = fma(-sl, q, e);
    return fma(r0, 0.5 * e, r0);
}

/* sin(atan(x)) = x/sqrt(1+x^2) */
SW_HD double sw_sin_atan(double x)
{
    double ax = x < 0 ? -x : x;
    if (ax != ax) return x;
    if (ax > 1e150) return x < 0 ? -1.0 : 1.0;
    double p = ax * ax;
    double pe = fma(ax, ax, -p);
    double sh = 1.0 + p;
    double bb = sh - 1.0;
    double sl = ((1.0 - (sh - bb)) + (p - bb)) + pe;
    double r0 = 1.0 / sqrt(sh);
    double q = r0 * r0;
    double qe = fma(r0, r0, -q);
    double e = fma(-sh, q, 1.0);
    e = fma(-sh, qe, e);
    e = fma(-sl, q, e);
    double d = r0 * (0.5 * e);
    return fma(x, r0, x * d);
}

#endif /* SWEHR_MATH_H */
