/*
 * bte_oracle_math.h -- ORACLE (test infrastructure only).
 *
 * Deterministic single-precision elementary functions for the CPU oracle.
 * Every function takes and returns float but evaluates internally in IEEE
 * double with an explicit, fixed sequence of operations (fma() where a fused
 * multiply-add is wanted, nothing contracted implicitly: this file must be
 * compiled with -ffp-contract=off).  The CUDA kernels of the product carry an
 * independently written copy of the same algorithms (bte_math.cuh); because
 * both sides perform the same IEEE-754 double operations, the two produce
 * bit-identical float results, which is what makes per-sample GPU-vs-oracle
 * comparisons exact.
 *
 * Methods (all published / from the mathematics, none taken from a vendor
 * math library):
 *   - argument reduction: W. J. Cody and W. Waite, "Software Manual for the
 *     Elementary Functions" (1980): x - k*C split into a three-part constant.
 *     The constant parts are pi/2 and ln 2 computed to 80 digits (Machin's
 *     formula for pi, 2*atanh(1/3) for ln 2) and split into doubles.
 *   - sin/cos: Taylor series on |r| <= pi/4 (degree 13 / 14).
 *   - exp: Taylor series of e^r on |r| <= ln2/2 (degree 12), scaled by 2^k.
 *   - log: log(m) = 2*atanh((m-1)/(m+1)) series, m in [sqrt(1/2), sqrt(2)).
 *   - atan: two half-angle reductions atan(z) = 2*atan(z/(1+sqrt(1+z^2)))
 *     followed by the Gregory series.
 *   - pow: exp(y*log|x|) evaluated in double, C99 Annex F special cases.
 * Accuracy: the double-evaluated result has relative error < 1e-13 before
 * the final rounding to float, so the returned float is the correctly
 * rounded value except in rare near-halfway cases (tests measure it against
 * long-double references).
 * Domain note: sin/cos/tan reduce accurately for |x| < 2^20; beyond that they
 * stay deterministic but lose accuracy (the renderer's angles are < 10).
 */
#ifndef BTE_ORACLE_MATH_H
#define BTE_ORACLE_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#define OM_PIO2_1 0x1.921fb54442d18p+0
#define OM_PIO2_2 0x1.1a62633145c07p-54
#define OM_PIO2_3 (-0x1.f1976b7ed8fbcp-110)
#define OM_PI_D 0x1.921fb54442d18p+1
#define OM_PIO4_D 0x1.921fb54442d18p-1
#define OM_TWO_OVER_PI 0.6366197723675814
#define OM_LN2_1 0x1.62e42fefa39efp-1
#define OM_LN2_2 0x1.abc9e3b39803fp-56
#define OM_INV_LN2 1.4426950408889634
#define OM_SQRT2 1.4142135623730951

static inline uint64_t om_dbits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
static inline double om_bitsd(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* ---- sin / cos of a reduced argument |r| <= pi/4 (double) ---- */
static inline double om_sin_poly(double r)
{
    const double s = r * r;
    double p = 1.0 / 6227020800.0;              /*  1/13! */
    p = fma(p, s, -1.0 / 39916800.0);           /* -1/11! */
    p = fma(p, s, 1.0 / 362880.0);              /*  1/9!  */
    p = fma(p, s, -1.0 / 5040.0);               /* -1/7!  */
    p = fma(p, s, 1.0 / 120.0);                 /*  1/5!  */
    p = fma(p, s, -1.0 / 6.0);                  /* -1/3!  */
    return fma(r * s, p, r);
}

static inline double om_cos_poly(double r)
{
    const double s = r * r;
    double p = -1.0 / 87178291200.0;            /* -1/14! */
    p = fma(p, s, 1.0 / 479001600.0);           /*  1/12! */
    p = fma(p, s, -1.0 / 3628800.0);            /* -1/10! */
    p = fma(p, s, 1.0 / 40320.0);               /*  1/8!  */
    p = fma(p, s, -1.0 / 720.0);                /* -1/6!  */
    p = fma(p, s, 1.0 / 24.0);                  /*  1/4!  */
    p = fma(p, s, -0.5);                        /* -1/2!  */
    return fma(p, s, 1.0);
}

/* Reduce x (finite) to r in [-pi/4, pi/4] and quadrant q = k mod 4. */
static inline double om_reduce_pio2(double x, int* q)
{
    const double k = rint(x * OM_TWO_OVER_PI);
    double r = fma(-k, OM_PIO2_1, x);
    r = fma(-k, OM_PIO2_2, r);
    r = fma(-k, OM_PIO2_3, r);
    const int64_t ki = (int64_t)k;
    *q = (int)(ki & 3);
    return r;
}

static inline double om_sin_d(double x)
{
    int q;
    const double r = om_reduce_pio2(x, &q);
    switch (q) {
    case 0: return om_sin_poly(r);
    case 1: return om_cos_poly(r);
    case 2: return -om_sin_poly(r);
    default: return -om_cos_poly(r);
    }
}

static inline double om_cos_d(double x)
{
    int q;
    const double r = om_reduce_pio2(x, &q);
    switch (q) {
    case 0: return om_cos_poly(r);
    case 1: return -om_sin_poly(r);
    case 2: return -om_cos_poly(r);
    default: return om_sin_poly(r);
    }
}

static inline float om_sinf(float x)
{
    if (x == 0.0f || x != x) return x + x * 0.0f; /* keeps -0, propagates NaN */
    if (isinf(x)) return NAN;
    return (float)om_sin_d((double)x);
}

static inline float om_cosf(float x)
{
    if (x != x) return x;
    if (isinf(x)) return NAN;
    return (float)om_cos_d((double)x);
}

static inline float om_tanf(float x)
{
    if (x == 0.0f || x != x) return x + x * 0.0f;
    if (isinf(x)) return NAN;
    int q;
    const double r = om_reduce_pio2((double)x, &q);
    const double s = om_sin_poly(r), c = om_cos_poly(r);
    return (float)((q & 1) ? (-c / s) : (s / c));
}

/* ---- exp ---- */
/* e^x for a double x with |x| < 1024*ln2 (no special cases). */
static inline double om_exp_d(double x)
{
    const double k = rint(x * OM_INV_LN2);
    double r = fma(-k, OM_LN2_1, x);
    r = fma(-k, OM_LN2_2, r);
    double p = 1.0 / 479001600.0;               /* 1/12! */
    p = fma(p, r, 1.0 / 39916800.0);            /* 1/11! */
    p = fma(p, r, 1.0 / 3628800.0);             /* 1/10! */
    p = fma(p, r, 1.0 / 362880.0);              /* 1/9!  */
    p = fma(p, r, 1.0 / 40320.0);               /* 1/8!  */
    p = fma(p, r, 1.0 / 5040.0);                /* 1/7!  */
    p = fma(p, r, 1.0 / 720.0);                 /* 1/6!  */
    p = fma(p, r, 1.0 / 120.0);                 /* 1/5!  */
    p = fma(p, r, 1.0 / 24.0);                  /* 1/4!  */
    p = fma(p, r, 1.0 / 6.0);                   /* 1/3!  */
    p = fma(p, r, 0.5);                         /* 1/2!  */
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    /* 2^k split in two factors so that k in [-1074, 1023] never overflows the
     * exponent field of either factor. */
    const int64_t ki = (int64_t)k;
    const int64_t k1 = ki / 2, k2 = ki - k1;
    const double s1 = om_bitsd((uint64_t)(k1 + 1023) << 52);
    const double s2 = om_bitsd((uint64_t)(k2 + 1023) << 52);
    return (p * s1) * s2;
}

static inline float om_expf(float x)
{
    if (x != x) return x;
    if (x > 89.0f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    return (float)om_exp_d((double)x);
}

/* ---- log ---- */
/* natural log of a finite, positive double (normal or subnormal float value) */
static inline double om_log_d(double x)
{
    uint64_t u = om_dbits(x);
    int e = (int)((u >> 52) & 0x7ff) - 1023;
    double m = om_bitsd((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL); /* [1,2) */
    if (m > OM_SQRT2) { m = m * 0.5; e += 1; }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double p = 1.0 / 21.0;
    p = fma(p, z, 1.0 / 19.0);
    p = fma(p, z, 1.0 / 17.0);
    p = fma(p, z, 1.0 / 15.0);
    p = fma(p, z, 1.0 / 13.0);
    p = fma(p, z, 1.0 / 11.0);
    p = fma(p, z, 1.0 / 9.0);
    p = fma(p, z, 1.0 / 7.0);
    p = fma(p, z, 1.0 / 5.0);
    p = fma(p, z, 1.0 / 3.0);
    const double twoS = 2.0 * s;
    const double lm = fma(twoS * z, p, twoS);
    const double ed = (double)e;
    return fma(ed, OM_LN2_1, fma(ed, OM_LN2_2, lm));
}

static inline float om_logf(float x)
{
    if (x != x) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (isinf(x)) return x;
    return (float)om_log_d((double)x);
}

/* ---- pow (C99 Annex F special cases) ---- */
static inline int om_is_int(float y) { return floorf(y) == y; }
static inline int om_is_odd_int(float y)
{
    if (!om_is_int(y) || fabsf(y) >= 16777216.0f) return 0;
    const int64_t i = (int64_t)y;
    return (int)(i & 1);
}

static inline float om_powf(float x, float y)
{
    if (y == 0.0f) return 1.0f;
    if (x == 1.0f) return 1.0f;
    if (x != x || y != y) return NAN;
    if (isinf(y)) {
        const float ax = fabsf(x);
        if (ax == 1.0f) return 1.0f;
        if ((ax < 1.0f) == (y < 0.0f)) return INFINITY;
        return 0.0f;
    }
    if (x == 0.0f) {
        const int odd = om_is_odd_int(y);
        if (y < 0.0f) return odd ? copysignf(INFINITY, x) : INFINITY;
        return odd ? x : 0.0f;
    }
    if (isinf(x)) {
        const int odd = om_is_odd_int(y);
        if (x < 0.0f) {
            if (y < 0.0f) return odd ? -0.0f : 0.0f;
            return odd ? -INFINITY : INFINITY;
        }
        return (y < 0.0f) ? 0.0f : INFINITY;
    }
    float sign = 1.0f;
    if (x < 0.0f) {
        if (!om_is_int(y)) return NAN;
        if (om_is_odd_int(y)) sign = -1.0f;
    }
    const double l = (double)y * om_log_d(fabs((double)x));
    if (l > 89.0) return sign * INFINITY;
    if (l < -104.0) return sign * 0.0f;
    return sign * (float)om_exp_d(l);
}

/* x^5 and x^2 (the reference's powf(x, 5) / powf(x, 2) call sites): double
 * products rounded once to float -- correctly rounded except in vanishingly
 * rare near-halfway cases; C99 pow special values for odd/even exponents. */
static inline float om_pow5f(float x)
{
    const double d = (double)x;
    const double d2 = d * d;
    const double d4 = d2 * d2;
    return (float)(d4 * d);
}
static inline float om_pow2f(float x)
{
    const double d = (double)x;
    return (float)(d * d);
}

/* ---- atan2 / acos ---- */
/* atan of z in [0, 1] (double) */
static inline double om_atan01_d(double z)
{
    double w = z / (1.0 + sqrt(fma(z, z, 1.0)));
    w = w / (1.0 + sqrt(fma(w, w, 1.0)));
    const double s = w * w;
    double p = -1.0 / 21.0;
    p = fma(p, s, 1.0 / 19.0);
    p = fma(p, s, -1.0 / 17.0);
    p = fma(p, s, 1.0 / 15.0);
    p = fma(p, s, -1.0 / 13.0);
    p = fma(p, s, 1.0 / 11.0);
    p = fma(p, s, -1.0 / 9.0);
    p = fma(p, s, 1.0 / 7.0);
    p = fma(p, s, -1.0 / 5.0);
    p = fma(p, s, 1.0 / 3.0);
    const double a = fma(-(w * s), p, w);
    return 4.0 * a;
}

/* atan2 for finite doubles with (y, x) != (0, 0) handled by the caller */
static inline double om_atan2_d(double y, double x)
{
    const double ay = fabs(y), ax = fabs(x);
    double a;
    if (ay <= ax) a = om_atan01_d(ay / ax);
    else          a = OM_PIO2_1 - om_atan01_d(ax / ay);
    if (x < 0.0) a = OM_PI_D - a;
    return (y < 0.0) ? -a : a;
}

static inline float om_atan2f(float y, float x)
{
    if (x != x || y != y) return NAN;
    if (y == 0.0f) {
        if (x > 0.0f || (x == 0.0f && !signbit(x))) return y;          /* +-0 */
        return signbit(y) ? -(float)OM_PI_D : (float)OM_PI_D;         /* x < 0 or -0 */
    }
    if (isinf(x) || isinf(y)) {
        double a;
        if (isinf(x) && isinf(y)) a = (x > 0.0f) ? OM_PIO4_D : 3.0 * OM_PIO4_D;
        else if (isinf(y))        a = OM_PIO2_1;
        else                      a = (x > 0.0f) ? 0.0 : OM_PI_D;
        return (float)(y < 0.0f ? -a : a);
    }
    if (x == 0.0f) return (y > 0.0f) ? (float)OM_PIO2_1 : -(float)OM_PIO2_1;
    return (float)om_atan2_d((double)y, (double)x);
}

static inline float om_acosf(float x)
{
    if (x != x) return x;
    if (x > 1.0f || x < -1.0f) return NAN;
    if (x == 1.0f) return 0.0f;
    const double xd = (double)x;
    const double s = sqrt((1.0 - xd) * (1.0 + xd));
    if (xd == 0.0) return (float)OM_PIO2_1;
    return (float)om_atan2_d(s, xd);
}

#endif /* BTE_ORACLE_MATH_H */
