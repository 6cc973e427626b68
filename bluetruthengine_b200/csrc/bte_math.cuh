// bte_math.cuh -- deterministic single-precision elementary functions.
//
// Every function takes and returns float and evaluates in IEEE double with a
// fixed sequence of operations: explicit fma() where a fused multiply-add is
// intended, nothing contracted implicitly (the library is compiled with
// -fmad=false).  Because IEEE double add/mul/div/sqrt/fma are correctly
// rounded on both the GPU and the host, a host compilation of the same
// algorithm reproduces these results bit-for-bit; the renderer relies on that
// for exact per-sample agreement with its CPU checker.
//
// Methods (published / from the mathematics; no vendor math-library code):
//   argument reduction: Cody & Waite, "Software Manual for the Elementary
//   Functions" (1980), constants pi/2 and ln 2 to 80 digits (Machin's
//   formula, 2*atanh(1/3)) split into doubles;
//   sin/cos: Taylor series on |r| <= pi/4 (degree 13 / 14);
//   exp: Taylor series on |r| <= ln2/2 (degree 12) scaled by 2^k;
//   log: 2*atanh((m-1)/(m+1)) series on m in [sqrt(1/2), sqrt(2));
//   atan: two half-angle reductions then the Gregory series;
//   pow: exp(y*log|x|) in double with the C99 Annex F special cases.
// The double result carries relative error < 1e-13, so the returned float
// is the correctly rounded value except in rare near-halfway cases.
// sin/cos/tan reduce accurately for |x| < 2^20 (renderer angles are < 10).
#pragma once

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define BTE_HD __host__ __device__ __forceinline__
// The public functions keep one out-of-line copy per kernel: inlined at every
// call site of the shading code they overflow the instruction cache.
#define BTE_HDN __host__ __device__ __noinline__ inline
#else
#define BTE_HD inline
#define BTE_HDN inline
#endif

// Product build (BTE_FAST_MATH, compiled with fused multiply-adds allowed): on
// the device the public float functions are CUDA's own single-precision
// functions -- the ones the reference's device code calls (sinf, cosf, tanf,
// expf, logf, powf, atan2f, acosf) -- and x^5, x^2 are float products, so
// shading runs in FP32 only.  The host keeps the portable functions below.
// The parity build (no BTE_FAST_MATH) evaluates every function as documented
// above on both sides.
#if defined(BTE_FAST_MATH) && defined(__CUDA_ARCH__)
#define BTE_FAST_DEVICE_MATH 1
#else
#define BTE_FAST_DEVICE_MATH 0
#endif
#ifdef BTE_FAST_MATH
#define BTE_MATHFN BTE_HD
#else
#define BTE_MATHFN BTE_HDN
#endif

namespace bte {
namespace m {

constexpr double kPio2_1 = 0x1.921fb54442d18p+0;
constexpr double kPio2_2 = 0x1.1a62633145c07p-54;
constexpr double kPio2_3 = -0x1.f1976b7ed8fbcp-110;
constexpr double kPi = 0x1.921fb54442d18p+1;
constexpr double kPio4 = 0x1.921fb54442d18p-1;
constexpr double kTwoOverPi = 0.6366197723675814;
constexpr double kLn2_1 = 0x1.62e42fefa39efp-1;
constexpr double kLn2_2 = 0x1.abc9e3b39803fp-56;
constexpr double kInvLn2 = 1.4426950408889634;
constexpr double kSqrt2 = 1.4142135623730951;

BTE_HD uint64_t dbits(double x)
{
#ifdef __CUDA_ARCH__
    return static_cast<uint64_t>(__double_as_longlong(x));
#else
    uint64_t u; __builtin_memcpy(&u, &x, 8); return u;
#endif
}
BTE_HD double bitsd(uint64_t u)
{
#ifdef __CUDA_ARCH__
    return __longlong_as_double(static_cast<long long>(u));
#else
    double x; __builtin_memcpy(&x, &u, 8); return x;
#endif
}
BTE_HD bool isnanf_(float x) { return x != x; }
BTE_HD bool isinff_(float x) { return x == INFINITY || x == -INFINITY; }
BTE_HD bool signbitf_(float x)
{
#ifdef __CUDA_ARCH__
    return (__float_as_uint(x) >> 31) != 0;
#else
    uint32_t u; __builtin_memcpy(&u, &x, 4); return (u >> 31) != 0;
#endif
}

BTE_HD double sinPoly(double r)
{
    const double s = r * r;
    double p = 1.0 / 6227020800.0;
    p = fma(p, s, -1.0 / 39916800.0);
    p = fma(p, s, 1.0 / 362880.0);
    p = fma(p, s, -1.0 / 5040.0);
    p = fma(p, s, 1.0 / 120.0);
    p = fma(p, s, -1.0 / 6.0);
    return fma(r * s, p, r);
}
BTE_HD double cosPoly(double r)
{
    const double s = r * r;
    double p = -1.0 / 87178291200.0;
    p = fma(p, s, 1.0 / 479001600.0);
    p = fma(p, s, -1.0 / 3628800.0);
    p = fma(p, s, 1.0 / 40320.0);
    p = fma(p, s, -1.0 / 720.0);
    p = fma(p, s, 1.0 / 24.0);
    p = fma(p, s, -0.5);
    return fma(p, s, 1.0);
}
BTE_HD double reducePio2(double x, int& q)
{
    const double k = rint(x * kTwoOverPi);
    double r = fma(-k, kPio2_1, x);
    r = fma(-k, kPio2_2, r);
    r = fma(-k, kPio2_3, r);
    q = static_cast<int>(static_cast<int64_t>(k) & 3);
    return r;
}
BTE_HD double sinD(double x)
{
    int q;
    const double r = reducePio2(x, q);
    switch (q) {
    case 0: return sinPoly(r);
    case 1: return cosPoly(r);
    case 2: return -sinPoly(r);
    default: return -cosPoly(r);
    }
}
BTE_HD double cosD(double x)
{
    int q;
    const double r = reducePio2(x, q);
    switch (q) {
    case 0: return cosPoly(r);
    case 1: return -sinPoly(r);
    case 2: return -cosPoly(r);
    default: return sinPoly(r);
    }
}
BTE_HD double expD(double x)
{
    const double k = rint(x * kInvLn2);
    double r = fma(-k, kLn2_1, x);
    r = fma(-k, kLn2_2, r);
    double p = 1.0 / 479001600.0;
    p = fma(p, r, 1.0 / 39916800.0);
    p = fma(p, r, 1.0 / 3628800.0);
    p = fma(p, r, 1.0 / 362880.0);
    p = fma(p, r, 1.0 / 40320.0);
    p = fma(p, r, 1.0 / 5040.0);
    p = fma(p, r, 1.0 / 720.0);
    p = fma(p, r, 1.0 / 120.0);
    p = fma(p, r, 1.0 / 24.0);
    p = fma(p, r, 1.0 / 6.0);
    p = fma(p, r, 0.5);
    p = fma(p, r, 1.0);
    p = fma(p, r, 1.0);
    const int64_t ki = static_cast<int64_t>(k);
    const int64_t k1 = ki / 2, k2 = ki - k1;
    const double s1 = bitsd(static_cast<uint64_t>(k1 + 1023) << 52);
    const double s2 = bitsd(static_cast<uint64_t>(k2 + 1023) << 52);
    return (p * s1) * s2;
}
BTE_HD double logD(double x)
{
    const uint64_t u = dbits(x);
    int e = static_cast<int>((u >> 52) & 0x7ff) - 1023;
    double mm = bitsd((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
    if (mm > kSqrt2) { mm = mm * 0.5; e += 1; }
    const double s = (mm - 1.0) / (mm + 1.0);
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
    const double ed = static_cast<double>(e);
    return fma(ed, kLn2_1, fma(ed, kLn2_2, lm));
}
BTE_HD double atan01D(double z)
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
BTE_HD double atan2D(double y, double x)
{
    const double ay = fabs(y), ax = fabs(x);
    double a;
    if (ay <= ax) a = atan01D(ay / ax);
    else a = kPio2_1 - atan01D(ax / ay);
    if (x < 0.0) a = kPi - a;
    return (y < 0.0) ? -a : a;
}

// ---- float entry points ----
BTE_MATHFN float sinf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::sinf(x);
#else
    if (x == 0.0f || isnanf_(x)) return x + x * 0.0f;
    if (isinff_(x)) return NAN;
    return static_cast<float>(sinD(static_cast<double>(x)));
#endif
}
BTE_MATHFN float cosf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::cosf(x);
#else
    if (isnanf_(x)) return x;
    if (isinff_(x)) return NAN;
    return static_cast<float>(cosD(static_cast<double>(x)));
#endif
}
BTE_MATHFN float tanf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::tanf(x);
#else
    if (x == 0.0f || isnanf_(x)) return x + x * 0.0f;
    if (isinff_(x)) return NAN;
    int q;
    const double r = reducePio2(static_cast<double>(x), q);
    const double s = sinPoly(r), c = cosPoly(r);
    return static_cast<float>((q & 1) ? (-c / s) : (s / c));
#endif
}
BTE_MATHFN float expf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::expf(x);
#else
    if (isnanf_(x)) return x;
    if (x > 89.0f) return INFINITY;
    if (x < -104.0f) return 0.0f;
    return static_cast<float>(expD(static_cast<double>(x)));
#endif
}
BTE_MATHFN float logf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::logf(x);
#else
    if (isnanf_(x)) return x;
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (isinff_(x)) return x;
    return static_cast<float>(logD(static_cast<double>(x)));
#endif
}
BTE_HD bool isIntF(float y) { return floorf(y) == y; }
BTE_HD bool isOddIntF(float y)
{
    if (!isIntF(y) || fabsf(y) >= 16777216.0f) return false;
    return (static_cast<int64_t>(y) & 1) != 0;
}
BTE_MATHFN float powf_(float x, float y)
{
#if BTE_FAST_DEVICE_MATH
    return ::powf(x, y);
#else
    if (y == 0.0f) return 1.0f;
    if (x == 1.0f) return 1.0f;
    if (isnanf_(x) || isnanf_(y)) return NAN;
    if (isinff_(y)) {
        const float ax = fabsf(x);
        if (ax == 1.0f) return 1.0f;
        if ((ax < 1.0f) == (y < 0.0f)) return INFINITY;
        return 0.0f;
    }
    if (x == 0.0f) {
        const bool odd = isOddIntF(y);
        if (y < 0.0f) return odd ? copysignf(INFINITY, x) : INFINITY;
        return odd ? x : 0.0f;
    }
    if (isinff_(x)) {
        const bool odd = isOddIntF(y);
        if (x < 0.0f) {
            if (y < 0.0f) return odd ? -0.0f : 0.0f;
            return odd ? -INFINITY : INFINITY;
        }
        return (y < 0.0f) ? 0.0f : INFINITY;
    }
    float sign = 1.0f;
    if (x < 0.0f) {
        if (!isIntF(y)) return NAN;
        if (isOddIntF(y)) sign = -1.0f;
    }
    const double l = static_cast<double>(y) * logD(fabs(static_cast<double>(x)));
    if (l > 89.0) return sign * INFINITY;
    if (l < -104.0) return sign * 0.0f;
    return sign * static_cast<float>(expD(l));
#endif
}
// x^5 and x^2 for the reference's powf(x, 5) / powf(x, 2) call sites: the
// double products (x*x exact, then two rounded products) carry relative error
// < 3e-16, so the single rounding to float gives the correctly rounded power
// except in vanishingly rare near-halfway cases; special values follow C99
// pow for odd/even integer exponents.
BTE_MATHFN float pow5f_(float x)
{
#if BTE_FAST_DEVICE_MATH
    const float x2 = x * x;
    return x2 * x2 * x;
#else
    const double d = static_cast<double>(x);
    const double d2 = d * d;
    const double d4 = d2 * d2;
    return static_cast<float>(d4 * d);
#endif
}
BTE_MATHFN float pow2f_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return x * x;
#else
    const double d = static_cast<double>(x);
    return static_cast<float>(d * d);
#endif
}
// sin and cos of one argument with a single reduction; bit-identical to
// sinf_(x) and cosf_(x).
BTE_MATHFN void sincosf_(float x, float& s, float& c)
{
#if BTE_FAST_DEVICE_MATH
    ::sincosf(x, &s, &c);
#else
    if (isnanf_(x)) { s = x + x * 0.0f; c = x; return; }
    if (isinff_(x)) { s = NAN; c = NAN; return; }
    if (x == 0.0f) { s = x + x * 0.0f; c = static_cast<float>(cosD(static_cast<double>(x))); return; }
    int q;
    const double r = reducePio2(static_cast<double>(x), q);
    const double sp = sinPoly(r), cp = cosPoly(r);
    switch (q) {
    case 0: s = static_cast<float>(sp); c = static_cast<float>(cp); break;
    case 1: s = static_cast<float>(cp); c = static_cast<float>(-sp); break;
    case 2: s = static_cast<float>(-sp); c = static_cast<float>(-cp); break;
    default: s = static_cast<float>(-cp); c = static_cast<float>(sp); break;
    }
#endif
}
BTE_MATHFN float atan2f_(float y, float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::atan2f(y, x);
#else
    if (isnanf_(x) || isnanf_(y)) return NAN;
    if (y == 0.0f) {
        if (x > 0.0f || (x == 0.0f && !signbitf_(x))) return y;
        return signbitf_(y) ? -static_cast<float>(kPi) : static_cast<float>(kPi);
    }
    if (isinff_(x) || isinff_(y)) {
        double a;
        if (isinff_(x) && isinff_(y)) a = (x > 0.0f) ? kPio4 : 3.0 * kPio4;
        else if (isinff_(y)) a = kPio2_1;
        else a = (x > 0.0f) ? 0.0 : kPi;
        return static_cast<float>(y < 0.0f ? -a : a);
    }
    if (x == 0.0f) return (y > 0.0f) ? static_cast<float>(kPio2_1) : -static_cast<float>(kPio2_1);
    return static_cast<float>(atan2D(static_cast<double>(y), static_cast<double>(x)));
#endif
}
BTE_MATHFN float acosf_(float x)
{
#if BTE_FAST_DEVICE_MATH
    return ::acosf(x);
#else
    if (isnanf_(x)) return x;
    if (x > 1.0f || x < -1.0f) return NAN;
    if (x == 1.0f) return 0.0f;
    const double xd = static_cast<double>(x);
    const double s = sqrt((1.0 - xd) * (1.0 + xd));
    if (xd == 0.0) return static_cast<float>(kPio2_1);
    return static_cast<float>(atan2D(s, xd));
#endif
}

}  // namespace m
}  // namespace bte
