// pmath64.cuh -- log and exp in FP64 built from IEEE + - * / only, for the plain path.
//
// The plain FP64 path must reproduce the oracle to the last bit, and the CPU and GPU math
// libraries' log/exp differ by up to an ulp; near the logarithmic-mean switch of the reference
// (|a-b| just above 1e-4) such an ulp is amplified over hundreds of stages.  Both sides therefore
// evaluate these two functions with the same construction (the oracle has its own copy):
//   log: x = 2^e m, m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1), |s| <= 0.1716,
//        atanh(s)/s = sum_k s^(2k)/(2k+1) to k = 10 (truncation < 2^-53); e ln2 with ln2 split
//        into a 32-bit head and a tail (Cody-Waite) so that e*LN2_HI is exact.
//   exp: y = k ln2 + r, k = rint(y / ln2), |r| <= ln2/2, e^r by its Taylor polynomial to
//        r^13/13! (truncation < 2^-56), 2^k applied through the exponent bits.
// Accuracy: within 3 ulp (log) and 2 ulp (exp), the order of the libraries they replace.
#pragma once

namespace nemo {

constexpr double PM_LN2_HI = 0x1.62e42feep-1;            // ln 2 with a 32-bit mantissa
constexpr double PM_LN2_LO = 0x1.a39ef35793c76p-33;      // ln 2 - PM_LN2_HI
constexpr double PM_INV_LN2 = 0x1.71547652b82fep+0;      // 1 / ln 2
constexpr double PM_SQRT2 = 1.4142135623730951;

__device__ __forceinline__ double plog64(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -__longlong_as_double(0x7ff0000000000000LL) : __longlong_as_double(0x7ff8000000000000LL);
    if (x == __longlong_as_double(0x7ff0000000000000LL)) return x;
    int shift = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; shift = 54; }  // 2^54
    const long long b = __double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7ff) - 1023 - shift;
    double m = __longlong_as_double((b & 0x000fffffffffffffLL) | 0x3ff0000000000000LL);
    if (m > PM_SQRT2) { m = 0.5 * m; e = e + 1; }
    const double s = (m - 1.0) / (m + 1.0);
    const double z = s * s;
    double p = 1.0 / 21.0;
    p = p * z + 1.0 / 19.0;
    p = p * z + 1.0 / 17.0;
    p = p * z + 1.0 / 15.0;
    p = p * z + 1.0 / 13.0;
    p = p * z + 1.0 / 11.0;
    p = p * z + 1.0 / 9.0;
    p = p * z + 1.0 / 7.0;
    p = p * z + 1.0 / 5.0;
    p = p * z + 1.0 / 3.0;
    p = p * z + 1.0;
    const double lm = (2.0 * s) * p;
    const double de = (double)e;
    return de * PM_LN2_HI + (lm + de * PM_LN2_LO);
}

__device__ __forceinline__ double pexp64(double y) {
    if (y != y) return y;
    if (y > 709.78) return __longlong_as_double(0x7ff0000000000000LL);
    if (y < -745.2) return 0.0;
    const double kd = rint(y * PM_INV_LN2);
    const double r = (y - kd * PM_LN2_HI) - kd * PM_LN2_LO;
    double p = 1.0 / 6227020800.0;
    p = p * r + 1.0 / 479001600.0;
    p = p * r + 1.0 / 39916800.0;
    p = p * r + 1.0 / 3628800.0;
    p = p * r + 1.0 / 362880.0;
    p = p * r + 1.0 / 40320.0;
    p = p * r + 1.0 / 5040.0;
    p = p * r + 1.0 / 720.0;
    p = p * r + 1.0 / 120.0;
    p = p * r + 1.0 / 24.0;
    p = p * r + 1.0 / 6.0;
    p = p * r + 0.5;
    p = p * r + 1.0;
    p = p * r + 1.0;
    int k = (int)kd;
    if (k > 1023) { p = p * 0x1p1023; k -= 1023; }
    if (k < -1022) { p = p * 0x1p-1022; k += 1022; if (k < -1022) return 0.0; }
    return p * __longlong_as_double((long long)(k + 1023) << 52);
}

}  // namespace nemo
