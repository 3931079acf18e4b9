// fastmath.cuh -- branch-free FP64 exponential, tanh on [0, 1] and square
// root for the per-pair arithmetic of the symmetry-function kernels.
//
// The library routines handle every argument range and special value, and
// their range tests are branches: inside a warp whose lanes hold different
// pairs the lanes can take different sides, and a branch also keeps the
// compiler from interleaving two independent sequences.  The arguments here
// are bounded by the cutoff geometry (exp of a non-positive number, tanh of
// u = 1 - r/rc in [0, 1], sqrt of a squared distance), so each function is
// one straight-line sequence:
//
//  * exp_clamped(x), x clamped to [-708, 709]: Cody-Waite argument
//    reduction x = k ln2 + r, |r| <= ln2/2 (W. J. Cody and W. Waite, "Software Manual for the
//    Elementary Functions", 1980), with the reduction done by fused
//    multiply-adds against ln2 split into its double rounding and the
//    remainder; e^r - 1 by its Taylor series to degree 13 evaluated with
//    Estrin's scheme (depth 4 instead of a 13-deep Horner chain), 1 added
//    last; 2^k applied through the exponent field (e^-708 ~ 3e-308, the
//    smallest result without a subnormal scale).  Error within 1 ulp of
//    libm (tests/test_fastmath.py emulates these operations on the host
//    with exact fused multiply-adds, and checks the device functions, run
//    through hdnnp_debug_math, against libm's exp, tanh and sqrt).
//  * tanh01(u) = (1 - e^(-2u)) / (1 + e^(-2u)) with the quotient from the
//    hardware reciprocal approximation refined by one third-order Newton
//    step and one residual correction (Newton-Raphson division, as in
//    P. Markstein, "IA-64 and Elementary Functions", 2000).  Absolute error
//    a few 1e-16; its relative error grows as u -> 0, where the cutoff
//    function tanh^3 and its derivative vanish.
//  * sqrt_rsqrt(x) and rsqrt_pos(x): the hardware reciprocal square-root
//    approximation refined by one third-order Newton step; the root as
//    x * rsqrt with one residual correction.  x = 0 gives 0 (the reciprocal
//    is taken of max(x, 1e-300)).
// The constants are ln 2 and 1/ln 2 rounded to double, the remainder
// ln 2 - double(ln 2), 1.5 * 2^52 (the round-to-integer shifter) and 1/n!.
#pragma once

namespace hdnnp {

__device__ __forceinline__ double rcp_approx(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    return y;
}

__device__ __forceinline__ double rsqrt_approx(double x) {
    double y;
    asm("rsqrt.approx.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

// e^x for x in [-708, 709] (arguments outside are clamped to the range)
__device__ __forceinline__ double exp_clamped(double x) {
    constexpr double kLog2e = 1.4426950408889634;
    constexpr double kLn2Hi = 0.6931471805599453;
    constexpr double kLn2Lo = 2.3190468138462996e-17;
    constexpr double kShift = 6755399441055744.0;  // 1.5 * 2^52
    x = fmin(fmax(x, -708.0), 709.0);
    const double t = fma(x, kLog2e, kShift);
    const int k = __double2loint(t);
    const double kd = t - kShift;
    double r = fma(kd, -kLn2Hi, x);
    r = fma(kd, -kLn2Lo, r);
    // e^r - 1 = sum_{n=1..13} r^n / n!, Estrin's scheme
    const double r2 = r * r, r4 = r2 * r2, r8 = r4 * r4;
    const double q0 = r;                                                  // r
    const double q1 = fma(0.16666666666666666, r, 0.5);                   // 1/2! + r/3!
    const double q2 = fma(0.008333333333333333, r, 0.041666666666666664);  // 1/4! + r/5!
    const double q3 = fma(0.0001984126984126984, r, 0.001388888888888889);
    const double q4 = fma(2.7557319223985893e-06, r, 2.48015873015873e-05);
    const double q5 = fma(2.505210838544172e-08, r, 2.755731922398589e-07);
    const double q6 = fma(1.6059043836821613e-10, r, 2.08767569878681e-09);
    const double s0 = fma(q1, r2, q0);
    const double s1 = fma(q3, r2, q2);
    const double s2 = fma(q5, r2, q4);
    const double t0 = fma(s1, r4, s0);
    const double t1 = fma(q6, r4, s2);
    const double p = 1.0 + fma(t1, r8, t0);
    return p * __hiloint2double((k + 1023) << 20, 0);
}

// 1 / d for d in [1, 2]
__device__ __forceinline__ double rcp_12(double d) {
    double y = rcp_approx(d);
    const double e = fma(-d, y, 1.0);
    return fma(y, fma(e, e, e), y);  // y (1 + e + e^2)
}

// tanh(u) for u in [0, 1]
__device__ __forceinline__ double tanh01(double u) {
    const double t = exp_clamped(-2.0 * u);
    const double n = 1.0 - t, d = 1.0 + t;
    const double y = rcp_12(d);
    const double q = n * y;
    return fma(y, fma(-d, q, n), q);
}

// 1 / sqrt(x) for x > 0 (x = 0 gives 1e150)
__device__ __forceinline__ double rsqrt_pos(double x) {
    const double xc = fmax(x, 1e-300);
    const double y = rsqrt_approx(xc);
    const double e = fma(-xc * y, y, 1.0);                     // 1 - x y^2
    return fma(y * e, fma(0.375, e, 0.5), y);                  // y (1 + e/2 + 3e^2/8)
}

// sqrt(x) and 1/sqrt(x) for x >= 0 (x = 0: r = 0, ir = 1e150)
__device__ __forceinline__ void sqrt_rsqrt(double x, double& r, double& ir) {
    ir = rsqrt_pos(x);
    const double s = x * ir;
    r = fma(0.5 * ir, fma(-s, s, x), s);
}

}  // namespace hdnnp
