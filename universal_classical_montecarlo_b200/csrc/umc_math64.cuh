// umc_math64.cuh -- FP64 sine and cosine for the accept decisions that the
// FP32 tests leave to FP64: branch-free, so that one thread evaluates all the
// angles of a site update in lockstep.  (With the library cos, the FP64
// settling of one XY update -- eight cosines and a logarithm -- took about
// 5,000 cycles of a thread.)
#pragma once

#include <cmath>

namespace umc {

// 1/n! in FP64 (n! is exact in FP64 up to 18!; 19! rounds once).
__host__ __device__ constexpr double inv_factorial(int n)
{
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= double(i);
    return 1.0 / f;
}

// sin x and cos x in FP64 for |x| <= 2^19, without branches, so that a
// thread can evaluate several in lockstep.  Cody-Waite reduction: k =
// rint(x 2/pi), r = x - k pi/2 with pi/2 = C1 + C2 + C3, C1 and C2 pi/2 and
// the rest rounded to 33 bits (k C1 and k C2 exact for |k| < 2^20; each step
// a fused multiply-add), C3 the next 53 bits: |r| <= pi/4 (1 + 2^-50), error a
// few units of 2^-53 |r|.  Then the Taylor series of sin r through r^17/17!
// and of cos r through r^16/16! (truncation below 2^-58 at |r| = pi/4), and
// the quadrant k mod 4.  Accuracy a few ulp.  The split constants are pi/2 in
// binary, derived from pi's decimal digits with exact rational arithmetic.
__host__ __device__ __forceinline__ void sincos_cw64(double x, double& s, double& c)
{
    constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;
    constexpr double kC1 = 0x1.921fb544p+0, kC2 = 0x1.0b4611a6p-34, kC3 = 0x1.3198a2e037073p-69;
    const double k = rint(x * kTwoOverPi);
    const double r = fma(-k, kC3, fma(-k, kC2, fma(-k, kC1, x)));
    const double z = r * r;
    // sin r = r + r z P(z), P = sum_{m=1..8} (-1)^m z^(m-1) / (2m+1)!
    // cos r = 1 + z Q(z),   Q = sum_{m=1..8} (-1)^m z^(m-1) / (2m)!
    double ps = inv_factorial(17), pc = inv_factorial(16);
#pragma unroll
    for (int m = 7; m >= 1; --m) {
        ps = fma(ps, z, (m & 1) ? -inv_factorial(2 * m + 1) : inv_factorial(2 * m + 1));
        pc = fma(pc, z, (m & 1) ? -inv_factorial(2 * m) : inv_factorial(2 * m));
    }
    const double sr = fma(r * z, ps, r);
    const double cr = fma(z, pc, 1.0);
    const int q = int(k) & 3;  // x = k pi/2 + r
    const double s0 = (q & 1) ? cr : sr, c0 = (q & 1) ? sr : cr;
    s = (q & 2) ? -s0 : s0;
    c = ((q + 1) & 2) ? -c0 : c0;
}

// Largest absolute error of __sincosf (sine and cosine) over every FP32
// argument with |x| <= kSincosfDomain: 0x1.43b5dcp-20 (2^-19.66), measured
// exhaustively on sm_100a against the FP64 library and rounded up here
// (tests/cpp/sincosf_bound.cu re-measures it on the GPU at hand; over
// |x| <= 4 it is 2^-20.55).  The FP32 XY decisions are bounded with it, so
// the engine keeps every angle inside the domain: draws lie in [0, 2 pi),
// proposals are wrapped into [-pi, pi], and uploaded angles outside it are
// reduced with wrap_angle.
constexpr float kSincosfDomain = 8.0f;
constexpr double kSincosfAbsErr = 0x1.44p-20;

// x itself when |x| <= kSincosfDomain, else the same angle in [-pi, pi]
// (reduced in FP64 and rounded once).  NaN stays NaN.
__host__ __device__ inline float wrap_angle(float x)
{
    return fabsf(x) > kSincosfDomain ? float(remainder(double(x), 0x1.921fb54442d18p+2)) : x;
}

}  // namespace umc
