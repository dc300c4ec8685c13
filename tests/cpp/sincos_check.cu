// Host check of sincos_cw64 (csrc/umc_math64.cuh): sin and cos against the
// x87 long-double library (64-bit significand) on FP32 angles in [-8, 8]
// (every value the FP64 settling of an XY or U(1) update can see), on
// multiples of pi/4 near the reduction's quadrant edges, and on FP64 values
// up to 2^19.  Prints the largest errors in units of 2^-53 and "ok" when
// all stay within 4.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "umc_math64.cuh"

static long double g_worst = 0.0L;

static void check(double x)
{
    double s, c;
    umc::sincos_cw64(x, s, c);
    const long double xs = sinl((long double)x), xc = cosl((long double)x);
    const long double es = fabsl((long double)s - xs), ec = fabsl((long double)c - xc);
    // error in units of 2^-53 relative to max(|value|, 2^-10): absolute near zeros
    const long double us = es / (ldexpl(1.0L, -53) * fmaxl(fabsl(xs), ldexpl(1.0L, -10)));
    const long double uc = ec / (ldexpl(1.0L, -53) * fmaxl(fabsl(xc), ldexpl(1.0L, -10)));
    if (us > g_worst) g_worst = us;
    if (uc > g_worst) g_worst = uc;
}

int main()
{
    uint64_t state = 0x9E3779B97F4A7C15ull;
    auto next = [&] {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        return state;
    };
    // FP32 angles in [-8, 8]
    for (int i = 0; i < 4000000; ++i) {
        const float f = float((double(next() >> 11) * 0x1.0p-53) * 16.0 - 8.0);
        check(double(f));
    }
    // near k pi/4 (quadrant and reduction edges)
    for (int k = -40; k <= 40; ++k)
        for (int d = -64; d <= 64; ++d) {
            // the FP32 value |d| steps from k pi/4 towards the sign of d
            float g = float(k * 0.78539816339744830962);
            for (int j = 0; j < (d < 0 ? -d : d); ++j) g = nextafterf(g, d < 0 ? -1e9f : 1e9f);
            check(double(g));
        }
    // FP64 values up to 2^19
    for (int i = 0; i < 1000000; ++i) {
        const double x = (double(next() >> 11) * 0x1.0p-53 * 2.0 - 1.0) * 524288.0;
        check(x);
    }
    printf("worst %.3Lf\n", g_worst);
    if (g_worst <= 4.0L) printf("ok\n");
    return 0;
}
