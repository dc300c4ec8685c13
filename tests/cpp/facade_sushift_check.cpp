// The facade's SUShift<N>::sample and SULink<N> (include/umc/dof.hpp) on the
// host, drawing from the keyed stream (seed, counter, tag, id) of
// include/umc/keyed_pcg.cuh.  Reads lines "N width seed counter tag id" and
// then N*N (re, im) pairs of the current link from stdin; writes the N*N
// (re, im) pairs of the proposed link, one line each, and after the last one
// the largest unitarity error seen.
#include <umc/umc.hpp>
#include <umc/keyed_pcg.cuh>

#include <cstdint>
#include <cstdio>

namespace {

struct KeyedUni
{
    umc::KeyedPcg g;
    double uni() { return umc::u_f64(g.next()); }
};

template <std::size_t N>
double run(double width, std::uint64_t seed, std::uint64_t counter, std::uint32_t tag, std::uint32_t id)
{
    umc::gpu::SULink<N> cur, out;
    for (std::size_t q = 0; q < N * N; ++q) {
        double re = 0, im = 0;
        if (std::scanf("%lf %lf", &re, &im) != 2) return -1.0;
        cur.m[q] = umc::gpu::Complex(re, im);
    }
    KeyedUni r{umc::KeyedPcg::open_key(seed, counter, tag, id)};
    umc::gpu::SUShift<N>{width}.sample(&cur, r, &out);
    for (std::size_t q = 0; q < N * N; ++q) std::printf("%.17g %.17g\n", out.m[q].real(), out.m[q].imag());
    return out.unitarity_error();
}

}  // namespace

int main()
{
    unsigned n = 0;
    double width = 0;
    unsigned long long seed = 0, counter = 0;
    unsigned tag = 0, id = 0;
    double worst = 0.0;
    while (std::scanf("%u %lf %llu %llu %u %u", &n, &width, &seed, &counter, &tag, &id) == 6) {
        const double e = n == 2 ? run<2>(width, seed, counter, tag, id) : run<3>(width, seed, counter, tag, id);
        if (e < 0) return 1;
        worst = e > worst ? e : worst;
    }
    std::printf("unitarity %.3e\n", worst);
    return 0;
}
