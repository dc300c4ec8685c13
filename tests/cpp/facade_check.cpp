// facade_check.cpp -- the C++23 facade (include/umc/umc.hpp) used the way the
// reference's own test programs use the reference library: concepts, table
// invariants, host-side energy finite differences, and GPU chains against
// exact answers (4x4 Ising by enumeration, the 2D U(1) torus plaquette by its
// character expansion).  Prints "ok" and exits 0 on success.
#include <umc/umc.hpp>

#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <tuple>
#include <vector>

#define CHECK(cond)                                                                  \
    do {                                                                             \
        if (!(cond)) {                                                               \
            std::fprintf(stderr, "check failed: %s (line %d)\n", #cond, __LINE__); \
            std::exit(1);                                                            \
        }                                                                            \
    } while (0)

static_assert(ModelLike<Ising>);
static_assert(WolffModel<Ising>);
static_assert(EnergyModel<Ising>);
static_assert(ModelLike<VectorSpin<3>>);
static_assert(WolffModel<VectorSpin<3>>);
static_assert(ModelLike<U1Gauge>);
static_assert(!WolffModel<U1Gauge>);
static_assert(ModelLike<SUGauge<3>>);
static_assert(Proposal<Flip, IsingSpin, Pcg32>);
static_assert(Proposal<U1Shift, U1Link, Pcg32>);
static_assert(Proposal<UniformSphereN<3>, double, Pcg32>);
static_assert(PairGraphLike<PairGraph<>>);
static_assert(CellComplexLike<CellComplex<4>>);

template <class M>
double total_energy(const M& m)
{
    double s = 0.0;
    for (std::size_t i = 0; i < m.sites(); ++i) s += m.energy_at(i);
    return 0.5 * s;
}

// Exact mean energy per site of the L x L periodic Ising model (J = 1) at beta.
double ising_exact(std::size_t L, double beta)
{
    const std::size_t n = L * L;
    double z = 0.0, e = 0.0;
    for (std::uint32_t c = 0; c < (1u << n); ++c) {
        int E = 0;
        for (std::size_t y = 0; y < L; ++y)
            for (std::size_t x = 0; x < L; ++x) {
                const int s = (c >> (y * L + x)) & 1u ? 1 : -1;
                const int r = (c >> (y * L + (x + 1) % L)) & 1u ? 1 : -1;
                const int u = (c >> (((y + 1) % L) * L + x)) & 1u ? 1 : -1;
                E -= s * (r + u);
            }
        const double w = std::exp(-beta * E);
        z += w;
        e += w * E;
    }
    return e / z / double(n);
}

// <cos theta_p> of 2D U(1) on a torus of n_plaq plaquettes:
// Z = sum_n I_n(beta)^n_plaq.
double torus_plaquette(double beta, int n_plaq)
{
    double num = 0.0, den = 0.0;
    const double i0 = std::cyl_bessel_i(0.0, beta);
    for (int k = -30; k <= 30; ++k) {
        const double a = std::cyl_bessel_i(double(std::abs(k)), beta) / i0;
        const double d = 0.5 * (std::cyl_bessel_i(double(std::abs(k - 1)), beta) +
                                std::cyl_bessel_i(double(std::abs(k + 1)), beta)) / i0;
        num += std::pow(a, n_plaq - 1) * d;
        den += std::pow(a, n_plaq);
    }
    return num / den;
}

int main()
{
    // ---- tables
    const auto graph = square_lattice(4, 4);
    CHECK(graph.sites() == 16);
    for (std::size_t i = 0; i < 16; ++i) CHECK(graph.degree(i) == 4);
    for (const auto& [Lx, Ly, deg] : {std::tuple{1u, 1u, 0u}, std::tuple{1u, 4u, 2u}, std::tuple{2u, 2u, 4u}}) {
        const auto g = square_lattice(Lx, Ly);
        for (std::size_t i = 0; i < g.sites(); ++i) CHECK(g.degree(i) == deg);
    }
    {
        bool threw = false;
        try {
            const std::array<PairGraph<>::Edge, 1> bad{PairGraph<>::Edge{1, 1}};
            PairGraph<> g(2, bad);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        CHECK(threw);
        threw = false;
        try {
            const std::array<PairGraph<>::Edge, 1> bad{PairGraph<>::Edge{0, 5}};
            PairGraph<> g(2, bad);
        } catch (const std::out_of_range&) {
            threw = true;
        }
        CHECK(threw);
    }
    {
        const auto cc = hypercubic_plaquettes(2);
        CHECK(cc.sites() == 4 * 16 && cc.cells() == 6 * 16);
        for (std::size_t i = 0; i < cc.sites(); ++i) CHECK(cc.incident(i).size() == 6);
    }

    // ---- host-side model functions (finite differences)
    {
        Ising model(graph);
        CHECK(std::abs(total_energy(model) / 16.0 + 2.0) < 1e-12);
        Pcg32 rng(7, 3);
        for (std::size_t i = 0; i < 16; ++i) {
            const IsingSpin s = rng.uni() < 0.5 ? IsingSpin(-1) : IsingSpin(1);
            model.update(i, &s);
        }
        const IsingSpin p = IsingSpin(-model.data()[5]);
        const double dE = model.energy_diff_at(5, &p), before = total_energy(model);
        model.update(5, &p);
        CHECK(std::abs(dE - (total_energy(model) - before)) < 1e-12);
    }
    {
        VectorSpin<3> model(graph);
        Pcg32 rng(8, 5);
        double v[3];
        for (std::size_t i = 0; i < 16; ++i) {
            UniformSphereN<3>{}.sample(nullptr, rng, v);
            model.update(i, v);
        }
        UniformSphereN<3>{}.sample(nullptr, rng, v);
        const double dE = model.energy_diff_at(2, v), before = total_energy(model);
        model.update(2, v);
        CHECK(std::abs(dE - (total_energy(model) - before)) < 1e-12);
    }

    // ---- Ising 4x4 at beta = 0.3 against exact enumeration
    const double exact = ising_exact(4, 0.3);
    {
        Ising model(graph);
        Metropolis metro(model, Flip{}, Pcg32(11, 1), 0.3);
        metro.run(2000);
        double sum = 0.0;
        metro.sample(2000, [&](const Ising& m) { sum += total_energy(m); });
        CHECK(std::abs(sum / (2000.0 * 16.0) - exact) < 0.03);
        metro.run(100000);  // the device records of one long run
        double r = 0.0;
        for (std::size_t k = 0; k < 100000; ++k) r += metro.records()[k * UMC_OBS_STRIDE];
        std::printf("Ising Metropolis %.5f exact %.5f\n", r / (100000.0 * 16.0), exact);
        CHECK(std::abs(r / (100000.0 * 16.0) - exact) < 0.01);
    }
    {
        Ising model(graph);
        Wolff wolff(model, FixedAxis{}, Pcg32(12, 1), 0.3);
        wolff.run(200);
        double sum = 0.0;
        wolff.sample(20000, [&](const Ising& m) { sum += total_energy(m); });
        std::printf("Ising Wolff %.5f (cluster %.2f)\n", sum / (20000.0 * 16.0), wolff.mean_cluster_size());
        CHECK(std::abs(sum / (20000.0 * 16.0) - exact) < 0.05);
        CHECK(wolff.mean_cluster_size() > 1.0);
    }

    // ---- Heisenberg 4x4 at beta = 0.3: Metropolis and Wolff agree
    double heis = 0.0;
    {
        VectorSpin<3> model(graph);
        Metropolis metro(model, UniformSphereN<3>{}, Pcg32(13, 1), 0.3);
        metro.run(2000);
        metro.run(100000);
        for (std::size_t k = 0; k < 100000; ++k) heis += metro.records()[k * UMC_OBS_STRIDE];
        heis /= 100000.0 * 16.0;
    }
    {
        VectorSpin<3> model(graph);
        Wolff wolff(model, UniformSphereN<3>{}, Pcg32(14, 1), 0.3);
        wolff.run(200);
        double sum = 0.0;
        wolff.sample(20000, [&](const VectorSpin<3>& m) { sum += total_energy(m); });
        std::printf("Heisenberg Metropolis %.5f Wolff %.5f\n", heis, sum / (20000.0 * 16.0));
        CHECK(std::abs(sum / (20000.0 * 16.0) - heis) < 0.05);
    }

    // ---- 2D U(1) on an 8 x 8 torus against the exact plaquette
    {
        const double beta = 2.0;
        U1Gauge g(square_plaquettes(8), beta);
        Metropolis metro(g, U1Shift{0.7}, Pcg32(15, 2), 1.0);
        metro.run(2000);
        const std::size_t n = 200000;
        metro.run(n);
        double s = 0.0, s2 = 0.0;
        const std::size_t bins = 100, per = n / bins;
        for (std::size_t b = 0; b < bins; ++b) {
            double m = 0.0;
            for (std::size_t k = b * per; k < (b + 1) * per; ++k) m += metro.records()[k * UMC_OBS_STRIDE + 1];
            m /= double(per);
            s += m;
            s2 += m * m;
        }
        const double mean = s / bins, err = std::sqrt((s2 / bins - mean * mean) / (bins - 1));
        const double ex = torus_plaquette(beta, 64);
        std::printf("U(1) 8x8 plaquette %.5f +- %.5f exact %.5f\n", mean, err, ex);
        CHECK(std::abs(mean - ex) < 4.0 * err + 1e-4);
        CHECK(std::abs(g.mean_plaquette() - metro.records()[(n - 1) * UMC_OBS_STRIDE + 1]) < 1e-5);
    }

    // ---- 4D U(1) reference model: host dE and the device chain agree on the state
    {
        U1Gauge g(3, 1.3);
        Pcg32 rng(3, 4);
        U1Shift shift{2.0};
        for (std::size_t i = 0; i < g.sites(); ++i) {
            U1Link p;
            shift.sample(g.data() + i, rng, &p);
            g.update(i, &p);
        }
        U1Link p;
        shift.sample(g.data() + 7, rng, &p);
        const double dE = g.energy_diff_at(7, &p), before = g.total_energy();
        g.update(7, &p);
        CHECK(std::abs(dE - (g.total_energy() - before)) < 1e-9);
        Metropolis metro(g, U1Shift{0.7}, Pcg32(5, 2), 1.3);
        metro.run(50);
        CHECK(std::abs(g.mean_plaquette() - metro.records()[49 * UMC_OBS_STRIDE + 1]) < 1e-5);
    }

    // ---- SU(3), cold start, multi-hit SUShift
    {
        SUGauge<3> g(2, 5.7);
        CHECK(std::abs(g.mean_plaquette() - 1.0) < 1e-12);
        Metropolis metro(g, Hits<SUShift<3>>{SUShift<3>{0.2}, 10}, Pcg32(21, 1), 1.0);
        metro.run(20);
        const double P = g.mean_plaquette();
        std::printf("SU(3) 2^4 plaquette after 20 sweeps %.5f\n", P);
        CHECK(P > 0.3 && P < 1.0);
        CHECK(std::abs(P - metro.records()[19 * UMC_OBS_STRIDE + 1]) < 1e-5);
    }

    std::puts("ok");
    return 0;
}
