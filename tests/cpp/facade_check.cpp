// facade_check.cpp -- the C++23 facade (include/umc/umc.hpp) used the way the
// reference's own test programs use the reference library: concepts, table
// invariants, host-side energy finite differences, and GPU chains against
// exact answers (4x4 Ising by enumeration, the 2D U(1) torus plaquette by its
// character expansion).  Prints "ok" and exits 0 on success.
#include <umc/umc.hpp>

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdio>
#include <string>
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
static_assert(PairGraphLike<PairGraph<double>>);
static_assert(sizeof(Bond<NoPayload>) == 4);
static_assert(CellComplexLike<CellComplex<4>>);
// the reference's table-driven models with its built-in terms (model/pair.hpp,
// model/cell.hpp, term/*.hpp)
using PairIsing = PairModel<IsingDof, IsingTerm, PairGraph<>>;
using PairHeis = PairModel<VectorDof<3>, HeisenbergTerm<3>, PairGraph<>>;
using CellU1 = CellModel<U1Dof, U1PlaquetteTerm, CellComplex<4>>;
using CellSU3 = CellModel<SUDof<3>, SUPlaquetteTerm<3>, CellComplex<4>>;
static_assert(CellTerm<IsingTerm, IsingDof> && CellTerm<U1PlaquetteTerm, U1Dof>);
static_assert(ModelLike<PairIsing> && WolffModel<PairIsing> && EnergyModel<PairIsing>);
static_assert(ModelLike<PairHeis> && WolffModel<PairHeis>);
static_assert(ModelLike<CellU1> && !WolffModel<CellU1>);
static_assert(ModelLike<CellSU3>);

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

// PairGraph<double>: the reference graph test's weighted 16 x 16 lattice
// (test/graph_check.cpp:86-127) with random couplings; each row carries its
// edges' couplings, so the row energy equals the edge sum.
void check_weighted_graph()
{
    constexpr std::uint32_t L = 16, N = L * L;
    std::vector<PairGraph<double>::Edge> edges;
    Pcg32 rng(77, 3);
    for (std::uint32_t y = 0; y < L; ++y)
        for (std::uint32_t x = 0; x < L; ++x) {
            edges.push_back({y * L + x, y * L + (x + 1) % L, 2.0 * rng.uni() - 1.0});
            edges.push_back({y * L + x, ((y + 1) % L) * L + x, 2.0 * rng.uni() - 1.0});
        }
    const PairGraph<double> g(N, edges);
    CHECK(g.sites() == N);
    std::vector<double> s(N);
    for (auto& v : s) v = rng.uni() < 0.5 ? -1.0 : 1.0;
    double row = 0.0, edge = 0.0;
    for (std::size_t i = 0; i < N; ++i) {
        CHECK(g.degree(i) == 4);
        for (std::size_t a = 0; a < g.degree(i); ++a) row += -g.bonds(i)[a].c * s[i] * s[g.bonds(i)[a].j];
    }
    for (const auto& e : edges) edge += -e.c * s[e.i] * s[e.j];
    CHECK(std::abs(0.5 * row - edge) < 1e-9);
    // the first edge's coupling sits in row 0 (slot 0) and in row 1
    CHECK(g.bonds(0)[0].j == 1 && g.bonds(0)[0].c == edges[0].c);
    bool found = false;
    for (std::size_t a = 0; a < g.degree(1); ++a) found |= g.bonds(1)[a].j == 0 && g.bonds(1)[a].c == edges[0].c;
    CHECK(found);
    // a copy shares the table; a directed graph keeps one entry per edge
    const PairGraph<double> copy = g;
    CHECK(copy.bonds(5)[2].c == g.bonds(5)[2].c);
    const std::array<PairGraph<double>::Edge, 1> one{PairGraph<double>::Edge{0, 1, 0.25}};
    const PairGraph<double> directed(2, one, false);
    CHECK(directed.degree(0) == 1 && directed.degree(1) == 0 && directed.bonds(0)[0].c == 0.25);
}

// su_project on links rounded to FP32, as the device stores them: the result
// is unitary with det 1 to FP64 rounding and within FP32 rounding of the link.
template <std::size_t N>
void check_su_project()
{
    Pcg32 rng(5 + N, 1);
    SULink<N> u = SULink<N>::identity();
    for (int k = 0; k < 200; ++k) {
        SUShift<N>{0.8}.sample(&u, rng, &u);
        SULink<N> v = u;
        for (auto& z : v.m) z = std::complex<double>(double(float(z.real())), double(float(z.imag())));
        CHECK(v.unitarity_error() > 1e-12);
        umc::gpu::su_project(v);
        CHECK(v.unitarity_error() < 1e-14);
        double d = 0.0;
        for (std::size_t q = 0; q < N * N; ++q) d = std::max(d, std::abs(v.m[q] - u.m[q]));
        CHECK(d < 1e-6);
        // det 1: the product of the pivots of v equals that of u (1) to rounding
        std::array<std::complex<double>, N * N> a = v.m;
        std::complex<double> det(1.0);
        for (std::size_t c = 0; c < N; ++c) {
            std::size_t p = c;
            for (std::size_t r = c + 1; r < N; ++r)
                if (std::abs(a[r * N + c]) > std::abs(a[p * N + c])) p = r;
            if (p != c) {
                for (std::size_t q = 0; q < N; ++q) std::swap(a[c * N + q], a[p * N + q]);
                det = -det;
            }
            det *= a[c * N + c];
            for (std::size_t r = c + 1; r < N; ++r) {
                const std::complex<double> f = a[r * N + c] / a[c * N + c];
                for (std::size_t q = c; q < N; ++q) a[r * N + q] -= f * a[c * N + q];
            }
        }
        CHECK(std::abs(det - std::complex<double>(1.0)) < 1e-14);
    }
    // sun_detail::norm (the reference's name): the largest absolute row sum
    umc::gpu::sun_detail::Mat<N> m{};
    for (std::size_t q = 0; q < N * N; ++q) m[q] = std::complex<double>(double(q % N) - 1.0, q == 0 ? 3.0 : 0.0);
    double want = 0.0;
    for (std::size_t r = 0; r < N; ++r) {
        double row = 0.0;
        for (std::size_t c = 0; c < N; ++c) row += std::abs(m[r * N + c]);
        want = std::max(want, row);
    }
    CHECK(umc::gpu::sun_detail::norm<N>(m) == want);
}

int main(int argc, char** argv)
{
    // ---- host-side tables and link algebra (no GPU needed)
    check_weighted_graph();
    check_su_project<2>();
    check_su_project<3>();
    if (argc > 1 && std::string(argv[1]) == "tables") {
        std::puts("facade_check tables: ok");
        return 0;
    }

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

    // ---- PairModel / CellModel: host dE by finite differences, and on the
    // device the same chains as the example models they map to
    {
        PairIsing pm(square_lattice(16, 16), IsingTerm{1});
        Ising em(square_lattice(16, 16), 1);
        Pcg32 rng(31, 2);
        for (std::size_t i = 0; i < pm.sites(); ++i) {
            const IsingSpin s = rng.uni() < 0.5 ? IsingSpin(-1) : IsingSpin(1);
            pm.update(i, &s);
            em.update(i, &s);
        }
        const IsingSpin p = IsingSpin(-pm.data()[9]);
        std::int32_t before = 0;
        for (std::size_t i = 0; i < pm.sites(); ++i) before += pm.energy_at(i);
        const std::int32_t dE = pm.energy_diff_at(9, &p);
        CHECK(double(dE) == em.energy_diff_at(9, &p));
        PairIsing q = pm;
        q.update(9, &p);
        std::int32_t after = 0;
        for (std::size_t i = 0; i < q.sites(); ++i) after += q.energy_at(i);
        CHECK(2 * dE == after - before);  // energy_at counts every bond from both ends
        Metropolis a(pm, Flip{}, Pcg32(41, 0), 0.44);
        Metropolis b(em, Flip{}, Pcg32(41, 0), 0.44);
        a.run(30);
        b.run(30);
        for (std::size_t i = 0; i < pm.sites(); ++i) CHECK(pm.data()[i] == em.data()[i]);
        Wolff wa(pm, FixedAxis{}, Pcg32(42, 0), 0.44);
        Wolff wb(em, FixedAxis{}, Pcg32(42, 0), 0.44);
        std::array<std::uint64_t, 20> sa{}, sb{};
        wa.flips(20, sa.data());
        wb.flips(20, sb.data());
        CHECK(sa == sb);
        for (std::size_t i = 0; i < pm.sites(); ++i) CHECK(pm.data()[i] == em.data()[i]);
    }
    {
        CellU1 cm(square_plaquettes(8), U1PlaquetteTerm{2.0});
        U1Gauge eg(square_plaquettes(8), 2.0);
        Pcg32 rng(33, 1);
        U1Shift shift{2.0};
        for (std::size_t i = 0; i < cm.sites(); ++i) {
            U1Link l;
            shift.sample(cm.data() + i, rng, &l);
            cm.update(i, &l);
            eg.update(i, &l);
        }
        U1Link l;
        shift.sample(cm.data() + 5, rng, &l);
        const double dE = cm.energy_diff_at(5, &l), before = cm.total_energy();
        CHECK(std::abs(dE - eg.energy_diff_at(5, &l)) < 1e-12);
        CellU1 q = cm;
        q.update(5, &l);
        CHECK(std::abs(dE - (q.total_energy() - before)) < 1e-9);
        Metropolis a(cm, U1Shift{0.7}, Pcg32(43, 0), 1.0);
        Metropolis b(eg, U1Shift{0.7}, Pcg32(43, 0), 1.0);
        a.run(40);
        b.run(40);
        for (std::size_t i = 0; i < cm.sites(); ++i) CHECK(cm.data()[i].theta == eg.data()[i].theta);
    }
    {
        CellSU3 cm(hypercubic_plaquettes(2), SUPlaquetteTerm<3>{5.7});
        SUGauge<3> eg(2, 5.7);
        for (std::size_t i = 0; i < cm.sites(); ++i) {
            const auto one = SULink<3>::identity();
            cm.update(i, &one);  // CellModel starts at zero, as the reference's does
        }
        CHECK(std::abs(cm.total_energy()) < 1e-12);
        Metropolis a(cm, SUShift<3>{0.2}, Pcg32(44, 0), 1.0);
        Metropolis b(eg, SUShift<3>{0.2}, Pcg32(44, 0), 1.0);
        a.run(5);
        b.run(5);
        for (std::size_t i = 0; i < cm.sites(); ++i)
            for (std::size_t k = 0; k < 9; ++k) CHECK(cm.data()[i].m[k] == eg.data()[i].m[k]);
    }

    std::puts("ok");
    return 0;
}
