// Host-side checks of include/umc/device.cuh that need no GPU: the fast
// division, RegularLattice's numbering and neighbours against a direct
// construction, the checkerboard colouring, Classes::from_colours, the Rng
// against a sequential reference Pcg32 seeded the keyed way, and
// PlaquetteLattice's numbering, cells and incidence against the library's
// plaquette complexes, and a model written on the Model base.  Prints "ok".
#include <umc/device.cuh>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <utility>
#include <vector>

using namespace umc::gpu::device;

#define CHECK(c)                                                            \
    do {                                                                    \
        if (!(c)) {                                                         \
            std::fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
            std::exit(1);                                                   \
        }                                                                   \
    } while (0)

// Pcg32(seed, 0) as rng.hpp:8-44 defines it.
struct RefPcg
{
    std::uint64_t state = 0, inc = 1;
    explicit RefPcg(std::uint64_t seed)
    {
        next();
        state += seed;
        next();
    }
    std::uint32_t next()
    {
        const std::uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        const auto x = std::uint32_t(((old >> 18u) ^ old) >> 27u);
        const auto r = std::uint32_t(old >> 59u);
        return (x >> r) | (x << ((32u - r) & 31u));
    }
};

static void check_fast_div()
{
    std::mt19937_64 g(7);
    const std::uint32_t ds[] = {1, 2, 3, 6, 7, 10, 64, 100, 255, 256, 1000, 4096, 65535, 65536, 123457, 1u << 31,
                                0xFFFFFFFFu};
    for (const auto d : ds) {
        const FastDiv f(d);
        const std::uint32_t ns[] = {0, 1, d - 1, d, d + 1, 0xFFFFFFFFu, 0xFFFFFFFEu};
        for (const auto n : ns) CHECK(f.div(n) == n / d);
        for (int k = 0; k < 20000; ++k) {
            const auto n = std::uint32_t(g());
            CHECK(f.div(n) == n / d);
        }
    }
}

static void check_lattice(std::uint32_t Lx, std::uint32_t Ly, std::uint32_t Lz)
{
    const RegularLattice l(Lx, Ly, Lz);
    const std::uint32_t n = l.sites(), deg = l.degree();
    CHECK(deg == 2u * ((Lx > 1) + (Ly > 1) + (Lz > 1)));
    std::vector<int> seen(n, 0);
    for (std::uint32_t z = 0; z < Lz; ++z)
        for (std::uint32_t y = 0; y < Ly; ++y)
            for (std::uint32_t x = 0; x < Lx; ++x) {
                const std::uint32_t k = l.index_of(x, y, z);
                CHECK(k < n);
                ++seen[k];
                std::uint32_t cx, cy, cz;
                l.coords(k, cx, cy, cz);
                CHECK(cx == x && cy == y && cz == z);
                std::uint32_t want[6], got[6], a = 0;
                want[a++] = l.index_of((x + 1) % Lx, y, z);
                want[a++] = l.index_of((x + Lx - 1) % Lx, y, z);
                if (Ly > 1) {
                    want[a++] = l.index_of(x, (y + 1) % Ly, z);
                    want[a++] = l.index_of(x, (y + Ly - 1) % Ly, z);
                }
                if (Lz > 1) {
                    want[a++] = l.index_of(x, y, (z + 1) % Lz);
                    want[a++] = l.index_of(x, y, (z + Lz - 1) % Lz);
                }
                CHECK(a == deg);
                l.neighbours(k, got);
                for (std::uint32_t b = 0; b < deg; ++b) {
                    CHECK(got[b] == want[b]);
                    CHECK((got[b] >= n / 2) != (k >= n / 2));  // the other colour
                    CHECK(l.neighbour(k, b) == want[b]);
                }
            }
    for (std::uint32_t k = 0; k < n; ++k) CHECK(seen[k] == 1);
    const auto c = detail::checkerboard(l);
    CHECK(c.count == 2 && c.begin() == (std::vector<std::uint32_t>{0, n / 2, n}));
    const auto order = c.order();
    for (std::uint32_t s = 0; s < n; ++s) CHECK(order[c.position[s]] == s);
}

static void check_lattice_refusals()
{
    const RegularLattice bad[] = {RegularLattice(3, 4, 1), RegularLattice(4, 3, 1), RegularLattice(4, 4, 5),
                                  RegularLattice(1, 4, 4), RegularLattice(0, 4, 4)};
    for (const auto& l : bad) {
        bool threw = false;
        try {
            (void)detail::checkerboard(l);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        CHECK(threw);
    }
}

static void check_classes()
{
    const std::vector<std::uint32_t> colour = {2, 0, 1, 0, 2, 1, 0};
    const auto k = Classes::from_colours(colour, 3);
    CHECK(k.count() == 3 && k.sites() == 7 && k.largest() == 3);
    CHECK(k.begin == (std::vector<std::uint32_t>{0, 3, 5, 7}));
    CHECK(k.order == (std::vector<std::uint32_t>{1, 3, 6, 2, 5, 0, 4}));
    bool threw = false;
    try {
        (void)Classes::from_colours({0, 3}, 3);
    } catch (const std::invalid_argument&) {
        threw = true;
    }
    CHECK(threw);
    const auto id = Classes::identity({0, 4, 9});
    CHECK(id.order.empty() && id.sites() == 9 && id.largest() == 5);
}

static void check_rng()
{
    for (std::uint64_t seed : {1ull, 42ull, 0xDEADBEEFull})
        for (std::uint64_t counter : {0ull, 7ull, 1000000ull})
            for (std::uint32_t id : {0u, 1u, 12345u}) {
                const std::uint64_t kb = umc::key_base(umc::key_seed(seed, counter, umc::tag_site(0)));
                Rng r(umc::KeyedPcg::open(kb, id));
                RefPcg ref(umc::id_seed(kb, id));
                for (int d = 0; d < 8; ++d) CHECK(r.uni() == double(ref.next()) * 0x1.0p-32);
            }
}

// A cell term that records which links a model hands it (host only).
struct Angle1
{
    using dtype = double;
    static constexpr std::size_t size = 1;
};
static std::vector<std::pair<std::array<std::uint32_t, 4>, std::size_t>> g_seen;
static const double* g_base = nullptr;
struct RecordingTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    __host__ __device__ double energy(const double* const*) const { return 0.0; }
    __host__ double delta(std::size_t which, const double*, const double*, const double* const* l) const
    {
        std::array<std::uint32_t, 4> c{};
        for (int k = 0; k < 4; ++k) c[k] = std::uint32_t(l[k] - g_base);
        g_seen.emplace_back(c, which);
        return 0.0;
    }
};

// Records the links cell_energy hands to energy (host only).
struct CellRecorder
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    __host__ __device__ double delta(std::size_t, const double*, const double*, const double* const*) const
    {
        return 0.0;
    }
    __host__ double energy(const double* const* ls) const
    {
        std::array<std::uint32_t, 4> cl{};
        for (int k = 0; k < 4; ++k) cl[k] = std::uint32_t(ls[k] - g_base);
        g_seen.emplace_back(cl, 0);
        return 0.0;
    }
};

// PlaquetteLattice against the library's plaquette complex: the numbering is
// the library's link colouring, and every link's computed (cell, slot) list is
// the library's incidence of that link, relabelled.
static void check_plaquettes(std::uint32_t L, std::uint32_t dim)
{
    umc_cells* cc = nullptr;
    umc_check(dim == 4 ? umc_cells_hypercubic(L, &cc) : umc_cells_square_plaquettes(L, &cc));
    const std::uint32_t n = std::uint32_t(umc_cells_sites(cc)), nc = std::uint32_t(umc_cells_count(cc));
    std::vector<std::uint32_t> colour(n), pos(n), cells(std::size_t(nc) * 4);
    std::uint32_t ncol = 0;
    umc_check(umc_cells_colouring(cc, &ncol, colour.data(), pos.data()));
    umc_check(umc_cells_table(cc, cells.data()));
    std::vector<std::uint64_t> off(n + 1);
    umc_check(umc_cells_incidence(cc, off.data(), nullptr, nullptr));
    std::vector<std::uint32_t> inc_cell(off.back());
    std::vector<std::uint8_t> inc_which(off.back());
    umc_check(umc_cells_incidence(cc, off.data(), inc_cell.data(), inc_which.data()));
    umc_cells_destroy(cc);

    const PlaquetteLattice l(L, dim);
    const auto c = detail::plaquette_colouring(l);
    CHECK(l.sites() == n && l.cells() == nc && c.count == ncol);
    for (std::uint32_t i = 0; i < n; ++i) CHECK(c.position[i] == pos[i]);
    std::vector<double> field(n, 0.0);
    g_base = field.data();
    const LatticeCellModel<Angle1, RecordingTerm> m{field.data(), l, RecordingTerm{}};
    for (std::uint32_t i = 0; i < n; ++i) {
        const std::uint32_t k = pos[i];
        std::uint32_t mu, x, par;
        l.decode(k, mu, x, par);
        CHECK(mu * l.V + x == i);
        g_seen.clear();
        const double p = 0.0;
        (void)m.energy_diff_at(k, &p);
        std::vector<std::pair<std::array<std::uint32_t, 4>, std::size_t>> want;
        for (std::uint64_t a = off[i]; a < off[i + 1]; ++a) {
            std::array<std::uint32_t, 4> cl{};
            for (int q = 0; q < 4; ++q) cl[q] = pos[cells[std::size_t(inc_cell[a]) * 4 + q]];
            want.emplace_back(cl, inc_which[a]);
        }
        std::sort(want.begin(), want.end());
        std::sort(g_seen.begin(), g_seen.end());
        CHECK(want == g_seen);
    }
    for (std::uint32_t q = 0; q < nc; ++q) {
        // cell_energy's links, read the same way
        g_seen.clear();
        const LatticeCellModel<Angle1, CellRecorder> mc{field.data(), l, CellRecorder{}};
        (void)mc.cell_energy(q);
        std::array<std::uint32_t, 4> want{};
        for (int k = 0; k < 4; ++k) want[k] = pos[cells[std::size_t(q) * 4 + k]];
        CHECK(g_seen.size() == 1 && g_seen[0].first == want);
    }
}

// A model written on the Model base (model.hpp:47-61): a Heisenberg ring of
// six sites, neighbours i - 1 and i + 1.
struct Ring : Model<double, 6, 3>
{
    using value_type = double;
    static constexpr std::size_t size = 3;
    using Model::Model;
    UMC_HD double energy_diff_at(std::size_t i, const double* p) const
    {
        const double* s = data();
        const std::size_t l = (i + 5) % 6, r = (i + 1) % 6;
        double d = 0.0;
        for (int c = 0; c < 3; ++c) d -= (p[c] - s[3 * i + c]) * (s[3 * l + c] + s[3 * r + c]);
        return d;
    }
};
static_assert(ModelLike<Ring>);
static_assert(std::is_trivially_copyable_v<Ring>);
static_assert(std::is_constructible_v<Ring, Field<double, 18>&>);
static_assert(!std::is_constructible_v<Ring, Field<double, 17>&>);

void check_model_base()
{
    std::vector<double> f(18);
    for (std::size_t k = 0; k < f.size(); ++k) f[k] = double(k);
    Ring m(f.data());
    CHECK(m.sites() == 6 && m.data() == f.data());
    const double p[3] = {-1.0, -2.0, -3.0};
    // site 2 holds (6, 7, 8), its neighbours 1 and 3 hold (3, 4, 5) and (9, 10, 11)
    const double want = -((-1.0 - 6.0) * (3.0 + 9.0) + (-2.0 - 7.0) * (4.0 + 10.0) + (-3.0 - 8.0) * (5.0 + 11.0));
    CHECK(m.energy_diff_at(2, p) == want);
    m.update(2, p);
    for (std::size_t k = 0; k < f.size(); ++k) CHECK(f[k] == (k / 3 == 2 ? p[k % 3] : double(k)));
}

int main()
{
    check_model_base();
    check_fast_div();
    const std::uint32_t dims[][3] = {{2, 2, 1}, {4, 2, 1}, {8, 8, 1}, {6, 4, 2}, {10, 6, 4}, {2, 1, 1},
                                     {8, 1, 1}, {4, 1, 6}, {12, 4, 10}, {16, 6, 1}, {2, 2, 2}};
    for (const auto& d : dims) check_lattice(d[0], d[1], d[2]);
    check_lattice_refusals();
    check_classes();
    check_rng();
    check_plaquettes(4, 4);
    check_plaquettes(6, 4);
    check_plaquettes(8, 2);
    check_plaquettes(2, 2);
    std::printf("ok\n");
    return 0;
}
