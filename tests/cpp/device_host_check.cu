// Host-side checks of include/umc/device.cuh that need no GPU: the fast
// division, RegularLattice's numbering and neighbours against a direct
// construction, the checkerboard colouring, Classes::from_colours, and the
// Rng against a sequential reference Pcg32 seeded the keyed way.  Prints "ok".
#include <umc/device.cuh>

#include <cstdio>
#include <cstdlib>
#include <random>
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

int main()
{
    check_fast_div();
    const std::uint32_t dims[][3] = {{2, 2, 1}, {4, 2, 1}, {8, 8, 1}, {6, 4, 2}, {10, 6, 4}, {2, 1, 1},
                                     {8, 1, 1}, {4, 1, 6}, {12, 4, 10}, {16, 6, 1}, {2, 2, 2}};
    for (const auto& d : dims) check_lattice(d[0], d[1], d[2]);
    check_lattice_refusals();
    check_classes();
    check_rng();
    std::printf("ok\n");
    return 0;
}
