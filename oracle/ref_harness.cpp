// ref_harness.cpp -- drives the UNMODIFIED reference library (TEST INFRASTRUCTURE).
//
// Compiled against the reference headers where they lie (oracle/Makefile passes
// -I<reference root>); nothing from the reference is copied here.  The adapters
// below are ordinary user types that satisfy the reference's own concepts
// (Proposal dof/proposal.hpp:8-12, ModelLike model.hpp:70-86, WolffModel
// driver.hpp:73-84).  They only choose WHICH random stream the reference
// driver reads from:
//
//   KeyState / KeyedRng  one reference Pcg32 (rng.hpp:8-44), re-seeded per key
//                        Pcg32(id_seed(key_seed(seed, counter, tag), id), 0);
//   Keyed<Q>             a proposal adapter that re-keys on the site index it is
//                        handed (cur - data(), driver.hpp:35-36) before calling
//                        the reference proposal;
//   KeyedWolff<M>        a model adapter that re-keys on the edge id inside
//                        energy_diff_bond, which the Wolff driver calls right
//                        before the activation draw (driver.hpp:150-151);
//   KeyedAxis<A>         re-keys the axis/seed draws of one flip (driver.hpp:110,114);
//   MultiHit<M>          exposes K pseudo-sites per link so that the reference
//                        driver performs K Metropolis hits on each link in turn.
//
// The exported extern "C" functions mirror oracle/umc_oracle.h with a ref_
// prefix, plus ref_bench_* entry points that time the reference's own stock
// path (plain Pcg32, no adapters) for the CPU baseline.

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <thread>
#include <vector>

#include <driver.hpp>
#include <dof/ising.hpp>
#include <dof/sun.hpp>
#include <dof/u1.hpp>
#include <dof/vector.hpp>
#include <example/ising.hpp>
#include <example/sun_gauge.hpp>
#include <example/u1_gauge.hpp>
#include <example/vector_spin.hpp>
#include <lattice/cell_complex.hpp>
#include <lattice/hypercubic.hpp>
#include <lattice/pair_graph.hpp>
#include <lattice/square.hpp>
#include <model/cell.hpp>
#include <model/pair.hpp>
#include <rng.hpp>
#include <term/heisenberg.hpp>
#include <term/plaquette.hpp>
#include <term/sun_plaquette.hpp>

#include "umc_oracle.h"

namespace {

constexpr std::uint32_t TAG_BOND = 1;
constexpr std::uint32_t TAG_AXIS = 2;
constexpr std::uint32_t tag_site(std::uint32_t h) { return 0x100u + h; }

std::uint64_t mix64(std::uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return z;
}
std::uint64_t key_seed(std::uint64_t seed, std::uint64_t counter, std::uint32_t tag)
{
    return mix64(mix64(seed ^ (std::uint64_t(tag) << 32)) + counter * 0x9E3779B97F4A7C15ULL);
}
struct KeyState
{
    std::uint64_t seed = 0;
    std::uint64_t counter = 0;
    Pcg32 gen{0, 0};
    void open(std::uint32_t tag, std::uint64_t id)
    {
        gen = Pcg32(mix64(key_seed(seed, counter, tag) + (std::uint64_t(static_cast<std::uint32_t>(id)) + 1) *
                                                              0x9E3779B97F4A7C15ULL),
                    0);
    }
};

struct KeyedRng
{
    KeyState* ks;
    double uni() { return ks->gen.uni(); }
};

template <class Q, class T>
struct Keyed
{
    Q inner;
    KeyState* ks;
    const T* base;
    std::size_t size;
    std::uint32_t tag;

    template <class R>
    void sample(const T* cur, R& rng, T* out) const
    {
        ks->open(tag, static_cast<std::size_t>(cur - base) / size);
        inner.sample(cur, rng, out);
    }
    double log_ratio(const T* a, const T* b) const { return inner.log_ratio(a, b); }
};

// One draw per site, 16 sites per stream: re-keys on site / 16 and skips to
// output site % 16 before the reference proposal runs (used with Flip, which
// draws nothing, so the driver's accept draw is that output).
template <class Q, class T>
struct KeyedGroup
{
    Q inner;
    KeyState* ks;
    const T* base;

    template <class R>
    void sample(const T* cur, R& rng, T* out) const
    {
        const std::size_t i = static_cast<std::size_t>(cur - base);
        ks->open(tag_site(0), i / 16);
        for (std::size_t q = 0; q < i % 16; ++q) (void)ks->gen.uni();
        inner.sample(cur, rng, out);
    }
    double log_ratio(const T* a, const T* b) const { return inner.log_ratio(a, b); }
};

template <class A>
struct KeyedAxis
{
    A inner;
    KeyState* ks;
    template <class C, class R, class T>
    void sample(C cur, R& rng, T* out) const
    {
        ks->open(TAG_AXIS, 0);
        inner.sample(cur, rng, out);
    }
};

template <class M>
struct KeyedWolff
{
    using value_type = typename M::value_type;
    using bond_type = typename M::bond_type;
    static constexpr std::size_t size = M::size;

    M* m;
    KeyState* ks;
    const std::uint32_t* slot_edge;

    std::size_t sites() const { return m->sites(); }
    const value_type* data() const { return m->data(); }
    double energy_diff_at(std::size_t i, const value_type* p) const { return m->energy_diff_at(i, p); }
    void update(std::size_t i, const value_type* p) { m->update(i, p); }
    std::size_t degree(std::size_t i) const { return m->degree(i); }
    const bond_type* bonds(std::size_t i) const { return m->bonds(i); }
    double energy_diff_bond(std::size_t i, const bond_type& b, const value_type* p) const
    {
        ks->open(TAG_BOND, slot_edge[static_cast<std::size_t>(&b - m->bonds(0))]);
        return m->energy_diff_bond(i, b, p);
    }
};

// K pseudo-sites per link; data() points at a K-times larger dummy buffer so that
// the driver's pointer arithmetic stays inside an allocation.
template <class M>
struct MultiHit
{
    using value_type = typename M::value_type;
    static constexpr std::size_t size = M::size;

    M* m;
    std::size_t K;
    std::vector<value_type> dummy;

    std::size_t sites() const { return m->sites() * K; }
    const value_type* data() const { return dummy.data(); }
    double energy_diff_at(std::size_t i, const value_type* p) const { return m->energy_diff_at(i / K, p); }
    void update(std::size_t i, const value_type* p) { m->update(i / K, p); }
};

// Proposal adapter for MultiHit: keys on (link, hit) and proposes from the
// inner model's current link rather than the dummy pointer.
template <class Q, class M>
struct KeyedHit
{
    Q inner;
    KeyState* ks;
    const MultiHit<M>* mh;

    template <class R, class T>
    void sample(const T* cur, R& rng, T* out) const
    {
        const std::size_t i = static_cast<std::size_t>(cur - mh->dummy.data()) / M::size;
        const std::size_t link = i / mh->K, hit = i % mh->K;
        ks->open(tag_site(static_cast<std::uint32_t>(hit)), link);
        inner.sample(mh->m->data() + link * M::size, rng, out);
    }
    template <class T>
    double log_ratio(const T* a, const T* b) const { return inner.log_ratio(a, b); }
};

// Pair term E = -J cos(theta_i - theta_j) for the XY model on angles; a user
// CellTerm of arity 2 (term/cell.hpp:10-25) for PairModel (model/pair.hpp).
struct XYAngleTerm
{
    using dtype = U1Link;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J = 1.0;

    energy_type energy(const dtype* const* links) const
    {
        return -J * std::cos(links[0]->theta - links[1]->theta);
    }
    energy_type delta(std::size_t which, const dtype* old, const dtype* nw,
                      const dtype* const* links) const
    {
        const dtype* fixed = links[which == 0 ? 1 : 0];
        return -J * (std::cos(nw->theta - fixed->theta) - std::cos(old->theta - fixed->theta));
    }
};
static_assert(CellTerm<XYAngleTerm, U1Dof>);

int status_of(const std::exception_ptr& e)
{
    try {
        std::rethrow_exception(e);
    } catch (const std::out_of_range&) {
        return -1;
    } catch (const std::invalid_argument&) {
        return -2;
    } catch (const std::overflow_error&) {
        return -3;
    } catch (...) {
        return -4;
    }
}

std::vector<PairGraph<>::Edge> make_edges(const std::uint32_t* ei, const std::uint32_t* ej,
                                          std::uint64_t m)
{
    std::vector<PairGraph<>::Edge> edges(m);
    for (std::uint64_t e = 0; e < m; ++e) edges[e] = {ei[e], ej[e], {}};
    return edges;
}

// Slot -> edge-list index, replaying PairGraph's scatter order
// (lattice/pair_graph.hpp:77-81).
std::vector<std::uint32_t> slot_edges(const PairGraph<>& g, const std::uint32_t* ei,
                                      const std::uint32_t* ej, std::uint64_t m, bool symmetric)
{
    const std::size_t n = g.sites();
    std::vector<std::uint32_t> slot;
    if (n == 0) return slot;
    const auto* base = g.bonds(0);
    std::vector<std::size_t> pos(n);
    std::size_t total = 0;
    for (std::size_t i = 0; i < n; ++i) {
        pos[i] = base ? static_cast<std::size_t>(g.bonds(i) - base) : 0;
        total += g.degree(i);
    }
    slot.assign(total, 0);
    for (std::uint64_t e = 0; e < m; ++e) {
        slot[pos[ei[e]]++] = static_cast<std::uint32_t>(e);
        if (symmetric) slot[pos[ej[e]]++] = static_cast<std::uint32_t>(e);
    }
    return slot;
}

template <class M>
double half_energy_sum(const M& m)
{
    double sum = 0.0;
    for (std::size_t i = 0; i < m.sites(); ++i) sum += m.energy_at(i);
    return 0.5 * sum;
}

}  // namespace

// ------------------------------------------------------------------------- RNG
extern "C" void ref_pcg32_draws(std::uint64_t seed, std::uint64_t stream, std::uint32_t n, std::uint32_t* out)
{
    Pcg32 g(seed, stream);
    for (std::uint32_t k = 0; k < n; ++k) out[k] = static_cast<std::uint32_t>(g.uni() * 0x1.0p32);
}

extern "C" void ref_key_draws(std::uint64_t seed, std::uint64_t counter, std::uint32_t tag, std::uint32_t id,
                   std::uint32_t n, std::uint32_t* out)
{
    KeyState ks;
    ks.seed = seed;
    ks.counter = counter;
    ks.open(tag, id);
    for (std::uint32_t k = 0; k < n; ++k) out[k] = static_cast<std::uint32_t>(ks.gen.uni() * 0x1.0p32);
}

// ---------------------------------------------------------------------- tables
extern "C" int ref_pair_graph(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                   std::uint64_t m, int symmetric, std::uint32_t* offset, std::uint32_t* bonds)
{
    try {
        const auto edges = make_edges(ei, ej, m);
        PairGraph<> g(n, edges, symmetric != 0);
        std::uint32_t acc = 0;
        for (std::size_t i = 0; i < g.sites(); ++i) {
            offset[i] = acc;
            for (std::size_t a = 0; a < g.degree(i); ++a) {
                if (bonds) bonds[acc] = g.bonds(i)[a].j;
                ++acc;
            }
        }
        offset[g.sites()] = acc;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" int ref_square_lattice(std::uint64_t Lx, std::uint64_t Ly, std::uint32_t* offset, std::uint32_t* bonds)
{
    try {
        const auto g = square_lattice(Lx, Ly);
        std::uint32_t acc = 0;
        for (std::size_t i = 0; i < g.sites(); ++i) {
            offset[i] = acc;
            for (std::size_t a = 0; a < g.degree(i); ++a) {
                if (bonds) bonds[acc] = g.bonds(i)[a].j;
                ++acc;
            }
        }
        offset[g.sites()] = acc;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Dumps hypercubic_plaquettes(L): cells (6L^4 x 4) and the incidence rows.
extern "C" int ref_hypercubic(std::uint64_t L, std::uint32_t* cells, std::uint64_t* offset,
                   std::uint32_t* inc_cell, std::uint8_t* inc_which)
{
    try {
        const auto cc = hypercubic_plaquettes(L);
        for (std::size_t c = 0; c < cc.cells(); ++c)
            for (std::size_t k = 0; k < 4; ++k) cells[4 * c + k] = cc.cell(c)[k];
        std::uint64_t acc = 0;
        for (std::size_t i = 0; i < cc.sites(); ++i) {
            offset[i] = acc;
            for (const auto inc : cc.incident(i)) {
                inc_cell[acc] = inc.cell;
                inc_which[acc] = inc.which;
                ++acc;
            }
        }
        offset[cc.sites()] = acc;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" int ref_cell_incidence(std::uint64_t n_sites, const std::uint32_t* cells, std::uint64_t n_cells,
                       std::uint64_t* offset, std::uint32_t* inc_cell, std::uint8_t* inc_which)
{
    try {
        std::vector<Cell<4>> cl(n_cells);
        for (std::uint64_t c = 0; c < n_cells; ++c)
            for (int k = 0; k < 4; ++k) cl[c].sites[k] = cells[4 * c + k];
        CellComplex<4> cc(n_sites, cl);
        std::uint64_t acc = 0;
        for (std::size_t i = 0; i < cc.sites(); ++i) {
            offset[i] = acc;
            for (const auto inc : cc.incident(i)) {
                inc_cell[acc] = inc.cell;
                inc_which[acc] = inc.which;
                ++acc;
            }
        }
        offset[cc.sites()] = acc;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ----------------------------------------------------------------------- Ising
extern "C" int ref_ising_metropolis(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                         std::uint64_t m, std::int32_t J, double beta, std::uint64_t seed,
                         std::uint64_t sweep0, std::uint64_t n_sweeps, std::int8_t* spins,
                         double* E_out, double* M_out)
{
    try {
        const auto edges = make_edges(ei, ej, m);
        Ising model(PairGraph<>(n, edges), J);
        for (std::size_t i = 0; i < n; ++i) model.update(i, spins + i);
        KeyState ks;
        ks.seed = seed;
        ks.counter = sweep0;
        KeyedGroup<Flip, IsingSpin> prop{Flip{}, &ks, model.data()};
        Metropolis<Ising, KeyedGroup<Flip, IsingSpin>, KeyedRng> mc(model, prop, KeyedRng{&ks}, beta);
        std::uint64_t k = 0;
        mc.sample(n_sweeps, [&](const Ising& mdl) {
            if (E_out) E_out[k] = half_energy_sum(mdl);
            if (M_out) {
                double s = 0.0;
                for (std::size_t i = 0; i < mdl.sites(); ++i) s += mdl.data()[i];
                M_out[k] = s;
            }
            ++k;
            ++ks.counter;
        });
        std::memcpy(spins, model.data(), n);
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" int ref_ising_wolff(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                    std::uint64_t m, std::int32_t J, double beta, std::uint64_t seed,
                    std::uint64_t flip0, std::uint64_t n_flips, std::int8_t* spins,
                    std::uint64_t* sizes, double* E_out, double* M_out)
{
    try {
        const auto edges = make_edges(ei, ej, m);
        Ising model(PairGraph<>(n, edges), J);
        for (std::size_t i = 0; i < n; ++i) model.update(i, spins + i);
        // The model's graph is a copy of this one; slot order is identical.
        const auto slots = slot_edges(PairGraph<>(n, edges), ei, ej, m, true);
        KeyState ks;
        ks.seed = seed;
        ks.counter = flip0;
        KeyedWolff<Ising> km{&model, &ks, slots.data()};
        Wolff<KeyedWolff<Ising>, KeyedAxis<FixedAxis>, KeyedRng> w(
            km, KeyedAxis<FixedAxis>{FixedAxis{}, &ks}, KeyedRng{&ks}, beta);
        for (std::uint64_t f = 0; f < n_flips; ++f) {
            const std::size_t c = w.flip();
            if (sizes) sizes[f] = c;
            if (E_out) E_out[f] = half_energy_sum(model);
            if (M_out) {
                double s = 0.0;
                for (std::size_t i = 0; i < n; ++i) s += model.data()[i];
                M_out[f] = s;
            }
            ++ks.counter;
        }
        std::memcpy(spins, model.data(), n);
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ----------------------------------------------------- weighted Ising (payload)
namespace {
// The model of the reference's graph test (test/graph_check.cpp:34-83): double
// spins, E = -sum over bonds of c s_i s_j, c carried by PairGraph<double>'s
// bonds; a ModelLike and WolffModel against the reference's own concepts and
// graph type, so the reference drivers run it unchanged.
class WeightedIsing
{
public:
    using value_type = double;
    static constexpr std::size_t size = 1;
    using bond_type = PairGraph<double>::bond_type;

    explicit WeightedIsing(PairGraph<double> g) : graph_(std::move(g)), spin_(graph_.sites(), 1.0) {}

    std::size_t sites() const noexcept { return graph_.sites(); }
    const double* data() const noexcept { return spin_.data(); }
    std::size_t degree(std::size_t i) const noexcept { return graph_.degree(i); }
    const bond_type* bonds(std::size_t i) const noexcept { return graph_.bonds(i); }
    double energy_at(std::size_t i) const noexcept
    {
        double e = 0.0;
        const bond_type* bs = graph_.bonds(i);
        for (std::size_t a = 0; a < graph_.degree(i); ++a) e += -bs[a].c * spin_[i] * spin_[bs[a].j];
        return e;
    }
    double energy_diff_at(std::size_t i, const double* p) const noexcept
    {
        double d = 0.0;
        const bond_type* bs = graph_.bonds(i);
        for (std::size_t a = 0; a < graph_.degree(i); ++a) d += -bs[a].c * (*p - spin_[i]) * spin_[bs[a].j];
        return d;
    }
    double energy_diff_bond(std::size_t i, const bond_type& b, const double* p) const noexcept
    {
        return -b.c * (*p - spin_[b.j]) * spin_[i];
    }
    void update(std::size_t i, const double* p) noexcept { spin_[i] = *p; }

private:
    PairGraph<double> graph_;
    std::vector<double> spin_;
};
static_assert(ModelLike<WeightedIsing>);
static_assert(WolffModel<WeightedIsing>);

// The graph test's Flip on double spins and its axis r = 1 (test/graph_check.cpp:15-32).
struct FlipDouble
{
    template <class R>
    void sample(const double* cur, R&, double* out) const { *out = *cur > 0.0 ? -1.0 : 1.0; }
    double log_ratio(const double*, const double*) const { return 0.0; }
};
struct AxisDouble
{
    template <class R>
    void sample(const double*, R&, double* out) const { out[0] = 1.0; }
};

WeightedIsing weighted_model(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej, const double* c,
                             std::uint64_t m, const double* spins)
{
    std::vector<PairGraph<double>::Edge> edges(m);
    for (std::uint64_t e = 0; e < m; ++e) edges[e] = {ei[e], ej[e], c[e]};
    WeightedIsing model(PairGraph<double>(n, edges));
    for (std::size_t i = 0; i < n; ++i) model.update(i, spins + i);
    return model;
}
}  // namespace

// The reference's Metropolis over the weighted Ising model with per-site keyed
// streams (site i: stream id i, the accept draw its first output); c[e] is
// edge e's coupling.  E_out: 0.5 sum_i energy_at(i) after every sweep.
extern "C" int ref_weighted_ising_metropolis(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                                             const double* c, std::uint64_t m, double beta, std::uint64_t seed,
                                             std::uint64_t sweep0, std::uint64_t n_sweeps, double* spins,
                                             double* E_out)
{
    try {
        WeightedIsing model = weighted_model(n, ei, ej, c, m, spins);
        KeyState ks;
        ks.seed = seed;
        ks.counter = sweep0;
        using Q = Keyed<FlipDouble, double>;
        Metropolis<WeightedIsing, Q, KeyedRng> mc(model, Q{FlipDouble{}, &ks, model.data(), 1, tag_site(0)},
                                                  KeyedRng{&ks}, beta);
        std::uint64_t k = 0;
        mc.sample(n_sweeps, [&](const WeightedIsing& mdl) {
            if (E_out) E_out[k] = half_energy_sum(mdl);
            ++k;
            ++ks.counter;
        });
        std::memcpy(spins, model.data(), n * sizeof(double));
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// The reference's Wolff over the weighted Ising model, the bond in CSR slot a
// drawing from key[a], the axis and seed site from the flip's axis key.
extern "C" int ref_weighted_ising_wolff(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                                        const double* c, std::uint64_t m, const std::uint32_t* key, double beta,
                                        std::uint64_t seed, std::uint64_t flip0, std::uint64_t n_flips, double* spins,
                                        std::uint64_t* sizes, double* E_out)
{
    try {
        WeightedIsing model = weighted_model(n, ei, ej, c, m, spins);
        KeyState ks;
        ks.seed = seed;
        ks.counter = flip0;
        KeyedWolff<WeightedIsing> km{&model, &ks, key};
        Wolff<KeyedWolff<WeightedIsing>, KeyedAxis<AxisDouble>, KeyedRng> w(
            km, KeyedAxis<AxisDouble>{AxisDouble{}, &ks}, KeyedRng{&ks}, beta);
        for (std::uint64_t f = 0; f < n_flips; ++f) {
            const std::size_t sz = w.flip();
            if (sizes) sizes[f] = sz;
            if (E_out) E_out[f] = half_energy_sum(model);
            ++ks.counter;
        }
        std::memcpy(spins, model.data(), n * sizeof(double));
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ------------------------------------------------------------------ VectorSpin
namespace {
template <std::size_t N>
void vector_obs(const VectorSpin<N>& m, double* obs)
{
    obs[0] = half_energy_sum(m);
    for (std::size_t k = 0; k < N; ++k) {
        double s = 0.0;
        for (std::size_t i = 0; i < m.sites(); ++i) s += m.data()[i * N + k];
        obs[1 + k] = s;
    }
}

template <std::size_t N, class Q>
void vector_metro_run(VectorSpin<N>& model, Q q, KeyState& ks, double beta, std::uint64_t n_sweeps,
                      double* obs_out)
{
    using KQ = Keyed<Q, double>;
    KQ prop{q, &ks, model.data(), N, tag_site(0)};
    Metropolis<VectorSpin<N>, KQ, KeyedRng> mc(model, prop, KeyedRng{&ks}, beta);
    std::uint64_t k = 0;
    mc.sample(n_sweeps, [&](const VectorSpin<N>& mdl) {
        if (obs_out) vector_obs<N>(mdl, obs_out + k * (N + 1));
        ++k;
        ++ks.counter;
    });
}

template <std::size_t N>
int vector_metropolis(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                      std::uint64_t m, double J, double beta, int proposal, double delta,
                      std::uint64_t seed, std::uint64_t sweep0, std::uint64_t n_sweeps,
                      double* spins, double* obs_out)
{
    const auto edges = make_edges(ei, ej, m);
    VectorSpin<N> model(PairGraph<>(n, edges), J);
    for (std::size_t i = 0; i < n; ++i) model.update(i, spins + i * N);
    KeyState ks;
    ks.seed = seed;
    ks.counter = sweep0;
    if (proposal == 0) {
        vector_metro_run<N>(model, UniformSphereN<N>{}, ks, beta, n_sweeps, obs_out);
    } else {
        if constexpr (N >= 2) vector_metro_run<N>(model, LocalRotation<N>{delta}, ks, beta, n_sweeps, obs_out);
        else throw std::invalid_argument("LocalRotation needs N >= 2");
    }
    std::memcpy(spins, model.data(), n * N * sizeof(double));
    return 0;
}

template <std::size_t N>
int vector_wolff(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                 std::uint64_t m, double J, double beta, std::uint64_t seed, std::uint64_t flip0,
                 std::uint64_t n_flips, double* spins, std::uint64_t* sizes, double* obs_out)
{
    const auto edges = make_edges(ei, ej, m);
    VectorSpin<N> model(PairGraph<>(n, edges), J);
    for (std::size_t i = 0; i < n; ++i) model.update(i, spins + i * N);
    const auto slots = slot_edges(PairGraph<>(n, edges), ei, ej, m, true);
    KeyState ks;
    ks.seed = seed;
    ks.counter = flip0;
    KeyedWolff<VectorSpin<N>> km{&model, &ks, slots.data()};
    using Ax = KeyedAxis<UniformSphereN<N>>;
    Wolff<KeyedWolff<VectorSpin<N>>, Ax, KeyedRng> w(km, Ax{UniformSphereN<N>{}, &ks}, KeyedRng{&ks}, beta);
    for (std::uint64_t f = 0; f < n_flips; ++f) {
        const std::size_t c = w.flip();
        if (sizes) sizes[f] = c;
        if (obs_out) vector_obs<N>(model, obs_out + f * (N + 1));
        ++ks.counter;
    }
    std::memcpy(spins, model.data(), n * N * sizeof(double));
    return 0;
}
}  // namespace

extern "C" int ref_vector_metropolis(std::uint32_t N, std::uint64_t n, const std::uint32_t* ei,
                          const std::uint32_t* ej, std::uint64_t m, double J, double beta,
                          int proposal, double delta, std::uint64_t seed, std::uint64_t sweep0,
                          std::uint64_t n_sweeps, double* spins, double* obs_out)
{
    try {
        switch (N) {
        case 1: return vector_metropolis<1>(n, ei, ej, m, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins, obs_out);
        case 2: return vector_metropolis<2>(n, ei, ej, m, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins, obs_out);
        case 3: return vector_metropolis<3>(n, ei, ej, m, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins, obs_out);
        case 4: return vector_metropolis<4>(n, ei, ej, m, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins, obs_out);
        default: return -2;
        }
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" int ref_vector_wolff(std::uint32_t N, std::uint64_t n, const std::uint32_t* ei,
                     const std::uint32_t* ej, std::uint64_t m, double J, double beta,
                     std::uint64_t seed, std::uint64_t flip0, std::uint64_t n_flips, double* spins,
                     std::uint64_t* sizes, double* obs_out)
{
    try {
        switch (N) {
        case 1: return vector_wolff<1>(n, ei, ej, m, J, beta, seed, flip0, n_flips, spins, sizes, obs_out);
        case 2: return vector_wolff<2>(n, ei, ej, m, J, beta, seed, flip0, n_flips, spins, sizes, obs_out);
        case 3: return vector_wolff<3>(n, ei, ej, m, J, beta, seed, flip0, n_flips, spins, sizes, obs_out);
        case 4: return vector_wolff<4>(n, ei, ej, m, J, beta, seed, flip0, n_flips, spins, sizes, obs_out);
        default: return -2;
        }
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" void ref_sphere_sample(std::uint32_t N, std::uint64_t seed, std::uint64_t counter, std::uint32_t tag,
                       std::uint32_t id, double* out)
{
    KeyState ks;
    ks.seed = seed;
    ks.counter = counter;
    ks.open(tag, id);
    KeyedRng r{&ks};
    switch (N) {
    case 1: UniformSphereN<1>{}.sample(nullptr, r, out); break;
    case 2: UniformSphereN<2>{}.sample(nullptr, r, out); break;
    case 3: UniformSphereN<3>{}.sample(nullptr, r, out); break;
    case 4: UniformSphereN<4>{}.sample(nullptr, r, out); break;
    default: break;
    }
}

// --------------------------------------------------------------------- XY angle
extern "C" int ref_xy_metropolis(std::uint64_t n, const std::uint32_t* ei, const std::uint32_t* ej,
                      std::uint64_t m, double J, double beta, double width, std::uint64_t seed,
                      std::uint64_t sweep0, std::uint64_t n_sweeps, double* theta, double* obs_out)
{
    try {
        using PM = PairModel<U1Dof, XYAngleTerm, PairGraph<>>;
        const auto edges = make_edges(ei, ej, m);
        PM model(PairGraph<>(n, edges), XYAngleTerm{J});
        for (std::size_t i = 0; i < n; ++i) {
            const U1Link l{theta[i]};
            model.update(i, &l);
        }
        KeyState ks;
        ks.seed = seed;
        ks.counter = sweep0;
        using KQ = Keyed<U1Shift, U1Link>;
        KQ prop{U1Shift{width}, &ks, model.data(), 1, tag_site(0)};
        Metropolis<PM, KQ, KeyedRng> mc(model, prop, KeyedRng{&ks}, beta);
        std::uint64_t k = 0;
        mc.sample(n_sweeps, [&](const PM& mdl) {
            if (obs_out) {
                obs_out[3 * k] = half_energy_sum(mdl);
                double mx = 0.0, my = 0.0;
                for (std::size_t i = 0; i < mdl.sites(); ++i) {
                    mx += std::cos(mdl.data()[i].theta);
                    my += std::sin(mdl.data()[i].theta);
                }
                obs_out[3 * k + 1] = mx;
                obs_out[3 * k + 2] = my;
            }
            ++k;
            ++ks.counter;
        });
        for (std::size_t i = 0; i < n; ++i) theta[i] = model.data()[i].theta;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ------------------------------------------------------------------------ U(1)
extern "C" int ref_u1_metropolis(std::uint64_t n_links, const std::uint32_t* cells, std::uint64_t n_cells,
                      double model_beta, double driver_beta, double width, std::uint32_t hits,
                      std::uint64_t seed, std::uint64_t sweep0, std::uint64_t n_sweeps,
                      double* theta, double* obs_out)
{
    try {
        using CM = CellModel<U1Dof, U1PlaquetteTerm, CellComplex<4>>;
        std::vector<Cell<4>> cl(n_cells);
        for (std::uint64_t c = 0; c < n_cells; ++c)
            for (int k = 0; k < 4; ++k) cl[c].sites[k] = cells[4 * c + k];
        CM model(CellComplex<4>(n_links, cl), U1PlaquetteTerm{model_beta});
        for (std::size_t i = 0; i < n_links; ++i) {
            const U1Link l{theta[i]};
            model.update(i, &l);
        }
        KeyState ks;
        ks.seed = seed;
        ks.counter = sweep0;
        MultiHit<CM> mh{&model, hits, std::vector<U1Link>(n_links * hits)};
        using KQ = KeyedHit<U1Shift, CM>;
        Metropolis<MultiHit<CM>, KQ, KeyedRng> mc(mh, KQ{U1Shift{width}, &ks, &mh}, KeyedRng{&ks}, driver_beta);
        std::uint64_t k = 0;
        mc.sample(n_sweeps, [&](const MultiHit<CM>&) {
            if (obs_out) {
                double sum = 0.0;
                for (std::size_t c = 0; c < model.cells(); ++c) {
                    const auto s = model.cell_sites(c);
                    const U1Link* ls[4] = {model.data() + s[0], model.data() + s[1], model.data() + s[2], model.data() + s[3]};
                    sum += model.term().cos_plaquette(ls);
                }
                const double P = sum / double(model.cells());
                obs_out[2 * k] = model_beta * double(model.cells()) * (1.0 - P);
                obs_out[2 * k + 1] = P;
            }
            ++k;
            ++ks.counter;
        });
        for (std::size_t i = 0; i < n_links; ++i) theta[i] = model.data()[i].theta;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ----------------------------------------------------------------------- SU(N)
namespace {
template <std::size_t N>
int su_metropolis(std::uint64_t n_links, const std::uint32_t* cells, std::uint64_t n_cells,
                  double model_beta, double driver_beta, double width, std::uint32_t hits,
                  std::uint64_t seed, std::uint64_t sweep0, std::uint64_t n_sweeps, double* links,
                  double* obs_out)
{
    using CM = CellModel<SUDof<N>, SUPlaquetteTerm<N>, CellComplex<4>>;
    std::vector<Cell<4>> cl(n_cells);
    for (std::uint64_t c = 0; c < n_cells; ++c)
        for (int k = 0; k < 4; ++k) cl[c].sites[k] = cells[4 * c + k];
    CM model(CellComplex<4>(n_links, cl), SUPlaquetteTerm<N>{model_beta});
    for (std::size_t i = 0; i < n_links; ++i) {
        SULink<N> u;
        for (std::size_t q = 0; q < N * N; ++q) u.m[q] = {links[(i * N * N + q) * 2], links[(i * N * N + q) * 2 + 1]};
        model.update(i, &u);
    }
    KeyState ks;
    ks.seed = seed;
    ks.counter = sweep0;
    MultiHit<CM> mh{&model, hits, std::vector<SULink<N>>(n_links * hits)};
    using KQ = KeyedHit<SUShift<N>, CM>;
    Metropolis<MultiHit<CM>, KQ, KeyedRng> mc(mh, KQ{SUShift<N>{width}, &ks, &mh}, KeyedRng{&ks}, driver_beta);
    std::uint64_t k = 0;
    mc.sample(n_sweeps, [&](const MultiHit<CM>&) {
        if (obs_out) {
            double sum = 0.0;
            for (std::size_t c = 0; c < model.cells(); ++c) {
                const auto s = model.cell_sites(c);
                const SULink<N>* ls[4] = {model.data() + s[0], model.data() + s[1], model.data() + s[2], model.data() + s[3]};
                sum += model.term().real_plaquette(ls);
            }
            const double P = sum / double(model.cells());
            obs_out[2 * k] = model_beta * double(model.cells()) * (1.0 - P);
            obs_out[2 * k + 1] = P;
        }
        ++k;
        ++ks.counter;
    });
    for (std::size_t i = 0; i < n_links; ++i)
        for (std::size_t q = 0; q < N * N; ++q) {
            links[(i * N * N + q) * 2] = model.data()[i].m[q].real();
            links[(i * N * N + q) * 2 + 1] = model.data()[i].m[q].imag();
        }
    return 0;
}
}  // namespace

extern "C" int ref_su_metropolis(std::uint32_t N, std::uint64_t n_links, const std::uint32_t* cells,
                      std::uint64_t n_cells, double model_beta, double driver_beta, double width,
                      std::uint32_t hits, std::uint64_t seed, std::uint64_t sweep0,
                      std::uint64_t n_sweeps, double* links, double* obs_out)
{
    try {
        switch (N) {
        case 2: return su_metropolis<2>(n_links, cells, n_cells, model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, links, obs_out);
        case 3: return su_metropolis<3>(n_links, cells, n_cells, model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, links, obs_out);
        default: return -2;
        }
    } catch (...) {
        return status_of(std::current_exception());
    }
}

extern "C" void ref_su_expm(std::uint32_t N, const double* a, double* out)
{
    if (N == 2) {
        sun_detail::Mat<2> m;
        for (int q = 0; q < 4; ++q) m[q] = {a[2 * q], a[2 * q + 1]};
        const auto r = sun_detail::expm<2>(m);
        for (int q = 0; q < 4; ++q) { out[2 * q] = r.m[q].real(); out[2 * q + 1] = r.m[q].imag(); }
    } else if (N == 3) {
        sun_detail::Mat<3> m;
        for (int q = 0; q < 9; ++q) m[q] = {a[2 * q], a[2 * q + 1]};
        const auto r = sun_detail::expm<3>(m);
        for (int q = 0; q < 9; ++q) { out[2 * q] = r.m[q].real(); out[2 * q + 1] = r.m[q].imag(); }
    }
}

extern "C" void ref_su_shift(std::uint32_t N, double width, std::uint64_t seed, std::uint64_t counter,
                  std::uint32_t tag, std::uint32_t id, const double* cur, double* out)
{
    KeyState ks;
    ks.seed = seed;
    ks.counter = counter;
    ks.open(tag, id);
    KeyedRng r{&ks};
    if (N == 2) {
        SULink<2> c, o;
        for (int q = 0; q < 4; ++q) c.m[q] = {cur[2 * q], cur[2 * q + 1]};
        SUShift<2>{width}.sample(&c, r, &o);
        for (int q = 0; q < 4; ++q) { out[2 * q] = o.m[q].real(); out[2 * q + 1] = o.m[q].imag(); }
    } else if (N == 3) {
        SULink<3> c, o;
        for (int q = 0; q < 9; ++q) c.m[q] = {cur[2 * q], cur[2 * q + 1]};
        SUShift<3>{width}.sample(&c, r, &o);
        for (int q = 0; q < 9; ++q) { out[2 * q] = o.m[q].real(); out[2 * q + 1] = o.m[q].imag(); }
    }
}

// -------------------------------------------------------------- CPU baseline
// Times the reference's stock path: VectorSpin<3> on a periodic L^3 PairGraph
// (edges built by hand, as a user of the reference would), Metropolis with
// UniformSphereN<3> and a plain Pcg32, alternating one sweep with one Wolff
// flip (UniformSphereN<3> axis).  One independent chain per thread, uniform
// random start; `warmup` untimed steps, then `steps` timed ones.  Reports the
// total site-updates (sweep sites + flipped cluster sites) and the wall time of
// the slowest thread.
extern "C" int ref_bench_o3(std::uint64_t L, double beta, std::uint64_t warmup, std::uint64_t steps,
                            std::uint32_t threads, std::uint64_t seed, double* site_updates, double* seconds)
{
    try {
        std::vector<PairGraph<>::Edge> edges;
        edges.reserve(3 * L * L * L);
        for (std::uint64_t z = 0; z < L; ++z)
            for (std::uint64_t y = 0; y < L; ++y)
                for (std::uint64_t x = 0; x < L; ++x) {
                    const auto i = static_cast<std::uint32_t>((z * L + y) * L + x);
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + y) * L + (x + 1) % L), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + (y + 1) % L) * L + x), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((((z + 1) % L) * L + y) * L + x), {}});
                }
        const std::size_t n = L * L * L;
        std::vector<double> upd(threads, 0.0), secs(threads, 0.0);
        std::vector<std::thread> pool;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                VectorSpin<3> model(PairGraph<>(n, edges), 1.0);
                Pcg32 init(seed + t, 7);
                double v[3];
                for (std::size_t i = 0; i < n; ++i) {
                    UniformSphereN<3>{}.sample(nullptr, init, v);
                    model.update(i, v);
                }
                Metropolis<VectorSpin<3>, UniformSphereN<3>, Pcg32> mc(model, UniformSphereN<3>{}, Pcg32(seed + t, 1), beta);
                Wolff<VectorSpin<3>, UniformSphereN<3>, Pcg32> w(model, UniformSphereN<3>{}, Pcg32(seed + t, 2), beta);
                for (std::uint64_t s = 0; s < warmup; ++s) {
                    (void)w.flip();
                    mc.sweep();
                }
                const auto t0 = std::chrono::steady_clock::now();
                double u = 0.0;
                for (std::uint64_t s = 0; s < steps; ++s) {
                    u += double(w.flip());
                    mc.sweep();
                    u += double(n);
                }
                const auto t1 = std::chrono::steady_clock::now();
                upd[t] = u;
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
            });
        for (auto& th : pool) th.join();
        double total = 0.0, worst = 0.0;
        for (std::uint32_t t = 0; t < threads; ++t) {
            total += upd[t];
            if (secs[t] > worst) worst = secs[t];
        }
        *site_updates = total;
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// The reference's stock O(3) chain as a user would run it (same set-up as
// ref_bench_o3, one chain): per step one Wolff flip then one Metropolis sweep,
// plain Pcg32 streams; after `warmup` steps it records [E, Mx, My, Mz] of every
// step into obs (steps x 4).  The statistical check against the GPU chain.
extern "C" int ref_stock_o3_chain(std::uint64_t L, double beta, std::uint64_t seed, std::uint64_t warmup,
                                  std::uint64_t steps, double* obs)
{
    try {
        std::vector<PairGraph<>::Edge> edges;
        edges.reserve(3 * L * L * L);
        for (std::uint64_t z = 0; z < L; ++z)
            for (std::uint64_t y = 0; y < L; ++y)
                for (std::uint64_t x = 0; x < L; ++x) {
                    const auto i = static_cast<std::uint32_t>((z * L + y) * L + x);
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + y) * L + (x + 1) % L), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + (y + 1) % L) * L + x), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((((z + 1) % L) * L + y) * L + x), {}});
                }
        const std::size_t n = L * L * L;
        VectorSpin<3> model(PairGraph<>(n, edges), 1.0);
        Pcg32 init(seed, 7);
        double v[3];
        for (std::size_t i = 0; i < n; ++i) {
            UniformSphereN<3>{}.sample(nullptr, init, v);
            model.update(i, v);
        }
        Metropolis<VectorSpin<3>, UniformSphereN<3>, Pcg32> mc(model, UniformSphereN<3>{}, Pcg32(seed, 1), beta);
        Wolff<VectorSpin<3>, UniformSphereN<3>, Pcg32> w(model, UniformSphereN<3>{}, Pcg32(seed, 2), beta);
        for (std::uint64_t s = 0; s < warmup + steps; ++s) {
            (void)w.flip();
            mc.sweep();
            if (s >= warmup) vector_obs<3>(model, obs + (s - warmup) * 4);
        }
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

namespace {
// A window of `links` links of a model, each visited K times in a row, for
// timing the reference's stock multi-hit Metropolis on a bounded sample:
// pseudo-site i is hit i % K of link i / K; data() points at a dummy buffer
// so the driver's pointer arithmetic stays inside an allocation.
template <class M>
struct HitWindow
{
    using value_type = typename M::value_type;
    static constexpr std::size_t size = M::size;

    M* m;
    std::size_t K, links;
    std::vector<value_type> dummy;

    std::size_t sites() const { return links * K; }
    const value_type* data() const { return dummy.data(); }
    double energy_diff_at(std::size_t i, const value_type* p) const { return m->energy_diff_at(i / K, p); }
    void update(std::size_t i, const value_type* p) { m->update(i / K, p); }
};

// The stock proposal on a HitWindow: proposes from the model's current link
// (not the dummy pointer) with the driver's plain Pcg32.
template <class Q, class M>
struct StockHit
{
    Q inner;
    const HitWindow<M>* w;

    template <class R, class T>
    void sample(const T* cur, R& rng, T* out) const
    {
        const std::size_t i = static_cast<std::size_t>(cur - w->dummy.data()) / M::size;
        inner.sample(w->m->data() + (i / w->K) * M::size, rng, out);
    }
    template <class T>
    double log_ratio(const T* a, const T* b) const { return inner.log_ratio(a, b); }
};
}  // namespace

// Times the reference's stock SU(3) path: SUGauge<3> (example/sun_gauge.hpp)
// on hypercubic_plaquettes(L) with model beta and a cold start, Metropolis
// with SUShift<3>{width}, driver beta 1 and a plain Pcg32, `hits` proposals per
// link in a row; one chain per thread, each sweeping a window of the first
// `window` links (the reference's link order) `sweeps` times after one
// untimed window sweep.  site_updates = threads x window x hits x sweeps.
extern "C" int ref_bench_su3(std::uint64_t L, double model_beta, double width, std::uint32_t hits, std::uint64_t window,
                             std::uint64_t sweeps, std::uint32_t threads, std::uint64_t seed, double* site_updates,
                             double* seconds)
{
    try {
        std::vector<double> secs(threads, 0.0);
        std::vector<std::thread> pool;
        std::atomic<int> failed{0};
        std::size_t used = 0;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                try {
                    SUGauge<3> model(L, model_beta);
                    const std::size_t w = std::min<std::size_t>(window, model.sites());
                    if (t == 0) used = w;
                    HitWindow<SUGauge<3>> hw{&model, hits, w, std::vector<SULink<3>>(w * hits)};
                    using Q = StockHit<SUShift<3>, SUGauge<3>>;
                    Metropolis<HitWindow<SUGauge<3>>, Q, Pcg32> mc(hw, Q{SUShift<3>{width}, &hw}, Pcg32(seed + t, 1), 1.0);
                    mc.sweep();
                    const auto t0 = std::chrono::steady_clock::now();
                    mc.run(sweeps);
                    const auto t1 = std::chrono::steady_clock::now();
                    secs[t] = std::chrono::duration<double>(t1 - t0).count();
                } catch (...) {
                    failed = 1;
                }
            });
        for (auto& th : pool) th.join();
        if (failed) return -1;
        double worst = 0.0;
        for (double x : secs) worst = x > worst ? x : worst;
        *site_updates = double(threads) * double(used) * double(hits) * double(sweeps);
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Independent copies of the reference's stock O(3) chain (set-up of
// ref_stock_o3_chain), one per thread: chain c starts from init + c n 3 (n x 3
// doubles per chain, the site order of the user edge list; NULL = the uniform
// random start of seed + c), runs `warmup` steps with plain Pcg32 streams seeded
// seed + c, then records [E, Mx, My, Mz] of every step into
// obs[(c * steps + k) * 4].  A start taken from another chain's equilibrium
// lets the reference's chains skip their own thermalisation.
extern "C" int ref_stock_o3_chains(std::uint64_t L, double beta, std::uint64_t seed, std::uint32_t chains,
                                   const double* init, std::uint64_t warmup, std::uint64_t steps, double* obs)
{
    try {
        std::vector<PairGraph<>::Edge> edges;
        edges.reserve(3 * L * L * L);
        for (std::uint64_t z = 0; z < L; ++z)
            for (std::uint64_t y = 0; y < L; ++y)
                for (std::uint64_t x = 0; x < L; ++x) {
                    const auto i = static_cast<std::uint32_t>((z * L + y) * L + x);
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + y) * L + (x + 1) % L), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + (y + 1) % L) * L + x), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((((z + 1) % L) * L + y) * L + x), {}});
                }
        const std::size_t n = L * L * L;
        std::vector<std::thread> pool;
        std::atomic<int> failed{0};
        for (std::uint32_t c = 0; c < chains; ++c)
            pool.emplace_back([&, c] {
                try {
                    VectorSpin<3> model(PairGraph<>(n, edges), 1.0);
                    Pcg32 init_rng(seed + c, 7);
                    double v[3];
                    for (std::size_t i = 0; i < n; ++i) {
                        if (init) {
                            model.update(i, init + (std::uint64_t(c) * n + i) * 3);
                        } else {
                            UniformSphereN<3>{}.sample(nullptr, init_rng, v);
                            model.update(i, v);
                        }
                    }
                    Metropolis<VectorSpin<3>, UniformSphereN<3>, Pcg32> mc(model, UniformSphereN<3>{}, Pcg32(seed + c, 1),
                                                                         beta);
                    Wolff<VectorSpin<3>, UniformSphereN<3>, Pcg32> w(model, UniformSphereN<3>{}, Pcg32(seed + c, 2), beta);
                    double* out = obs + std::uint64_t(c) * steps * 4;
                    for (std::uint64_t s = 0; s < warmup + steps; ++s) {
                        (void)w.flip();
                        mc.sweep();
                        if (s >= warmup) vector_obs<3>(model, out + (s - warmup) * 4);
                    }
                } catch (...) {
                    failed = 1;
                }
            });
        for (auto& th : pool) th.join();
        return failed ? -1 : 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// The reference's stock SU(3) chains: example/sun_gauge.hpp's SUGauge<3> on
// hypercubic_plaquettes(L) (cold start, model beta), Metropolis with
// SUShift<3>{width}, one hit per link, driver beta 1 and a plain Pcg32 (seed +
// c for chain c), one chain per thread; after `warmup` sweeps each records the
// mean plaquette of every sweep into plaq[c * sweeps + k].
extern "C" int ref_stock_su3_chain(std::uint64_t L, double beta, double width, std::uint64_t seed,
                                   std::uint32_t chains, std::uint64_t warmup, std::uint64_t sweeps, double* plaq)
{
    try {
        std::vector<std::thread> pool;
        std::atomic<int> failed{0};
        for (std::uint32_t c = 0; c < chains; ++c)
            pool.emplace_back([&, c] {
                try {
                    SUGauge<3> model(L, beta);
                    Metropolis<SUGauge<3>, SUShift<3>, Pcg32> mc(model, SUShift<3>{width}, Pcg32(seed + c, 1), 1.0);
                    mc.run(warmup);
                    double* out = plaq + std::uint64_t(c) * sweeps;
                    std::uint64_t k = 0;
                    mc.sample(sweeps, [&](const SUGauge<3>& m) { out[k++] = m.mean_plaquette(); });
                } catch (...) {
                    failed = 1;
                }
            });
        for (auto& th : pool) th.join();
        return failed ? -1 : 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Times the reference's stock Ising Metropolis on an L x L square_lattice
// (example/ising.hpp + Flip + Pcg32), one chain per thread, cold start.
extern "C" int ref_bench_ising(std::uint64_t L, double beta, std::uint64_t warmup, std::uint64_t sweeps,
                               std::uint32_t threads, std::uint64_t seed, double* site_updates, double* seconds)
{
    try {
        std::vector<double> secs(threads, 0.0);
        std::vector<std::thread> pool;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                Ising model(square_lattice(L, L), 1);
                Metropolis<Ising, Flip, Pcg32> mc(model, Flip{}, Pcg32(seed + t, 1), beta);
                mc.run(warmup);
                const auto t0 = std::chrono::steady_clock::now();
                mc.run(sweeps);
                const auto t1 = std::chrono::steady_clock::now();
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
            });
        for (auto& th : pool) th.join();
        double worst = 0.0;
        for (double s : secs) worst = s > worst ? s : worst;
        *site_updates = double(threads) * double(L * L) * double(sweeps);
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Times the reference's stock Ising Wolff: Ising on an L x L square_lattice
// (cold start, then `warmup` flips) with FixedAxis and a plain Pcg32, one
// chain per thread; site_updates = the flipped sites of the timed flips.
extern "C" int ref_bench_ising_wolff(std::uint64_t L, double beta, std::uint64_t warmup, std::uint64_t flips,
                                     std::uint32_t threads, std::uint64_t seed, double* site_updates, double* seconds)
{
    try {
        std::vector<double> secs(threads, 0.0), sites(threads, 0.0);
        std::vector<std::thread> pool;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                Ising model(square_lattice(L, L), 1);
                Wolff<Ising, FixedAxis, Pcg32> w(model, FixedAxis{}, Pcg32(seed + t, 2), beta);
                for (std::uint64_t f = 0; f < warmup; ++f) (void)w.flip();
                double u = 0.0;
                const auto t0 = std::chrono::steady_clock::now();
                for (std::uint64_t f = 0; f < flips; ++f) u += double(w.flip());
                const auto t1 = std::chrono::steady_clock::now();
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
                sites[t] = u;
            });
        for (auto& th : pool) th.join();
        double worst = 0.0, total = 0.0;
        for (std::uint32_t t = 0; t < threads; ++t) {
            worst = secs[t] > worst ? secs[t] : worst;
            total += sites[t];
        }
        *site_updates = total;
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Times the reference's generic cell model: CellModel<U1Dof, U1PlaquetteTerm,
// CellComplex<4>> (model/cell.hpp, term/plaquette.hpp) on hypercubic_plaquettes(L)
// with U1Shift{width} and a plain Pcg32, one chain per thread, uniform random
// start; site_updates = links x sweeps x threads.
extern "C" int ref_bench_u1_cells(std::uint64_t L, double model_beta, double beta, double width, std::uint64_t warmup,
                                  std::uint64_t sweeps, std::uint32_t threads, std::uint64_t seed,
                                  double* site_updates, double* seconds)
{
    try {
        using CM = CellModel<U1Dof, U1PlaquetteTerm, CellComplex<4>>;
        std::vector<double> secs(threads, 0.0);
        std::vector<std::thread> pool;
        std::size_t links = 0;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                CM model(hypercubic_plaquettes(L), U1PlaquetteTerm{model_beta});
                Pcg32 init(seed + t, 9);
                for (std::size_t i = 0; i < model.sites(); ++i) {
                    const U1Link l{6.283185307179586 * init.uni() - 3.141592653589793};
                    model.update(i, &l);
                }
                if (t == 0) links = model.sites();
                Metropolis<CM, U1Shift, Pcg32> mc(model, U1Shift{width}, Pcg32(seed + t, 1), beta);
                mc.run(warmup);
                const auto t0 = std::chrono::steady_clock::now();
                mc.run(sweeps);
                const auto t1 = std::chrono::steady_clock::now();
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
            });
        for (auto& th : pool) th.join();
        double worst = 0.0;
        for (double x : secs) worst = x > worst ? x : worst;
        *site_updates = double(threads) * double(links) * double(sweeps);
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Times the reference's stock XY model on angles: PairModel<U1Dof, -J cos> on an
// L x L square_lattice with U1Shift{width} and a plain Pcg32, one chain per
// thread, uniform random start.
extern "C" int ref_bench_xy(std::uint64_t L, double beta, double width, std::uint64_t warmup, std::uint64_t sweeps,
                            std::uint32_t threads, std::uint64_t seed, double* site_updates, double* seconds)
{
    try {
        using PM = PairModel<U1Dof, XYAngleTerm, PairGraph<>>;
        std::vector<double> secs(threads, 0.0);
        std::vector<std::thread> pool;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                PM model(square_lattice(L, L), XYAngleTerm{1.0});
                Pcg32 init(seed + t, 9);
                for (std::size_t i = 0; i < model.sites(); ++i) {
                    const U1Link l{6.283185307179586 * init.uni()};
                    model.update(i, &l);
                }
                Metropolis<PM, U1Shift, Pcg32> mc(model, U1Shift{width}, Pcg32(seed + t, 1), beta);
                mc.run(warmup);
                const auto t0 = std::chrono::steady_clock::now();
                mc.run(sweeps);
                const auto t1 = std::chrono::steady_clock::now();
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
            });
        for (auto& th : pool) th.join();
        double worst = 0.0;
        for (double x : secs) worst = x > worst ? x : worst;
        *site_updates = double(threads) * double(L * L) * double(sweeps);
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// Times the reference's generic table-driven O(3) model: PairModel<VectorDof<3>,
// HeisenbergTerm<3>, PairGraph<>> (model/pair.hpp, term/heisenberg.hpp) on the
// periodic L^3 cubic edge list, Metropolis with UniformSphereN<3> and a plain
// Pcg32, one chain per thread, uniform random start.
extern "C" int ref_bench_pair_o3(std::uint64_t L, double beta, std::uint64_t warmup, std::uint64_t sweeps,
                                 std::uint32_t threads, std::uint64_t seed, double* site_updates, double* seconds)
{
    try {
        using PM = PairModel<VectorDof<3>, HeisenbergTerm<3>, PairGraph<>>;
        std::vector<PairGraph<>::Edge> edges;
        edges.reserve(3 * L * L * L);
        for (std::uint64_t z = 0; z < L; ++z)
            for (std::uint64_t y = 0; y < L; ++y)
                for (std::uint64_t x = 0; x < L; ++x) {
                    const auto i = static_cast<std::uint32_t>((z * L + y) * L + x);
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + y) * L + (x + 1) % L), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((z * L + (y + 1) % L) * L + x), {}});
                    edges.push_back({i, static_cast<std::uint32_t>((((z + 1) % L) * L + y) * L + x), {}});
                }
        const std::size_t n = L * L * L;
        std::vector<double> secs(threads, 0.0);
        std::vector<std::thread> pool;
        for (std::uint32_t t = 0; t < threads; ++t)
            pool.emplace_back([&, t] {
                PM model(PairGraph<>(n, edges), HeisenbergTerm<3>{1.0});
                Pcg32 init(seed + t, 7);
                double v[3];
                for (std::size_t i = 0; i < n; ++i) {
                    UniformSphereN<3>{}.sample(nullptr, init, v);
                    model.update(i, v);
                }
                Metropolis<PM, UniformSphereN<3>, Pcg32> mc(model, UniformSphereN<3>{}, Pcg32(seed + t, 1), beta);
                mc.run(warmup);
                const auto t0 = std::chrono::steady_clock::now();
                mc.run(sweeps);
                const auto t1 = std::chrono::steady_clock::now();
                secs[t] = std::chrono::duration<double>(t1 - t0).count();
            });
        for (auto& th : pool) th.join();
        double worst = 0.0;
        for (double x : secs) worst = x > worst ? x : worst;
        *site_updates = double(threads) * double(n) * double(sweeps);
        *seconds = worst;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}

// ------------------------------------------------------- learned U(1) proposal
// A user Proposal (dof/proposal.hpp:8-12) whose density depends on the link's
// staple.  It finds the link from cur - data() (the driver hands it the model's
// own storage, driver.hpp:35-36), evaluates the oracle's network and mixture
// for that staple, samples with the oracle's Best-Fisher trial fed by the
// reference Pcg32 (each uni() is k 2^-32, so k is recovered exactly), and
// returns log q(old) - log q(new).  The reference Metropolis driver supplies
// dE (CellModel::energy_diff_at) and the accept step, so this pins the
// learned update's composition against the reference driver itself.
struct LearnedU1
{
    KeyState* ks;
    const U1Link* base;
    const std::uint32_t* cells;
    const std::uint64_t* inc_off;
    const std::uint32_t* inc_cell;
    const std::uint8_t* inc_which;
    const double* params;
    mutable double w[4], mu[4], kappa[4], li[4];
    mutable bool moved = false;

    static std::uint32_t raw(double u) { return static_cast<std::uint32_t>(u * 4294967296.0); }

    template <class R>
    void sample(const U1Link* cur, R& rng, U1Link* out) const
    {
        const std::size_t i = static_cast<std::size_t>(cur - base);
        ks->open(6u, i);
        double Sr = 0.0, Si = 0.0;
        for (std::uint64_t a = inc_off[i]; a < inc_off[i + 1]; ++a) {
            const std::uint32_t* q = cells + 4 * std::uint64_t(inc_cell[a]);
            const double t0 = base[q[0]].theta, t1 = base[q[1]].theta, t2 = base[q[2]].theta,
                         t3 = base[q[3]].theta;
            double phi;
            switch (inc_which[a]) {
            case 0: phi = t1 - t2 - t3; break;
            case 1: phi = t0 - t2 - t3; break;
            case 2: phi = t3 - t0 - t1; break;
            default: phi = t2 - t0 - t1; break;
            }
            Sr += std::cos(phi);
            Si += std::sin(phi);
        }
        double x[3], o[16];
        orc_u1_features(Sr, Si, x);
        orc_mlp_forward(params, 1, x, 1, o);
        orc_vm_mixture(o, w, mu, kappa, li);
        const int k = orc_vm_pick(w, raw(rng.uni()));
        moved = false;
        out->theta = cur->theta;
        for (int t = 0; t < ORC_VM_TRIES; ++t) {
            const std::uint32_t d1 = raw(rng.uni()), d2 = raw(rng.uni()), d3 = raw(rng.uni());
            double a;
            if (orc_vm_trial(kappa[k], d1, d2, d3, &a)) {
                out->theta = std::remainder(mu[k] + a, 2.0 * 3.14159265358979323846);
                moved = true;
                break;
            }
        }
    }
    double log_ratio(const U1Link* cur, const U1Link* prop) const
    {
        if (!moved) return 0.0;
        return orc_vm_mixture_logpdf(w, mu, kappa, li, cur->theta) -
               orc_vm_mixture_logpdf(w, mu, kappa, li, prop->theta);
    }
};

extern "C" int ref_u1_learned_metropolis(std::uint64_t n_links, const std::uint32_t* cells,
                                         std::uint64_t n_cells, const std::uint64_t* inc_off,
                                         const std::uint32_t* inc_cell, const std::uint8_t* inc_which,
                                         const double* params, double model_beta, double driver_beta,
                                         std::uint64_t seed, std::uint64_t sweep0, std::uint64_t n_sweeps,
                                         double* theta, double* obs_out)
{
    try {
        using CM = CellModel<U1Dof, U1PlaquetteTerm, CellComplex<4>>;
        std::vector<Cell<4>> cl(n_cells);
        for (std::uint64_t c = 0; c < n_cells; ++c)
            for (int k = 0; k < 4; ++k) cl[c].sites[k] = cells[4 * c + k];
        CM model(CellComplex<4>(n_links, cl), U1PlaquetteTerm{model_beta});
        for (std::size_t i = 0; i < n_links; ++i) {
            const U1Link l{theta[i]};
            model.update(i, &l);
        }
        KeyState ks;
        ks.seed = seed;
        ks.counter = sweep0;
        LearnedU1 prop{&ks, model.data(), cells, inc_off, inc_cell, inc_which, params, {}, {}, {}, {}};
        Metropolis<CM, LearnedU1, KeyedRng> mc(model, prop, KeyedRng{&ks}, driver_beta);
        std::uint64_t k = 0;
        mc.sample(n_sweeps, [&](const CM& m) {
            if (obs_out) {
                double sum = 0.0;
                for (std::size_t c = 0; c < m.cells(); ++c) {
                    const auto s = m.cell_sites(c);
                    const U1Link* ls[4] = {m.data() + s[0], m.data() + s[1], m.data() + s[2], m.data() + s[3]};
                    sum += m.term().cos_plaquette(ls);
                }
                obs_out[k] = sum / double(m.cells());
            }
            ++k;
            ++ks.counter;
        });
        for (std::size_t i = 0; i < n_links; ++i) theta[i] = model.data()[i].theta;
        return 0;
    } catch (...) {
        return status_of(std::current_exception());
    }
}
