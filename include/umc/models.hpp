// umc/models.hpp -- the reference's example models (example/ising.hpp,
// example/vector_spin.hpp, example/u1_gauge.hpp, example/sun_gauge.hpp) with
// their interface: value_type, size, sites(), data(), update(), energy_at(),
// energy_diff_at() and, for pair models, degree()/bonds()/energy_diff_bond().
//
// Each model holds its field on the host in the reference's data() layout
// (Ising int8, O(N) doubles, U1Link angles, SULink<N> complex matrices) and
// describes the device chain a driver builds for it.  After a driver ran,
// data() and update() first copy the device field back; a driver uploads the
// host field before it runs whenever the host copy is the newer one.
#pragma once

#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <utility>

#include "detail.hpp"
#include "dof.hpp"
#include "lattice.hpp"

namespace umc::gpu {

// Concepts of model.hpp:70-93 and driver.hpp:73-84.
template <class M>
concept ModelLike = requires(const M cm, M m, std::size_t loc, const typename M::value_type* proposal) {
    typename M::value_type;
    { M::size } -> std::convertible_to<std::size_t>;
    { cm.sites() } -> std::convertible_to<std::size_t>;
    { cm.data() } -> std::convertible_to<const typename M::value_type*>;
    { cm.energy_diff_at(loc, proposal) } -> std::convertible_to<double>;
    { m.update(loc, proposal) } -> std::same_as<void>;
};

template <class M>
concept EnergyModel = ModelLike<M> && requires(const M cm, std::size_t loc) {
    { cm.energy_at(loc) } -> std::convertible_to<double>;
};

template <class M>
concept WolffModel = ModelLike<M> && requires(const M cm, std::size_t loc, const typename M::value_type* proposal,
                                             const typename M::bond_type& bond) {
    typename M::bond_type;
    { cm.degree(loc) } -> std::convertible_to<std::size_t>;
    { cm.bonds(loc) } -> std::convertible_to<const typename M::bond_type*>;
    { cm.energy_diff_bond(loc, bond, proposal) } -> std::convertible_to<double>;
};

namespace detail {
inline umc_chain_desc base_desc(int32_t model, int32_t components)
{
    umc_chain_desc d{};
    d.model = model;
    d.components = components;
    d.hits = 1;
    d.device = 0;
    d.max_records = 4096;
    return d;
}
}  // namespace detail

// ---- Ising: E = -J sum_<ij> s_i s_j, cold start all +1 ------------------------
class Ising : public detail::Field<IsingSpin, std::int8_t>
{
public:
    using value_type = IsingSpin;
    using bond_type = Bond<>;
    using energy_type = double;
    static constexpr std::size_t size = 1;

    explicit Ising(PairGraph<> graph, std::int32_t J = 1) : graph_(std::move(graph)), J_(J)
    {
        host_.assign(graph_.sites(), IsingSpin(1));
    }

    std::size_t sites() const noexcept { return graph_.sites(); }
    const IsingSpin* data() const
    {
        ensure_host();
        return host_.data();
    }
    void update(std::size_t i, const IsingSpin* p)
    {
        ensure_host();
        host_[i] = *p;
        host_written();
    }
    std::size_t degree(std::size_t i) const noexcept { return graph_.degree(i); }
    const bond_type* bonds(std::size_t i) const noexcept { return graph_.bonds(i); }

    double energy_at(std::size_t i) const { return -double(J_) * double(data()[i]) * double(field_sum(i)); }
    double energy_diff_at(std::size_t i, const IsingSpin* p) const
    {
        return -double(J_) * double(int32_t(*p) - int32_t(data()[i])) * double(field_sum(i));
    }
    double energy_diff_bond(std::size_t i, const bond_type& b, const IsingSpin* p) const
    {
        return -double(J_) * double(data()[i]) * double(int32_t(*p) - int32_t(data()[b.j]));
    }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(UMC_MODEL_ISING, 1);
        d.graph = graph_.handle();
        d.coupling = double(J_);
        return d;
    }

private:
    int32_t field_sum(std::size_t i) const
    {
        const IsingSpin* s = data();
        int32_t h = 0;
        for (std::size_t a = 0; a < graph_.degree(i); ++a) h += s[graph_.bonds(i)[a].j];
        return h;
    }

    PairGraph<> graph_;
    std::int32_t J_;
};

// ---- VectorSpin<N>: E = -J sum_<ij> S_i . S_j, cold start along the last axis ----
template <std::size_t N>
class VectorSpin : public detail::Field<double, float>
{
public:
    using value_type = double;
    using bond_type = Bond<>;
    using energy_type = double;
    static constexpr std::size_t size = N;

    explicit VectorSpin(PairGraph<> graph, double J = 1.0) : graph_(std::move(graph)), J_(J)
    {
        host_.assign(graph_.sites() * N, 0.0);
        for (std::size_t i = 0; i < graph_.sites(); ++i) host_[i * N + N - 1] = 1.0;
    }

    std::size_t sites() const noexcept { return graph_.sites(); }
    const double* data() const
    {
        ensure_host();
        return host_.data();
    }
    void update(std::size_t i, const double* p)
    {
        ensure_host();
        for (std::size_t k = 0; k < N; ++k) host_[i * N + k] = p[k];
        host_written();
    }
    std::size_t degree(std::size_t i) const noexcept { return graph_.degree(i); }
    const bond_type* bonds(std::size_t i) const noexcept { return graph_.bonds(i); }

    double energy_at(std::size_t i) const
    {
        const double* s = data();
        double e = 0.0;
        for (std::size_t a = 0; a < graph_.degree(i); ++a) e += -J_ * dot(s + i * N, s + graph_.bonds(i)[a].j * N);
        return e;
    }
    double energy_diff_at(std::size_t i, const double* p) const
    {
        const double* s = data();
        double d = 0.0;
        for (std::size_t a = 0; a < graph_.degree(i); ++a) {
            const double* t = s + graph_.bonds(i)[a].j * N;
            d += -J_ * (dot(p, t) - dot(s + i * N, t));
        }
        return d;
    }
    double energy_diff_bond(std::size_t i, const bond_type& b, const double* p) const
    {
        const double* s = data();
        return -J_ * (dot(s + i * N, p) - dot(s + i * N, s + b.j * N));
    }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(UMC_MODEL_VECTOR, int32_t(N));
        d.graph = graph_.handle();
        d.coupling = J_;
        return d;
    }

private:
    static double dot(const double* a, const double* b) noexcept
    {
        double s = 0.0;
        for (std::size_t k = 0; k < N; ++k) s += a[k] * b[k];
        return s;
    }

    PairGraph<> graph_;
    double J_;
};

using XY = VectorSpin<2>;
using Heisenberg = VectorSpin<3>;

// ---- U1Gauge: S = beta sum_p (1 - cos theta_p) on a plaquette complex -------------
class U1Gauge : public detail::Field<double, float>
{
public:
    using value_type = U1Link;
    static constexpr std::size_t size = 1;

    // The reference's 4D lattice (hypercubic_plaquettes(L)), cold start.
    explicit U1Gauge(std::size_t L, double beta = 1.0) : U1Gauge(hypercubic_plaquettes(L), beta) { L_ = L; }
    // Any plaquette complex (e.g. square_plaquettes(L) in 2D).
    U1Gauge(CellComplex<4> cells, double beta) : cells_(std::move(cells)), beta_(beta)
    {
        host_.assign(cells_.sites(), 0.0);
    }

    std::size_t sites() const noexcept { return cells_.sites(); }
    std::size_t cells() const noexcept { return cells_.cells(); }
    std::size_t length() const noexcept { return L_; }
    const U1Link* data() const
    {
        ensure_host();
        return reinterpret_cast<const U1Link*>(host_.data());
    }
    void update(std::size_t i, const U1Link* p)
    {
        ensure_host();
        host_[i] = p->theta;
        host_written();
    }

    double energy_diff_at(std::size_t i, const U1Link* p) const
    {
        const double* t = (data(), host_.data());
        double d = 0.0;
        for (const auto inc : cells_.incident(i)) {
            const auto s = cells_.cell(inc.cell);
            double a[4] = {t[s[0]], t[s[1]], t[s[2]], t[s[3]]};
            const double before = plaquette(a[0], a[1], a[2], a[3]);
            a[inc.which] = p->theta;
            d += beta_ * (before - plaquette(a[0], a[1], a[2], a[3]));
        }
        return d;
    }
    double total_energy() const { return beta_ * double(cells_.cells()) * (1.0 - mean_plaquette()); }
    double mean_plaquette() const
    {
        const double* t = (data(), host_.data());
        double sum = 0.0;
        for (std::size_t c = 0; c < cells_.cells(); ++c) {
            const auto s = cells_.cell(c);
            sum += plaquette(t[s[0]], t[s[1]], t[s[2]], t[s[3]]);
        }
        return sum / double(cells_.cells());
    }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(UMC_MODEL_U1, 1);
        d.cells = cells_.handle();
        d.coupling = beta_;
        return d;
    }

private:
    CellComplex<4> cells_;
    double beta_;
    std::size_t L_ = 0;
};

// ---- SUGauge<N>: S = beta sum_p (1 - ReTr U_p / N), cold start identity ----------
template <std::size_t N>
class SUGauge : public detail::Field<double, float>
{
public:
    using value_type = SULink<N>;
    static constexpr std::size_t size = 1;
    static constexpr std::size_t kScalars = 2 * N * N;

    explicit SUGauge(std::size_t L, double beta = 1.0) : SUGauge(hypercubic_plaquettes(L), beta) { L_ = L; }
    SUGauge(CellComplex<4> cells, double beta) : cells_(std::move(cells)), beta_(beta)
    {
        host_.assign(cells_.sites() * kScalars, 0.0);
        for (std::size_t l = 0; l < cells_.sites(); ++l)
            for (std::size_t i = 0; i < N; ++i) host_[l * kScalars + 2 * (i * N + i)] = 1.0;
    }

    std::size_t sites() const noexcept { return cells_.sites(); }
    std::size_t cells() const noexcept { return cells_.cells(); }
    std::size_t length() const noexcept { return L_; }
    const SULink<N>* data() const
    {
        host_links();
        return reinterpret_cast<const SULink<N>*>(host_.data());
    }
    void update(std::size_t i, const SULink<N>* p)
    {
        host_links();
        const double* s = reinterpret_cast<const double*>(p->m.data());
        for (std::size_t k = 0; k < kScalars; ++k) host_[i * kScalars + k] = s[k];
        host_written();
    }

    double energy_diff_at(std::size_t i, const SULink<N>* p) const
    {
        const SULink<N>* u = data();
        double d = 0.0;
        for (const auto inc : cells_.incident(i)) {
            const auto s = cells_.cell(inc.cell);
            const SULink<N>* l[4] = {u + s[0], u + s[1], u + s[2], u + s[3]};
            const double before = plaq(l);
            l[inc.which] = p;
            d += beta_ * (before - plaq(l));
        }
        return d;
    }
    double mean_plaquette() const
    {
        const SULink<N>* u = data();
        double sum = 0.0;
        for (std::size_t c = 0; c < cells_.cells(); ++c) {
            const auto s = cells_.cell(c);
            const SULink<N>* l[4] = {u + s[0], u + s[1], u + s[2], u + s[3]};
            sum += plaq(l);
        }
        return sum / double(cells_.cells());
    }
    double total_energy() const { return beta_ * double(cells_.cells()) * (1.0 - mean_plaquette()); }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(UMC_MODEL_SU, int32_t(N));
        d.cells = cells_.handle();
        d.coupling = beta_;
        return d;
    }

private:
    // ReTr(U0 U1 U2^dag U3^dag) / N
    static double plaq(const SULink<N>* const l[4]) { return plaquette(*l[0], *l[1], *l[2], *l[3]); }

    // The host copy of the links.  The device holds them in FP32, unitary to
    // about 1e-7; after a read-back each link is replaced by its projection
    // onto SU(N) in FP64 (su_project_all), so that the host sees links as unitary
    // as the reference's FP64 chain keeps them.
    void host_links() const
    {
        ensure_host();
        if (!downloaded_) return;
        su_project_all(reinterpret_cast<SULink<N>*>(host_.data()), cells_.sites());
        downloaded_ = false;
    }

    CellComplex<4> cells_;
    double beta_;
    std::size_t L_ = 0;
};

// example/sun_gauge.hpp:85-86
using SU2Gauge = SUGauge<2>;
using SU3Gauge = SUGauge<3>;

}  // namespace umc::gpu
