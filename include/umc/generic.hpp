// umc/generic.hpp -- the reference's table-driven models with its built-in
// terms: PairModel<D, Term, G> (model/pair.hpp:17-83), CellModel<D, Term, List>
// (model/cell.hpp:16-99), the CellTerm concept (term/cell.hpp:10-25) and
// IsingTerm, HeisenbergTerm<N>, U1PlaquetteTerm, SUPlaquetteTerm<N>
// (term/ising.hpp, term/heisenberg.hpp, term/plaquette.hpp,
// term/sun_plaquette.hpp).
//
// The host-side members (energy, delta, energy_at, energy_diff_at,
// energy_diff_bond) follow the reference's arithmetic.  A driver runs these
// models on the device kernels of the matching example model: IsingTerm ->
// Ising, HeisenbergTerm<N> -> VectorSpin<N>, U1PlaquetteTerm -> U(1) links,
// SUPlaquetteTerm<N> -> SU(N) links.  Any other term is a user-written one:
// in a file compiled by nvcc, whose term members are __host__ __device__,
// the drivers run it through umc/device.cuh (the generic device Metropolis
// and Wolff); under g++ it is a compile-time error, since g++ cannot build
// device code and there is no CPU fallback.  As in the reference, every
// component starts at zero.
#pragma once

#include <array>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <span>
#include <type_traits>
#include <utility>
#include <vector>

#include "detail.hpp"
#include "dof.hpp"
#include "lattice.hpp"
#include "models.hpp"

namespace umc::gpu {

// term/cell.hpp:10-25
template <class Term, class D>
concept CellTerm = requires {
    typename D::dtype;
    typename Term::dtype;
    typename Term::energy_type;
    { Term::arity } -> std::convertible_to<std::size_t>;
    requires(Term::arity >= 1);
    requires std::same_as<typename Term::dtype, typename D::dtype>;
} && requires(const Term term, const typename D::dtype* const* links, const typename D::dtype* old,
              const typename D::dtype* nw) {
    { term.energy(links) } -> std::convertible_to<typename Term::energy_type>;
    { term.delta(std::size_t{}, old, nw, links) } -> std::convertible_to<typename Term::energy_type>;
};

// ---- built-in terms --------------------------------------------------------------
// E = -J s_i s_j (term/ising.hpp)
struct IsingTerm
{
    using dtype = IsingSpin;
    using energy_type = std::int32_t;
    static constexpr std::size_t arity = 2;
    energy_type J = 1;

    energy_type energy(const dtype* const* links) const noexcept
    {
        return -J * std::int32_t(*links[0]) * std::int32_t(*links[1]);
    }
    energy_type delta(std::size_t which, const dtype* old, const dtype* nw, const dtype* const* links) const noexcept
    {
        const dtype* fixed = links[which == 0 ? 1 : 0];
        return -J * (std::int32_t(*nw) * std::int32_t(*fixed) - std::int32_t(*old) * std::int32_t(*fixed));
    }
};

// E = -J S_i . S_j (term/heisenberg.hpp)
template <std::size_t N>
struct HeisenbergTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J = 1.0;

    static double dot(const double* a, const double* b) noexcept
    {
        double s = 0.0;
        for (std::size_t k = 0; k < N; ++k) s += a[k] * b[k];
        return s;
    }
    energy_type energy(const dtype* const* links) const noexcept { return -J * dot(links[0], links[1]); }
    energy_type delta(std::size_t which, const dtype* old, const dtype* nw, const dtype* const* links) const noexcept
    {
        const dtype* fixed = links[which == 0 ? 1 : 0];
        return -J * (dot(nw, fixed) - dot(old, fixed));
    }
};

// S_p = beta (1 - cos theta_p), theta_p = t0 + t1 - t2 - t3 (term/plaquette.hpp)
struct U1PlaquetteTerm
{
    using dtype = U1Link;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta = 1.0;

    static double cos_plaquette(const dtype* const* l) noexcept
    {
        return plaquette(l[0]->theta, l[1]->theta, l[2]->theta, l[3]->theta);
    }
    energy_type energy(const dtype* const* links) const noexcept { return beta * (1.0 - cos_plaquette(links)); }
    energy_type delta(std::size_t which, const dtype*, const dtype* nw, const dtype* const* links) const noexcept
    {
        std::array<const dtype*, arity> p{links[0], links[1], links[2], links[3]};
        const double before = cos_plaquette(p.data());
        p[which] = nw;
        return beta * (before - cos_plaquette(p.data()));
    }
};

// S_p = beta (1 - Re Tr(U0 U1 U2^dag U3^dag) / N) (term/sun_plaquette.hpp)
template <std::size_t N>
struct SUPlaquetteTerm
{
    using dtype = SULink<N>;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta = 1.0;

    static double real_plaquette(const dtype* const* l) { return plaquette(*l[0], *l[1], *l[2], *l[3]); }
    energy_type energy(const dtype* const* links) const { return beta * (1.0 - real_plaquette(links)); }
    energy_type delta(std::size_t which, const dtype*, const dtype* nw, const dtype* const* links) const
    {
        std::array<const dtype*, arity> p{links[0], links[1], links[2], links[3]};
        const double before = real_plaquette(p.data());
        p[which] = nw;
        return beta * (before - real_plaquette(p.data()));
    }
};

namespace detail {
// Which device model runs a (degree of freedom, term) pair, and the host
// scalars of one site in the reference's data() layout.
// No built-in device model: a user-written term.  Under nvcc it runs through
// umc/device.cuh with the field in the dtype itself; g++ builds refuse it.
template <class D, class Term>
struct DeviceTerm
{
    static constexpr bool ok = false;
    using HS = typename D::dtype;
    using DevT = typename D::dtype;
    static constexpr std::size_t scalars = D::size;
};

#if defined(__CUDACC__)
inline constexpr bool kUserTermsOnDevice = true;
#else
inline constexpr bool kUserTermsOnDevice = false;
#endif

// A PairModel or CellModel whose term has no built-in device model.
template <class M>
concept UserTermModel = requires { typename M::term_type; typename M::dof_type; } &&
                        !DeviceTerm<typename M::dof_type, typename M::term_type>::ok;
template <>
struct DeviceTerm<IsingDof, IsingTerm>
{
    static constexpr bool ok = true;
    using HS = IsingSpin;
    using DevT = std::int8_t;
    static constexpr std::size_t scalars = 1;
    static constexpr int32_t model = UMC_MODEL_ISING, comps = 1;
    static double coupling(const IsingTerm& t) { return double(t.J); }
};
template <std::size_t N>
struct DeviceTerm<VectorDof<N>, HeisenbergTerm<N>>
{
    static constexpr bool ok = true;
    using HS = double;
    using DevT = float;
    static constexpr std::size_t scalars = N;
    static constexpr int32_t model = UMC_MODEL_VECTOR, comps = int32_t(N);
    static double coupling(const HeisenbergTerm<N>& t) { return t.J; }
};
template <>
struct DeviceTerm<U1Dof, U1PlaquetteTerm>
{
    static constexpr bool ok = true;
    using HS = double;
    using DevT = float;
    static constexpr std::size_t scalars = 1;
    static constexpr int32_t model = UMC_MODEL_U1, comps = 1;
    static double coupling(const U1PlaquetteTerm& t) { return t.beta; }
};
template <std::size_t N>
struct DeviceTerm<SUDof<N>, SUPlaquetteTerm<N>>
{
    static constexpr bool ok = true;
    using HS = double;
    using DevT = float;
    static constexpr std::size_t scalars = 2 * N * N;
    static constexpr int32_t model = UMC_MODEL_SU, comps = int32_t(N);
    static double coupling(const SUPlaquetteTerm<N>& t) { return t.beta; }
};

template <class D, class Term>
using TermField = Field<typename DeviceTerm<D, Term>::HS, typename DeviceTerm<D, Term>::DevT>;
}  // namespace detail

// ---- PairModel (model/pair.hpp:17-83) ---------------------------------------------
template <class D, class Term, class G>
    requires Dof<D> && CellTerm<Term, D> && PairGraphLike<G> && (Term::arity == 2)
class PairModel : public detail::TermField<D, Term>
{
    using DT = detail::DeviceTerm<D, Term>;
    static_assert(DT::ok || detail::kUserTermsOnDevice,
                  "a user-written pair term runs on the device when this file is compiled by nvcc "
                  "(umc/device.cuh); g++ builds run IsingTerm and HeisenbergTerm<N>");
    static_assert(std::is_same_v<G, PairGraph<>>, "the device engine takes the unweighted PairGraph<>");

public:
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    static constexpr std::size_t size = D::size;
    using bond_type = typename G::bond_type;
    using dof_type = D;
    using term_type = Term;

    PairModel(G graph, Term term) : graph_(std::move(graph)), term_(std::move(term))
    {
        this->host_.assign(graph_.sites() * DT::scalars, typename DT::HS{});
    }

    std::size_t sites() const noexcept { return graph_.sites(); }
    const dtype* data() const
    {
        this->ensure_host();
        return reinterpret_cast<const dtype*>(this->host_.data());
    }
    std::size_t degree(std::size_t i) const noexcept { return graph_.degree(i); }
    const bond_type* bonds(std::size_t i) const noexcept { return graph_.bonds(i); }
    const Term& term() const noexcept { return term_; }
    const G& graph() const noexcept { return graph_; }

    energy_type energy_at(std::size_t i) const
    {
        const dtype* f = data();
        energy_type e = 0;
        for (std::size_t a = 0; a < graph_.degree(i); ++a) {
            const std::array<const dtype*, 2> l{f + i * size, f + graph_.bonds(i)[a].j * size};
            e += term_.energy(l.data());
        }
        return e;
    }
    energy_type energy_diff_at(std::size_t i, const dtype* p) const
    {
        const dtype* f = data();
        energy_type d = 0;
        for (std::size_t a = 0; a < graph_.degree(i); ++a) {
            const std::array<const dtype*, 2> l{f + i * size, f + graph_.bonds(i)[a].j * size};
            d += term_.delta(0, f + i * size, p, l.data());
        }
        return d;
    }
    energy_type energy_diff_bond(std::size_t i, const bond_type& b, const dtype* p) const
    {
        const dtype* f = data();
        const std::array<const dtype*, 2> l{f + b.j * size, f + i * size};
        return term_.delta(0, f + b.j * size, p, l.data());
    }
    void update(std::size_t i, const dtype* p)
    {
        this->ensure_host();
        const auto* s = reinterpret_cast<const typename DT::HS*>(p);
        for (std::size_t k = 0; k < DT::scalars; ++k) this->host_[i * DT::scalars + k] = s[k];
        this->host_written();
    }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(DT::model, DT::comps);
        d.graph = graph_.handle();
        d.coupling = DT::coupling(term_);
        return d;
    }

private:
    G graph_;
    Term term_;
};

// ---- CellModel (model/cell.hpp:16-99) ---------------------------------------------
template <class D, class Term, class List>
    requires Dof<D> && CellTerm<Term, D> && CellComplexLike<List> && (Term::arity == List::arity)
class CellModel : public detail::TermField<D, Term>
{
    using DT = detail::DeviceTerm<D, Term>;
    static_assert(DT::ok || detail::kUserTermsOnDevice,
                  "a user-written cell term runs on the device when this file is compiled by nvcc "
                  "(umc/device.cuh); g++ builds run U1PlaquetteTerm and SUPlaquetteTerm<N>");
    static_assert(std::is_same_v<List, CellComplex<List::arity>>, "the device engine takes CellComplex<A> lists");
    static_assert(!DT::ok || List::arity == 4, "the built-in cell terms are plaquettes of CellComplex<4>");

public:
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    static constexpr std::size_t size = D::size;
    static constexpr std::size_t arity = List::arity;
    using dof_type = D;
    using term_type = Term;

    CellModel(List list, Term term) : list_(std::move(list)), term_(std::move(term))
    {
        this->host_.assign(list_.sites() * DT::scalars, typename DT::HS{});
    }

    std::size_t sites() const noexcept { return list_.sites(); }
    std::size_t cells() const noexcept { return list_.cells(); }
    const dtype* data() const
    {
        host_view();
        return reinterpret_cast<const dtype*>(this->host_.data());
    }
    const Term& term() const noexcept { return term_; }
    const List& list() const noexcept { return list_; }
    std::span<const std::uint32_t, arity> cell_sites(std::size_t c) const { return list_.cell(c); }

    energy_type cell_energy(std::size_t c) const
    {
        const auto l = links(c);
        return term_.energy(l.data());
    }
    energy_type total_energy() const
    {
        energy_type e = 0;
        for (std::size_t c = 0; c < cells(); ++c) e += cell_energy(c);
        return e;
    }
    energy_type energy_diff_at(std::size_t i, const dtype* p) const
    {
        const dtype* f = data();
        energy_type d = 0;
        for (const auto inc : list_.incident(i)) {
            const auto s = list_.cell(inc.cell);
            std::array<const dtype*, arity> l{};
            for (std::size_t k = 0; k < arity; ++k) l[k] = f + s[k] * size;
            d += term_.delta(inc.which, f + i * size, p, l.data());
        }
        return d;
    }
    void update(std::size_t i, const dtype* p)
    {
        host_view();
        const auto* s = reinterpret_cast<const typename DT::HS*>(p);
        for (std::size_t k = 0; k < DT::scalars; ++k) this->host_[i * DT::scalars + k] = s[k];
        this->host_written();
    }

    umc_chain_desc chain_desc() const
    {
        auto d = detail::base_desc(DT::model, DT::comps);
        d.cells = list_.handle();
        d.coupling = DT::coupling(term_);
        return d;
    }

private:
    std::array<const dtype*, arity> links(std::size_t c) const
    {
        const dtype* f = data();
        const auto s = list_.cell(c);
        std::array<const dtype*, arity> l{};
        for (std::size_t k = 0; k < arity; ++k) l[k] = f + s[k] * size;
        return l;
    }
    // The host copy.  The built-in SU(N) term keeps its links in FP32 on the
    // device; after a read-back the host copy holds their FP64 projections
    // onto SU(N) (su_project_all), as SUGauge's does.
    void host_view() const
    {
        this->ensure_host();
        if constexpr (DT::ok) {
            if constexpr (DT::model == UMC_MODEL_SU) {
                if (!this->downloaded_) return;
                su_project_all(reinterpret_cast<dtype*>(this->host_.data()), list_.sites());
                this->downloaded_ = false;
            }
        }
    }

    List list_;
    Term term_;
};

}  // namespace umc::gpu
