// umc/lattice.hpp -- PairGraph / CellComplex with the reference's interface
// (lattice/pair_graph.hpp:13-116, lattice/cell_complex.hpp:13-97) over the
// engine's device tables (umc_graph_*, umc_cells_*).  The host keeps a copy of
// the CSR / incidence for degree(), bonds(), cell() and incident(); copies of a
// graph share one device table.
#pragma once

#include <array>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <span>
#include <stdexcept>
#include <type_traits>
#include <vector>

#include "detail.hpp"

namespace umc::gpu {

struct NoPayload
{};

template <class P = NoPayload>
struct Bond
{
    std::uint32_t j;
    [[no_unique_address]] P c;
};

// P is the per-bond payload (lattice/pair_graph.hpp:13-22): NoPayload, or a
// trivially copyable record of at most UMC_MAX_PAYLOAD_BYTES bytes (a coupling,
// a vector of couplings, ...) that the engine keeps beside the CSR and hands
// to device code (umc/device.cuh BondTables<P>).
template <class P = NoPayload>
class PairGraph
{
    static_assert(std::is_same_v<P, NoPayload> ||
                      (std::is_trivially_copyable_v<P> && sizeof(P) <= UMC_MAX_PAYLOAD_BYTES),
                  "a bond payload must be trivially copyable and at most UMC_MAX_PAYLOAD_BYTES bytes");

public:
    using bond_type = Bond<P>;

    struct Edge
    {
        std::uint32_t i;
        std::uint32_t j;
        P c{};
    };

    PairGraph() = default;

    // Same rules and exceptions as the reference constructor; c is copied into
    // both directed entries when symmetric.
    PairGraph(std::size_t n, std::span<const Edge> edges, bool symmetric = true)
    {
        std::vector<std::uint32_t> ei(edges.size()), ej(edges.size());
        for (std::size_t k = 0; k < edges.size(); ++k) {
            ei[k] = edges[k].i;
            ej[k] = edges[k].j;
        }
        umc_graph* g = nullptr;
        if constexpr (std::is_same_v<P, NoPayload>) {
            detail::check(umc_graph_create(n, ei.data(), ej.data(), edges.size(), symmetric ? 1 : 0, &g));
        } else {
            std::vector<unsigned char> blob(edges.size() * sizeof(P));
            for (std::size_t k = 0; k < edges.size(); ++k) std::memcpy(blob.data() + k * sizeof(P), &edges[k].c, sizeof(P));
            detail::check(umc_graph_create_payload(n, ei.data(), ej.data(), edges.size(), symmetric ? 1 : 0,
                                                   blob.data(), std::uint32_t(sizeof(P)), &g));
        }
        adopt(g);
    }

    // Wraps a table the engine built (square_lattice, cubic_lattice).
    static PairGraph from_handle(umc_graph* g)
    {
        PairGraph p;
        p.adopt(g);
        return p;
    }

    std::size_t sites() const noexcept { return offset_.empty() ? 0 : offset_.size() - 1; }
    std::size_t degree(std::size_t i) const noexcept { return std::size_t(offset_[i + 1] - offset_[i]); }
    const bond_type* bonds(std::size_t i) const noexcept
    {
        return bonds_.empty() ? nullptr : bonds_.data() + offset_[i];
    }
    const umc_graph* handle() const noexcept { return g_.get(); }

private:
    void adopt(umc_graph* g)
    {
        g_ = std::shared_ptr<umc_graph>(g, detail::GraphFree{});
        const std::size_t n = umc_graph_sites(g), m = umc_graph_slots(g);
        offset_.resize(n + 1);
        std::vector<std::uint32_t> b(m);
        detail::check(umc_graph_csr(g, offset_.data(), b.data()));
        bonds_.resize(m);
        for (std::size_t k = 0; k < m; ++k) bonds_[k] = bond_type{b[k], {}};
        if constexpr (!std::is_same_v<P, NoPayload>) {
            if (umc_graph_payload_bytes(g) != sizeof(P)) throw std::invalid_argument("PairGraph: payload size differs");
            std::vector<unsigned char> blob(m * sizeof(P));
            if (m) detail::check(umc_graph_payloads(g, blob.data()));
            for (std::size_t k = 0; k < m; ++k) std::memcpy(&bonds_[k].c, blob.data() + k * sizeof(P), sizeof(P));
        }
    }

    std::shared_ptr<umc_graph> g_;
    std::vector<std::uint32_t> offset_;
    std::vector<bond_type> bonds_;
};

template <class G>
concept PairGraphLike = requires(const G g, std::size_t i) {
    typename G::bond_type;
    { g.sites() } -> std::convertible_to<std::size_t>;
    { g.degree(i) } -> std::convertible_to<std::size_t>;
    { g.bonds(i) } -> std::convertible_to<const typename G::bond_type*>;
};

// square_lattice(Lx, Ly), lattice/square.hpp:15-38.
inline PairGraph<> square_lattice(std::size_t Lx, std::size_t Ly)
{
    umc_graph* g = nullptr;
    detail::check(umc_graph_square(Lx, Ly, &g));
    return PairGraph<>::from_handle(g);
}

// Periodic cubic lattice with square_lattice's conventions (no reference builder).
inline PairGraph<> cubic_lattice(std::size_t Lx, std::size_t Ly, std::size_t Lz)
{
    umc_graph* g = nullptr;
    detail::check(umc_graph_cubic(Lx, Ly, Lz, &g));
    return PairGraph<>::from_handle(g);
}

template <std::size_t A>
struct Cell
{
    std::array<std::uint32_t, A> sites;
};

template <std::size_t A>
class CellComplex
{
    static_assert(A >= 1 && A <= 255, "CellComplex arity must fit uint8_t");

public:
    struct Incident
    {
        std::uint32_t cell;
        std::uint8_t which;
    };
    static constexpr std::size_t arity = A;

    explicit CellComplex(std::size_t sites, std::span<const Cell<A>> cells)
    {
        std::vector<std::uint32_t> flat(cells.size() * A);
        for (std::size_t c = 0; c < cells.size(); ++c)
            for (std::size_t k = 0; k < A; ++k) flat[c * A + k] = cells[c].sites[k];
        umc_cells* h = nullptr;
        detail::check(umc_cells_create(sites, std::uint32_t(A), flat.data(), cells.size(), &h));
        adopt(h);
    }

    static CellComplex from_handle(umc_cells* h)
    {
        CellComplex c;
        c.adopt(h);
        return c;
    }

    std::size_t sites() const noexcept { return sites_; }
    std::size_t cells() const noexcept { return cells_.size(); }
    std::span<const std::uint32_t, A> cell(std::size_t c) const
    {
        if (c >= cells_.size()) throw std::out_of_range("CellComplex: cell out of range");
        return cells_[c].sites;
    }
    std::span<const Incident> incident(std::size_t i) const
    {
        if (i >= sites_) throw std::out_of_range("CellComplex: site out of range");
        return {incident_.data() + offset_[i], std::size_t(offset_[i + 1] - offset_[i])};
    }
    const umc_cells* handle() const noexcept { return h_.get(); }

private:
    CellComplex() = default;

    void adopt(umc_cells* h)
    {
        h_ = std::shared_ptr<umc_cells>(h, detail::CellsFree{});
        sites_ = umc_cells_sites(h);
        const std::size_t nc = umc_cells_count(h);
        std::vector<std::uint32_t> flat(nc * A);
        detail::check(umc_cells_table(h, flat.data()));
        cells_.resize(nc);
        for (std::size_t c = 0; c < nc; ++c)
            for (std::size_t k = 0; k < A; ++k) cells_[c].sites[k] = flat[c * A + k];
        offset_.resize(sites_ + 1);
        std::vector<std::uint32_t> ic(nc * A);
        std::vector<std::uint8_t> iw(nc * A);
        detail::check(umc_cells_incidence(h, offset_.data(), ic.data(), iw.data()));
        incident_.resize(nc * A);
        for (std::size_t k = 0; k < incident_.size(); ++k) incident_[k] = Incident{ic[k], iw[k]};
    }

    std::shared_ptr<umc_cells> h_;
    std::size_t sites_ = 0;
    std::vector<Cell<A>> cells_;
    std::vector<std::uint64_t> offset_;
    std::vector<Incident> incident_;
};

template <class L>
concept CellComplexLike = requires(const L list, std::size_t i, std::size_t c) {
    { L::arity } -> std::convertible_to<std::size_t>;
    { list.sites() } -> std::convertible_to<std::size_t>;
    { list.cells() } -> std::convertible_to<std::size_t>;
    list.cell(c);
    list.incident(i);
};

// hypercubic_plaquettes(L), lattice/hypercubic.hpp:15-64.
inline CellComplex<4> hypercubic_plaquettes(std::size_t L)
{
    umc_cells* h = nullptr;
    detail::check(umc_cells_hypercubic(L, &h));
    return CellComplex<4>::from_handle(h);
}

// 2D periodic plaquettes with the same orientation rule (links mu L^2 + y L + x).
inline CellComplex<4> square_plaquettes(std::size_t L)
{
    umc_cells* h = nullptr;
    detail::check(umc_cells_square_plaquettes(L, &h));
    return CellComplex<4>::from_handle(h);
}

}  // namespace umc::gpu
