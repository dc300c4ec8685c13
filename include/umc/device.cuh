// umc/device.cuh -- user-written models on the GPU.
//
// The reference's ModelLike concept (model.hpp:65-88) keeps a model a plain
// struct "so the same definition can be copied to a device and driven by a
// kernel".  This header is that kernel: a translation unit compiled by nvcc
// includes it, writes its terms, proposals or whole models with __host__
// __device__ members (UMC_HD), and drives them with device::Metropolis, the
// single-site driver of driver.hpp:17-66 run over colour classes, and with
// device::Wolff (driver.hpp:85-210) when they are WolffModels.  Tables
// (PairGraph CSR, CellComplex cells and incidence, colourings) come from
// libumc_b200.so; the update loop is instantiated for the user's types here.
//
//   * PairModel<D, Term>   -- model/pair.hpp:18-80 over a CSR bond table, for any
//                             arity-2 CellTerm (term/cell.hpp:10-25);
//   * CellModel<D, Term>   -- model/cell.hpp:16-99 over a cell table;
//   * any other M          -- a user struct with value_type, size, sites(),
//                             data(), energy_diff_at(loc, p) and update(loc, p)
//                             (model.hpp:65-88), e.g. neighbours computed from
//                             the site index instead of read from a table;
//   * proposals            -- sample(cur, rng, out) and log_ratio(cur, out)
//                             (dof/proposal.hpp:5-11); rng.uni() is Pcg32::uni
//                             (rng.hpp:22-26).
//
// Update order and random numbers.  The reference sweeps sites 0..n-1 from one
// sequential Pcg32.  Here a sweep visits the colour classes in order (no two
// sites of a class interact, so a class updates in parallel) and site i draws
// from its own counter-keyed stream Pcg32(id_seed(key_seed(seed, sweep,
// tag_site(0)), k), 0), k = i's colour-major index.  The result equals the
// reference driver run on the graph relabelled to colour-major order with
// that keying, which is how the library's own chains are checked.
//
// Layout.  PairTables and CellTables number sites colour-major on the device
// (a class is a contiguous range; table rows and field entries of a class are
// read with unit stride) and move fields to and from the host in the
// reference's site order, permuting on the device.  A model that numbers its
// own sites (any other M) keeps its numbering; its classes list the sites.
//
// One launch runs any number of sweeps: a cooperative persistent kernel whose
// blocks meet at a grid barrier between classes.  The barrier's waits are
// bounded; a wait that runs out sets a status bit, every block returns, and
// the host call throws.
#pragma once

#include <cuda_runtime.h>
#include <umc_b200.h>
#include <umc/keyed_pcg.cuh>

#include <algorithm>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace umc::gpu::device {

// ------------------------------------------------------------------ errors

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

inline void umc_check(int status)
{
    if (status != UMC_OK) throw std::runtime_error("umc status " + std::to_string(status) + ": " + umc_last_error());
}

// ------------------------------------------------------------------ buffers

// Device array of n T, freed on destruction; moved, never copied.
template <class T>
class Buffer
{
public:
    Buffer() = default;
    explicit Buffer(std::size_t n) : n_(n)
    {
        if (n) cuda_check(cudaMalloc(&p_, n * sizeof(T)), "cudaMalloc");
    }
    explicit Buffer(const std::vector<T>& host) : Buffer(host.size()) { upload(host.data()); }
    ~Buffer()
    {
        if (p_) cudaFree(p_);
    }
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    Buffer(Buffer&& o) noexcept : p_(std::exchange(o.p_, nullptr)), n_(std::exchange(o.n_, 0)) {}
    Buffer& operator=(Buffer&& o) noexcept
    {
        if (this != &o) {
            if (p_) cudaFree(p_);
            p_ = std::exchange(o.p_, nullptr);
            n_ = std::exchange(o.n_, 0);
        }
        return *this;
    }

    T* data() noexcept { return p_; }
    const T* data() const noexcept { return p_; }
    std::size_t size() const noexcept { return n_; }

    void upload(const T* host) { cuda_check(cudaMemcpy(p_, host, n_ * sizeof(T), cudaMemcpyHostToDevice), "upload"); }
    void download(T* host) const
    {
        cuda_check(cudaMemcpy(host, p_, n_ * sizeof(T), cudaMemcpyDeviceToHost), "download");
    }
    // Ordered on stream s; host must stay valid (pinned for overlap) until then.
    void upload_async(const T* host, cudaStream_t s)
    {
        cuda_check(cudaMemcpyAsync(p_, host, n_ * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
    }
    void download_async(T* host, cudaStream_t s) const
    {
        cuda_check(cudaMemcpyAsync(host, p_, n_ * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
    }
    std::vector<T> to_host() const
    {
        std::vector<T> h(n_);
        download(h.data());
        return h;
    }

private:
    T* p_ = nullptr;
    std::size_t n_ = 0;
};

// Field<T, N> of model.hpp:9-41: the owning buffer of one lattice, N values,
// allocated once, moved but never copied; here in device memory.
template <class T, std::size_t N>
class Field : public Buffer<T>
{
public:
    Field() : Buffer<T>(N) {}
};

// Model<T, Sites, Dof> of model.hpp:47-61: sites(), data() and the write-back
// update() of a model whose state is one field of Sites sites with Dof values
// each, so that a model only writes its energy terms.  The reference's Model
// owns its Field; a model driven by a kernel must be trivially copyable, so
// this one points at a Field<T, Sites * Dof> (or any device array of that
// many T) that the caller owns and passes at construction.
template <class T, std::size_t Sites, std::size_t Dof>
class Model
{
public:
    Model() = default;
    explicit Model(T* field) : field_(field) {}
    template <std::size_t N>
        requires(N == Sites * Dof)
    explicit Model(Field<T, N>& f) : field_(f.data())
    {
    }

    UMC_HD std::size_t sites() const noexcept { return Sites; }
    UMC_HD const T* data() const noexcept { return field_; }
    UMC_HD T* data() noexcept { return field_; }

    // Writes proposal into loc, leaving every other site untouched.
    UMC_HD void update(std::size_t loc, const T* proposal)
    {
        for (std::size_t c = 0; c < Dof; ++c) field_[loc * Dof + c] = proposal[c];
    }

private:
    T* field_ = nullptr;
};

// ------------------------------------------------------------------ random numbers

// The proposal's rng argument: one counter-keyed reference Pcg32.
class Rng
{
public:
    UMC_HD explicit Rng(KeyedPcg g) : g_(g) {}
    // Pcg32::uni, rng.hpp:22-26: k * 2^-32, in [0, 1).
    UMC_HD double uni() { return double(g_.next()) * 0x1.0p-32; }

private:
    KeyedPcg g_;
};

// ------------------------------------------------------------------ concepts

// dof/dof.hpp:8-12
template <class D>
concept Dof = requires {
    typename D::dtype;
    { D::size } -> std::convertible_to<std::size_t>;
};

// term/cell.hpp:10-25; the members must be callable on the device.
template <class Term, class D>
concept CellTerm = Dof<D> && requires {
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

// model.hpp:65-88.  A model crosses to the device by value: it holds device
// pointers, never owning containers.
template <class M>
concept ModelLike = std::is_trivially_copyable_v<M> &&
                    requires(const M cm, M m, std::size_t loc, const typename M::value_type* p) {
                        typename M::value_type;
                        { M::size } -> std::convertible_to<std::size_t>;
                        { cm.sites() } -> std::convertible_to<std::size_t>;
                        { cm.data() } -> std::convertible_to<const typename M::value_type*>;
                        { cm.energy_diff_at(loc, p) } -> std::convertible_to<double>;
                        { m.update(loc, p) } -> std::same_as<void>;
                    };

// dof/proposal.hpp:5-11 with this header's Rng.
template <class Q, class T>
concept Proposal = std::is_trivially_copyable_v<Q> && requires(const Q& q, const T* cur, T* out, Rng& rng) {
    { q.sample(cur, rng, out) };
    { q.log_ratio(cur, out) } -> std::convertible_to<double>;
};

// Wolff's axis argument (driver.hpp:108-109): only sample(cur, rng, out) is
// used, with cur == nullptr; FixedAxis (dof/ising.hpp:41-49) has nothing else.
template <class A, class T>
concept Axis = std::is_trivially_copyable_v<A> && requires(const A& a, const T* cur, T* out, Rng& rng) {
    { a.sample(cur, rng, out) };
};

// model.hpp:93-96
template <class M>
concept EnergyModel = ModelLike<M> && requires(const M cm, std::size_t loc) {
    { cm.energy_at(loc) } -> std::convertible_to<double>;
};

// model/cell.hpp:52-62: per-cell energies that sum to the total.
template <class M>
concept CellEnergyModel = ModelLike<M> && requires(const M cm, std::size_t c) {
    { cm.cells() } -> std::convertible_to<std::size_t>;
    { cm.cell_energy(c) } -> std::convertible_to<double>;
};

// driver.hpp:69-83, plus bond_id(i, a): the key of the a-th bond of i's row.
// The device tests each bond once, from its lower endpoint, with a draw keyed
// by that id, so the ids of the bonds i tests (those with j > i) must be
// distinct.  bond_type has a member j, the neighbour.
//
// A model without bond storage (a lattice that computes its neighbours) gives
// bond(i, a) by value instead of the row pointer bonds(i).
template <class M>
concept WolffModel =
    ModelLike<M> &&
    requires(const M cm, std::size_t loc, const typename M::value_type* p, const typename M::bond_type& b,
             std::size_t a) {
        typename M::bond_type;
        { cm.degree(loc) } -> std::convertible_to<std::size_t>;
        { cm.energy_diff_bond(loc, b, p) } -> std::convertible_to<double>;
        { cm.bond_id(loc, a) } -> std::convertible_to<std::uint32_t>;
        { b.j } -> std::convertible_to<std::size_t>;
    } &&
    (requires(const M cm, std::size_t loc) { { cm.bonds(loc) } -> std::convertible_to<const typename M::bond_type*>; } ||
     requires(const M cm, std::size_t loc, std::size_t a) {
         { cm.bond(loc, a) } -> std::convertible_to<typename M::bond_type>;
     });

// ------------------------------------------------------------------ colour classes

// Sites grouped by colour: order[begin[c] .. begin[c+1]) are the sites of
// colour c.  The index k of a site in order is its colour-major position, the
// id of its random stream.  An empty order is the identity: the model numbers
// its sites colour-major already (the table models below do).
struct Classes
{
    std::vector<std::uint32_t> order;
    std::vector<std::uint32_t> begin;

    std::uint32_t count() const { return std::uint32_t(begin.size() - 1); }
    std::uint64_t sites() const { return begin.back(); }
    std::uint32_t largest() const
    {
        std::uint32_t m = 0;
        for (std::uint32_t c = 0; c + 1 < begin.size(); ++c) m = std::max(m, begin[c + 1] - begin[c]);
        return m;
    }

    // From colour[i] in [0, n_colours): within a colour, ascending site index.
    static Classes from_colours(const std::vector<std::uint32_t>& colour, std::uint32_t n_colours)
    {
        Classes k;
        k.begin.assign(std::size_t(n_colours) + 1, 0);
        for (const auto c : colour) {
            if (c >= n_colours) throw std::invalid_argument("colour out of range");
            ++k.begin[c + 1];
        }
        for (std::uint32_t c = 0; c < n_colours; ++c) k.begin[c + 1] += k.begin[c];
        std::vector<std::uint32_t> next(k.begin.begin(), k.begin.end() - 1);
        k.order.resize(colour.size());
        for (std::uint32_t i = 0; i < colour.size(); ++i) k.order[next[colour[i]]++] = i;
        return k;
    }
    // Contiguous classes [begin[c], begin[c+1]) of a colour-major numbering.
    static Classes identity(std::vector<std::uint32_t> begin)
    {
        Classes k;
        k.begin = std::move(begin);
        return k;
    }
};

// Classes on the device.  Must outlive the drivers that use it.
class ClassTable
{
public:
    explicit ClassTable(Classes k) : host_(std::move(k))
    {
        const auto& b = host_.begin;
        if (b.size() < 2 || b.front() != 0 || !std::is_sorted(b.begin(), b.end()))
            throw std::invalid_argument("class table: begin must rise from 0");
        if (!host_.order.empty() && host_.order.size() != b.back())
            throw std::invalid_argument("class table: begin does not cover order");
        begin_ = Buffer<std::uint32_t>(b);
        if (!host_.order.empty()) order_ = Buffer<std::uint32_t>(host_.order);
    }
    const Classes& host() const noexcept { return host_; }
    // nullptr for the identity order
    const std::uint32_t* order() const noexcept { return host_.order.empty() ? nullptr : order_.data(); }
    const std::uint32_t* begin() const noexcept { return begin_.data(); }

private:
    Classes host_;
    Buffer<std::uint32_t> order_, begin_;
};

// ------------------------------------------------------------------ colour-major numbering

namespace detail {

constexpr int kThreads = 256;

// dst[k] = src[order[k]] (device numbering from site order), per_site scalars
// per site; scatter_sites is the inverse.
template <class T>
__global__ void __launch_bounds__(kThreads) gather_sites(T* __restrict__ dst, const T* __restrict__ src,
                                                         const std::uint32_t* __restrict__ order, std::uint64_t n,
                                                         std::uint32_t per_site)
{
    for (std::uint64_t x = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; x < n * per_site;
         x += std::uint64_t(gridDim.x) * blockDim.x)
        dst[x] = src[std::uint64_t(order[x / per_site]) * per_site + x % per_site];
}

template <class T>
__global__ void __launch_bounds__(kThreads) scatter_sites(T* __restrict__ dst, const T* __restrict__ src,
                                                          const std::uint32_t* __restrict__ order, std::uint64_t n,
                                                          std::uint32_t per_site)
{
    for (std::uint64_t x = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; x < n * per_site;
         x += std::uint64_t(gridDim.x) * blockDim.x)
        dst[std::uint64_t(order[x / per_site]) * per_site + x % per_site] = src[x];
}

inline unsigned permute_grid(std::uint64_t count)
{
    return unsigned(std::max<std::uint64_t>(1, std::min<std::uint64_t>(148 * 16, (count + kThreads - 1) / kThreads)));
}

// The library's colouring of a table: colour and colour-major position of
// every site (umc_graph_colouring / umc_cells_colouring).
struct Colouring
{
    std::vector<std::uint32_t> colour, position;
    std::uint32_t count = 0;

    std::vector<std::uint32_t> order() const
    {
        std::vector<std::uint32_t> o(position.size());
        for (std::uint32_t i = 0; i < position.size(); ++i) o[position[i]] = i;
        return o;
    }
    std::vector<std::uint32_t> begin() const
    {
        std::vector<std::uint32_t> b(std::size_t(count) + 1, 0);
        for (const auto c : colour) ++b[c + 1];
        for (std::uint32_t c = 0; c < count; ++c) b[c + 1] += b[c];
        return b;
    }
};

inline Colouring colouring_of(const umc_graph* g)
{
    Colouring c;
    c.colour.resize(umc_graph_sites(g));
    c.position.resize(c.colour.size());
    umc_check(umc_graph_colouring(g, &c.count, c.colour.data(), c.position.data()));
    return c;
}

inline Colouring colouring_of(const umc_cells* cc)
{
    Colouring c;
    c.colour.resize(umc_cells_sites(cc));
    c.position.resize(c.colour.size());
    umc_check(umc_cells_colouring(cc, &c.count, c.colour.data(), c.position.data()));
    return c;
}

}  // namespace detail

// The device numbering of the table models.  Site i of the library's table
// is device site position[i] (colour-major), so a colour class is one
// contiguous range and its sites, their table rows and their field entries
// are read with unit stride.  Fields cross to and from the host in the
// reference's site order (data() of model/pair.hpp and model/cell.hpp) and
// are permuted on the device.
class ColourMajor
{
public:
    explicit ColourMajor(const detail::Colouring& c)
        : position_(c.position), order_(c.order()), begin_(c.begin()), order_dev_(order_), position_dev_(position_)
    {}

    std::uint32_t sites() const noexcept { return std::uint32_t(position_.size()); }
    const std::vector<std::uint32_t>& position() const noexcept { return position_; }
    const std::vector<std::uint32_t>& order() const noexcept { return order_; }
    const std::vector<std::uint32_t>& class_begin() const noexcept { return begin_; }
    // On the device: the reference site of each device site, and the device
    // site of each reference site (Wolff's site-order tiles use both).
    const std::uint32_t* device_order() const noexcept { return order_dev_.data(); }
    const std::uint32_t* device_position() const noexcept { return position_dev_.data(); }

    // field (sites * per_site, device numbering) <- host (site order).  Ordered
    // on stream s; a pinned host buffer must stay valid until s passes the copy.
    // Transfers through one object share a staging buffer: issue them on one
    // stream.
    template <class T>
    void upload(Buffer<T>& field, const T* host, std::size_t per_site, cudaStream_t s = nullptr) const
    {
        const std::uint64_t count = std::uint64_t(sites()) * per_site;
        if (field.size() != count) throw std::invalid_argument("upload: field size differs from sites * per_site");
        T* stage = staging<T>(count);
        cuda_check(cudaMemcpyAsync(stage, host, count * sizeof(T), cudaMemcpyHostToDevice, s), "upload");
        detail::gather_sites<T><<<detail::permute_grid(count), detail::kThreads, 0, s>>>(
            field.data(), stage, order_dev_.data(), sites(), std::uint32_t(per_site));
        cuda_check(cudaGetLastError(), "upload permute");
    }
    // host (site order) <- field; returns when the host copy is complete.
    template <class T>
    void download(const Buffer<T>& field, T* host, std::size_t per_site, cudaStream_t s = nullptr) const
    {
        const std::uint64_t count = std::uint64_t(sites()) * per_site;
        if (field.size() != count) throw std::invalid_argument("download: field size differs from sites * per_site");
        T* stage = staging<T>(count);
        detail::scatter_sites<T><<<detail::permute_grid(count), detail::kThreads, 0, s>>>(
            stage, field.data(), order_dev_.data(), sites(), std::uint32_t(per_site));
        cuda_check(cudaGetLastError(), "download permute");
        cuda_check(cudaMemcpyAsync(host, stage, count * sizeof(T), cudaMemcpyDeviceToHost, s), "download");
        cuda_check(cudaStreamSynchronize(s), "download");
    }

private:
    template <class T>
    T* staging(std::uint64_t count) const
    {
        if (stage_.size() < count * sizeof(T)) stage_ = Buffer<unsigned char>(count * sizeof(T));
        return reinterpret_cast<T*>(stage_.data());
    }

    std::vector<std::uint32_t> position_, order_, begin_;
    Buffer<std::uint32_t> order_dev_, position_dev_;
    mutable Buffer<unsigned char> stage_;
};

// ------------------------------------------------------------------ table models

// One entry of a bond row: PairGraph's Bond<NoPayload> (lattice/pair_graph.hpp)
// on the device, the neighbour's device index.
struct Bond
{
    std::uint32_t j;
};

// PairModel (model/pair.hpp:18-80) as a device view: the field and the CSR
// bond table live on the device; Term is any arity-2 CellTerm.
template <class D, class Term>
    requires CellTerm<Term, D> && (Term::arity == 2)
struct PairModel
{
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    using bond_type = Bond;
    static constexpr std::size_t size = D::size;

    dtype* field;
    const std::uint32_t* offset;  // sites + 1
    const Bond* row;              // offset[sites]
    std::uint32_t n;
    Term term;

    UMC_HD std::size_t sites() const { return n; }
    UMC_HD const dtype* data() const { return field; }
    UMC_HD dtype* data() { return field; }
    UMC_HD std::size_t degree(std::size_t i) const { return offset[i + 1] - offset[i]; }
    UMC_HD const Bond* bonds(std::size_t i) const { return row + offset[i]; }
    // Key of the a-th bond of i's row: its CSR slot.
    UMC_HD std::uint32_t bond_id(std::size_t i, std::size_t a) const { return offset[i] + std::uint32_t(a); }

    // model/pair.hpp:38-49: bonds incident to i, each counted once.
    UMC_HD energy_type energy_at(std::size_t i) const
    {
        energy_type e = 0;
        const dtype* si = field + i * size;
        for (std::uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
            const dtype* links[2] = {si, field + std::size_t(row[a].j) * size};
            e += term.energy(links);
        }
        return e;
    }
    // model/pair.hpp:52-63
    UMC_HD energy_type energy_diff_at(std::size_t i, const dtype* p) const
    {
        energy_type d = 0;
        const dtype* si = field + i * size;
        for (std::uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
            const dtype* links[2] = {si, field + std::size_t(row[a].j) * size};
            d += term.delta(0, si, p, links);
        }
        return d;
    }
    // model/pair.hpp:66-72: the bond's energy change when b.j takes p, i fixed.
    UMC_HD energy_type energy_diff_bond(std::size_t i, const Bond& b, const dtype* p) const
    {
        const dtype* sj = field + std::size_t(b.j) * size;
        const dtype* links[2] = {sj, field + i * size};
        return term.delta(0, sj, p, links);
    }
    UMC_HD void update(std::size_t i, const dtype* p)
    {
        for (std::size_t k = 0; k < size; ++k) field[i * size + k] = p[k];
    }
};

// CellModel (model/cell.hpp:16-99) as a device view over a cell table and the
// per-site incidence (cell, slot) lists.
template <class D, class Term>
    requires CellTerm<Term, D>
struct CellModel
{
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    static constexpr std::size_t size = D::size;
    static constexpr std::size_t arity = Term::arity;

    dtype* field;
    const std::uint32_t* cell_sites;   // n_cells * arity
    const std::uint64_t* inc_offset;   // sites + 1
    const std::uint32_t* inc_cell;
    const std::uint8_t* inc_which;
    std::uint32_t n, n_cells;
    Term term;

    UMC_HD std::size_t sites() const { return n; }
    UMC_HD std::size_t cells() const { return n_cells; }
    UMC_HD const dtype* data() const { return field; }
    UMC_HD dtype* data() { return field; }

    // model/cell.hpp:52-56
    UMC_HD energy_type cell_energy(std::size_t c) const
    {
        const dtype* ls[arity];
        for (std::size_t k = 0; k < arity; ++k) ls[k] = field + std::size_t(cell_sites[c * arity + k]) * size;
        return term.energy(ls);
    }
    // model/cell.hpp:64-78
    UMC_HD energy_type energy_diff_at(std::size_t i, const dtype* p) const
    {
        energy_type d = 0;
        const dtype* old = field + i * size;
        const dtype* ls[arity];
        for (std::uint64_t a = inc_offset[i]; a < inc_offset[i + 1]; ++a) {
            const std::uint32_t* cs = cell_sites + std::size_t(inc_cell[a]) * arity;
            for (std::size_t k = 0; k < arity; ++k) ls[k] = field + std::size_t(cs[k]) * size;
            d += term.delta(inc_which[a], old, p, ls);
        }
        return d;
    }
    // model/cell.hpp:80-83
    UMC_HD void update(std::size_t i, const dtype* p)
    {
        for (std::size_t k = 0; k < size; ++k) field[i * size + k] = p[k];
    }
};

// A pair graph's CSR in the colour-major device numbering: row k holds the
// bonds of site order[k], each as the neighbour's device index.
class PairTables : public ColourMajor
{
public:
    explicit PairTables(const umc_graph* g) : PairTables(g, detail::colouring_of(g)) {}

    const ClassTable& classes() const noexcept { return classes_; }
    // Bond slots of the CSR (each bond appears in both endpoints' rows).
    std::uint64_t bond_slots() const noexcept { return bonds_.size(); }

    // A PairModel view over field (sites * D::size device scalars, device numbering).
    template <class D, class Term>
    PairModel<D, Term> model(typename D::dtype* field, Term term) const
    {
        return PairModel<D, Term>{field, offset_.data(), reinterpret_cast<const Bond*>(bonds_.data()), sites(), term};
    }

private:
    PairTables(const umc_graph* g, const detail::Colouring& c)
        : ColourMajor(c), classes_(Classes::identity(class_begin()))
    {
        const std::uint32_t n = sites();
        std::vector<std::uint32_t> off(std::size_t(n) + 1), bonds(umc_graph_slots(g));
        umc_check(umc_graph_csr(g, off.data(), bonds.data()));
        std::vector<std::uint32_t> doff(std::size_t(n) + 1, 0), dbonds(bonds.size());
        for (std::uint32_t k = 0; k < n; ++k) {
            const std::uint32_t i = order()[k];
            std::uint32_t w = doff[k];
            for (std::uint32_t a = off[i]; a < off[i + 1]; ++a) dbonds[w++] = position()[bonds[a]];
            doff[k + 1] = w;
        }
        offset_ = Buffer<std::uint32_t>(doff);
        bonds_ = Buffer<std::uint32_t>(dbonds);
    }

    ClassTable classes_;
    Buffer<std::uint32_t> offset_, bonds_;
};

// One entry of a bond row with a payload: PairGraph's Bond<P> (lattice/
// pair_graph.hpp:16-22) on the device, the neighbour's device index and the
// bond's payload c (a coupling, for instance).
template <class P>
struct BondOf
{
    std::uint32_t j;
    P c;
};

// A PairGraphLike view of a weighted graph on the device (lattice/
// pair_graph.hpp:86-116): sites(), degree(i), bonds(i) over rows of BondOf<P>
// in the colour-major device numbering, and bond_id(i, a), the key of the
// a-th bond of i's row (its CSR slot).  Trivially copyable: a user model
// holds one as a member, as the reference's models hold their PairGraph.
template <class P>
struct PairRows
{
    using bond_type = BondOf<P>;
    const std::uint32_t* offset;  // sites + 1
    const BondOf<P>* row;         // offset[sites]
    std::uint32_t n;

    UMC_HD std::size_t sites() const { return n; }
    UMC_HD std::size_t degree(std::size_t i) const { return offset[i + 1] - offset[i]; }
    UMC_HD const BondOf<P>* bonds(std::size_t i) const { return row + offset[i]; }
    UMC_HD std::uint32_t bond_id(std::size_t i, std::size_t a) const { return offset[i] + std::uint32_t(a); }
};

// PairTables plus each slot's payload: the CSR of a PairGraph<P> built with a
// payload (umc_graph_create_payload, or the facade's PairGraph<P>) in the
// colour-major device numbering, slot for slot the rows of PairTables, each
// bond carrying the payload the reference copies into it from its Edge.
// rows() is the device view a weighted user model reads; the rest (classes,
// upload/download, the Wolff tiles) is PairTables'.
template <class P>
class BondTables : public PairTables
{
    static_assert(std::is_trivially_copyable_v<P>, "a bond payload must be trivially copyable");

public:
    explicit BondTables(const umc_graph* g) : PairTables(g)
    {
        if (umc_graph_payload_bytes(g) != sizeof(P))
            throw std::invalid_argument("BondTables<P>: the graph's payload size differs from sizeof(P)");
        const std::uint32_t n = sites();
        const std::size_t m = umc_graph_slots(g);
        std::vector<std::uint32_t> off(std::size_t(n) + 1), bonds(m);
        umc_check(umc_graph_csr(g, off.data(), bonds.data()));
        std::vector<P> pay(m);
        if (m) umc_check(umc_graph_payloads(g, pay.data()));
        std::vector<std::uint32_t> doff(std::size_t(n) + 1, 0);
        std::vector<BondOf<P>> rows(m);
        for (std::uint32_t k = 0; k < n; ++k) {
            const std::uint32_t i = order()[k];
            std::uint32_t w = doff[k];
            for (std::uint32_t a = off[i]; a < off[i + 1]; ++a, ++w) rows[w] = BondOf<P>{position()[bonds[a]], pay[a]};
            doff[k + 1] = w;
        }
        woffset_ = Buffer<std::uint32_t>(doff);
        wrows_ = Buffer<BondOf<P>>(rows);
    }

    PairRows<P> rows() const noexcept { return PairRows<P>{woffset_.data(), wrows_.data(), sites()}; }

private:
    Buffer<std::uint32_t> woffset_;
    Buffer<BondOf<P>> wrows_;
};

// A cell complex in the colour-major device numbering: cell c lists its
// sites' device indices; incidence row k is that of site order[k].
class CellTables : public ColourMajor
{
public:
    explicit CellTables(const umc_cells* cc) : CellTables(cc, detail::colouring_of(cc)) {}

    std::uint32_t cells() const noexcept { return n_cells_; }
    const ClassTable& classes() const noexcept { return classes_; }

    template <class D, class Term>
    CellModel<D, Term> model(typename D::dtype* field, Term term) const
    {
        if (Term::arity != arity_) throw std::invalid_argument("term arity differs from the cell table's");
        return CellModel<D, Term>{field, cells_.data(), inc_offset_.data(), inc_cell_.data(), inc_which_.data(),
                                  sites(), n_cells_, term};
    }

private:
    CellTables(const umc_cells* cc, const detail::Colouring& c)
        : ColourMajor(c), classes_(Classes::identity(class_begin()))
    {
        const std::uint32_t n = sites();
        n_cells_ = std::uint32_t(umc_cells_count(cc));
        arity_ = umc_cells_arity(cc);
        std::vector<std::uint32_t> cells(std::size_t(n_cells_) * arity_);
        umc_check(umc_cells_table(cc, cells.data()));
        for (auto& s : cells) s = position()[s];
        std::vector<std::uint64_t> off(std::size_t(n) + 1);
        umc_check(umc_cells_incidence(cc, off.data(), nullptr, nullptr));
        std::vector<std::uint32_t> inc_cell(off.back());
        std::vector<std::uint8_t> inc_which(off.back());
        umc_check(umc_cells_incidence(cc, off.data(), inc_cell.data(), inc_which.data()));
        std::vector<std::uint64_t> doff(std::size_t(n) + 1, 0);
        std::vector<std::uint32_t> dcell(inc_cell.size());
        std::vector<std::uint8_t> dwhich(inc_which.size());
        for (std::uint32_t k = 0; k < n; ++k) {
            const std::uint32_t i = order()[k];
            std::uint64_t w = doff[k];
            for (std::uint64_t a = off[i]; a < off[i + 1]; ++a, ++w) {
                dcell[w] = inc_cell[a];
                dwhich[w] = inc_which[a];
            }
            doff[k + 1] = w;
        }
        cells_ = Buffer<std::uint32_t>(cells);
        inc_offset_ = Buffer<std::uint64_t>(doff);
        inc_cell_ = Buffer<std::uint32_t>(dcell);
        inc_which_ = Buffer<std::uint8_t>(dwhich);
    }

    ClassTable classes_;
    std::uint32_t n_cells_ = 0, arity_ = 0;
    Buffer<std::uint32_t> cells_;
    Buffer<std::uint64_t> inc_offset_;
    Buffer<std::uint32_t> inc_cell_;
    Buffer<std::uint8_t> inc_which_;
};

// ------------------------------------------------------------------ tables without storage

// n / d for 32-bit n and a fixed d >= 1 without a divide: the high 64 bits of
// n * ceil(2^64 / d).  The rounding error is below 2^-32 <= 1/d, so the
// quotient is exact for every 32-bit n.
struct FastDiv
{
    std::uint32_t d = 1;
    std::uint64_t m = 0;

    FastDiv() = default;
    explicit FastDiv(std::uint32_t divisor) : d(divisor)
    {
        if (d == 0) throw std::invalid_argument("FastDiv: divisor 0");
        // ceil(2^64 / d) = floor((2^64 - 1) / d) + 1 for every d >= 2
        m = d == 1 ? 0 : ~std::uint64_t(0) / d + 1;
    }
    UMC_HD std::uint32_t div(std::uint32_t n) const
    {
        if (d == 1) return n;
#if defined(__CUDA_ARCH__)
        return std::uint32_t(__umul64hi(std::uint64_t(n), m));
#else
        return std::uint32_t((unsigned __int128)n * m >> 64);
#endif
    }
};

// A periodic Lx x Ly x Lz lattice whose bonds are computed, not stored
// (square_lattice's and cubic_lattice's sites and bonds; Lz = 1 in 2D).
// Lx is even and Ly, Lz are even or 1, so the checkerboard is a proper
// 2-colouring and sites 2r, 2r + 1 share a row; device site k is the
// colour-major position ((x+y+z)&1) n/2 + s/2 of reference site
// s = (z Ly + y) Lx + x.  The bonds of k, in the order +x, -x, +y, -y, +z, -z
// over the extents above 1, are the neighbours' device sites.
class RegularLattice
{
public:
    static constexpr std::uint32_t kMaxDegree = 6;

    RegularLattice(std::uint32_t lx, std::uint32_t ly, std::uint32_t lz)
        : Lx(lx), Ly(ly), Lz(lz), div_x(lx ? lx : 1), div_y(ly ? ly : 1)
    {}

    std::uint32_t Lx, Ly, Lz;

    UMC_HD std::uint32_t sites() const { return Lx * Ly * Lz; }
    UMC_HD std::uint32_t degree() const { return 2u * ((Lx > 1) + (Ly > 1) + (Lz > 1)); }
    UMC_HD std::uint32_t index_of(std::uint32_t x, std::uint32_t y, std::uint32_t z) const
    {
        const std::uint32_t s = (z * Ly + y) * Lx + x;
        return ((x + y + z) & 1u) * (sites() / 2) + s / 2;
    }
    // Coordinates of device site k.
    UMC_HD void coords(std::uint32_t k, std::uint32_t& x, std::uint32_t& y, std::uint32_t& z) const
    {
        const std::uint32_t half = sites() / 2;
        const std::uint32_t c = k >= half ? 1u : 0u;
        const std::uint32_t s0 = 2u * (k - c * half);  // the even site of the pair; same row as s0 + 1
        const std::uint32_t row = div_x.div(s0);
        z = div_y.div(row);
        y = row - z * Ly;
        const std::uint32_t x0 = s0 - row * Lx;
        x = x0 + ((c + y + z) & 1u);
    }
    // All degree() neighbours of device site k, in bond order.  Site k is
    // s = 2r + b (rank r in its colour c); every neighbour has the other
    // colour, and s +- 1, s +- Lx, s +- Lx Ly have ranks r + b or r + b - 1,
    // r +- Lx/2, r +- Lx Ly/2 (Lx even), shifted by one period at a wrap.
    // Unsigned wrap-around in the intermediate sums is harmless: every result
    // is a valid rank.
    UMC_HD void neighbours(std::uint32_t k, std::uint32_t* nb) const
    {
        const std::uint32_t half = sites() / 2, hx = Lx / 2, ha = Lx * Ly / 2;
        const std::uint32_t c = k >= half ? 1u : 0u;
        const std::uint32_t r = k - c * half;
        const std::uint32_t row = div_x.div(2u * r);
        const std::uint32_t z = div_y.div(row), y = row - z * Ly;
        const std::uint32_t b = (c + y + z) & 1u;
        const std::uint32_t x = 2u * r - row * Lx + b;
        const std::uint32_t o = (1u - c) * half;
        std::uint32_t a = 0;
        nb[a++] = o + (x + 1 == Lx ? r + 1 - hx : r + b);
        nb[a++] = o + (x == 0 ? r + hx - 1 : r + b - 1);
        if (Ly > 1) {
            nb[a++] = o + (y + 1 == Ly ? r + hx - ha : r + hx);
            nb[a++] = o + (y == 0 ? r - hx + ha : r - hx);
        }
        if (Lz > 1) {
            nb[a++] = o + (z + 1 == Lz ? r + ha - half : r + ha);
            nb[a++] = o + (z == 0 ? r - ha + half : r - ha);
        }
    }
    UMC_HD std::uint32_t neighbour(std::uint32_t k, std::uint32_t a) const
    {
        std::uint32_t nb[kMaxDegree];
        neighbours(k, nb);
        return nb[a];
    }

private:
    FastDiv div_x, div_y;
};

namespace detail {
inline Colouring checkerboard(const RegularLattice& l)
{
    if (l.Lx < 2 || l.Lx % 2 || l.Ly < 1 || l.Lz < 1 || (l.Ly > 1 && l.Ly % 2) || (l.Lz > 1 && l.Lz % 2))
        throw std::invalid_argument("RegularLattice: Lx must be even, Ly and Lz even or 1");
    if (std::uint64_t(l.Lx) * l.Ly * l.Lz * l.degree() >= (std::uint64_t(1) << 32))
        throw std::invalid_argument("RegularLattice: sites x degree must stay below 2^32");
    Colouring c;
    c.count = 2;
    c.colour.resize(l.sites());
    c.position.resize(l.sites());
    for (std::uint32_t z = 0, s = 0; z < l.Lz; ++z)
        for (std::uint32_t y = 0; y < l.Ly; ++y)
            for (std::uint32_t x = 0; x < l.Lx; ++x, ++s) {
                c.colour[s] = (x + y + z) & 1u;
                c.position[s] = l.index_of(x, y, z);
            }
    return c;
}
}  // namespace detail

// PairModel over a RegularLattice: neighbours computed from the device index,
// no CSR bytes read.  A ModelLike, EnergyModel and WolffModel (bond(i, a) by
// value; bond_id(i, a) = i * degree + a).
template <class D, class Term>
    requires CellTerm<Term, D> && (Term::arity == 2)
struct LatticePairModel
{
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    using bond_type = Bond;
    static constexpr std::size_t size = D::size;

    dtype* field;
    RegularLattice lattice;
    Term term;

    UMC_HD std::size_t sites() const { return lattice.sites(); }
    UMC_HD const dtype* data() const { return field; }
    UMC_HD dtype* data() { return field; }
    UMC_HD std::size_t degree(std::size_t) const { return lattice.degree(); }
    UMC_HD Bond bond(std::size_t i, std::size_t a) const
    {
        return Bond{lattice.neighbour(std::uint32_t(i), std::uint32_t(a))};
    }
    UMC_HD std::uint32_t bond_id(std::size_t i, std::size_t a) const
    {
        return std::uint32_t(i) * lattice.degree() + std::uint32_t(a);
    }

    // model/pair.hpp:38-49
    UMC_HD energy_type energy_at(std::size_t i) const
    {
        std::uint32_t nb[RegularLattice::kMaxDegree];
        lattice.neighbours(std::uint32_t(i), nb);
        energy_type e = 0;
        const dtype* si = field + i * size;
        for (std::uint32_t a = 0; a < lattice.degree(); ++a) {
            const dtype* links[2] = {si, field + std::size_t(nb[a]) * size};
            e += term.energy(links);
        }
        return e;
    }
    // model/pair.hpp:52-63
    UMC_HD energy_type energy_diff_at(std::size_t i, const dtype* p) const
    {
        std::uint32_t nb[RegularLattice::kMaxDegree];
        lattice.neighbours(std::uint32_t(i), nb);
        energy_type d = 0;
        const dtype* si = field + i * size;
        for (std::uint32_t a = 0; a < lattice.degree(); ++a) {
            const dtype* links[2] = {si, field + std::size_t(nb[a]) * size};
            d += term.delta(0, si, p, links);
        }
        return d;
    }
    // model/pair.hpp:66-72
    UMC_HD energy_type energy_diff_bond(std::size_t i, const Bond& b, const dtype* p) const
    {
        const dtype* sj = field + std::size_t(b.j) * size;
        const dtype* links[2] = {sj, field + i * size};
        return term.delta(0, sj, p, links);
    }
    UMC_HD void update(std::size_t i, const dtype* p)
    {
        for (std::size_t k = 0; k < size; ++k) field[i * size + k] = p[k];
    }
};

// The two colour classes of a RegularLattice and the site-order transfers;
// nothing about its bonds is stored.
class LatticeTables : public ColourMajor
{
public:
    explicit LatticeTables(RegularLattice l)
        : LatticeTables(l, detail::checkerboard(l))
    {}

    const RegularLattice& lattice() const noexcept { return lattice_; }
    const ClassTable& classes() const noexcept { return classes_; }
    std::uint64_t bond_slots() const noexcept { return std::uint64_t(lattice_.sites()) * lattice_.degree(); }

    template <class D, class Term>
    LatticePairModel<D, Term> model(typename D::dtype* field, Term term) const
    {
        return LatticePairModel<D, Term>{field, lattice_, term};
    }

private:
    LatticeTables(RegularLattice l, const detail::Colouring& c)
        : ColourMajor(c), lattice_(l), classes_(Classes::identity(class_begin()))
    {}

    RegularLattice lattice_;
    ClassTable classes_;
};

// A periodic L^dim plaquette complex whose cells and incidence are computed,
// not stored: hypercubic_plaquettes (dim 4, lattice/hypercubic.hpp:15-64:
// link mu L^4 + ((t L + z) L + y) L + x, direction 0 along t) and the library's
// 2D square_plaquettes (dim 2: link mu L^2 + y L + x, direction 0 along x).
// Plaquette (a < b) at site c is [U_a(c), U_b(c + a), U_a(c + b), U_b(c)], in
// the reference's cell order (pairs (a, b) ascending, then sites).  L is even,
// so the device numbering is the library's closed-form link colouring:
// class 2 mu + parity(site), position class V/2 + site/2, and every unit step
// flips a site's parity.
class PlaquetteLattice
{
public:
    static constexpr std::uint32_t kMaxDim = 4;

    PlaquetteLattice(std::uint32_t l, std::uint32_t d) : L(l), dim(d), div_l(l ? l : 1)
    {
        V = 1;
        for (std::uint32_t k = 0; k < dim; ++k) V *= L;
    }

    std::uint32_t L, dim, V;

    UMC_HD std::uint32_t sites() const { return dim * V; }
    UMC_HD std::uint32_t cells() const { return V * dim * (dim - 1) / 2; }
    // Base-L digit (0 = fastest) that direction mu moves, and its stride.
    UMC_HD std::uint32_t digit_of(std::uint32_t mu) const { return dim == 2 ? mu : dim - 1 - mu; }
    UMC_HD std::uint32_t stride_of(std::uint32_t mu) const
    {
        std::uint32_t st = 1;
        for (std::uint32_t k = 0; k < digit_of(mu); ++k) st *= L;
        return st;
    }
    UMC_HD void digits(std::uint32_t s, std::uint32_t* dg) const
    {
        for (std::uint32_t k = 0; k < dim; ++k) {
            const std::uint32_t q = div_l.div(s);
            dg[k] = s - q * L;
            s = q;
        }
    }
    UMC_HD std::uint32_t parity(std::uint32_t s) const
    {
        std::uint32_t dg[kMaxDim], p = 0;
        digits(s, dg);
        for (std::uint32_t k = 0; k < dim; ++k) p += dg[k];
        return p & 1u;
    }
    // Device index of link (mu, site s) whose site parity is par.
    UMC_HD std::uint32_t link(std::uint32_t mu, std::uint32_t s, std::uint32_t par) const
    {
        return (2u * mu + par) * (V / 2) + s / 2;
    }
    // Site s moved by one step (+1 or -1) along direction mu; dg are s's digits.
    UMC_HD std::uint32_t step(std::uint32_t s, const std::uint32_t* dg, std::uint32_t mu, bool up) const
    {
        const std::uint32_t st = stride_of(mu), x = dg[digit_of(mu)];
        if (up) return x + 1 == L ? s - (L - 1) * st : s + st;
        return x == 0 ? s + (L - 1) * st : s - st;
    }
    // Direction and site of device link k.
    UMC_HD void decode(std::uint32_t k, std::uint32_t& mu, std::uint32_t& s, std::uint32_t& par) const
    {
        const std::uint32_t half = V / 2, cls = k / half;
        mu = cls >> 1;
        par = cls & 1u;
        const std::uint32_t s0 = 2u * (k - cls * half);  // s0 and s0 + 1 differ in the fastest digit only
        s = s0 + ((par + parity(s0)) & 1u);
    }

private:
    FastDiv div_l;
};

namespace detail {
inline Colouring plaquette_colouring(const PlaquetteLattice& l)
{
    if (!(l.dim == 2 || l.dim == 4) || l.L < 2 || l.L % 2)
        throw std::invalid_argument("PlaquetteLattice: dim 2 or 4 and an even L");
    if (std::uint64_t(l.V) * l.dim >= (std::uint64_t(1) << 32))
        throw std::invalid_argument("PlaquetteLattice: links must stay below 2^32");
    Colouring c;
    c.count = 2 * l.dim;
    c.colour.resize(l.sites());
    c.position.resize(l.sites());
    for (std::uint32_t mu = 0; mu < l.dim; ++mu)
        for (std::uint32_t s = 0; s < l.V; ++s) {
            const std::uint32_t par = l.parity(s);
            c.colour[mu * l.V + s] = 2 * mu + par;
            c.position[mu * l.V + s] = l.link(mu, s, par);
        }
    return c;
}
}  // namespace detail

// CellModel over a PlaquetteLattice: cells and incidence computed from the
// device index, no tables read.  A ModelLike and CellEnergyModel.
template <class D, class Term>
    requires CellTerm<Term, D> && (Term::arity == 4)
struct LatticeCellModel
{
    using dtype = typename D::dtype;
    using value_type = dtype;
    using energy_type = typename Term::energy_type;
    static constexpr std::size_t size = D::size;
    static constexpr std::size_t arity = 4;

    dtype* field;
    PlaquetteLattice lattice;
    Term term;

    UMC_HD std::size_t sites() const { return lattice.sites(); }
    UMC_HD std::size_t cells() const { return lattice.cells(); }
    UMC_HD const dtype* data() const { return field; }
    UMC_HD dtype* data() { return field; }
    UMC_HD const dtype* at(std::uint32_t k) const { return field + std::size_t(k) * size; }

    // model/cell.hpp:52-56; cell c = pair index * V + site, pairs (a < b) ascending.
    UMC_HD energy_type cell_energy(std::size_t c) const
    {
        const PlaquetteLattice& l = lattice;
        std::uint32_t pi = std::uint32_t(c / l.V), a = 0, b = 1;
        for (std::uint32_t q = 0; q < pi; ++q)
            if (++b == l.dim) b = ++a + 1;
        const std::uint32_t x = std::uint32_t(c - std::size_t(pi) * l.V);
        std::uint32_t dg[PlaquetteLattice::kMaxDim];
        l.digits(x, dg);
        const std::uint32_t par = l.parity(x);
        const dtype* ls[4] = {at(l.link(a, x, par)), at(l.link(b, l.step(x, dg, a, true), par ^ 1u)),
                              at(l.link(a, l.step(x, dg, b, true), par ^ 1u)), at(l.link(b, x, par))};
        return term.energy(ls);
    }
    // model/cell.hpp:64-78 over the 2 (dim - 1) plaquettes that hold link k.
    UMC_HD energy_type energy_diff_at(std::size_t k, const dtype* p) const
    {
        const PlaquetteLattice& l = lattice;
        std::uint32_t mu, x, par;
        l.decode(std::uint32_t(k), mu, x, par);
        std::uint32_t dg[PlaquetteLattice::kMaxDim];
        l.digits(x, dg);
        const dtype* old = at(std::uint32_t(k));
        energy_type d = 0;
        for (std::uint32_t nu = 0; nu < l.dim; ++nu) {
            if (nu == mu) continue;
            const std::uint32_t xm = l.step(x, dg, nu, false);  // x - nu
            std::uint32_t dm[PlaquetteLattice::kMaxDim];
            l.digits(xm, dm);
            if (mu < nu) {
                // (mu, nu) at x, slot 0; at x - nu, slot 2
                const dtype* c1[4] = {old, at(l.link(nu, l.step(x, dg, mu, true), par ^ 1u)),
                                      at(l.link(mu, l.step(x, dg, nu, true), par ^ 1u)), at(l.link(nu, x, par))};
                d += term.delta(0, old, p, c1);
                const dtype* c2[4] = {at(l.link(mu, xm, par ^ 1u)), at(l.link(nu, l.step(xm, dm, mu, true), par)), old,
                                      at(l.link(nu, xm, par ^ 1u))};
                d += term.delta(2, old, p, c2);
            } else {
                // (nu, mu) at x - nu, slot 1; at x, slot 3
                const dtype* c3[4] = {at(l.link(nu, xm, par ^ 1u)), old, at(l.link(nu, l.step(xm, dm, mu, true), par)),
                                      at(l.link(mu, xm, par ^ 1u))};
                d += term.delta(1, old, p, c3);
                const dtype* c4[4] = {at(l.link(nu, x, par)), at(l.link(mu, l.step(x, dg, nu, true), par ^ 1u)),
                                      at(l.link(nu, l.step(x, dg, mu, true), par ^ 1u)), old};
                d += term.delta(3, old, p, c4);
            }
        }
        return d;
    }
    UMC_HD void update(std::size_t i, const dtype* p)
    {
        for (std::size_t k = 0; k < size; ++k) field[i * size + k] = p[k];
    }
};

// The 2 dim colour classes of a PlaquetteLattice and the transfers in the
// reference's link order; nothing about its cells is stored.
class PlaquetteTables : public ColourMajor
{
public:
    PlaquetteTables(std::uint32_t L, std::uint32_t dim) : PlaquetteTables(PlaquetteLattice(L, dim)) {}
    explicit PlaquetteTables(PlaquetteLattice l) : PlaquetteTables(l, detail::plaquette_colouring(l)) {}

    const PlaquetteLattice& lattice() const noexcept { return lattice_; }
    const ClassTable& classes() const noexcept { return classes_; }
    std::uint32_t cells() const noexcept { return lattice_.cells(); }

    template <class D, class Term>
    LatticeCellModel<D, Term> model(typename D::dtype* field, Term term) const
    {
        return LatticeCellModel<D, Term>{field, lattice_, term};
    }

private:
    PlaquetteTables(PlaquetteLattice l, const detail::Colouring& c)
        : ColourMajor(c), lattice_(l), classes_(Classes::identity(class_begin()))
    {}

    PlaquetteLattice lattice_;
    ClassTable classes_;
};

// ------------------------------------------------------------------ kernels

namespace detail {

constexpr unsigned kSpinLimit = 1u << 24;  // about a second of 64 ns sleeps

struct Control
{
    unsigned count;       // blocks arrived at the current barrier
    unsigned generation;  // barriers completed
    unsigned status;      // bit 0: a barrier wait ran out
    unsigned pad;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier of a cooperative launch.  Returns false in every thread of
// every block once any block's wait has run out.
__device__ __forceinline__ bool grid_sync(Control* ctl)
{
    int fail = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned gen = ld_acquire(&ctl->generation);
        __threadfence();
        if (atomicAdd(&ctl->count, 1u) == gridDim.x - 1) {
            atomicExch(&ctl->count, 0u);
            st_release(&ctl->generation, gen + 1);
        } else {
            unsigned spins = 0;
            while (ld_acquire(&ctl->generation) == gen) {
                if (ld_acquire(&ctl->status) != 0u || ++spins > kSpinLimit) {
                    atomicOr(&ctl->status, 1u);
                    fail = 1;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    return __syncthreads_or(fail) == 0;
}

// log(u) < log_p, decided as the FP64 test decides it.  logf(float(u)) is
// within 2^-24 + 2^-23 |log u| of log(u): rounding u to float moves log u by
// at most 2^-24, and logf is accurate to 1 ulp.  The FP32 answer is taken
// when it clears log_p by 2^-21 (1 + |logf|), at least four times that error;
// otherwise the FP64 log decides.
__device__ __forceinline__ bool log_below(double u, double log_p)
{
    const float lf = logf(float(u));
    const double gap = double(lf) - log_p;
    const double bound = 0x1.0p-21 * (1.0 + fabs(double(lf)));
    if (gap > bound) return false;
    if (gap < -bound) return true;
    return log(u) < log_p;
}

// The failure path of grid_sync: block 0 waits at a barrier that block 1
// never reaches, so its bounded wait runs out, sets the status bit and
// returns false.  status[0] = the status word, status[1] = what grid_sync
// returned in block 0.
__global__ void barrier_timeout_probe(Control* ctl, unsigned* status)
{
    if (blockIdx.x != 0) return;  // block 1 leaves without arriving
    const bool ok = grid_sync(ctl);
    if (threadIdx.x == 0) {
        status[0] = ld_acquire(&ctl->status);
        status[1] = ok ? 1u : 0u;
    }
}

// No per-sweep observable.
struct NoObservable
{};

// Sum over the block of v; the result is valid in thread 0.
__device__ __forceinline__ double block_total(double v)
{
    __shared__ double sh[kThreads];
    __syncthreads();
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    return sh[0];
}

// n_sweeps Metropolis sweeps (driver.hpp:29-43) over the colour classes.
// With an observable O, record after sweep s the FP64 sum of obs(m, x) over
// x < obs_count into records[s]: per-block partials, then block 0 adds them in
// block order (deterministic for a given grid).  This is sample(n, observe)
// (driver.hpp:54-61) with the observation on the device, inside the launch.
template <class M, class Q, class O = NoObservable>
__global__ void __launch_bounds__(kThreads) metropolis_sweeps(M m, Q q, const std::uint32_t* __restrict__ order,
                                                              const std::uint32_t* __restrict__ begin,
                                                              std::uint32_t n_classes, double beta, std::uint64_t seed,
                                                              std::uint64_t sweep0, std::uint32_t n_sweeps,
                                                              Control* ctl, O obs = {}, std::uint64_t obs_count = 0,
                                                              double* partial = nullptr, double* records = nullptr)
{
    using T = typename M::value_type;
    constexpr bool kObserve = !std::is_same_v<O, NoObservable>;
    const std::uint32_t stride = gridDim.x * blockDim.x;
    const std::uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    for (std::uint32_t s = 0; s < n_sweeps; ++s) {
        const std::uint64_t kbase = key_base(key_seed(seed, sweep0 + s, tag_site(0)));
        for (std::uint32_t c = 0; c < n_classes; ++c) {
            const std::uint32_t end = begin[c + 1];
            for (std::uint32_t k = begin[c] + t; k < end; k += stride) {
                const std::uint32_t i = order ? order[k] : k;
                Rng rng(KeyedPcg::open(kbase, k));
                T cand[M::size];
                const T* cur = m.data() + std::size_t(i) * M::size;
                q.sample(cur, rng, cand);
                const double dE = m.energy_diff_at(i, cand);
                const double log_p = -beta * dE + q.log_ratio(cur, cand);
                if (log_p >= 0.0 || log_below(rng.uni(), log_p)) m.update(i, cand);
            }
            if ((kObserve || s + 1 < n_sweeps || c + 1 < n_classes) && !grid_sync(ctl)) return;
        }
        if constexpr (kObserve) {
            double v = 0.0;
            for (std::uint64_t x = t; x < obs_count; x += stride) v += double(obs(m, x));
            const double b = block_total(v);
            if (threadIdx.x == 0) partial[blockIdx.x] = b;
            if (!grid_sync(ctl)) return;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                double e = 0.0;
                for (std::uint32_t k = 0; k < gridDim.x; ++k) e += __ldcg(partial + k);
                records[s] = e;
            }
        }
    }
}

// Per-block FP64 sums of f(m, x) over x < count; the host adds the blocks'
// partials in block order.
template <class M, class F>
__global__ void __launch_bounds__(kThreads) block_sums(M m, std::uint64_t count, F f, double* partial)
{
    __shared__ double sh[kThreads];
    double v = 0.0;
    for (std::uint64_t x = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; x < count;
         x += std::uint64_t(gridDim.x) * blockDim.x)
        v += double(f(m, x));
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

struct CellEnergyOf
{
    template <class M>
    __device__ double operator()(const M& m, std::uint64_t c) const
    {
        return double(m.cell_energy(c));
    }
};
struct EnergyAtOf
{
    template <class M>
    __device__ double operator()(const M& m, std::uint64_t i) const
    {
        return double(m.energy_at(i));
    }
};

// FP64 sum of f(m, x) over x < count: per-block partials, added on the host
// in block order (deterministic for a given count).  partial is the caller's
// reusable buffer (grown here), so a sum allocates nothing after the first.
template <class M, class F>
double device_sum(const M& m, std::uint64_t count, F f, cudaStream_t s, Buffer<double>& partial)
{
    const std::uint32_t blocks =
        std::uint32_t(std::max<std::uint64_t>(1, std::min<std::uint64_t>(1024, (count + kThreads - 1) / kThreads)));
    if (partial.size() < blocks) partial = Buffer<double>(1024);
    block_sums<M, F><<<blocks, kThreads, 0, s>>>(m, count, f, partial.data());
    cuda_check(cudaGetLastError(), "sum launch");
    std::vector<double> h(blocks);
    cuda_check(cudaMemcpyAsync(h.data(), partial.data(), blocks * sizeof(double), cudaMemcpyDeviceToHost, s),
               "sum read");
    cuda_check(cudaStreamSynchronize(s), "sum read");
    double e = 0.0;
    for (const double v : h) e += v;
    return e;
}

// Blocks of a cooperative launch of kernel: all resident at once, no more
// than `need`.
inline std::uint32_t cooperative_grid(const void* kernel, std::uint64_t need)
{
    int dev = 0, sms = 0, per_sm = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0), "occupancy");
    if (per_sm < 1) throw std::runtime_error("kernel does not fit on an SM");
    return std::uint32_t(std::max<std::uint64_t>(1, std::min<std::uint64_t>(need, std::uint64_t(per_sm) * sms)));
}

// ---- Wolff: bond activation, union-find labelling, flip of the seed's cluster

constexpr unsigned kUfLimit = 1u << 26;  // steps of one find or union before giving up

struct WolffControl
{
    Control bar;
    unsigned long long touched;  // sites flipped by this launch
    unsigned done;               // flips completed by this launch
    unsigned uf_status;          // bit 1: a find or union ran past kUfLimit; bit 2: crossing list full
    unsigned long long xcount;   // active bonds between tiles in this flip (tiled kernel)
};

__device__ __forceinline__ std::uint32_t uf_load(const std::uint32_t* p) { return *(const volatile std::uint32_t*)p; }

// Linking order of the union-find: a root is linked under a root of higher
// priority, the priority of site x being stream_id(x) (a bijection of 32-bit
// words, so the order is strict).  Random priorities keep the trees shallow
// and spread the roots, and so the CAS traffic, over memory; linking by index
// piled the unions of a large cluster onto a few low-index roots.
__device__ __forceinline__ bool uf_below(std::uint32_t a, std::uint32_t b) { return stream_id(a) < stream_id(b); }

// Root of x with path halving.  The links form a forest (a union links a root
// under another root; the tiled kernel also points sites at their tile's
// root), so a walk ends within n steps; kUfLimit guards it all the same.
__device__ __forceinline__ std::uint32_t uf_root(std::uint32_t* parent, std::uint32_t x, unsigned* status)
{
    for (unsigned it = 0; it < kUfLimit; ++it) {
        const std::uint32_t p = uf_load(parent + x);
        if (p == x) return x;
        const std::uint32_t gp = uf_load(parent + p);
        if (gp != p) *(volatile std::uint32_t*)(parent + x) = gp;
        x = gp;
    }
    atomicOr(status, 2u);
    return x;
}

// Joins the sets of a and b: the root of lower priority is linked under the other.
__device__ __forceinline__ void uf_unite(std::uint32_t* parent, std::uint32_t a, std::uint32_t b, unsigned* status)
{
    for (unsigned it = 0; it < kUfLimit; ++it) {
        a = uf_root(parent, a, status);
        b = uf_root(parent, b, status);
        if (a == b) return;
        if (uf_below(a, b)) {
            const std::uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(parent + b, b, a) == b) return;
    }
    atomicOr(status, 2u);
}

// The a-th bond of i: from the row pointer, or by value from a model that
// computes its bonds.
template <class M>
__device__ __forceinline__ typename M::bond_type bond_of(const M& m, std::uint32_t i, std::size_t a)
{
    if constexpr (requires { m.bond(std::size_t(i), a); })
        return m.bond(i, a);
    else
        return m.bonds(i)[a];
}

// u < 1 - exp(-x) for x > 0, decided as the FP64 test decides it.
// 1 - expf(-float(x)) is within 2^-22 of 1 - exp(-x): rounding x to float
// moves exp(-x) by at most x e^-x 2^-24 < 2^-24, and expf's 2-ulp error is at
// most 2^-23 for a result below 1.  The FP32 answer is taken when it clears u
// by 2^-19, eight times that; otherwise FP64 decides.
__device__ __forceinline__ bool activates(double u, double x)
{
    const double p32 = 1.0 - double(expf(-float(x)));
    const double gap = u - p32;
    if (gap > 0x1.0p-19) return false;
    if (gap < -0x1.0p-19) return true;
    return u < 1.0 - exp(-x);
}

// out = s - 2 (s . r) r, in T arithmetic as Wolff::flip does (driver.hpp:127-130).
template <class T, std::size_t D>
__device__ __forceinline__ void reflect(const T* s, const T* r, T* out)
{
    T dot = 0;
    for (std::size_t k = 0; k < D; ++k) dot += s[k] * r[k];
    for (std::size_t k = 0; k < D; ++k) out[k] = s[k] - T(2) * dot * r[k];
}

// Wolff::flip (driver.hpp:104-162) for flips flip0, flip0 + 1, ...: stops
// after max_flips, or once the flipped sites reach `target` when target > 0.
// Per flip: the axis and seed site from the key (seed, flip, kTagAxis); every
// bond (i, j > i) active with probability 1 - exp(-beta dE), dE =
// energy_diff_bond(i, b, reflected s_j), its uniform keyed (seed, flip,
// kTagBond, bond_id); the seed's component of the active bonds reflected.
// With a reflection-invariant pair energy the bond test is the same from
// either end, so this is the reference's cluster for those draws.
template <class M, class A>
__global__ void __launch_bounds__(kThreads) wolff_flips(M m, A axis, double beta, std::uint64_t seed,
                                                        std::uint64_t flip0, std::uint32_t max_flips,
                                                        std::uint64_t target, std::uint32_t* parent,
                                                        unsigned long long* sizes, WolffControl* ctl,
                                                        const std::uint32_t*, const std::uint32_t*, uint2*,
                                                        unsigned long long)  // the tiled kernel's; unused
{
    using T = typename M::value_type;
    constexpr std::size_t D = M::size;
    __shared__ unsigned long long block_count;
    const std::uint32_t n = std::uint32_t(m.sites());
    const std::uint32_t stride = gridDim.x * blockDim.x;
    const std::uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long touched = 0;
    for (std::uint32_t f = 0; f < max_flips; ++f) {
        const std::uint64_t counter = flip0 + f;
        Rng g(KeyedPcg::open_key(seed, counter, kTagAxis, 0));
        T r[D];
        axis.sample(static_cast<const T*>(nullptr), g, r);
        const std::uint32_t seed_site = std::uint32_t(g.uni() * double(n));
        for (std::uint32_t i = t; i < n; i += stride) parent[i] = i;
        if (threadIdx.x == 0) block_count = 0;
        if (!grid_sync(&ctl->bar)) return;

        const std::uint64_t kbond = key_base(key_seed(seed, counter, kTagBond));
        for (std::uint32_t i = t; i < n; i += stride) {
            const std::size_t deg = m.degree(i);
            for (std::size_t a = 0; a < deg; ++a) {
                const auto b = bond_of(m, i, a);
                const std::uint32_t j = std::uint32_t(b.j);
                if (j <= i) continue;
                T nb[D];
                reflect<T, D>(m.data() + std::size_t(j) * D, r, nb);
                const double dE = m.energy_diff_bond(i, b, nb);
                if (!(beta * dE > 0.0)) continue;  // p = 1 - exp(-beta dE) <= 0: never active
                Rng u(KeyedPcg::open(kbond, m.bond_id(i, a)));
                if (activates(u.uni(), beta * dE)) uf_unite(parent, i, j, &ctl->uf_status);
            }
        }
        if (!grid_sync(&ctl->bar)) return;

        // the seed's root, found once per block (the trees are fixed in this phase)
        __shared__ std::uint32_t root_sh;
        if (threadIdx.x == 0) root_sh = uf_root(parent, seed_site, &ctl->uf_status);
        __syncthreads();
        const std::uint32_t root = root_sh;
        unsigned long long mine = 0;
        for (std::uint32_t i = t; i < n; i += stride) {
            if (uf_root(parent, i, &ctl->uf_status) != root) continue;
            T prop[D];
            reflect<T, D>(m.data() + std::size_t(i) * D, r, prop);
            m.update(i, prop);
            ++mine;
        }
        if (mine) atomicAdd(&block_count, mine);
        __syncthreads();
        if (threadIdx.x == 0 && block_count) atomicAdd(sizes + f, block_count);
        if (!grid_sync(&ctl->bar)) return;
        touched += __ldcg(sizes + f);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctl->done = f + 1;
            ctl->touched = touched;
        }
        if (target > 0 && touched >= target) return;
    }
}

// Whether the a-th bond of i (j > i) is active in this flip: the same test,
// draw and key as wolff_flips.
template <class M, class T, std::size_t D>
__device__ __forceinline__ bool bond_active(const M& m, std::uint32_t i, std::size_t a,
                                            const typename M::bond_type& b, const T* r, double beta,
                                            std::uint64_t kbond)
{
    T nb[D];
    reflect<T, D>(m.data() + std::size_t(b.j) * D, r, nb);
    const double dE = m.energy_diff_bond(i, b, nb);
    if (!(beta * dE > 0.0)) return false;
    Rng u(KeyedPcg::open(kbond, m.bond_id(i, a)));
    return activates(u.uni(), beta * dE);
}

// Reference sites per shared-memory tile (16-bit local labels, 8 KB).  Larger
// tiles cut the crossing bonds but leave blocks without a tile, smaller ones
// send more bonds to the global list: on a 2048^2 flip, 16,384 took 0.68 ms,
// 2,048 took 0.57 ms and 4,096 0.42 ms.
constexpr std::uint32_t kWolffTile = 4096;

// Local root of t in a tile's shared-memory forest (links point to smaller t).
__device__ __forceinline__ std::uint32_t tile_root(unsigned short* lab, std::uint32_t t)
{
    for (std::uint32_t it = 0; it < kWolffTile; ++it) {
        const std::uint32_t p = *(volatile unsigned short*)(lab + t);
        if (p == t) return t;
        const std::uint32_t gp = *(volatile unsigned short*)(lab + p);
        if (gp != p) *(volatile unsigned short*)(lab + t) = (unsigned short)gp;
        t = gp;
    }
    return t;  // unreachable: each step moves to a smaller index
}

__device__ __forceinline__ void tile_unite(unsigned short* lab, std::uint32_t a, std::uint32_t b)
{
    for (std::uint32_t it = 0; it < 4 * kWolffTile; ++it) {
        a = tile_root(lab, a);
        b = tile_root(lab, b);
        if (a == b) return;
        if (a > b) {
            const std::uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(lab + b, (unsigned short)b, (unsigned short)a) == b) return;
    }
}

// wolff_flips with the labelling done in two levels.  Each block takes tiles
// of kWolffTile consecutive reference sites (site_of / dev_of translate to and
// from the device numbering): the active bonds inside a tile are united in
// shared memory, every site's global parent is set to its tile root, and the
// active bonds between tiles go to a list that a second phase unites in
// global memory.  Same bonds, draws and keys as wolff_flips, so the same
// clusters; far fewer global unions and shallow global trees.
template <class M, class A>
__global__ void __launch_bounds__(kThreads) wolff_flips_tiled(M m, A axis, double beta, std::uint64_t seed,
                                                              std::uint64_t flip0, std::uint32_t max_flips,
                                                              std::uint64_t target, std::uint32_t* parent,
                                                              unsigned long long* sizes, WolffControl* ctl,
                                                              const std::uint32_t* __restrict__ site_of,
                                                              const std::uint32_t* __restrict__ dev_of,
                                                              uint2* xlist, unsigned long long xcap)
{
    using T = typename M::value_type;
    constexpr std::size_t D = M::size;
    __shared__ unsigned short lab[kWolffTile];
    __shared__ unsigned long long block_count;
    __shared__ std::uint32_t root_sh;
    const std::uint32_t n = std::uint32_t(m.sites());
    const std::uint32_t tiles = (n + kWolffTile - 1) / kWolffTile;
    unsigned long long touched = 0;
    for (std::uint32_t f = 0; f < max_flips; ++f) {
        const std::uint64_t counter = flip0 + f;
        Rng g(KeyedPcg::open_key(seed, counter, kTagAxis, 0));
        T r[D];
        axis.sample(static_cast<const T*>(nullptr), g, r);
        const std::uint32_t seed_site = std::uint32_t(g.uni() * double(n));
        const std::uint64_t kbond = key_base(key_seed(seed, counter, kTagBond));
        if (threadIdx.x == 0) block_count = 0;

        // tiles: local unions in shared memory, crossing bonds to the list
        for (std::uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
            const std::uint32_t s0 = tile * kWolffTile;
            const std::uint32_t len = min(kWolffTile, n - s0);
            for (std::uint32_t t = threadIdx.x; t < len; t += blockDim.x) lab[t] = (unsigned short)t;
            __syncthreads();
            for (std::uint32_t t = threadIdx.x; t < len; t += blockDim.x) {
                const std::uint32_t i = dev_of[s0 + t];
                const std::size_t deg = m.degree(i);
                for (std::size_t a = 0; a < deg; ++a) {
                    const auto b = bond_of(m, i, a);
                    const std::uint32_t j = std::uint32_t(b.j);
                    if (j <= i || !bond_active<M, T, D>(m, i, a, b, r, beta, kbond)) continue;
                    const std::uint32_t sj = site_of[j];
                    if (sj - s0 < len) {
                        tile_unite(lab, t, sj - s0);
                    } else {
                        const unsigned long long at = atomicAdd(&ctl->xcount, 1ull);
                        if (at < xcap) xlist[at] = make_uint2(i, j);
                        else atomicOr(&ctl->uf_status, 4u);
                    }
                }
            }
            __syncthreads();
            for (std::uint32_t t = threadIdx.x; t < len; t += blockDim.x)
                parent[dev_of[s0 + t]] = dev_of[s0 + tile_root(lab, t)];
            __syncthreads();
        }
        if (!grid_sync(&ctl->bar)) return;

        // crossing bonds: global unions
        const unsigned long long xn = min(__ldcg(&ctl->xcount), xcap);
        for (unsigned long long e = blockIdx.x * std::uint64_t(blockDim.x) + threadIdx.x; e < xn;
             e += std::uint64_t(gridDim.x) * blockDim.x) {
            const uint2 bj = xlist[e];
            uf_unite(parent, bj.x, bj.y, &ctl->uf_status);
        }
        if (!grid_sync(&ctl->bar)) return;

        // the seed's cluster, as in wolff_flips
        if (threadIdx.x == 0) root_sh = uf_root(parent, seed_site, &ctl->uf_status);
        __syncthreads();
        const std::uint32_t root = root_sh;
        unsigned long long mine = 0;
        for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            if (uf_root(parent, i, &ctl->uf_status) != root) continue;
            T prop[D];
            reflect<T, D>(m.data() + std::size_t(i) * D, r, prop);
            m.update(i, prop);
            ++mine;
        }
        if (mine) atomicAdd(&block_count, mine);
        __syncthreads();
        if (threadIdx.x == 0 && block_count) atomicAdd(sizes + f, block_count);
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->xcount = 0;  // read by no one until the next flip's list
        if (!grid_sync(&ctl->bar)) return;
        touched += __ldcg(sizes + f);
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            ctl->done = f + 1;
            ctl->touched = touched;
        }
        if (target > 0 && touched >= target) return;
    }
}

}  // namespace detail

// ------------------------------------------------------------------ driver

// Runs the barrier's failure path once (a second or two): true when the wait
// ran out, set the status bit that the drivers turn into an exception, and
// returned instead of hanging.
inline bool barrier_timeout_selftest()
{
    Buffer<detail::Control> ctl(1);
    Buffer<unsigned> status(2);
    cuda_check(cudaMemset(ctl.data(), 0, sizeof(detail::Control)), "reset");
    cuda_check(cudaMemset(status.data(), 0, 2 * sizeof(unsigned)), "reset");
    detail::barrier_timeout_probe<<<2, detail::kThreads>>>(ctl.data(), status.data());
    cuda_check(cudaGetLastError(), "probe launch");
    cuda_check(cudaDeviceSynchronize(), "probe");
    unsigned h[2] = {0, 0};
    cuda_check(cudaMemcpy(h, status.data(), sizeof h, cudaMemcpyDeviceToHost), "probe status");
    return (h[0] & 1u) != 0u && h[1] == 0u;
}

// Metropolis (driver.hpp:17-66) for a device model M and proposal Q.  The
// reference's rng argument becomes a seed: every sweep keys its own streams
// from (seed, sweep counter), so a chain continues exactly after
// set_sweeps() and runs the same on any grid size.
template <ModelLike M, class Q>
    requires Proposal<Q, typename M::value_type>
class Metropolis
{
public:
    // The driver keeps a reference to classes: a temporary is refused.
    Metropolis(M, Q, ClassTable&&, std::uint64_t, double, cudaStream_t = nullptr) = delete;
    Metropolis(M model, Q proposal, const ClassTable& classes, std::uint64_t seed, double beta,
               cudaStream_t stream = nullptr)
        : model_(model), proposal_(proposal), classes_(classes), seed_(seed), beta_(beta), stream_(stream),
          ctl_(1)
    {
        if (classes.host().sites() != model.sites())
            throw std::invalid_argument("colour classes do not cover the model's sites");
        grid_ = detail::cooperative_grid(reinterpret_cast<const void*>(&detail::metropolis_sweeps<M, Q>),
                                         (classes.host().largest() + detail::kThreads - 1) / detail::kThreads);
    }

    // One pass over every site (driver.hpp:29-43).
    void sweep() { run(1); }

    // n passes (driver.hpp:46-50) in one launch; returns when they are done.
    void run(std::size_t sweeps)
    {
        enqueue(sweeps);
        cuda_check(cudaStreamSynchronize(stream_), "Metropolis::run");
        check();
    }

    // Runs n sweeps, calling observe(*this) after each (driver.hpp:55-62).
    template <class F>
    void sample(std::size_t sweeps, F&& observe)
    {
        for (std::size_t k = 0; k < sweeps; ++k) {
            run(1);
            observe(std::as_const(*this));
        }
    }

    // The launch alone, ordered on the stream; check() after a sync.
    void enqueue(std::size_t sweeps)
    {
        while (sweeps > 0) {
            const std::uint32_t chunk = std::uint32_t(std::min<std::size_t>(sweeps, 1u << 30));
            cuda_check(cudaMemsetAsync(ctl_.data(), 0, sizeof(detail::Control), stream_), "reset barrier");
            M m = model_;
            Q q = proposal_;
            const std::uint32_t* order = classes_.order();
            const std::uint32_t* begin = classes_.begin();
            std::uint32_t nc = classes_.host().count();
            double beta = beta_;
            std::uint64_t seed = seed_, sweep0 = sweeps_;
            std::uint32_t n = chunk;
            detail::Control* ctl = ctl_.data();
            detail::NoObservable obs;
            std::uint64_t obs_count = 0;
            double* partial = nullptr;
            double* records = nullptr;
            // every kernel parameter, the unused observable ones included
            void* args[] = {&m, &q, &order, &begin, &nc, &beta, &seed, &sweep0, &n, &ctl, &obs, &obs_count, &partial,
                            &records};
            cuda_check(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&detail::metropolis_sweeps<M, Q>),
                                                   dim3(grid_), dim3(detail::kThreads), args, 0, stream_),
                       "Metropolis launch");
            sweeps_ += chunk;
            sweeps -= chunk;
        }
    }

    // Throws if a barrier wait of an earlier launch ran out.
    void check() const
    {
        detail::Control h{};
        cuda_check(cudaMemcpyAsync(&h, ctl_.data(), sizeof h, cudaMemcpyDeviceToHost, stream_), "read status");
        cuda_check(cudaStreamSynchronize(stream_), "read status");
        if (h.status != 0u) throw std::runtime_error("Metropolis: a grid barrier wait ran out");
    }

    // n sweeps in one launch, observing on the device: after sweep s,
    // records[s] (host, n entries) = FP64 sum of obs(model, x) over x < count.
    // obs is a device functor double(const M&, std::uint64_t).  The
    // observation is driver.hpp:54-61's observe hook without a host round
    // trip per sweep.
    template <class O>
    void record(std::size_t sweeps, O obs, std::uint64_t count, double* records)
    {
        if (sweeps == 0) return;
        if (sweeps >= (std::size_t(1) << 30)) throw std::invalid_argument("record: at most 2^30 sweeps per call");
        const void* k = reinterpret_cast<const void*>(&detail::metropolis_sweeps<M, Q, O>);
        const std::uint32_t grid =
            detail::cooperative_grid(k, (classes_.host().largest() + detail::kThreads - 1) / detail::kThreads);
        if (rec_partial_.size() < grid) rec_partial_ = Buffer<double>(grid);
        if (rec_out_.size() < sweeps) rec_out_ = Buffer<double>(std::max<std::size_t>(sweeps, 64));
        cuda_check(cudaMemsetAsync(ctl_.data(), 0, sizeof(detail::Control), stream_), "reset barrier");
        M m = model_;
        Q q = proposal_;
        const std::uint32_t* order = classes_.order();
        const std::uint32_t* begin = classes_.begin();
        std::uint32_t nc = classes_.host().count();
        double beta = beta_;
        std::uint64_t seed = seed_, sweep0 = sweeps_;
        std::uint32_t n = std::uint32_t(sweeps);
        detail::Control* ctl = ctl_.data();
        std::uint64_t cnt = count;
        double* part = rec_partial_.data();
        double* out = rec_out_.data();
        void* args[] = {&m, &q, &order, &begin, &nc, &beta, &seed, &sweep0, &n, &ctl, &obs, &cnt, &part, &out};
        cuda_check(cudaLaunchCooperativeKernel(k, dim3(grid), dim3(detail::kThreads), args, 0, stream_),
                   "Metropolis launch");
        sweeps_ += sweeps;
        cuda_check(cudaMemcpyAsync(records, out, sweeps * sizeof(double), cudaMemcpyDeviceToHost, stream_), "records");
        cuda_check(cudaStreamSynchronize(stream_), "Metropolis::record");
        check();
    }
    // The energy after each of n sweeps: sum of energy_at (EnergyModel; a
    // pair model counts every bond twice) or of cell_energy (CellEnergyModel).
    void record_energy(std::size_t sweeps, double* records)
        requires EnergyModel<M> || CellEnergyModel<M>
    {
        if constexpr (CellEnergyModel<M>)
            record(sweeps, detail::CellEnergyOf{}, model_.cells(), records);
        else
            record(sweeps, detail::EnergyAtOf{}, model_.sites(), records);
    }

    // Sum over cells of cell_energy (model/cell.hpp:58-62), FP64.
    double total_energy() const
        requires CellEnergyModel<M>
    {
        return detail::device_sum(model_, model_.cells(), detail::CellEnergyOf{}, stream_, sum_partial_);
    }
    // Sum over sites of energy_at (model.hpp:93-96), FP64; for a pair model
    // every bond appears twice.
    double energy_at_sum() const
        requires EnergyModel<M>
    {
        return detail::device_sum(model_, model_.sites(), detail::EnergyAtOf{}, stream_, sum_partial_);
    }

    const M& model() const noexcept { return model_; }
    std::uint64_t sweeps() const noexcept { return sweeps_; }
    void set_sweeps(std::uint64_t s) noexcept { sweeps_ = s; }
    double beta() const noexcept { return beta_; }
    void set_beta(double b) noexcept { beta_ = b; }
    std::uint32_t grid() const noexcept { return grid_; }

private:
    M model_;
    Q proposal_;
    const ClassTable& classes_;
    std::uint64_t seed_;
    double beta_;
    cudaStream_t stream_;
    Buffer<detail::Control> ctl_;
    mutable Buffer<double> sum_partial_;  // energy sums' block partials, reused
    Buffer<double> rec_partial_, rec_out_;  // record()'s partials and records, reused
    std::uint32_t grid_ = 1;
    std::uint64_t sweeps_ = 0;
};

// Wolff (driver.hpp:85-210) for a device WolffModel M and axis proposal A.
// Flip f keys its draws by (seed, f), so set_flips() continues a chain
// exactly.  The device needs no stack: every bond is tested at once, a
// union-find labels the active bonds' components, and the seed's component is
// reflected, in one cooperative launch for many flips.
template <WolffModel M, class A>
    requires Axis<A, typename M::value_type>
class Wolff
{
public:
    Wolff(M model, A axis, std::uint64_t seed, double beta, cudaStream_t stream = nullptr)
        : model_(model), axis_(axis), seed_(seed), beta_(beta), stream_(stream), parent_(model.sites()),
          sizes_(kCapacity), ctl_(1)
    {
        if (model.sites() == 0 || model.sites() >= (std::uint64_t(1) << 32))
            throw std::invalid_argument("Wolff: the model needs 1 to 2^32 - 1 sites");
        grid_ = detail::cooperative_grid(kernel(), (model.sites() + detail::kThreads - 1) / detail::kThreads);
    }
    // With the tables the model was made from (PairTables, LatticeTables):
    // the labelling runs in shared-memory tiles of consecutive reference
    // sites first (wolff_flips_tiled), with the same clusters.  The driver
    // keeps pointers into the tables, which must outlive it (a temporary is
    // refused).
    template <class Tables>
        requires(!std::is_lvalue_reference_v<Tables>)
    Wolff(M, A, Tables&&, std::uint64_t, double, cudaStream_t = nullptr) = delete;
    template <class Tables>
        requires requires(const Tables& t) {
            { t.device_order() } -> std::convertible_to<const std::uint32_t*>;
            { t.device_position() } -> std::convertible_to<const std::uint32_t*>;
            { t.bond_slots() } -> std::convertible_to<std::uint64_t>;
        }
    Wolff(M model, A axis, const Tables& layout, std::uint64_t seed, double beta, cudaStream_t stream = nullptr)
        : Wolff(model, axis, seed, beta, stream)
    {
        if (layout.sites() != model.sites()) throw std::invalid_argument("Wolff: tables of another size");
        site_of_ = layout.device_order();
        dev_of_ = layout.device_position();
        xlist_ = Buffer<uint2>(std::max<std::uint64_t>(1, layout.bond_slots()));
        grid_ = detail::cooperative_grid(kernel(), (model.sites() + detail::kThreads - 1) / detail::kThreads);
    }

    // One cluster flip; returns how many sites it flipped (driver.hpp:104-162).
    std::size_t flip()
    {
        std::uint64_t size = 0;
        launch(1, 0, &size);
        return std::size_t(size);
    }

    // n flips in launches of up to 65,536; sizes (n entries) may be null.
    void flips(std::size_t n, std::uint64_t* sizes = nullptr)
    {
        while (n > 0) {
            const std::uint32_t chunk = std::uint32_t(std::min<std::size_t>(n, kCapacity));
            launch(chunk, 0, sizes);
            if (sizes) sizes += chunk;
            n -= chunk;
        }
    }

    // Flips until the flipped sites add up to the lattice (driver.hpp:163-173);
    // returns the sites flipped.
    std::uint64_t sweep()
    {
        std::uint64_t need = model_.sites(), total = 0;
        while (need > 0) {
            const std::uint64_t got = launch(kCapacity, need, nullptr);
            total += got;
            need = got >= need ? 0 : need - got;
        }
        return total;
    }

    // n sweeps (driver.hpp:175-180).
    void run(std::size_t sweeps)
    {
        for (std::size_t k = 0; k < sweeps; ++k) sweep();
    }

    // Flips n clusters, calling observe(*this) after each (driver.hpp:182-190).
    template <class F>
    void sample(std::size_t flips, F&& observe)
    {
        for (std::size_t k = 0; k < flips; ++k) {
            flip();
            observe(std::as_const(*this));
        }
    }

    // Mean cluster size over every flip so far (driver.hpp:193-197).
    double mean_cluster_size() const { return flips_ == 0 ? 0.0 : size_sum_ / double(flips_); }

    double total_energy() const
        requires CellEnergyModel<M>
    {
        return detail::device_sum(model_, model_.cells(), detail::CellEnergyOf{}, stream_, sum_partial_);
    }
    double energy_at_sum() const
        requires EnergyModel<M>
    {
        return detail::device_sum(model_, model_.sites(), detail::EnergyAtOf{}, stream_, sum_partial_);
    }

    const M& model() const noexcept { return model_; }
    std::uint64_t flips_done() const noexcept { return flips_; }
    void set_flips(std::uint64_t f) noexcept { flips_ = f; }
    double beta() const noexcept { return beta_; }
    void set_beta(double b) noexcept { beta_ = b; }
    std::uint32_t grid() const noexcept { return grid_; }

private:
    static constexpr std::uint32_t kCapacity = 1u << 16;
    const void* kernel() const
    {
        return site_of_ ? reinterpret_cast<const void*>(&detail::wolff_flips_tiled<M, A>)
                        : reinterpret_cast<const void*>(&detail::wolff_flips<M, A>);
    }

    // Up to max_flips flips (fewer once target sites are flipped, target > 0);
    // returns the sites flipped and writes one size per flip to sizes_out.
    std::uint64_t launch(std::uint32_t max_flips, std::uint64_t target, std::uint64_t* sizes_out)
    {
        cuda_check(cudaMemsetAsync(ctl_.data(), 0, sizeof(detail::WolffControl), stream_), "reset control");
        cuda_check(cudaMemsetAsync(sizes_.data(), 0, max_flips * sizeof(unsigned long long), stream_), "reset sizes");
        M m = model_;
        A a = axis_;
        double beta = beta_;
        std::uint64_t seed = seed_, flip0 = flips_;
        std::uint32_t nf = max_flips;
        std::uint64_t tgt = target;
        std::uint32_t* parent = parent_.data();
        unsigned long long* sizes = sizes_.data();
        detail::WolffControl* ctl = ctl_.data();
        const std::uint32_t* site_of = site_of_;
        const std::uint32_t* dev_of = dev_of_;
        uint2* xlist = xlist_.data();
        unsigned long long xcap = xlist_.size();
        void* args[] = {&m, &a, &beta, &seed, &flip0, &nf, &tgt, &parent, &sizes, &ctl, &site_of, &dev_of, &xlist, &xcap};
        cuda_check(cudaLaunchCooperativeKernel(kernel(), dim3(grid_), dim3(detail::kThreads), args, 0, stream_),
                   "Wolff launch");
        detail::WolffControl h{};
        cuda_check(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, stream_), "read control");
        cuda_check(cudaStreamSynchronize(stream_), "Wolff");
        if (h.bar.status != 0u) throw std::runtime_error("Wolff: a grid barrier wait ran out");
        if (h.uf_status & 4u) throw std::runtime_error("Wolff: the crossing-bond list overflowed");
        if (h.uf_status != 0u) throw std::runtime_error("Wolff: a union-find walk ran past its limit");
        std::vector<unsigned long long> sz(h.done);
        if (h.done)
            cuda_check(cudaMemcpy(sz.data(), sizes, h.done * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                       "read sizes");
        for (std::uint32_t k = 0; k < h.done; ++k) {
            size_sum_ += double(sz[k]);
            if (sizes_out) sizes_out[k] = sz[k];
        }
        flips_ += h.done;
        return h.touched;
    }

    M model_;
    A axis_;
    std::uint64_t seed_;
    double beta_;
    cudaStream_t stream_;
    Buffer<std::uint32_t> parent_;
    Buffer<unsigned long long> sizes_;
    Buffer<detail::WolffControl> ctl_;
    const std::uint32_t* site_of_ = nullptr;  // tiled labelling (with tables)
    const std::uint32_t* dev_of_ = nullptr;
    Buffer<uint2> xlist_;
    mutable Buffer<double> sum_partial_;  // energy sums' block partials, reused
    std::uint32_t grid_ = 1;
    std::uint64_t flips_ = 0;
    double size_sum_ = 0.0;
};

}  // namespace umc::gpu::device
