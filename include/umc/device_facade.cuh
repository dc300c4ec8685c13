// umc/device_facade.cuh -- the facade's Metropolis and Wolff on user-written
// terms (nvcc builds; umc/umc.hpp includes this file when __CUDACC__ is set).
//
// A reference program that builds PairModel<D, Term, PairGraph<>> or
// CellModel<D, Term, CellComplex<A>> with a term of its own (term/cell.hpp:
// 10-25) keeps its code; the term's energy and delta, and the proposal or
// axis, are marked __host__ __device__.  The facade's drivers then hand the
// model to umc/device.cuh: its tables (colour-major on the device), a device
// copy of the field, and the generic Metropolis or Wolff kernel instantiated
// for the user's types.  The model's host field (data()) follows the device
// copy as it does for the engine's chains.
#pragma once

#include "device.cuh"
#include "driver.hpp"
#include "generic.hpp"

#include <memory>

namespace umc::gpu::detail {

// The umc/device.cuh side of a facade model with a user-written term.
template <class M>
struct UserDevice;

template <class D, class Term, class G>
struct UserDevice<PairModel<D, Term, G>>
{
    using Tables = device::PairTables;
    using View = device::PairModel<D, Term>;
    static const umc_graph* handle(const PairModel<D, Term, G>& m) { return m.graph().handle(); }
};

template <class D, class Term, class L>
struct UserDevice<CellModel<D, Term, L>>
{
    using Tables = device::CellTables;
    using View = device::CellModel<D, Term>;
    static const umc_cells* handle(const CellModel<D, Term, L>& m) { return m.list().handle(); }
};

// Tables and the device copy of the field, in the model's data() layout on
// the host and the colour-major numbering on the device.
template <class M>
class UserField : public UserRunner
{
protected:
    using U = UserDevice<M>;
    using D = typename M::dof_type;
    using T = typename D::dtype;

    explicit UserField(const M& m) : tables_(U::handle(m)), field_(std::size_t(tables_.sites()) * D::size) {}

    typename U::View view(const M& m) { return tables_.template model<D>(field_.data(), m.term()); }

public:
    void push(const void* host) override { tables_.upload(field_, static_cast<const T*>(host), D::size); }
    void pull(void* host) const override { tables_.download(field_, static_cast<T*>(host), D::size); }

protected:
    typename U::Tables tables_;
    device::Buffer<T> field_;
};

template <class M, class Q>
class UserMetropolis final : public UserField<M>
{
public:
    UserMetropolis(const M& m, const Q& q, std::uint64_t key, double beta)
        : UserField<M>(m), mc_(this->view(m), q, this->tables_.classes(), key, beta)
    {}
    void run(std::size_t n, std::uint64_t*) override { mc_.run(n); }
    void wolff_sweep(std::size_t&, double&) override { throw std::logic_error("a Metropolis runner has no Wolff sweep"); }
    // E after each sweep: half the sum of energy_at for a pair model (every
    // bond counted at both ends), the sum of cell_energy for a cell model.
    void run_energy(std::size_t n, double* energy) override
    {
        mc_.record_energy(n, energy);
        if constexpr (!device::CellEnergyModel<typename UserDevice<M>::View>)
            for (std::size_t k = 0; k < n; ++k) energy[k] *= 0.5;
    }

private:
    device::Metropolis<typename UserDevice<M>::View, Q> mc_;
};

template <class M, class A>
class UserWolff final : public UserField<M>
{
public:
    UserWolff(const M& m, const A& a, std::uint64_t key, double beta)
        : UserField<M>(m), w_(this->view(m), a, this->tables_, key, beta)
    {}
    void run(std::size_t n, std::uint64_t* sizes) override { w_.flips(n, sizes); }
    void run_energy(std::size_t, double*) override { throw std::logic_error("Wolff records no energies"); }
    void wolff_sweep(std::size_t& flips, double& sites) override
    {
        const std::uint64_t f0 = w_.flips_done();
        sites += double(w_.sweep());
        flips += std::size_t(w_.flips_done() - f0);
    }

private:
    device::Wolff<typename UserDevice<M>::View, A> w_;
};

template <class M, class Q>
std::unique_ptr<UserRunner> make_user_metropolis(M& model, const Q& proposal, std::uint64_t key, double beta)
{
    return std::make_unique<UserMetropolis<M, Q>>(model, proposal, key, beta);
}

template <class M, class A>
std::unique_ptr<UserRunner> make_user_wolff(M& model, const A& axis, std::uint64_t key, double beta)
{
    return std::make_unique<UserWolff<M, A>>(model, axis, key, beta);
}

}  // namespace umc::gpu::detail
