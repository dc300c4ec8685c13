// umc/driver.hpp -- Metropolis<M,Q,R> and Wolff<M,A,R> with the reference's
// constructors and members (driver.hpp:17-68, :92-210), running on the GPU.
// A PairModel/CellModel with a user-written term, in a file compiled by nvcc,
// runs through umc/device.cuh instead of an engine chain.
//
// A driver owns one device chain (umc_chain) built from the model, its
// proposal or axis, and the key of its Pcg32.  run() and the Wolff flips go to
// the device; sample() calls observe(model) after every sweep or flip, and the
// model's data() then reads the device field back.  For long measurements
// without per-step host work, records() returns the chain's FP64 observables
// (E, magnetisation or S, plaquette, Q; see UMC_OBS_STRIDE) of the last run.
#pragma once

#include <cstddef>
#include <cstdint>
#include <limits>
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

#include "detail.hpp"
#include "dof.hpp"
#include "generic.hpp"
#include "models.hpp"
#include "rng.hpp"

namespace umc::gpu {

namespace detail {

template <class Q>
struct ProposalKind;

template <>
struct ProposalKind<Flip>
{
    static void set(umc_chain_desc& d, const Flip&) { d.proposal = UMC_PROPOSAL_FLIP; }
};
template <std::size_t N, class T>
struct ProposalKind<UniformSphereN<N, T>>
{
    static void set(umc_chain_desc& d, const UniformSphereN<N, T>&) { d.proposal = UMC_PROPOSAL_SPHERE; }
};
template <std::size_t N, class T>
struct ProposalKind<LocalRotation<N, T>>
{
    static void set(umc_chain_desc& d, const LocalRotation<N, T>& q)
    {
        d.proposal = UMC_PROPOSAL_ROTATION;
        d.width = double(q.delta);
    }
};
template <>
struct ProposalKind<U1Shift>
{
    static void set(umc_chain_desc& d, const U1Shift& q)
    {
        d.proposal = UMC_PROPOSAL_U1SHIFT;
        d.width = q.width;
    }
};
template <std::size_t N>
struct ProposalKind<SUShift<N>>
{
    static void set(umc_chain_desc& d, const SUShift<N>& q)
    {
        d.proposal = UMC_PROPOSAL_SUSHIFT;
        d.width = q.width;
    }
};
template <class Q>
struct ProposalKind<Hits<Q>>
{
    static void set(umc_chain_desc& d, const Hits<Q>& q)
    {
        ProposalKind<Q>::set(d, q.inner);
        d.hits = q.hits;
    }
};

template <class A>
struct AxisKind;
template <>
struct AxisKind<FixedAxis>
{
    static constexpr int32_t value = UMC_AXIS_FIXED;
};
template <std::size_t N, class T>
struct AxisKind<UniformSphereN<N, T>>
{
    static constexpr int32_t value = UMC_AXIS_SPHERE;
};

template <class R>
std::uint64_t key_of(const R& rng)
{
    return rng.key();
}

// Drivers of umc/device.cuh for models with a user-written term; defined in
// umc/device_facade.cuh, which umc/umc.hpp includes in nvcc builds.
template <class M, class Q>
std::unique_ptr<UserRunner> make_user_metropolis(M& model, const Q& proposal, std::uint64_t key, double beta);
template <class M, class A>
std::unique_ptr<UserRunner> make_user_wolff(M& model, const A& axis, std::uint64_t key, double beta);

// A model the engine runs itself: the example models and the PairModel /
// CellModel of the built-in terms describe their chain.
template <class M>
concept EngineModel = requires(const M& m) { m.chain_desc(); };

}  // namespace detail

#define UMC_DRIVER_MODEL_CHECK(M)                                                                          \
    static_assert(detail::EngineModel<M> || detail::UserTermModel<M>,                                     \
                  "the facade's drivers run the engine's models and PairModel / CellModel with any term; " \
                  "a model type of your own runs on the device through umc/device.cuh "                   \
                  "(umc::gpu::device::Metropolis / Wolff, built by nvcc)")

template <class M, class Q, class R>
class Metropolis
{
public:
    Metropolis(M& model, Q proposal, R rng, double beta)
        : model_(model), proposal_(std::move(proposal)), rng_(std::move(rng)), beta_(beta)
    {
        UMC_DRIVER_MODEL_CHECK(M);
        if constexpr (detail::UserTermModel<M>) {
            user_ = detail::make_user_metropolis(model_, proposal_, detail::key_of(rng_), beta_);
        } else {
            umc_chain_desc d = model_.chain_desc();
            detail::ProposalKind<Q>::set(d, proposal_);
            d.seed = detail::key_of(rng_);
            chain_ = detail::make_chain(d);
        }
    }
    Metropolis(const Metropolis&) = delete;
    Metropolis& operator=(const Metropolis&) = delete;
    ~Metropolis()
    {
        if constexpr (detail::UserTermModel<M>)
            model_.detach(static_cast<detail::DeviceCopy*>(user_.get()));
        else
            model_.detach(chain_.get());
    }

    // One pass over every site.
    void sweep() { run(1); }

    // n sweeps (one call into the engine).  A user-written term runs in one
    // launch of umc/device.cuh's Metropolis, which records the energy after
    // every sweep (records() slot 0; the other slots are NaN).
    void run(std::size_t sweeps)
    {
        if (!sweeps) return;
        if constexpr (detail::UserTermModel<M>) {
            auto* copy = static_cast<detail::DeviceCopy*>(user_.get());
            model_.attach(copy);
            std::vector<double> e(sweeps);
            user_->run_energy(sweeps, e.data());
            model_.mark_device(copy);
            // the energy only: a user term defines no magnetisation or plaquette
            records_.assign(sweeps * UMC_OBS_STRIDE, std::numeric_limits<double>::quiet_NaN());
            for (std::size_t k = 0; k < sweeps; ++k) records_[k * UMC_OBS_STRIDE] = e[k];
        } else {
            model_.attach(chain_.get());
            records_.assign(sweeps * UMC_OBS_STRIDE, 0.0);
            detail::check(umc_metropolis_run(chain_.get(), beta_, sweeps, records_.data()));
            model_.mark_device(chain_.get());
        }
    }

    // n sweeps, observe(model) after each.
    template <class F>
    void sample(std::size_t sweeps, F&& observe)
    {
        for (std::size_t k = 0; k < sweeps; ++k) {
            run(1);
            observe(std::as_const(model_));
        }
    }

    // FP64 observables of the sweeps of the last run() (UMC_OBS_STRIDE each).
    const std::vector<double>& records() const noexcept { return records_; }
    umc_chain* chain() const noexcept { return chain_.get(); }

private:
    M& model_;
    Q proposal_;
    R rng_;
    double beta_;
    detail::ChainPtr chain_;
    std::unique_ptr<detail::UserRunner> user_;
    std::vector<double> records_;
};

template <class M, class A, class R>
class Wolff
{
public:
    Wolff(M& model, A axis, R rng, double beta) : model_(model), axis_(std::move(axis)), rng_(std::move(rng)), beta_(beta)
    {
        static_assert(WolffModel<M>, "Wolff needs a pair model (degree, bonds, energy_diff_bond)");
        UMC_DRIVER_MODEL_CHECK(M);
        if constexpr (detail::UserTermModel<M>) {
            user_ = detail::make_user_wolff(model_, axis_, detail::key_of(rng_), beta_);
        } else {
            umc_chain_desc d = model_.chain_desc();
            d.proposal = std::is_same_v<A, FixedAxis> ? UMC_PROPOSAL_FLIP : UMC_PROPOSAL_SPHERE;
            d.wolff_axis = detail::AxisKind<A>::value;
            d.seed = detail::key_of(rng_);
            chain_ = detail::make_chain(d);
        }
    }
    Wolff(const Wolff&) = delete;
    Wolff& operator=(const Wolff&) = delete;
    ~Wolff()
    {
        if constexpr (detail::UserTermModel<M>)
            model_.detach(static_cast<detail::DeviceCopy*>(user_.get()));
        else
            model_.detach(chain_.get());
    }

    // One cluster flip; returns how many sites it flipped.
    std::size_t flip()
    {
        std::uint64_t size = 0;
        flips(1, &size);
        return std::size_t(size);
    }

    // Flips until the flipped sites add up to one lattice.  A user-written
    // term does this in the device Wolff's own launch, which stops there.
    void sweep()
    {
        if constexpr (detail::UserTermModel<M>) {
            auto* copy = static_cast<detail::DeviceCopy*>(user_.get());
            model_.attach(copy);
            std::size_t f = 0;
            double s = 0.0;
            user_->wolff_sweep(f, s);
            model_.mark_device(copy);
            n_flips_ += f;
            size_sum_ += s;
        } else {
            std::size_t touched = 0;
            do {
                touched += flip();
            } while (touched < model_.sites());
        }
    }

    void run(std::size_t sweeps)
    {
        for (std::size_t k = 0; k < sweeps; ++k) sweep();
    }

    // n flips, observe(model) after each.
    template <class F>
    void sample(std::size_t n, F&& observe)
    {
        for (std::size_t k = 0; k < n; ++k) {
            flip();
            observe(std::as_const(model_));
        }
    }

    // n flips in one engine call; sizes (n entries) may be null.
    void flips(std::size_t n, std::uint64_t* sizes)
    {
        if (!n) return;
        std::vector<std::uint64_t> s(n);
        if constexpr (detail::UserTermModel<M>) {
            auto* copy = static_cast<detail::DeviceCopy*>(user_.get());
            model_.attach(copy);
            user_->run(n, s.data());
            model_.mark_device(copy);
        } else {
            model_.attach(chain_.get());
            detail::check(umc_wolff_run(chain_.get(), beta_, n, s.data(), nullptr));
            model_.mark_device(chain_.get());
        }
        for (std::size_t k = 0; k < n; ++k) {
            size_sum_ += double(s[k]);
            if (sizes) sizes[k] = s[k];
        }
        n_flips_ += n;
    }

    double mean_cluster_size() const { return n_flips_ == 0 ? 0.0 : size_sum_ / double(n_flips_); }
    umc_chain* chain() const noexcept { return chain_.get(); }

private:
    M& model_;
    A axis_;
    R rng_;
    double beta_;
    detail::ChainPtr chain_;
    std::unique_ptr<detail::UserRunner> user_;
    std::size_t n_flips_ = 0;
    double size_sum_ = 0.0;
};

}  // namespace umc::gpu

#undef UMC_DRIVER_MODEL_CHECK
