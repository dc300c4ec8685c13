// umc/detail.hpp -- status codes -> the reference's exception types, handle
// ownership, and the host/device field synchronisation shared by the models
// (with a device chain of the engine, or with a device copy kept by a driver
// of umc/device.cuh for user-written terms).
#pragma once

#include <umc_b200.h>

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace umc::gpu::detail {

// Builder errors keep the reference's exception classes (lattice/*.hpp);
// everything else (CUDA, device timeouts, misuse) is a runtime_error.
inline void check(int status)
{
    if (status == UMC_OK) return;
    const std::string msg = umc_last_error();
    switch (status) {
    case UMC_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case UMC_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
    case UMC_ERR_OVERFLOW: throw std::overflow_error(msg);
    default: throw std::runtime_error("umc status " + std::to_string(status) + ": " + msg);
    }
}

struct GraphFree
{
    void operator()(umc_graph* g) const noexcept { umc_graph_destroy(g); }
};
struct CellsFree
{
    void operator()(umc_cells* c) const noexcept { umc_cells_destroy(c); }
};
struct ChainFree
{
    void operator()(umc_chain* c) const noexcept { umc_chain_destroy(c); }
};
using ChainPtr = std::unique_ptr<umc_chain, ChainFree>;

inline ChainPtr make_chain(const umc_chain_desc& d)
{
    umc_chain* c = nullptr;
    check(umc_chain_create(&d, &c));
    return ChainPtr(c);
}

// Host/device member marker for code that a user's nvcc translation unit may
// run on the device (proposals, axes, plaquette helpers); empty under g++.
#if defined(__CUDACC__)
#define UMC_FACADE_HD __host__ __device__
#else
#define UMC_FACADE_HD
#endif

// A device copy of a model's field kept by a driver of umc/device.cuh (user
// terms, nvcc builds): push() writes the host field (data() layout) to the
// device, pull() reads it back.
struct DeviceCopy
{
    virtual void push(const void* host) = 0;
    virtual void pull(void* host) const = 0;

protected:
    ~DeviceCopy() = default;
};

// A driver of umc/device.cuh behind a facade driver: Metropolis sweeps or
// Wolff flips on its own device copy of the field.
struct UserRunner : DeviceCopy
{
    virtual ~UserRunner() = default;
    virtual void run(std::size_t n, std::uint64_t* sizes) = 0;
    // n Metropolis sweeps with the total energy after each (observed on the
    // device); a Wolff runner has none.
    virtual void run_energy(std::size_t n, double* energy) = 0;
    // One Wolff sweep (flips until the flipped sites reach the lattice) in as
    // few launches as possible; adds its flips and flipped sites.
    virtual void wolff_sweep(std::size_t& flips, double& sites) = 0;
};

// A model's field on the host as scalars HS in the reference's data() layout,
// plus which device chain (or device copy) holds the newest copy.  Drivers call attach() before
// they run and mark_device() after; data() and update() call ensure_host()
// first.  DevT is the scalar type of the C ABI's set_field/get_field layout
// (int8 Ising spins, FP32 otherwise).
template <class HS, class DevT>
class Field
{
public:
    void attach(umc_chain* c) const
    {
        if (owner_ == c) return;
        ensure_host();
        std::vector<DevT> dev(host_.size());
        for (std::size_t k = 0; k < host_.size(); ++k) dev[k] = static_cast<DevT>(host_[k]);
        check(umc_chain_set_field(c, dev.data()));
        owner_ = c;
        copy_ = nullptr;
        host_valid_ = true;
    }
    void mark_device(umc_chain* c) const
    {
        owner_ = c;
        host_valid_ = false;
    }
    // A driver going away keeps its results in the host copy.
    void detach(umc_chain* c) const noexcept
    {
        if (owner_ != c) return;
        try {
            ensure_host();
        } catch (...) {
        }
        owner_ = nullptr;
        host_valid_ = true;
    }

    // The same for a device copy (user terms; HS is then the dtype itself).
    void attach(DeviceCopy* d) const
    {
        if (copy_ == d) return;
        ensure_host();
        d->push(host_.data());
        copy_ = d;
        owner_ = nullptr;
        host_valid_ = true;
    }
    void mark_device(DeviceCopy* d) const
    {
        copy_ = d;
        host_valid_ = false;
    }
    void detach(DeviceCopy* d) const noexcept
    {
        if (copy_ != d) return;
        try {
            ensure_host();
        } catch (...) {
        }
        copy_ = nullptr;
        host_valid_ = true;
    }

protected:
    void ensure_host() const
    {
        if (host_valid_) return;
        if (owner_) {
            std::vector<DevT> dev(host_.size());
            check(umc_chain_get_field(owner_, dev.data()));
            for (std::size_t k = 0; k < host_.size(); ++k) host_[k] = static_cast<HS>(dev[k]);
            downloaded_ = true;
        } else if (copy_) {
            copy_->pull(host_.data());
            downloaded_ = true;
        }
        host_valid_ = true;
    }
    // After a host-side write the host copy is the newest.
    void host_written() const
    {
        owner_ = nullptr;
        copy_ = nullptr;
    }

    mutable std::vector<HS> host_;
    mutable umc_chain* owner_ = nullptr;
    mutable DeviceCopy* copy_ = nullptr;
    mutable bool host_valid_ = true;
    // set by each read-back from the device (a model may post-process it)
    mutable bool downloaded_ = false;
};

}  // namespace umc::gpu::detail
