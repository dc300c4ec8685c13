// umc/rng.hpp -- the driver's RNG argument (rng.hpp:8-44).
//
// Pcg32 is the PCG-XSH-RR 64/32 generator (O'Neill 2014): LCG multiplier
// 6364136223846793005, increment 2 * stream + 1, output rotr32(((s >> 18) ^ s)
// >> 27, s >> 59), seeding "advance, add seed, advance", uni() = k * 2^-32.
// Host code may draw from it (start configurations and the like).  Handed to a
// driver it only supplies the key of the device chain's counter-keyed streams:
// key() = seed ^ (stream * 0x9E3779B97F4A7C15).
#pragma once

#include <cstdint>

namespace umc::gpu {

class Pcg32
{
public:
    explicit Pcg32(std::uint64_t seed, std::uint64_t stream = 0) noexcept
        : seed_(seed), stream_(stream), state_(0), inc_((stream << 1u) | 1u)
    {
        next();
        state_ += seed;
        next();
    }

    [[nodiscard]] double uni() noexcept { return next() * 0x1.0p-32; }

    // Key of the device chain's random streams.
    std::uint64_t key() const noexcept { return seed_ ^ (stream_ * 0x9E3779B97F4A7C15ULL); }

private:
    std::uint32_t next() noexcept
    {
        const std::uint64_t old = state_;
        state_ = old * 6364136223846793005ULL + inc_;
        const auto x = static_cast<std::uint32_t>(((old >> 18u) ^ old) >> 27u);
        const auto r = static_cast<std::uint32_t>(old >> 59u);
        return (x >> r) | (x << ((32u - r) & 31u));
    }

    std::uint64_t seed_, stream_;
    std::uint64_t state_, inc_;
};

}  // namespace umc::gpu
