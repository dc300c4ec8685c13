// umc/dof.hpp -- degrees of freedom and proposals with the reference's names
// (dof/ising.hpp, dof/vector.hpp, dof/u1.hpp, dof/sun.hpp, dof/proposal.hpp).
//
// Handed to a driver, a proposal selects and parameterises the device update
// (UMC_PROPOSAL_*); its draws then come from the chain's counter-keyed
// streams.  Flip, UniformSphereN and U1Shift can also sample on the host with
// any generator that has uni() (start configurations, tests); LocalRotation
// and SUShift only parameterise the device update.
#pragma once

#include <array>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <numbers>

#include "detail.hpp"

namespace umc::gpu {

// dof/dof.hpp:9-13: a degree of freedom names its scalar type and how many of
// them one site holds.
template <class D>
concept Dof = requires {
    typename D::dtype;
    { D::size } -> std::convertible_to<std::size_t>;
};

// Proposal contract of dof/proposal.hpp:8-12.
template <typename Q, typename T, typename R>
concept Proposal = requires(const Q& q, const T* cur, T* out, R& rng) {
    { q.sample(cur, rng, out) };
    { q.log_ratio(cur, out) } -> std::convertible_to<double>;
};

// ---- Ising ---------------------------------------------------------------
using IsingSpin = std::int8_t;

struct IsingDof
{
    using dtype = IsingSpin;
    static constexpr std::size_t size = 1;
};

struct Flip
{
    template <class R>
    UMC_FACADE_HD void sample(const IsingSpin* cur, R&, IsingSpin* out) const noexcept
    {
        *out = IsingSpin(-*cur);
    }
    UMC_FACADE_HD double log_ratio(const IsingSpin*, const IsingSpin*) const noexcept { return 0.0; }
};

// Wolff reflection axis r = +1 (the only reflection of an Ising spin).
struct FixedAxis
{
    template <class C, class R>
    UMC_FACADE_HD void sample(C, R&, IsingSpin* out) const noexcept
    {
        *out = 1;
    }
};

// ---- O(N) ------------------------------------------------------------------
template <std::size_t N>
struct VectorDof
{
    using dtype = double;
    static constexpr std::size_t size = N;
};

// Uniform point on S^(N-1) by the height method: N = 1 a random sign, N = 2
// (cos, sin) of 2 pi u, N >= 3 height z = 2u - 1 and the rest a scaled point
// of S^(N-2).  Also the Wolff axis of O(N) models.
template <std::size_t N, class T = double>
struct UniformSphereN
{
    template <class C, class R>
    UMC_FACADE_HD void sample(C, R& rng, T* out) const
    {
        fill<N>(rng, out);
    }
    UMC_FACADE_HD double log_ratio(const T*, const T*) const noexcept { return 0.0; }

private:
    template <std::size_t M, class R>
    UMC_FACADE_HD static void fill(R& rng, T* out)
    {
        if constexpr (M == 1) {
            out[0] = rng.uni() < 0.5 ? T(-1) : T(1);
        } else if constexpr (M == 2) {
            const double a = 2.0 * std::numbers::pi * rng.uni();
            out[0] = T(std::cos(a));
            out[1] = T(std::sin(a));
        } else {
            const double z = 2.0 * rng.uni() - 1.0;
            const double r = std::sqrt(1.0 - z * z);
            fill<M - 1>(rng, out);
            for (std::size_t k = 0; k + 1 < M; ++k) out[k] = T(out[k] * r);
            out[M - 1] = T(z);
        }
    }
};

// Rotation by an angle in [-delta, delta] in a uniform random oriented
// 2-plane (dof/vector.hpp:62-122): u on the sphere, a second sphere point made
// orthogonal to u and normalised (redrawn while |v - (v.u) u|^2 <= 64 eps),
// then the rotation of cur in the (u, v) plane.  The engine's chains run it in
// their own kernels; sample() serves user-written terms (nvcc builds) and
// host code.  The redraw is capped at 64 tries, a limit that a draw reaches
// with probability below 1e-800.
template <std::size_t N, class T = double>
struct LocalRotation
{
    static_assert(N >= 2, "LocalRotation needs at least two components");
    T delta = T(0.5);

    template <class R>
    UMC_FACADE_HD void sample(const T* cur, R& rng, T* out) const
    {
        T u[N] = {}, v[N] = {};
        UniformSphereN<N, T>{}.sample(nullptr, rng, u);
        const T eps = T(64) * std::numeric_limits<T>::epsilon();
        for (int tries = 0; tries < 64; ++tries) {
            UniformSphereN<N, T>{}.sample(nullptr, rng, v);
            T proj = 0;
            for (std::size_t k = 0; k < N; ++k) proj += v[k] * u[k];
            T r2 = 0;
            for (std::size_t k = 0; k < N; ++k) {
                v[k] -= proj * u[k];
                r2 += v[k] * v[k];
            }
            if (r2 > eps) {
                const T inv = T(1) / std::sqrt(r2);
                for (std::size_t k = 0; k < N; ++k) v[k] *= inv;
                break;
            }
        }
        const T th = delta * (T(2) * static_cast<T>(rng.uni()) - T(1));
        const T c = std::cos(th);
        const T s = std::sin(th);
        T cu = 0, cv = 0;
        for (std::size_t k = 0; k < N; ++k) {
            cu += u[k] * cur[k];
            cv += v[k] * cur[k];
        }
        for (std::size_t k = 0; k < N; ++k) out[k] = cur[k] + (c - T(1)) * (cu * u[k] + cv * v[k]) + s * (cu * v[k] - cv * u[k]);
    }
    UMC_FACADE_HD double log_ratio(const T*, const T*) const noexcept { return 0.0; }
};

// ---- U(1) --------------------------------------------------------------------
struct U1Link
{
    double theta = 0.0;
    static constexpr U1Link identity() noexcept { return {}; }
};

struct U1Dof
{
    using dtype = U1Link;
    static constexpr std::size_t size = 1;
};

UMC_FACADE_HD inline double plaquette(double t0, double t1, double t2, double t3) noexcept
{
    return std::cos(t0 + t1 - t2 - t3);
}

// theta -> remainder(theta + width (2u - 1), 2 pi).
struct U1Shift
{
    double width = 0.5;

    template <class R>
    UMC_FACADE_HD void sample(const U1Link* cur, R& rng, U1Link* out) const
    {
        out->theta = std::remainder(cur->theta + width * (2.0 * rng.uni() - 1.0), 2.0 * std::numbers::pi);
    }
    UMC_FACADE_HD double log_ratio(const U1Link*, const U1Link*) const noexcept { return 0.0; }
};

// ---- SU(N) ---------------------------------------------------------------------
// N x N row-major complex matrix (the reference's SULink<N> layout).
template <std::size_t N>
struct SULink
{
    std::array<std::complex<double>, N * N> m{};
    static SULink identity() noexcept
    {
        SULink u;
        for (std::size_t i = 0; i < N; ++i) u.m[i * N + i] = 1.0;
        return u;
    }
};

template <std::size_t N>
struct SUDof
{
    using dtype = SULink<N>;
    static constexpr std::size_t size = 1;
};

// U -> U exp(i X), X traceless Hermitian of scale `width` (device only).
template <std::size_t N>
struct SUShift
{
    double width = 0.2;
    double log_ratio(const SULink<N>*, const SULink<N>*) const noexcept { return 0.0; }
};

// Engine extension: `hits` Metropolis hits per site and sweep with the inner
// proposal (multi-hit; one hit is the reference sweep).
template <class Q>
struct Hits
{
    Q inner;
    std::uint32_t hits = 1;
};

}  // namespace umc::gpu
