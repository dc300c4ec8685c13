// umc/dof.hpp -- degrees of freedom and proposals with the reference's names
// (dof/ising.hpp, dof/vector.hpp, dof/u1.hpp, dof/sun.hpp, dof/proposal.hpp).
//
// Handed to a driver, a proposal selects and parameterises the device update
// (UMC_PROPOSAL_*); its draws then come from the chain's counter-keyed
// streams.  Flip, UniformSphereN and U1Shift can also sample on the host with
// any generator that has uni() (start configurations, tests); LocalRotation
// and SUShift only parameterise the device update.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <limits>
#include <numbers>
#include <system_error>
#include <thread>
#include <vector>

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

// dof/ising.hpp:20-24: the bilinear s_i s_j of two Ising spins.
UMC_FACADE_HD constexpr std::int32_t dot(IsingSpin a, IsingSpin b) noexcept
{
    return std::int32_t(a) * std::int32_t(b);
}

// dof/vector.hpp:23-31: the dot product of two N-component vectors, summed in
// component order.
template <std::size_t N>
UMC_FACADE_HD constexpr double dot(const double* a, const double* b) noexcept
{
    static_assert(N >= 1, "dot needs at least one component");
    double s = 0.0;
    for (std::size_t k = 0; k < N; ++k) s += a[k] * b[k];
    return s;
}

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
// The entries of an SU(N) link.  In a g++ translation unit, which has no
// device code, they are the reference's own std::complex<double>, so that host
// code such as std::abs(u.m[k] - v.m[k]) compiles unchanged.  In an nvcc
// translation unit they are Complex below: the layout of std::complex<double>
// (real part, then imaginary part) in a type that device code can use, which
// std::complex cannot.  It converts to and from std::complex on the host;
// conj, abs and norm are found by argument-dependent lookup, and the
// arithmetic is the textbook one ((a + bi)(c + di) = (ac - bd) + (ad + bc)i).
#if defined(__CUDACC__)
struct Complex
{
    double re = 0.0, im = 0.0;

    Complex() = default;
    UMC_FACADE_HD constexpr Complex(double r, double i = 0.0) noexcept : re(r), im(i) {}
    Complex(const std::complex<double>& z) noexcept : re(z.real()), im(z.imag()) {}
    operator std::complex<double>() const noexcept { return {re, im}; }

    UMC_FACADE_HD constexpr double real() const noexcept { return re; }
    UMC_FACADE_HD constexpr double imag() const noexcept { return im; }

    UMC_FACADE_HD constexpr Complex& operator+=(const Complex& z) noexcept
    {
        re += z.re;
        im += z.im;
        return *this;
    }
    UMC_FACADE_HD constexpr Complex& operator-=(const Complex& z) noexcept
    {
        re -= z.re;
        im -= z.im;
        return *this;
    }
    UMC_FACADE_HD constexpr Complex& operator*=(const Complex& z) noexcept
    {
        const double r = re * z.re - im * z.im, i = re * z.im + im * z.re;
        re = r;
        im = i;
        return *this;
    }
    UMC_FACADE_HD constexpr Complex& operator*=(double x) noexcept
    {
        re *= x;
        im *= x;
        return *this;
    }
    UMC_FACADE_HD constexpr Complex& operator/=(double x) noexcept
    {
        re /= x;
        im /= x;
        return *this;
    }
    UMC_FACADE_HD friend constexpr Complex operator+(Complex a, const Complex& b) noexcept { return a += b; }
    UMC_FACADE_HD friend constexpr Complex operator-(Complex a, const Complex& b) noexcept { return a -= b; }
    UMC_FACADE_HD friend constexpr Complex operator*(Complex a, const Complex& b) noexcept { return a *= b; }
    UMC_FACADE_HD friend constexpr Complex operator*(Complex a, double x) noexcept { return a *= x; }
    UMC_FACADE_HD friend constexpr Complex operator*(double x, Complex a) noexcept { return a *= x; }
    UMC_FACADE_HD friend constexpr Complex operator/(Complex a, double x) noexcept { return a /= x; }
    UMC_FACADE_HD friend constexpr Complex operator-(const Complex& a) noexcept { return {-a.re, -a.im}; }
    UMC_FACADE_HD friend constexpr bool operator==(const Complex& a, const Complex& b) noexcept
    {
        return a.re == b.re && a.im == b.im;
    }
    UMC_FACADE_HD friend constexpr Complex conj(const Complex& z) noexcept { return {z.re, -z.im}; }
    UMC_FACADE_HD friend constexpr double norm(const Complex& z) noexcept { return z.re * z.re + z.im * z.im; }
    UMC_FACADE_HD friend double abs(const Complex& z) noexcept { return std::hypot(z.re, z.im); }
};
#else
using Complex = std::complex<double>;
#endif
static_assert(sizeof(Complex) == sizeof(std::complex<double>) && alignof(Complex) == alignof(std::complex<double>));

// One SU(N) link: an N x N complex matrix, row-major (dof/sun.hpp:14-76), with
// the reference's group operations.  Host and device code (nvcc builds) can
// both use it, so a user's SU(N) term written against this interface runs on
// the device unchanged.
template <std::size_t N>
struct SULink
{
    static_assert(N >= 2, "SU(N) needs N >= 2");
    static constexpr std::size_t dim = N;
    using Mat = std::array<Complex, N * N>;

    Mat m{};

    SULink() = default;
    UMC_FACADE_HD explicit SULink(const Mat& mat) : m(mat) {}

    UMC_FACADE_HD static SULink identity() noexcept
    {
        SULink u;
        for (std::size_t i = 0; i < N; ++i) u.m[i * N + i] = 1.0;
        return u;
    }
    UMC_FACADE_HD SULink dagger() const noexcept
    {
        SULink u;
        for (std::size_t i = 0; i < N; ++i)
            for (std::size_t j = 0; j < N; ++j) u.m[i * N + j] = conj(m[j * N + i]);
        return u;
    }
    // Re Tr U; the plaquette action divides it by N.
    UMC_FACADE_HD double real_trace() const noexcept
    {
        double t = 0.0;
        for (std::size_t i = 0; i < N; ++i) t += m[i * N + i].real();
        return t;
    }
    // max_ij |(U^dagger U - I)_ij|
    UMC_FACADE_HD double unitarity_error() const noexcept
    {
        const SULink u = dagger() * (*this);
        double e = 0.0;
        for (std::size_t i = 0; i < N; ++i)
            for (std::size_t j = 0; j < N; ++j) {
                const double d = abs(u.m[i * N + j] - Complex(i == j ? 1.0 : 0.0));
                e = d > e ? d : e;
            }
        return e;
    }
    UMC_FACADE_HD friend SULink operator*(const SULink& a, const SULink& b) noexcept
    {
        SULink r;
        for (std::size_t i = 0; i < N; ++i)
            for (std::size_t j = 0; j < N; ++j) {
                Complex s = 0.0;
                for (std::size_t k = 0; k < N; ++k) s += a.m[i * N + k] * b.m[k * N + j];
                r.m[i * N + j] = s;
            }
        return r;
    }
};

// Re Tr(U0 U1 U2^dagger U3^dagger) / N, the oriented plaquette (dof/sun.hpp:78-84).
template <std::size_t N>
UMC_FACADE_HD double plaquette(const SULink<N>& u0, const SULink<N>& u1, const SULink<N>& u2,
                               const SULink<N>& u3) noexcept
{
    return (u0 * u1 * u2.dagger() * u3.dagger()).real_trace() / double(N);
}

// The nearest-by-construction SU(N) matrix to a link that is unitary only to
// a few ulp of FP32, in FP64 on the host: Gram-Schmidt over the rows (each row
// minus its projections on the rows before it, then normalised), then the
// last row multiplied by conj(det) / |det| so that det U = 1.  A link already
// in SU(N) to FP64 rounding moves by a few ulp.
template <std::size_t N>
void su_project(SULink<N>& u)
{
    for (std::size_t r = 0; r < N; ++r) {
        for (std::size_t q = 0; q < r; ++q) {
            Complex c(0.0);
            for (std::size_t k = 0; k < N; ++k) c += conj(u.m[q * N + k]) * u.m[r * N + k];
            for (std::size_t k = 0; k < N; ++k) u.m[r * N + k] -= c * u.m[q * N + k];
        }
        double s = 0.0;
        for (std::size_t k = 0; k < N; ++k) s += norm(u.m[r * N + k]);
        const double inv = 1.0 / std::sqrt(s);
        for (std::size_t k = 0; k < N; ++k) u.m[r * N + k] *= inv;
    }
    // det by Gaussian elimination with partial pivoting on a copy
    std::array<Complex, N * N> a = u.m;
    Complex det(1.0);
    for (std::size_t c = 0; c < N; ++c) {
        std::size_t p = c;
        for (std::size_t r = c + 1; r < N; ++r)
            if (abs(a[r * N + c]) > abs(a[p * N + c])) p = r;
        if (p != c) {
            for (std::size_t k = 0; k < N; ++k) std::swap(a[c * N + k], a[p * N + k]);
            det = -det;
        }
        det *= a[c * N + c];
        for (std::size_t r = c + 1; r < N; ++r) {
            const Complex f = a[r * N + c] * conj(a[c * N + c]) / norm(a[c * N + c]);
            for (std::size_t k = c; k < N; ++k) a[r * N + k] -= f * a[c * N + k];
        }
    }
    const Complex phase = conj(det) / abs(det);
    for (std::size_t k = 0; k < N; ++k) u.m[(N - 1) * N + k] *= phase;
}

// su_project of n links, split into contiguous ranges over the host's
// hardware threads when n is large; every link is projected on its own, so
// the result does not depend on the split.  A thread that cannot be started
// leaves its range to the calling thread.
template <std::size_t N>
void su_project_all(SULink<N>* u, std::size_t n)
{
    constexpr std::size_t kMinPerThread = 16384;
    const std::size_t hw = std::max<std::size_t>(1, std::thread::hardware_concurrency());
    const std::size_t parts = std::min<std::size_t>(hw, (n + kMinPerThread - 1) / kMinPerThread);
    const auto range = [u, n, parts](std::size_t p) {
        for (std::size_t i = n * p / parts; i < n * (p + 1) / parts; ++i) su_project(u[i]);
    };
    if (parts <= 1) {
        for (std::size_t i = 0; i < n; ++i) su_project(u[i]);
        return;
    }
    std::vector<std::thread> threads;
    std::vector<std::size_t> left;
    for (std::size_t p = 1; p < parts; ++p) {
        try {
            threads.emplace_back(range, p);
        } catch (const std::system_error&) {
            left.push_back(p);
        }
    }
    range(0);
    for (std::size_t p : left) range(p);
    for (auto& t : threads) t.join();
}

namespace sun_detail {
template <std::size_t N>
using Mat = std::array<Complex, N * N>;

template <std::size_t N>
UMC_FACADE_HD Mat<N> mul(const Mat<N>& a, const Mat<N>& b) noexcept
{
    Mat<N> r{};
    for (std::size_t i = 0; i < N; ++i)
        for (std::size_t j = 0; j < N; ++j) {
            Complex s = 0.0;
            for (std::size_t k = 0; k < N; ++k) s += a[i * N + k] * b[k * N + j];
            r[i * N + j] = s;
        }
    return r;
}

// Largest absolute row sum (each entry's modulus).
template <std::size_t N>
UMC_FACADE_HD double norm_inf(const Mat<N>& a) noexcept
{
    double n = 0.0;
    for (std::size_t i = 0; i < N; ++i) {
        double row = 0.0;
        for (std::size_t j = 0; j < N; ++j) row += abs(a[i * N + j]);
        n = row > n ? row : n;
    }
    return n;
}

// The same norm under its dof/sun.hpp:104-114 name.
template <std::size_t N>
UMC_FACADE_HD double norm(const Mat<N>& a) noexcept
{
    return norm_inf<N>(a);
}

// exp(A) as dof/sun.hpp:118-146 computes it: halve A until its norm is at most
// 1/2, sum the Taylor series until a term's norm drops below 1e-16 (at most 30
// terms), square back.  The steps are kept so that a chain on the device
// proposes what the reference proposes, to rounding.
template <std::size_t N>
UMC_FACADE_HD SULink<N> expm(const Mat<N>& a) noexcept
{
    double n = norm_inf<N>(a);
    int squarings = 0;
    while (n > 0.5) {
        n *= 0.5;
        ++squarings;
    }
    const double scale = std::ldexp(1.0, -squarings);
    Mat<N> b = a;
    for (auto& z : b) z *= scale;
    Mat<N> result{}, term{};
    for (std::size_t i = 0; i < N; ++i) result[i * N + i] = 1.0;
    for (std::size_t i = 0; i < N; ++i) term[i * N + i] = 1.0;
    for (std::size_t k = 1; k <= 30; ++k) {
        term = mul<N>(term, b);
        for (auto& z : term) z /= double(k);
        for (std::size_t i = 0; i < N * N; ++i) result[i] += term[i];
        if (norm_inf<N>(term) < 1e-16) break;
    }
    for (int k = 0; k < squarings; ++k) result = mul<N>(result, result);
    return SULink<N>(result);
}
}  // namespace sun_detail

template <std::size_t N>
struct SUDof
{
    using dtype = SULink<N>;
    static constexpr std::size_t size = 1;
};

// U -> U exp(i X), X traceless Hermitian with independent uniform entries of
// scale `width` (dof/sun.hpp:160-204; the proposal is symmetric).  The draws
// come in the reference's order: the N diagonal entries, then the real and
// imaginary parts of each entry above the diagonal, row by row.  The engine's
// own SU(N) chains only take the width from it; sample() runs for user
// SU(N) terms (on the device in nvcc builds) and on the host.
template <std::size_t N>
struct SUShift
{
    static_assert(N >= 2, "SUShift needs N >= 2");
    double width = 0.3;

    template <class R>
    UMC_FACADE_HD void sample(const SULink<N>* cur, R& rng, SULink<N>* out) const
    {
        sun_detail::Mat<N> x{};
        double tr = 0.0;
        for (std::size_t i = 0; i < N; ++i) {
            const double d = width * (2.0 * rng.uni() - 1.0);
            x[i * N + i] = d;
            tr += d;
        }
        for (std::size_t i = 0; i < N; ++i)
            for (std::size_t j = i + 1; j < N; ++j) {
                const double a = width * (2.0 * rng.uni() - 1.0);
                const double b = width * (2.0 * rng.uni() - 1.0);
                x[i * N + j] = Complex(a, b);
                x[j * N + i] = Complex(a, -b);
            }
        for (std::size_t i = 0; i < N; ++i) x[i * N + i] -= Complex(tr / double(N));
        // A = i X is anti-Hermitian, so exp(A) is unitary
        sun_detail::Mat<N> a{};
        for (std::size_t k = 0; k < N * N; ++k) a[k] = Complex(-x[k].imag(), x[k].real());
        *out = (*cur) * sun_detail::expm<N>(a);
    }
    UMC_FACADE_HD double log_ratio(const SULink<N>*, const SULink<N>*) const noexcept { return 0.0; }
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
