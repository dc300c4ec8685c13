// umc_spin_kernels.cuh -- colour-pass Metropolis and Wolff kernels for the
// spin models (Ising, VectorSpin<N>, XY on angles).
//
// Layout in HBM: one array per field component, sites in colour-major order
// (colour class 0 first, then class 1, ...; inside a class by ascending site
// id).  A colour pass reads its own class and the neighbouring classes and
// writes its own class once; nothing else is staged through memory.
//
// Each kernel is the body of the reference's Metropolis::sweep loop
// (driver.hpp:34-42) for the sites of one colour class:
//   propose (dof/*.hpp) -> dE (example/*.hpp energy_diff_at) ->
//   accept iff log_p >= 0 or log(u) < log_p -> update,
// with every draw taken from the site's keyed stream.  Ising acceptance is an
// integer comparison against thresholds the host derived with the same
// std::log, so Ising chains are bit-exact with the reference driver.
#pragma once

#include <cmath>
#include <type_traits>

#include "umc_device.cuh"
#include "umc_math64.cuh"

namespace umc {

// ----------------------------------------------------------------- topology

// Colour-major CSR of a PairGraph.  Neighbours below early_end belong to
// colour classes already final in this sweep.
struct CsrTopo
{
    const uint32_t* off;
    const uint32_t* adj;
    uint32_t early_end;
    template <class F>
    __device__ __forceinline__ void neighbours(uint32_t k, F&& f) const
    {
        const uint32_t a0 = off[k], a1 = off[k + 1];
        for (uint32_t a = a0; a < a1; ++a) {
            const uint32_t j = adj[a];
            f(j, j < early_end);
        }
    }
};

// Periodic Lx x Ly x Lz lattice (Lx even, Ly and Lz 1 or even) in the
// two-colour layout: colour c = (x+y+z)&1, index c*half + site/2.  Rows of a
// colour class hold H = Lx/2 sites; site (row, i) sits at x = 2i + ((y+z+c)&1).
// Extents equal to 2 revisit the same neighbour twice, which reproduces the
// duplicated periodic bonds of square_lattice (lattice/square.hpp:11-14).
struct StencilTopo
{
    uint32_t H, Ly, Lz, half, colour;
    uint32_t hasy, hasz;
    uint32_t hshift, yshift;  // log2(H), log2(Ly) when both are powers of two, else 0xFF
    template <class F>
    __device__ __forceinline__ void neighbours(uint32_t k, F&& f) const
    {
        const uint32_t j = k - colour * half;
        uint32_t row, i, y, z;
        if (hshift != 0xFFu) {  // uniform branch: shifts instead of integer division
            row = j >> hshift;
            i = j & (H - 1);
            y = row & (Ly - 1);
            z = row >> yshift;
        } else {
            row = j / H;
            i = j - row * H;
            y = row % Ly;
            z = row / Ly;
        }
        const uint32_t p = (y + z + colour) & 1u;
        const uint32_t ob = (1u - colour) * half;
        const bool early = colour == 1u;
        f(ob + row * H + i, early);
        const uint32_t i2 = p ? (i + 1 == H ? 0u : i + 1) : (i == 0 ? H - 1 : i - 1);
        f(ob + row * H + i2, early);
        if (hasy) {
            const uint32_t ym = y == 0 ? Ly - 1 : y - 1, yp = y + 1 == Ly ? 0u : y + 1;
            f(ob + (z * Ly + ym) * H + i, early);
            f(ob + (z * Ly + yp) * H + i, early);
        }
        if (hasz) {
            const uint32_t zm = z == 0 ? Lz - 1 : z - 1, zp = z + 1 == Lz ? 0u : z + 1;
            f(ob + (zm * Ly + y) * H + i, early);
            f(ob + (zp * Ly + y) * H + i, early);
        }
    }
};

// --------------------------------------------------- Ising, packed 2D stencil

// 16 sites per thread: one 16-byte load of the own class and three of the
// other class (rows y-1, y, y+1), plus one byte for the ragged horizontal
// neighbour.  Requires Lx/2 to be a multiple of 16 and Ly even.
struct IsingPackedArgs
{
    int8_t* spins;
    uint32_t H, Ly, half, colour;
    uint64_t kbase;
    uint32_t tm1[5];  // accept iff draw <= tm1[(s*h + 4) / 2]
    int32_t J;
    PassOut out;
};

__device__ __forceinline__ uint32_t down_bits(uint32_t w) { return (w >> 1) & 0x01010101u; }
__device__ __forceinline__ uint32_t byte_sum(uint32_t w) { return (w * 0x01010101u) >> 24; }

static __global__ void __launch_bounds__(kBlock) ising_packed_pass(IsingPackedArgs a)
{
    __shared__ uint32_t tm1[5];
    if (threadIdx.x < 5) tm1[threadIdx.x] = a.tm1[threadIdx.x];
    __syncthreads();
    int64_t e_acc = 0, m_acc = 0, n_acc = 0;
    const uint32_t nvec = a.half >> 4;
    const int8_t* other = a.spins + (1u - a.colour) * a.half;
    int8_t* own = a.spins + a.colour * a.half;
    const uint32_t idbase = a.colour * a.half;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nvec; v += gridDim.x * blockDim.x) {
        const uint32_t base = v << 4;
        const uint32_t y = base / a.H, i0 = base - y * a.H;
        const uint32_t p = (y + a.colour) & 1u;
        const uint32_t ym = y == 0 ? a.Ly - 1 : y - 1, yp = y + 1 == a.Ly ? 0u : y + 1;
        const uint4 s4 = *reinterpret_cast<const uint4*>(own + base);
        const uint4 m4 = *reinterpret_cast<const uint4*>(other + y * a.H + i0);
        const uint4 u4 = *reinterpret_cast<const uint4*>(other + yp * a.H + i0);
        const uint4 d4 = *reinterpret_cast<const uint4*>(other + ym * a.H + i0);
        const uint32_t xe = p ? (i0 + 16 == a.H ? 0u : i0 + 16) : (i0 == 0 ? a.H - 1 : i0 - 1);
        const uint32_t extra = uint32_t(uint8_t(other[y * a.H + xe]));
        const uint32_t sw[4] = {s4.x, s4.y, s4.z, s4.w};
        const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
        const uint32_t uw[4] = {u4.x, u4.y, u4.z, u4.w};
        const uint32_t dw[4] = {d4.x, d4.y, d4.z, d4.w};
        uint32_t out[4];
        // the 16 sites of this vector are one group: consecutive outputs of the
        // stream of id (class offset + base) / 16
        KeyedPcg rng = KeyedPcg::open(a.kbase, (idbase + base) / kGroupSites);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            // second horizontal neighbour: byte k-1 (p == 0) or k+1 (p == 1)
            const uint32_t h2 = p ? __byte_perm(mw[w], w == 3 ? extra : mw[w + 1], 0x4321)
                                  : __byte_perm(w == 0 ? (extra << 24) : mw[w - 1], mw[w], 0x6543);
            const uint32_t nd = down_bits(uw[w]) + down_bits(dw[w]) + down_bits(mw[w]) + down_bits(h2);
            const uint32_t di = down_bits(sw[w]);
            const uint32_t mask = di * 0xFFu;
            // t = (s*h + 4)/2 with h = 4 - 2*nd: nd if s = -1, 4 - nd if s = +1
            const uint32_t t = (nd & mask) | ((0x04040404u - nd) & ~mask);
            uint32_t fm = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const uint32_t tb = (t >> (8 * b)) & 0xFFu;
                const uint32_t r = rng.next();
                fm |= (r <= tm1[tb] ? 0xFEu : 0u) << (8 * b);
            }
            const uint32_t ns = sw[w] ^ fm;
            out[w] = ns;
            const uint32_t dn = down_bits(ns);
            const int32_t ndown = __popc(dn);
            m_acc += 4 - 2 * ndown;
            n_acc += __popc(fm) / 7;
            // sum_k s_k h_k = 16 - 2 sum nd - 8 sum d + 4 sum d*nd  (per 4 bytes)
            const int32_t sh = 16 - 2 * int32_t(byte_sum(nd)) - 8 * ndown + 4 * int32_t(byte_sum(nd & (dn * 0xFFu)));
            e_acc += sh;
        }
        *reinterpret_cast<uint4*>(own + base) = make_uint4(out[0], out[1], out[2], out[3]);
    }
    // every bond joins the two classes: count it once, in the pass of class 1
    double v[kObs] = {a.colour == 1u ? double(-int64_t(a.J) * e_acc) : 0.0, double(m_acc), 0, 0, 0, 0, 0, double(n_acc)};
    finish_pass<kObs>(v, a.out);
}

// --------------------------------------- Ising, packed 2D stencil, J > 0
//
// The same pass for the usual sign of J (ferromagnet): only a site with at
// most one anti-aligned neighbour can be rejected (dE = 8J with none, 4J with
// one), so the decision per site is
//     flip  <=>  anti + [r <= T(dE=4J)] + [r <= T(dE=8J)] >= 2,
// evaluated four sites at a time on bytes.  The arithmetic is arranged for the
// FMA pipe where it can be (multiply-high shifts, wide multiply-adds for the
// comparisons), the integer ALU being the limiting pipe of this kernel.
struct IsingFastArgs
{
    int8_t* spins;
    uint32_t H, Ly, half, colour, vpr;
    uint64_t vmagic;  // row of vector v = (v * vmagic) >> 40 (exact for v < 2^25, vpr < 2^15)
    uint64_t kbase;
    uint32_t T3, T4;  // accept iff draw <= T for dE = 4J, 8J (T4 <= T3)
    int32_t J;
    // 2^(8b+1) and -2^(8b+2) for byte b: kernel parameters rather than
    // literals, so that the per-site accumulation stays three integer
    // multiply-adds on the FMA pipe instead of shifts and adds on the ALU
    uint32_t m1[4], m2[4];
    PassOut out;
};

// XSH-RR output of state (hi:lo): rotr32(uint32(s >> 27) ^ uint32(s >> 45), s >> 59),
// with the right shifts of hi as multiply-highs.
__device__ __forceinline__ uint32_t pcg_output_split(uint32_t lo, uint32_t hi)
{
    const uint32_t xs = __funnelshift_r(lo, hi, 27) ^ __umulhi(hi, 1u << 19);
    return __funnelshift_r(xs, xs, __umulhi(hi, 32u));
}

// One Pcg32 step (rng.hpp:34, increment 1) on the state's 32-bit halves:
// lo * A_lo + 1 as one wide multiply-add (the +1 rides in its addend), then
// the high word from two multiply-adds and that product's carry word.
__device__ __forceinline__ void pcg_step_split(uint32_t& lo, uint32_t& hi)
{
    constexpr uint32_t aL = uint32_t(kPcgMult), aH = uint32_t(kPcgMult >> 32);
    uint64_t w;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(w) : "r"(lo), "r"(aL), "l"(1ull));
    hi = hi * aL + lo * aH + uint32_t(w >> 32);
    lo = uint32_t(w);
}

// hi32(a * b + c) with one wide multiply-add.
__device__ __forceinline__ uint32_t mad_wide_hi(uint32_t a, uint32_t b, uint32_t c)
{
    uint64_t w;
    asm("mad.wide.u32 %0, %1, %2, %3;" : "=l"(w) : "r"(a), "r"(b), "l"(uint64_t(c)));
    return uint32_t(w >> 32);
}

// ENERGY: the pass of class 1, which also sums s_k h_k (every bond once).
template <bool ENERGY>
__global__ void __launch_bounds__(kBlock) ising_fast_pass(IsingFastArgs a)
{
    int64_t e_acc = 0, m_acc = 0, n_acc = 0;
    const uint32_t nvec = a.half >> 4;
    const int8_t* other = a.spins + (1u - a.colour) * a.half;
    int8_t* own = a.spins + a.colour * a.half;
    const uint32_t gbase = (a.colour * a.half) >> 4;  // stream id of this class's first vector
    constexpr uint32_t M2 = 0x02020202u;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nvec; v += gridDim.x * blockDim.x) {
        const uint32_t y = uint32_t((uint64_t(v) * a.vmagic) >> 40);
        const uint32_t i0 = (v - y * a.vpr) << 4;
        const uint32_t base = v << 4;
        const uint32_t p = (y + a.colour) & 1u;
        const uint32_t ym = y == 0 ? a.Ly - 1 : y - 1, yp = y + 1 == a.Ly ? 0u : y + 1;
        const uint4 s4 = *reinterpret_cast<const uint4*>(own + base);
        const uint4 m4 = *reinterpret_cast<const uint4*>(other + base);
        const uint4 u4 = *reinterpret_cast<const uint4*>(other + yp * a.H + i0);
        const uint4 d4 = *reinterpret_cast<const uint4*>(other + ym * a.H + i0);
        const uint32_t xe = p ? (i0 + 16 == a.H ? 0u : i0 + 16) : (i0 == 0 ? a.H - 1 : i0 - 1);
        const uint32_t extra = uint32_t(uint8_t(other[y * a.H + xe]));
        const uint32_t sw[4] = {s4.x, s4.y, s4.z, s4.w};
        const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
        const uint32_t uw[4] = {u4.x, u4.y, u4.z, u4.w};
        const uint32_t dw[4] = {d4.x, d4.y, d4.z, d4.w};
        const uint64_t st0 = first_state(id_seed(a.kbase, gbase + v));
        uint32_t slo = uint32_t(st0), shi = uint32_t(st0 >> 32);
        uint32_t out[4], acc_f = 0, acc_dn = 0, acc_e = 0;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint32_t h2 = p ? __byte_perm(mw[w], w == 3 ? extra : mw[w + 1], 0x4321)
                                  : __byte_perm(w == 0 ? (extra << 24) : mw[w - 1], mw[w], 0x6543);
            const uint32_t s = sw[w];
            // twice the number of neighbours whose spin differs from the site's
            const uint32_t A2 = ((mw[w] ^ s) & M2) + ((h2 ^ s) & M2) + ((uw[w] ^ s) & M2) + ((dw[w] ^ s) & M2);
            // byte b: A2 + 16 - 2 ([r > T3] + [r > T4]), flip iff >= 16
            uint32_t X = A2 + 0x10101010u;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const uint32_t r = pcg_output_split(slo, shi);
                pcg_step_split(slo, shi);
                // hi32(r (2^32 - 1) + T) = r - [r > T]: byte b gains
                // 2 (h3 + h4 - 2 r) = -2 ([r > T3] + [r > T4])
                const uint32_t h3 = mad_wide_hi(r, 0xFFFFFFFFu, a.T3);
                const uint32_t h4 = mad_wide_hi(r, 0xFFFFFFFFu, a.T4);
                X = h3 * a.m1[b] + X;
                X = h4 * a.m1[b] + X;
                X = r * a.m2[b] + X;
            }
            const uint32_t g = (X & 0x10101010u) >> 4;  // 1 per flipped site
            const uint32_t gm = g * 0xFFu;
            const uint32_t ns = s ^ (gm - g);           // flipped bytes ^= 0xFE
            out[w] = ns;
            acc_f += g;
            acc_dn += ns & M2;                          // twice the new down count
            if constexpr (ENERGY) {
                // twice the anti-aligned count of the new spin
                acc_e += (A2 & ~gm) | ((0x08080808u - A2) & gm);
            }
        }
        *reinterpret_cast<uint4*>(own + base) = make_uint4(out[0], out[1], out[2], out[3]);
        n_acc += byte_sum(acc_f);
        m_acc += 16 - int32_t(byte_sum(acc_dn));
        // sum_k s_k h_k = sum_k (4 - 2 anti_k)
        if constexpr (ENERGY) e_acc += 64 - int32_t(byte_sum(acc_e));
    }
    double v[kObs] = {ENERGY ? double(-int64_t(a.J) * e_acc) : 0.0, double(m_acc), 0, 0, 0, 0, 0, double(n_acc)};
    finish_pass<kObs>(v, a.out);
}

// ----------------------------------------------------- Ising, any topology

struct IsingArgs
{
    int8_t* spins;
    uint32_t first, count;
    uint64_t kbase;
    const uint32_t* tm1;  // 2*D+1 thresholds, index s*h + D
    uint32_t D;
    int32_t J;
    PassOut out;
};

template <class Topo>
__global__ void __launch_bounds__(kBlock) ising_pass(IsingArgs a, Topo t)
{
    extern __shared__ uint32_t tm1s[];
    for (uint32_t q = threadIdx.x; q < 2 * a.D + 1; q += blockDim.x) tm1s[q] = a.tm1[q];
    __syncthreads();
    int64_t e_acc = 0, m_acc = 0, n_acc = 0;
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < a.count; q += gridDim.x * blockDim.x) {
        const uint32_t k = a.first + q;
        int32_t h = 0, he = 0;
        t.neighbours(k, [&](uint32_t j, bool early) {
            const int32_t sj = a.spins[j];
            h += sj;
            he += early ? sj : 0;
        });
        const int32_t s = a.spins[k];
        const uint32_t r = group_draw(a.kbase, k);
        const bool flip = r <= tm1s[s * h + int32_t(a.D)];
        const int32_t ns = flip ? -s : s;
        if (flip) a.spins[k] = int8_t(ns);
        m_acc += ns;
        n_acc += flip;
        e_acc += ns * he;
    }
    double v[kObs] = {double(-int64_t(a.J) * e_acc), double(m_acc), 0, 0, 0, 0, 0, double(n_acc)};
    finish_pass<kObs>(v, a.out);
}

// ------------------------------------------------------------- proposals

// UniformSphereN<N>::sample (dof/vector.hpp:35-61) in FP32 from keyed draws.
template <int N>
__device__ __forceinline__ void sphere_sample(KeyedPcg& g, float* out)
{
    if constexpr (N == 1) {
        out[0] = g.next() < 0x80000000u ? -1.0f : 1.0f;  // u < 0.5
    } else if constexpr (N == 2) {
        // angle 2 pi u = a + pi with a = pi (2u - 1) in [-pi, pi), where the
        // hardware sine/cosine are accurate to ~4e-7
        float sn, cs;
        __sincosf(3.14159265358979f * sym_f32(g.next()), &sn, &cs);
        out[0] = -cs;
        out[1] = -sn;
    } else {
        const float z = sym_f32(g.next());
        const float w = (1.0f - z) * (1.0f + z);
        const float r = w > 0.0f ? w * rsqrtf(w) : 0.0f;
        sphere_sample<N - 1>(g, out);
#pragma unroll
        for (int k = 0; k < N - 1; ++k) out[k] *= r;
        out[N - 1] = z;
    }
}

template <int N>
__device__ __forceinline__ float vdot(const float* a, const float* b)
{
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < N; ++k) s = fmaf(a[k], b[k], s);
    return s;
}

// Wolff reflection s - 2 (s.r) r in FP32, rounded the same way wherever a
// cluster is flipped (one fused multiply-add per component).
template <int N>
__device__ __forceinline__ void reflect(float* s, const float* r)
{
    const float d2 = 2.0f * vdot<N>(s, r);
#pragma unroll
    for (int c = 0; c < N; ++c) s[c] = __fmaf_rn(-d2, r[c], s[c]);
}

// LocalRotation<N>::sample (dof/vector.hpp:70-122) in FP32.  The retry loop
// is bounded; running out flags the chain and leaves the site unchanged.
template <int N>
__device__ __forceinline__ bool local_rotation(KeyedPcg& g, float delta, const float* cur, float* out)
{
    float u[N], v[N];
    sphere_sample<N>(g, u);
    bool ok = false;
    for (int tries = 0; tries < 64 && !ok; ++tries) {
        sphere_sample<N>(g, v);
        const float proj = vdot<N>(v, u);
        float r2 = 0.0f;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            v[k] -= proj * u[k];
            r2 += v[k] * v[k];
        }
        if (r2 > 64.0f * 2.220446049250313e-16f) {
            const float inv = rsqrtf(r2);
#pragma unroll
            for (int k = 0; k < N; ++k) v[k] *= inv;
            ok = true;
        }
    }
    if (!ok) return false;
    const float th = delta * sym_f32(g.next());
    float sn, cs;
    __sincosf(th, &sn, &cs);
    const float cu = vdot<N>(u, cur), cv = vdot<N>(v, cur);
#pragma unroll
    for (int k = 0; k < N; ++k) out[k] = cur[k] + (cs - 1.0f) * (cu * u[k] + cv * v[k]) + sn * (cu * v[k] - cv * u[k]);
    return true;
}

// U1Shift::sample (dof/u1.hpp:35-50): theta + width*(2u-1) wrapped into [-pi, pi].
__device__ __forceinline__ float u1_shift(KeyedPcg& g, float width, float cur)
{
    return remainderf(cur + width * sym_f32(g.next()), 6.283185307179586f);
}

// ------------------------------------ accept and activation decisions in FP64

// N floats by value (arguments of the out-of-line FP64 decisions).
template <int N>
struct SpinVal
{
    float v[N];
};


// Metropolis accept (driver.hpp:39-40): log_p >= 0 || log(u) < log_p, with the
// uniform drawn only when needed, as the reference draws it (the keyed stream
// makes a skipped draw harmless).  lp is the kernel's FP32 log-ratio and err
// bounds its distance from lp64(), the same log-ratio recomputed in FP64 from
// the same FP32 state.  The FP32 test compares u_f32(k) (within 2^-24 of u,
// relatively) with __expf(lp) (within (2 + 1.173 |lp|) ulps of exp(lp)); with
// the rounding of the band edge it misplaces log u - log_p by at most
// err + 2^-23 (3 + 1.2 |lp|).  Outside twice that band the FP32 answer is the
// FP64 one; inside it lp64() and the FP64 log decide.  So every decision is
// the reference's FP64 test applied to the kernel's FP32 values.
template <class F64>
__device__ __forceinline__ bool metropolis_accept(KeyedPcg& g, float lp, float err, F64&& lp64)
{
    const float tol = 2.0f * (err + 0x1.0p-23f * (3.0f + 1.2f * fabsf(lp)));
    if (lp >= tol) return true;
    const uint32_t k = g.next();
    if (lp <= -tol) {
        const float u = u_f32(k), e = __expf(lp);
        if (u < e * (1.0f - tol)) return true;
        if (u > e * (1.0f + tol)) return false;
    }
    const double l = lp64();
    return l >= 0.0 || log(u_f64(k)) < l;
}

// Wolff bond activation (driver.hpp:151): u < 1 - exp(-x), x = beta dE.  x is
// the kernel's FP32 value and err bounds its distance from x64(), the same
// quantity in FP64 from the same FP32 state.  For x >= 0, 1 - __expf(-x) is
// within err + 2^-23 (3 + 1.2 x) of 1 - exp(-x64) (exp(-x) <= 1 turns the
// relative error of __expf into an absolute one), and u_f32(k) within 2^-25
// of u.  Outside twice that band the FP32 comparison decides; inside it x64()
// and FP64 do.  A negative x never activates: 1 - exp(-x) < 0 <= u.
template <class F64>
__device__ __forceinline__ bool wolff_activates(uint32_t k, float x, float err, F64&& x64)
{
    const float tol = 2.0f * (err + 0x1.0p-23f * (3.0f + 1.2f * fabsf(x)));
    if (x <= -tol) return false;
    if (x >= tol) {
        const float p = 1.0f - __expf(-x), u = u_f32(k);
        if (u < p - tol) return true;
        if (u > p + tol) return false;
    }
    return u_f64(k) < 1.0 - exp(-x64());
}

// Error bounds (in units of log_p, resp. x) of the FP32 forms below, for the
// host to pass with each launch.  u = 2^-24; spins are unit vectors, so every
// component and every neighbour term is at most 1 in magnitude.
//  * VectorSpin<N> Metropolis over deg neighbours: h_c sums deg terms
//    ((deg - 1) deg u), each dot takes N fused products (N sqrt(N) deg u),
//    their difference, J, beta and the FP32 beta add 3 u |lp| <= 6 u beta |J|
//    sqrt(N) deg:  beta |J| u sqrt(N) deg (2 (N + deg - 1) + 8).
//  * Wolff on VectorSpin<N>: x = 2 beta J (r.s_i)(r.s_j), each dot within N u,
//    three products and the FP32 beta: beta |J| u (4 N + 8).
inline float vector_metropolis_err(double beta, double J, int N, uint32_t deg)
{
    return float(std::fabs(beta * J) * 0x1.0p-24 * std::sqrt(double(N)) * double(deg) * (2.0 * (N + deg - 1.0) + 8.0));
}
inline float vector_wolff_err(double beta, double J, int N)
{
    return float(std::fabs(beta * J) * 0x1.0p-24 * (4.0 * N + 8.0));
}
// XY on angles over d neighbours (xy_pass; the batched chains with d = 4):
// lp = -beta J ((cos p - cos t) C + (sin p - sin t) S) from __sincosf values
// within e = kSincosfAbsErr of the exact ones (every angle within
// kSincosfDomain) and FP32 roundings of at most u = 2^-24 of each result:
//   C, S (d values, sums up to d):          dC = d e + u (d (d + 1) / 2 - 1)
//   cos p - cos t, sin p - sin t (<= 2):    da = 2 e + 2 u
//   each product (<= 2 d, rounded):         dP = 2 dC + d da + 2 d u
//   their sum (<= 4 d), J and beta (each rounded to FP32 and multiplied):
//   beta |J| (2 dP + 4 d u (sum) + 8 d u (J) + 8 d u (beta)).
// The factor 1 + 2^-10 covers the second-order terms.  For d = 4:
// beta |J| (32 e + 148 u), about 4.8e-5 beta |J|.
inline float xy_metropolis_err(double beta, double J, uint32_t deg)
{
    const double e = kSincosfAbsErr, u = 0x1.0p-24, d = double(deg);
    const double dC = d * e + u * (d * (d + 1.0) / 2.0 - 1.0);
    const double da = 2.0 * e + 2.0 * u;
    const double dP = 2.0 * dC + d * da + 2.0 * d * u;
    return float(std::fabs(beta * J) * (2.0 * dP + 20.0 * d * u) * (1.0 + 0x1.0p-10));
}
// The U(1) gauge passes (umc_gauge_kernels.cuh, and the plain batched U(1)
// chains), deg = cells per link: a cell's staple angle sums three FP32 angles
// of at most 2 pi (38 u), sincosf adds 2 u, deg of them make Sr and Si; with
// the old and new cos/sin and the products: driver_beta model_beta u deg
// (4 (40 + deg) + 24).
inline float u1_metropolis_err(double driver_beta, double model_beta, uint32_t deg)
{
    return float(std::fabs(driver_beta * model_beta) * 0x1.0p-24 * double(deg) * (4.0 * (40.0 + deg) + 24.0));
}

// ------------------------------------------------------ VectorSpin<N> pass

constexpr int kPropSphere = 0;
constexpr int kPropRotation = 1;

struct VecArgs
{
    float* f;  // component c of colour-major site k at f[c * n + k]
    uint32_t n, first, count;
    uint64_t kbase;
    float J, beta, delta;
    PassOut out;
    double J64, beta64;  // the coupling and beta of the FP64 decisions
    float err;           // vector_metropolis_err
};

// -beta dE of site k taking cand (energy_diff_at, example/vector_spin.hpp:50-60:
// sum over bonds of -J (cand.s_j - s.s_j)) in FP64 on the FP32 state.  Out of
// line: it runs only for decisions the FP32 test cannot call.
template <int N, class Topo>
__device__ __noinline__ double vector_log_ratio64(const VecArgs& a, Topo t, uint32_t k, SpinVal<N> cand, SpinVal<N> s)
{
    double d = 0.0;
    t.neighbours(k, [&](uint32_t j, bool) {
        double pj = 0.0, oj = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c) {
            const double v = a.f[c * a.n + j];
            pj += double(cand.v[c]) * v;
            oj += double(s.v[c]) * v;
        }
        d += -a.J64 * (pj - oj);
    });
    return -a.beta64 * d;
}

// (kBlock, 4): at most 64 registers, the occupancy of the FP32 path; the
// out-of-line FP64 decision spills inside itself instead of widening it.
template <int N, int PROP, class Topo>
__global__ void __launch_bounds__(kBlock, 4) vector_pass(VecArgs a, Topo t)
{
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < a.count; q += gridDim.x * blockDim.x) {
        const uint32_t k = a.first + q;
        float s[N], h[N], he[N];
#pragma unroll
        for (int c = 0; c < N; ++c) {
            s[c] = a.f[c * a.n + k];
            h[c] = 0.0f;
            he[c] = 0.0f;
        }
        t.neighbours(k, [&](uint32_t j, bool early) {
#pragma unroll
            for (int c = 0; c < N; ++c) {
                const float v = a.f[c * a.n + j];
                h[c] += v;
                he[c] += early ? v : 0.0f;
            }
        });
        KeyedPcg g = KeyedPcg::open(a.kbase, k);
        float cand[N];
        bool ok = true;
        if constexpr (PROP == kPropSphere) sphere_sample<N>(g, cand);
        else ok = local_rotation<N>(g, a.delta, s, cand);
        bool acc_ok = false;
        if (ok) {
            // energy_diff_at, example/vector_spin.hpp:50-60: -J (p.h - s.h)
            const float dE = -a.J * (vdot<N>(cand, h) - vdot<N>(s, h));
            acc_ok = metropolis_accept(g, -a.beta * dE, a.err, [&] {
                SpinVal<N> cv, sv;
#pragma unroll
                for (int c = 0; c < N; ++c) {
                    cv.v[c] = cand[c];
                    sv.v[c] = s[c];
                }
                return vector_log_ratio64<N>(a, t, k, cv, sv);
            });
        }
        if (acc_ok) {
#pragma unroll
            for (int c = 0; c < N; ++c) {
                s[c] = cand[c];
                a.f[c * a.n + k] = cand[c];
            }
        }
        acc[0] += double(-a.J * vdot<N>(s, he));
#pragma unroll
        for (int c = 0; c < N; ++c) acc[1 + c] += double(s[c]);
        acc[7] += acc_ok ? 1.0 : 0.0;
    }
    finish_pass<kObs>(acc, a.out);
}

// --------------------------------------------------------- XY on angles

// PairModel<U1Dof, -J cos(ti - tj)> (model/pair.hpp:53-64) with U1Shift.
// sum_j cos(t - tj) = cos(t) C + sin(t) S with C, S the neighbour sums.
struct XYArgs
{
    float* th;
    uint32_t first, count;
    uint64_t kbase;
    float J, beta, width;
    PassOut out;
    double J64, beta64;  // the coupling and beta of the FP64 decisions
    float err;           // xy_metropolis_err
};

// -beta dE of angle site k going from t0 to p: -J sum_j (cos(p - t_j) -
// cos(t0 - t_j)) (PairModel with the XY term, model/pair.hpp:53-64), in FP64 on
// the FP32 angles.  Out of line: it runs only for decisions the FP32 test
// cannot call.
template <class Topo>
__device__ __noinline__ double xy_log_ratio64(const XYArgs& a, Topo t, uint32_t k, float t0, float p)
{
    // sum_j cos(x - t_j) = cos x C + sin x S, C and S the neighbours' sums
    double C = 0.0, S = 0.0;
    t.neighbours(k, [&](uint32_t j, bool) {
        double sn, cs;
        sincos_cw64(double(a.th[j]), sn, cs);
        C += cs;
        S += sn;
    });
    double s0, c0, s1, c1;
    sincos_cw64(double(t0), s0, c0);
    sincos_cw64(double(p), s1, c1);
    return a.beta64 * a.J64 * ((c1 - c0) * C + (s1 - s0) * S);
}

// (kBlock, 5): at most 48 registers (see vector_pass).
template <class Topo>
__global__ void __launch_bounds__(kBlock, 5) xy_pass(XYArgs a, Topo t)
{
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < a.count; q += gridDim.x * blockDim.x) {
        const uint32_t k = a.first + q;
        float C = 0.f, S = 0.f, Ce = 0.f, Se = 0.f;
        t.neighbours(k, [&](uint32_t j, bool early) {
            float sn, cs;
            __sincosf(a.th[j], &sn, &cs);
            C += cs;
            S += sn;
            Ce += early ? cs : 0.f;
            Se += early ? sn : 0.f;
        });
        float th = a.th[k];
        KeyedPcg g = KeyedPcg::open(a.kbase, k);
        const float p = u1_shift(g, a.width, th);
        float so, co, sp, cp;
        __sincosf(th, &so, &co);
        __sincosf(p, &sp, &cp);
        const float dE = -a.J * ((cp - co) * C + (sp - so) * S);
        const bool ok = metropolis_accept(g, -a.beta * dE, a.err, [&] { return xy_log_ratio64(a, t, k, th, p); });
        if (ok) {
            a.th[k] = p;
            th = p;
            co = cp;
            so = sp;
        }
        acc[0] += double(-a.J * (co * Ce + so * Se));
        acc[1] += double(co);
        acc[2] += double(so);
        acc[7] += ok ? 1.0 : 0.0;
    }
    finish_pass<kObs>(acc, a.out);
}

// ------------------------------------------------------------- observables

// E = 0.5 * sum_i energy_at(i) (example/ising.hpp:35-43,
// example/vector_spin.hpp:39-47) and M = sum_i s_i over a colour-major CSR.
// MODEL: 0 Ising (int8), N >= 1 VectorSpin<N> (FP32 SoA), -1 XY angles.
template <int MODEL>
__global__ void __launch_bounds__(kBlock) observe_csr(const void* field, uint32_t n, const uint32_t* off,
                                                      const uint32_t* adj, float J, PassOut out,
                                                      const unsigned long long* size_slot)
{
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if constexpr (MODEL == 0) {
            const int8_t* s = static_cast<const int8_t*>(field);
            int32_t e = 0;
            for (uint32_t a = off[i]; a < off[i + 1]; ++a) e += int32_t(s[i]) * int32_t(s[adj[a]]);
            acc[0] += 0.5 * double(-J) * double(e);
            acc[1] += double(s[i]);
        } else if constexpr (MODEL > 0) {
            const float* f = static_cast<const float*>(field);
            float si[MODEL];
#pragma unroll
            for (int c = 0; c < MODEL; ++c) si[c] = f[c * n + i];
            double e = 0.0;
            for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
                float sj[MODEL];
#pragma unroll
                for (int c = 0; c < MODEL; ++c) sj[c] = f[c * n + adj[a]];
                e += double(-J * vdot<MODEL>(si, sj));
            }
            acc[0] += 0.5 * e;
#pragma unroll
            for (int c = 0; c < MODEL; ++c) acc[1 + c] += double(si[c]);
        } else {
            const float* th = static_cast<const float*>(field);
            double e = 0.0;
            for (uint32_t a = off[i]; a < off[i + 1]; ++a) e += double(-J * cosf(th[i] - th[adj[a]]));
            acc[0] += 0.5 * e;
            float sn, cs;
            sincosf(th[i], &sn, &cs);
            acc[1] += double(cs);
            acc[2] += double(sn);
        }
    }
    if (size_slot && blockIdx.x == 0 && threadIdx.x == 0) acc[7] = double(*size_slot);
    finish_pass<kObs>(acc, out);
}

// ----------------------------------------------------------------- Wolff

// Wolff::flip (driver.hpp:104-162) as bond activation + connected components:
// the reference's depth-first growth adds exactly the sites reachable from the
// seed over activated bonds, because every bond it tests gets the same keyed
// draw whichever end reaches it first and every bond leaving the final cluster
// is tested and rejected.  MODEL: 0 Ising with FixedAxis, N >= 1 VectorSpin<N>
// with a UniformSphereN<N> axis.
struct WolffArgs
{
    void* field;
    uint32_t n;
    const uint32_t* off;
    const uint32_t* adj;
    const uint32_t* slot;  // edge-list index of each colour-major CSR slot
    uint32_t* lab;
    uint32_t* lab_next;
    uint64_t seed, flip;
    float J, beta;
    unsigned long long cw[2];  // Ising: activate iff draw < cw[s_i s_j > 0]
    DevCtl* ctl;
    unsigned long long* size_slot;
    double J64, beta64;  // VectorSpin: the coupling and beta of the FP64 decisions
    float err;           // VectorSpin: vector_wolff_err
};

// Activation of one bond (driver.hpp:150-151): uni() < 1 - exp(-beta dE).
// The reference's energy_diff_bond, -J (nb.s_i - s_j.s_i) with the reflected
// nb = s_j - 2 (s_j.r) r, equals 2 J (r.s_i)(r.s_j); that symmetric form is
// used in FP32 so the decision does not depend on which end reaches the bond
// first.  Near the threshold the reference's own form decides in FP64
// (wolff_activates), on the FP32 spins and axis, and is symmetric to within
// 1e-16.  Ising compares the draw with integer thresholds (exact).
__device__ __forceinline__ bool ising_bond_active(const unsigned long long* cw, int si, int sj, uint32_t k)
{
    return uint64_t(k) < cw[si * sj > 0 ? 1 : 0];
}

// beta dE of bond (i, j) with s_j reflected: energy_diff_bond
// (example/vector_spin.hpp:62-68) with nb = s_j - 2 (s_j.r) r (driver.hpp:
// 142-146), in FP64 on the FP32 spins and axis.  Out of line: it runs only for
// decisions the FP32 test cannot call.
template <int N>
__device__ __noinline__ double vector_bond_x64(SpinVal<N> si, SpinVal<N> sj, SpinVal<N> r, double J64, double beta64)
{
    double d = 0.0;
#pragma unroll
    for (int c = 0; c < N; ++c) d += double(sj.v[c]) * double(r.v[c]);
    double pn = 0.0, po = 0.0;
#pragma unroll
    for (int c = 0; c < N; ++c) {
        const double nb = double(sj.v[c]) - 2.0 * d * double(r.v[c]);
        pn += nb * double(si.v[c]);
        po += double(sj.v[c]) * double(si.v[c]);
    }
    return beta64 * (-J64 * (pn - po));
}

template <int N>
__device__ __forceinline__ bool vector_bond_active(float J, float beta, double J64, double beta64, float err,
                                                   const float* si, const float* sj, const float* r, uint32_t k)
{
    const float x = beta * (2.0f * J * (vdot<N>(si, r) * vdot<N>(sj, r)));
    return wolff_activates(k, x, err, [&] {
        SpinVal<N> a, b, c;
#pragma unroll
        for (int q = 0; q < N; ++q) {
            a.v[q] = si[q];
            b.v[q] = sj[q];
            c.v[q] = r[q];
        }
        return vector_bond_x64<N>(a, b, c, J64, beta64);
    });
}

// Axis and seed site of one flip (driver.hpp:110-115), from the axis key.
template <int MODEL>
__device__ __forceinline__ uint32_t wolff_axis(const WolffArgs& a, float* r)
{
    KeyedPcg g = KeyedPcg::open_key(a.seed, a.flip, kTagAxis, 0);
    if constexpr (MODEL == 0) r[0] = 1.0f;
    else sphere_sample<MODEL>(g, r);
    return uint32_t(u_f64(g.next()) * double(a.n));  // same double product as the reference
}

// (kBlock, 8): at most 32 registers (see vector_pass).
template <int MODEL>
__global__ void __launch_bounds__(kBlock, 8) wolff_union(WolffArgs a)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    __shared__ float r_sh[4];
    if (threadIdx.x == 0) {
        float r[N];
        wolff_axis<MODEL>(a, r);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
        if (blockIdx.x == 0) *a.size_slot = 0ull;
    }
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint64_t kb = key_base(key_seed(a.seed, a.flip, kTagBond));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        const uint32_t a0 = a.off[i], a1 = a.off[i + 1];
        if constexpr (MODEL == 0) {
            const int8_t* s = static_cast<const int8_t*>(a.field);
            const int32_t si = s[i];
            for (uint32_t q = a0; q < a1; ++q) {
                const uint32_t j = a.adj[q];
                if (j <= i) continue;
                const uint32_t k = first_draw(kb, a.slot[q]);
                if (ising_bond_active(a.cw, si, s[j], k)) uf_union(a.lab, i, j, a.n + 1, &a.ctl->status);
            }
        } else {
            const float* f = static_cast<const float*>(a.field);
            float si[N];
#pragma unroll
            for (int c = 0; c < N; ++c) si[c] = f[c * a.n + i];
            for (uint32_t q = a0; q < a1; ++q) {
                const uint32_t j = a.adj[q];
                if (j <= i) continue;
                float t[N];
#pragma unroll
                for (int c = 0; c < N; ++c) t[c] = f[c * a.n + j];
                const uint32_t k = first_draw(kb, a.slot[q]);
                if (vector_bond_active<N>(a.J, a.beta, a.J64, a.beta64, a.err, si, t, r, k))
                    uf_union(a.lab, i, j, a.n + 1, &a.ctl->status);
            }
        }
    }
}

template <int MODEL>
__global__ void __launch_bounds__(kBlock) wolff_flip(WolffArgs a)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    __shared__ float r_sh[4];
    __shared__ uint32_t root_sh;
    if (threadIdx.x == 0) {
        float r[N];
        const uint32_t seed = wolff_axis<MODEL>(a, r);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
        root_sh = seed < a.n ? uf_find(a.lab, seed, a.n + 1, &a.ctl->status) : 0xFFFFFFFFu;
    }
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint32_t root = root_sh;
    double cnt[1] = {0.0};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
        if (uf_find(a.lab, i, a.n + 1, &a.ctl->status) == root) {
            cnt[0] += 1.0;
            if constexpr (MODEL == 0) {
                int8_t* s = static_cast<int8_t*>(a.field);
                s[i] = int8_t(-s[i]);
            } else {
                float* f = static_cast<float*>(a.field);
                float si[N];
#pragma unroll
                for (int c = 0; c < N; ++c) si[c] = f[c * a.n + i];
                reflect<N>(si, r);
#pragma unroll
                for (int c = 0; c < N; ++c) f[c * a.n + i] = si[c];
            }
        }
        a.lab_next[i] = i;
    }
    block_sum<1>(cnt);
    if (threadIdx.x == 0 && cnt[0] > 0.0) atomicAdd(a.size_slot, (unsigned long long)cnt[0]);
}

static __global__ void iota_u32(uint32_t* p, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = i;
}

// ------------------------------------------------- layout conversion / start

// Colour-major index of site i: closed form on the regular lattices, a table
// otherwise.
struct Placement
{
    const uint32_t* position;  // null on regular lattices
    uint32_t Lx, Ly, half;
    __device__ __forceinline__ uint32_t operator()(uint32_t i) const
    {
        if (position) return position[i];
        const uint32_t x = i % Lx, r = i / Lx, y = r % Ly, z = r / Ly;
        return ((x + y + z) & 1u) * half + (i >> 1);
    }
};

// site-order AoS (the reference's data()) <-> colour-major SoA
template <class T>
__global__ void scatter_field(const T* src, T* dst, uint32_t n, uint32_t comps, Placement pl, bool angles)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = pl(i);
        for (uint32_t c = 0; c < comps; ++c) {
            T v = src[uint64_t(i) * comps + c];
            // XY angles: kept within the domain of the FP32 decisions' sincos bound
            if constexpr (std::is_same_v<T, float>)
                if (angles) v = wrap_angle(v);
            dst[uint64_t(c) * n + k] = v;
        }
    }
}

template <class T>
__global__ void gather_field(const T* src, T* dst, uint32_t n, uint32_t comps, Placement pl)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = pl(i);
        for (uint32_t c = 0; c < comps; ++c) dst[uint64_t(i) * comps + c] = src[uint64_t(c) * n + k];
    }
}

// Random start from keyed draws (tag kTagInit, id = site).  MODEL: 0 Ising
// (sign from u < 0.5), N >= 1 uniform on S^(N-1), -1 angle 2 pi u.
template <int MODEL>
__global__ void randomize_spins(void* field, uint32_t n, uint64_t seed, Placement pl)
{
    const uint64_t kb = key_base(key_seed(seed, 0, kTagInit));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = pl(i);
        KeyedPcg g = KeyedPcg::open(kb, i);
        if constexpr (MODEL == 0) {
            static_cast<int8_t*>(field)[k] = g.next() < 0x80000000u ? int8_t(-1) : int8_t(1);
        } else if constexpr (MODEL > 0) {
            float v[MODEL];
            sphere_sample<MODEL>(g, v);
            for (int c = 0; c < MODEL; ++c) static_cast<float*>(field)[uint64_t(c) * n + k] = v[c];
        } else {
            static_cast<float*>(field)[k] = twice_u_f32(g.next()) * 3.14159265358979f;
        }
    }
}

}  // namespace umc
