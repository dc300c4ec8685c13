// umc/keyed_pcg.cuh -- counter-keyed PCG32, identical on host and device.
//
// The reference draws every random number from one sequential Pcg32
// (rng.hpp:8-44), and how many it draws depends on the data (the accept draw is
// skipped when log_p >= 0, driver.hpp:40; Wolff draws once per tested bond,
// driver.hpp:151).  A sequential stream cannot be replayed by thousands of
// threads, so every update here opens its OWN reference-semantics Pcg32:
//
//     Pcg32(id_seed(key_seed(seed, counter, tag), id), 0)
//
//     key_seed(s, c, t) = mix64(mix64(s ^ (t << 32)) + c * 0x9E3779B97F4A7C15)
//     id_seed(k, id)    = mix64(k + (id + 1) * 0x9E3779B97F4A7C15)
//     mix64             = splitmix64 finaliser (Steele, Lea & Flood, 2014)
//
// and consumes its draws in the same order the reference driver would.  With
// stream 0 the constructor (rng.hpp:14-20) leaves state = (s + 1) * A + 1 and
// increment 1.
//
// Why the id goes into the seed: an earlier keying gave every id of a key the
// SAME seed and a per-id increment (stream = a 32-bit hash of id).  Then the
// first states of two ids differ by an offset that depends on the two ids only,
// identical at every sweep, and the small correlation between the XSH-RR
// outputs of states a fixed offset apart never averages out: plain U(1)
// Metropolis on a 4 x 4 torus at beta = 1 settled 2.5e-3 (7 sigma) below the
// exact plaquette.  Hashing (key, id) into the seed gives every update an
// independent state at every sweep.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define UMC_HD __host__ __device__ __forceinline__
#else
#define UMC_HD inline
#endif

namespace umc {

constexpr uint64_t kPcgMult = 6364136223846793005ULL;  // rng.hpp:34
constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ULL;

// Key tags: which kind of update a key belongs to.
constexpr uint32_t kTagBond = 1;   // Wolff bond activation, id = edge index
constexpr uint32_t kTagAxis = 2;   // Wolff axis + seed draw, id = 0
constexpr uint32_t kTagInit = 3;   // random start, id = site
constexpr uint32_t kTagSwap = 4;   // replica exchange, id = ladder slot
constexpr uint32_t kTagLearn = 5;  // learned-proposal training minibatch
UMC_HD constexpr uint32_t tag_site(uint32_t hit) { return 0x100u + hit; }  // Metropolis hit

UMC_HD uint64_t mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return z;
}

UMC_HD uint64_t key_seed(uint64_t seed, uint64_t counter, uint32_t tag)
{
    return mix64(mix64(seed ^ (uint64_t(tag) << 32)) + counter * kGolden);
}

// lowbias32 (Wellons, 2018), a bijection on 32 bits; the union-find linking
// priority of a site (umc_device.cuh).
UMC_HD uint32_t stream_id(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

// Per-key base of the ids' seeds (the key seed itself).
UMC_HD uint64_t key_base(uint64_t kseed) { return kseed; }

// Seed of id's stream under a key.
UMC_HD uint64_t id_seed(uint64_t kbase, uint32_t id) { return mix64(kbase + (uint64_t(id) + 1ULL) * kGolden); }

// First state of Pcg32(seed, 0): (seed + 1) * A + 1.
UMC_HD uint64_t first_state(uint64_t seed) { return (seed + 1ULL) * kPcgMult + 1ULL; }

// XSH-RR output of a state (rng.hpp:36-39).
UMC_HD uint32_t pcg_output(uint64_t old)
{
#if defined(__CUDA_ARCH__)
    const uint32_t lo = uint32_t(old), hi = uint32_t(old >> 32);
    // x = old ^ (old >> 18) restricted to the bits the output uses
    const uint32_t xlo = lo ^ __funnelshift_r(lo, hi, 18);
    const uint32_t xhi = hi ^ (hi >> 18);
    const uint32_t xs = __funnelshift_r(xlo, xhi, 27);
    const uint32_t rot = hi >> 27;
    return __funnelshift_r(xs, xs, rot);
#else
    const uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = uint32_t(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
#endif
}

// One keyed stream: the reference Pcg32 after construction.
struct KeyedPcg
{
    uint64_t state;
    uint64_t inc;

    UMC_HD static KeyedPcg open(uint64_t kbase, uint32_t id)
    {
        KeyedPcg g;
        g.state = first_state(id_seed(kbase, id));
        g.inc = 1ULL;
        return g;
    }
    UMC_HD static KeyedPcg open_key(uint64_t seed, uint64_t counter, uint32_t tag, uint32_t id)
    {
        return open(key_base(key_seed(seed, counter, tag)), id);
    }
    // Pcg32::next (rng.hpp:31-40)
    UMC_HD uint32_t next()
    {
        const uint64_t old = state;
        state = old * kPcgMult + inc;
        return pcg_output(old);
    }
};

// First draw of a key without materialising the stream (one draw per site).
UMC_HD uint32_t first_draw(uint64_t kbase, uint32_t id) { return pcg_output(first_state(id_seed(kbase, id))); }

// ---- one draw per site, 16 sites per stream ------------------------------------
// Ising Metropolis draws exactly one uniform per site (Flip proposes without a
// draw).  There site k reads output (k % 16) of the stream of id k / 16: one
// hash per 16 sites, and consecutive outputs of one Pcg32 within a group.
constexpr uint32_t kGroupSites = 16;

// Jump table of Pcg32 stream 0 (increment 1): state_j = A^j state_0 + C_j with
// C_j = A^0 + ... + A^(j-1), all mod 2^64.
struct PcgJump
{
    uint64_t mul[kGroupSites], add[kGroupSites];
    constexpr PcgJump() : mul(), add()
    {
        uint64_t m = 1, c = 0;
        for (uint32_t j = 0; j < kGroupSites; ++j) {
            mul[j] = m;
            add[j] = c;
            c = c * kPcgMult + 1ULL;
            m = m * kPcgMult;
        }
    }
};
constexpr PcgJump kPcgJump{};

// Advance a stream-0 state by j < 16 outputs: four conditional jumps by 1, 2,
// 4 and 8 steps with compile-time constants (no table in memory).
UMC_HD uint64_t pcg_advance(uint64_t st, uint32_t j)
{
    constexpr uint64_t m1 = kPcgJump.mul[1], a1 = kPcgJump.add[1];
    constexpr uint64_t m2 = kPcgJump.mul[2], a2 = kPcgJump.add[2];
    constexpr uint64_t m4 = kPcgJump.mul[4], a4 = kPcgJump.add[4];
    constexpr uint64_t m8 = kPcgJump.mul[8], a8 = kPcgJump.add[8];
    if (j & 1u) st = st * m1 + a1;
    if (j & 2u) st = st * m2 + a2;
    if (j & 4u) st = st * m4 + a4;
    if (j & 8u) st = st * m8 + a8;
    return st;
}

// The draw of site k under a key (one draw per site).
UMC_HD uint32_t group_draw(uint64_t kbase, uint32_t k)
{
    return pcg_output(pcg_advance(first_state(id_seed(kbase, k / kGroupSites)), k % kGroupSites));
}

// ---- conversions of a 32-bit draw k (the reference uses u = k * 2^-32) ----
// u in FP64, exactly the reference's value.
UMC_HD double u_f64(uint32_t k) { return double(k) * 0x1.0p-32; }
// 2u - 1 in FP32 with a single rounding: 2k - 2^32 = 2 (k - 2^31).
UMC_HD float sym_f32(uint32_t k) { return float(int32_t(k ^ 0x80000000u)) * 0x1.0p-31f; }
// 2u in FP32 (argument of sincospif for an angle 2 pi u).
UMC_HD float twice_u_f32(uint32_t k) { return float(k) * 0x1.0p-31f; }
// u in FP32.
UMC_HD float u_f32(uint32_t k) { return float(k) * 0x1.0p-32f; }

}  // namespace umc
