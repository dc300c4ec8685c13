// umc_batch.cu -- many independent XY chains with replica-exchange ladders.
//
// The reference drives one chain per driver object (driver.hpp:17-68) and has
// no notion of batching or parallel tempering; this is the engine's batched
// form of its XY angle model (PairModel<U1Dof, -J cos(ti - tj)> + U1Shift).
//
// Layout: every chain is a periodic L x L lattice (L even, one L per ladder) in
// the two-colour layout of umc_spin_kernels.cuh (colour c, site/2); all chains
// sit back to back in one FP32 buffer.  Chain c belongs to ladder c / R and
// starts at temperature slot c % R.
//
// One segment = S sweeps of every chain (each chain at the beta of the slot it
// holds) followed by one exchange round per ladder.  A segment is one kernel
// per lattice-size group -- the groups run as parallel branches of a CUDA
// graph -- plus one swap kernel.  Within a group a CTA either owns several
// small chains (chains per CTA, cpc) or a cluster of CTAs shares one large
// chain (CTAs per chain, cpk) and synchronises with the hardware cluster
// barrier.  cpc / cpk / block size come from a short autotuning run per group.
//
// Keys: site k of chain c at sweep s draws from (chain_seed[c], s, site tag, k),
// exactly the stream a single XY chain with seed chain_seed[c] would use, so a
// chain's trajectory can be replayed by the single-chain oracle.  The swap of
// slots (k, k+1) in ladder l at round r draws from (ladder_seed[l], r, 4, k).

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "umc_chain.hpp"
#include "umc_spin_kernels.cuh"
#include "umc_nvtx.hpp"

namespace cg = cooperative_groups;

namespace umc {
namespace {

constexpr uint32_t kMaxCpc = 64;       // chains per CTA
constexpr uint32_t kMaxRungs = 64;     // replicas per ladder
constexpr uint32_t kMaxShares = 8;     // CTAs per chain (cluster size)
constexpr unsigned kBatchErrRecords = 1u;

struct BatchCounters
{
    unsigned long long sweep;     // sweeps done by every chain
    unsigned long long round;     // exchange rounds done
    unsigned long long rec;       // records written since the last fetch
    unsigned long long capacity;  // record slots
    unsigned int status;
    unsigned int pad;
};

struct SegArgs
{
    float* theta;
    const unsigned long long* off;  // per chain
    const uint32_t* chains;         // chain ids of this group
    uint32_t n_chains;              // in this group
    uint32_t L, H, half;
    uint32_t cpc, cpk;
    uint32_t sweeps;
    const BatchCounters* ctr;
    const uint32_t* slot_of_chain;
    const double* betas;  // betas[ladder * R + slot]
    uint32_t R;
    const unsigned long long* chain_seed;
    float J, width;
    double* part;  // per chain, kMaxShares shares: [E, Mx, My, accepted]
    double J64;    // the coupling of the FP64 decisions
    float err_per_beta;  // xy_metropolis_err(1, J, 4): the bound scales with beta
};

template <bool CG>
__device__ __forceinline__ float ldf(const float* p)
{
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

// -beta dE of an XY site with four neighbour angles going from t to p, in
// FP64 on the FP32 angles: dE = -J sum_q (cos(p - n_q) - cos(t - n_q))
// = -J ((cos p - cos t) C + (sin p - sin t) S), C and S the sums of the
// neighbours' cosines and sines (the six sincos in lockstep).  Out of line:
// it runs only for decisions the FP32 test cannot call.
__device__ __noinline__ double xy4_log_ratio64(double J64, double beta64, float t, float p, float n0, float n1, float n2,
                                               float n3)
{
    const float v[6] = {n0, n1, n2, n3, t, p};
    double sn[6], cs[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) sincos_cw64(double(v[q]), sn[q], cs[q]);
    const double C = (cs[0] + cs[1]) + (cs[2] + cs[3]), S = (sn[0] + sn[1]) + (sn[2] + sn[3]);
    return beta64 * J64 * ((cs[5] - cs[4]) * C + (sn[5] - sn[4]) * S);
}

// One XY site update (the body of xy_pass in umc_spin_kernels.cuh) on chain
// data `th`; neighbours through L1 inside one CTA, through L2 in a cluster.
// In a cluster, rows [row_lo, row_lo + row_n) of both colours are written by
// this CTA alone, so they are read through L1; the two halo rows belong to
// other CTAs of the cluster and are read through L2.
// other / own: the chain's two colour classes (the one read, the one
// updated); err: beta * err_per_beta, the FP32 test's bound at this beta.
template <bool CLUSTER>
__device__ __forceinline__ bool xy_update(const SegArgs& a, const float* other, float* own, uint32_t colour,
                                          uint32_t y, uint32_t i, uint64_t kbase, float beta, double beta64,
                                          float err, uint32_t row_lo, uint32_t row_n)
{
    const uint32_t L = a.L, H = a.H;
    const uint32_t p = (y + colour) & 1u;
    const uint32_t ym = y == 0 ? L - 1 : y - 1, yp = y + 1 == L ? 0u : y + 1;
    const uint32_t i2 = p ? (i + 1 == H ? 0u : i + 1) : (i == 0 ? H - 1 : i - 1);
    const bool l2m = CLUSTER && ym - row_lo >= row_n, l2p = CLUSTER && yp - row_lo >= row_n;
    const float nb[4] = {other[y * H + i], other[y * H + i2],
                         l2m ? __ldcg(other + ym * H + i) : other[ym * H + i],
                         l2p ? __ldcg(other + yp * H + i) : other[yp * H + i]};
    float C = 0.f, S = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        float sn, cs;
        __sincosf(nb[q], &sn, &cs);
        C += cs;
        S += sn;
    }
    const uint32_t k = colour * a.half + y * H + i;
    const float t = own[y * H + i];
    KeyedPcg g = KeyedPcg::open(kbase, k);
    const float prop = u1_shift(g, a.width, t);
    float so, co, sp, cp;
    __sincosf(t, &so, &co);
    __sincosf(prop, &sp, &cp);
    const float dE = -a.J * ((cp - co) * C + (sp - so) * S);
    const bool ok = metropolis_accept(g, -beta * dE, err, [&] {
        return xy4_log_ratio64(a.J64, beta64, t, prop, nb[0], nb[1], nb[2], nb[3]);
    });
    if (!ok) return false;
    own[y * H + i] = prop;
    return true;
}

// Per-CTA staging of the chains a CTA updates: per owned chain and sweep the
// key base, beta and field offset (computed once per CTA instead of once per
// site update), and its accepted-update count.
struct SegShared
{
    unsigned int accepted[kMaxCpc];
    uint64_t kb[kMaxCpc];
    float beta[kMaxCpc];
    double beta64[kMaxCpc];
    unsigned long long off[kMaxCpc];
};

// a.sweeps sweeps of chain_n chains (ids chains[0..chain_n)) of side a.L, rows
// [row_lo, row_lo + row_n) of each (all of them unless a cluster shares the
// chains), then their observables into a.part (share `share`).  CLUSTER: the
// CTAs of a thread-block cluster share the chains and meet at the cluster
// barrier between colour passes; else one CTA and __syncthreads.
template <bool CLUSTER>
__device__ __forceinline__ void run_share(const SegArgs& a, SegShared& sh, const uint32_t* chains, uint32_t chain_n,
                                          uint32_t row_lo, uint32_t row_n, uint32_t share)
{
    const uint64_t sweep0 = a.ctr->sweep;
    const uint32_t H = a.H, half = a.half;
    if (threadIdx.x < kMaxCpc) sh.accepted[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t per_chain = row_n * H;  // sites of one colour per chain share
    const uint32_t work = chain_n * per_chain;
    // H and per_chain are powers of two for the usual sides: shifts instead of
    // integer divisions (uniform branch)
    const bool pow2 = (H & (H - 1)) == 0 && (per_chain & (per_chain - 1)) == 0;
    const uint32_t hs = __ffs(H) - 1, ps = __ffs(per_chain) - 1;
    for (uint32_t s = 0; s < a.sweeps; ++s) {
        for (uint32_t ci = threadIdx.x; ci < chain_n; ci += blockDim.x) {
            const uint32_t chain = chains[ci];
            sh.kb[ci] = key_base(key_seed(a.chain_seed[chain], sweep0 + s, tag_site(0)));
            sh.beta64[ci] = a.betas[(chain / a.R) * a.R + a.slot_of_chain[chain]];
            sh.beta[ci] = float(sh.beta64[ci]);
            sh.off[ci] = a.off[chain];
        }
        __syncthreads();
        const auto site_of = [&](uint32_t w, uint32_t& ci, uint32_t& y, uint32_t& i) {
            if (pow2) {
                ci = w >> ps;
                const uint32_t r = w & (per_chain - 1);
                y = row_lo + (r >> hs);
                i = r & (H - 1);
            } else {
                ci = w / per_chain;
                const uint32_t r = w - ci * per_chain;
                y = row_lo + r / H;
                i = r % H;
            }
        };
        for (uint32_t colour = 0; colour < 2; ++colour) {
            // accepted updates counted in a register while the thread stays
            // on one chain (its items change chain every per_chain / blockDim
            // iterations at most), added to the chain's count on a change
            // (the chain's field, key base and betas likewise stay in registers)
            uint32_t cur = 0xFFFFFFFFu, cnt = 0;
            const float* other = nullptr;
            float* own = nullptr;
            uint64_t kb = 0;
            float beta = 0.f, err = 0.f;
            double beta64 = 0.0;
            for (uint32_t w = threadIdx.x; w < work; w += blockDim.x) {
                uint32_t ci, y, i;
                site_of(w, ci, y, i);
                if (ci != cur) {
                    if (cnt) atomicAdd(&sh.accepted[cur], cnt);
                    cur = ci;
                    cnt = 0;
                    float* th = a.theta + sh.off[ci];
                    other = th + (1u - colour) * half;
                    own = th + colour * half;
                    kb = sh.kb[ci];
                    beta = sh.beta[ci];
                    beta64 = sh.beta64[ci];
                    err = beta * a.err_per_beta;
                }
                cnt += xy_update<CLUSTER>(a, other, own, colour, y, i, kb, beta, beta64, err, row_lo, row_n) ? 1u : 0u;
            }
            if (cnt) atomicAdd(&sh.accepted[cur], cnt);
            if constexpr (CLUSTER) cg::this_cluster().sync();
            else __syncthreads();
        }
    }
    // observables of this CTA's share, per chain, in FP64 (fixed-order sums)
    for (uint32_t ci = 0; ci < chain_n; ++ci) {
        const uint32_t chain = chains[ci];
        const float* th = a.theta + a.off[chain];
        double v[3] = {0, 0, 0};
        for (uint32_t r = threadIdx.x; r < per_chain; r += blockDim.x) {
            const uint32_t y = row_lo + r / H, i = r % H;
            // colour-1 site: its four bonds, all to colour 0, carry every bond once
            const uint32_t p = (y + 1u) & 1u;
            const uint32_t ym = y == 0 ? a.L - 1 : y - 1, yp = y + 1 == a.L ? 0u : y + 1;
            const uint32_t i2 = p ? (i + 1 == H ? 0u : i + 1) : (i == 0 ? H - 1 : i - 1);
            const float t1 = ldf<CLUSTER>(th + half + y * H + i);
            const float e = cosf(t1 - ldf<CLUSTER>(th + y * H + i)) + cosf(t1 - ldf<CLUSTER>(th + y * H + i2)) +
                            cosf(t1 - ldf<CLUSTER>(th + ym * H + i)) + cosf(t1 - ldf<CLUSTER>(th + yp * H + i));
            v[0] += double(-a.J * e);
            float sn, cs;
            sincosf(t1, &sn, &cs);
            v[1] += double(cs);
            v[2] += double(sn);
            sincosf(ldf<CLUSTER>(th + y * H + i), &sn, &cs);
            v[1] += double(cs);
            v[2] += double(sn);
        }
        block_sum<3>(v);
        if (threadIdx.x == 0) {
            double* out = a.part + (uint64_t(chain) * kMaxShares + share) * 4;
            out[0] = v[0];
            out[1] = v[1];
            out[2] = v[2];
            out[3] = double(sh.accepted[ci]);
        }
    }
}

template <bool CLUSTER>
__global__ void __launch_bounds__(1024) xy_batch_segment(SegArgs a)
{
    __shared__ SegShared sh;
    uint32_t chain_lo, chain_n, row_lo, row_n, share = 0;
    if (CLUSTER) {
        chain_lo = blockIdx.x / a.cpk;
        chain_n = 1;
        share = blockIdx.x % a.cpk;
        row_n = a.L / a.cpk;
        row_lo = share * row_n;
    } else {
        chain_lo = blockIdx.x * a.cpc;
        chain_n = min(a.cpc, a.n_chains - chain_lo);
        row_lo = 0;
        row_n = a.L;
    }
    run_share<CLUSTER>(a, sh, a.chains + chain_lo, chain_n, row_lo, row_n, share);
}

// Ladder l's record of the segment [E, Mx, My, chain, beta, swap accepted,
// accepted updates, 0] for every temperature slot, then its exchange round:
// slots (k, k+1), k of the round's parity, swap their chains iff
// (beta_k - beta_{k+1})(E_k - E_{k+1}) >= 0 or log(u) < that product.  One
// warp: lane q sums the energy of the ladder's chains q and q + 32, writes
// the records of slots q and q + 32, and decides the pairs starting at
// parity + 2 q (+ 64): the pairs of a round are disjoint, so their swaps
// are independent.  Every sum runs over the shares in the same order as a
// single thread would.  part holds each chain's share partials (read
// through L2: another CTA may have written them in this launch); E is 64
// doubles of shared memory for this warp.
__device__ void exchange_ladder(uint32_t l, uint32_t R, unsigned long long round, unsigned long long rec, bool keep,
                                uint32_t n_ladders, const uint32_t* cpk_of_chain, const double* part,
                                const double* betas, uint32_t* holder, uint32_t* slot_of_chain,
                                const unsigned long long* ladder_seed, double* records, unsigned long long* swaps,
                                double* E)
{
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t q = lane; q < R; q += 32) {
        const uint32_t c = l * R + q, k = cpk_of_chain[c];
        double e = 0.0;
        for (uint32_t r = 0; r < k; ++r) e += __ldcg(part + (uint64_t(c) * kMaxShares + r) * 4);
        E[q] = e;
    }
    __syncwarp();
    for (uint32_t k = lane; k < R && keep; k += 32) {
        const uint32_t c = holder[l * R + k], nk = cpk_of_chain[c];
        double mx = 0.0, my = 0.0, acc = 0.0;
        for (uint32_t r = 0; r < nk; ++r) {
            mx += __ldcg(part + (uint64_t(c) * kMaxShares + r) * 4 + 1);
            my += __ldcg(part + (uint64_t(c) * kMaxShares + r) * 4 + 2);
            acc += __ldcg(part + (uint64_t(c) * kMaxShares + r) * 4 + 3);
        }
        double* out = records + ((rec * n_ladders + l) * R + k) * kObs;
        out[0] = E[c - l * R];
        out[1] = mx;
        out[2] = my;
        out[3] = double(c);
        out[4] = betas[l * R + k];
        out[5] = 0.0;
        out[6] = acc;
        out[7] = 0.0;
    }
    __syncwarp();  // every slot's holder read before any pair swaps
    const uint32_t parity = uint32_t(round & 1ull);
    const uint64_t kb = key_base(key_seed(ladder_seed[l], round, kTagSwap));
    for (uint32_t k = parity + 2 * lane; k + 1 < R; k += 64) {
        const uint32_t a = holder[l * R + k], b = holder[l * R + k + 1];
        const double delta = (betas[l * R + k] - betas[l * R + k + 1]) * (E[a - l * R] - E[b - l * R]);
        const bool acc = delta >= 0.0 || log(u_f64(first_draw(kb, k))) < delta;
        if (keep) records[((rec * n_ladders + l) * R + k) * kObs + 5] = acc ? 1.0 : 0.0;
        if (acc) {
            holder[l * R + k] = b;
            holder[l * R + k + 1] = a;
            slot_of_chain[a] = k + 1;
            slot_of_chain[b] = k;
            atomicAdd(swaps, 1ull);
        }
    }
    __syncwarp();
}

// The segment's bookkeeping once every ladder has exchanged: counters advance
// (or the record ring reports overflow).
__device__ __forceinline__ void close_segment(BatchCounters* ctr, unsigned long long round, unsigned long long rec,
                                              bool keep, uint32_t sweeps)
{
    ctr->round = round + 1;
    ctr->sweep += sweeps;
    if (keep) ctr->rec = rec + 1;
    else ctr->status |= kBatchErrRecords;
}

// One exchange round per ladder: one warp per ladder, up to 32 warps.
constexpr uint32_t kSwapWarps = 32;
__global__ void __launch_bounds__(kSwapWarps * 32) xy_batch_swap(BatchCounters* ctr, uint32_t n_ladders, uint32_t R,
                                                                 const uint32_t* cpk_of_chain, const double* part,
                                                                 const double* betas, uint32_t* holder,
                                                                 uint32_t* slot_of_chain,
                                                                 const unsigned long long* ladder_seed,
                                                                 double* records, unsigned long long* swaps,
                                                                 uint32_t sweeps)
{
    __shared__ double E[kSwapWarps][kMaxRungs];
    const unsigned long long round = ctr->round;
    const unsigned long long rec = ctr->rec;
    const bool keep = rec < ctr->capacity;
    __syncthreads();
    const uint32_t w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (uint32_t l = w; l < n_ladders; l += nw)
        exchange_ladder(l, R, round, rec, keep, n_ladders, cpk_of_chain, part, betas, holder, slot_of_chain,
                        ladder_seed, records, swaps, E[w]);
    __syncthreads();
    if (threadIdx.x == 0) close_segment(ctr, round, rec, keep, sweeps);
}

// ---------------------------------------------------- one persistent kernel
// The whole segment -- every chain's sweeps and every ladder's exchange -- in
// one launch of resident CTAs grouped in clusters of KC (1, 4 or 8).  Work
// items, largest first: a "big" chain is swept by a whole cluster (one row
// band per CTA, the cluster barrier between colour passes; with KC = 1 by one
// CTA, as the grouped form sweeps it); smaller chains are
// packed into CTA items of up to kPersistSites sites per colour.  CTAs take
// items from two atomic counters (big, then small), so the long items start
// first and the short ones fill the gaps.  The CTA that completes the last
// share of a ladder runs its exchange; the one that completes the last ladder
// advances the counters.  No CTA ever waits for another: the scheduler is
// atomics only, and the cluster barrier joins CTAs that are co-scheduled.
// cluster sizes the autotuner chooses between (a big chain's bands)
constexpr uint32_t kPersistClusters[3] = {1, 4, 8};
constexpr uint32_t kPersistSites = 8192;   // sites per colour of a CTA item
constexpr uint32_t kPersistBlock = 1024;

struct PersistArgs
{
    SegArgs seg;                // fields common to all items (seg.L/H/half set per item)
    const uint4* items;         // {first index into chains, chains, L, shares}
    const uint32_t* chains;     // chain ids in item order
    uint32_t n_big, n_items;
    unsigned* sched;            // [0] next big item, [1] next small item, [2] ladders exchanged
    unsigned* ladder_done;      // per ladder: chain shares completed
    const uint32_t* cpk_of_chain;
    uint32_t n_ladders;
    double* records;
    uint32_t* holder;
    const unsigned long long* ladder_seed;
    unsigned long long* swaps;
};

// Counts the item's chain shares as done; the CTA that completes a ladder
// exchanges it (its first warp), and the one that completes the last ladder
// closes the segment.
__device__ void complete_item(const PersistArgs& p, const uint32_t* chains, uint32_t chain_n, uint32_t shares,
                              double* E)
{
    if (threadIdx.x >= 32) return;
    const uint32_t lane = threadIdx.x;
    if (lane == 0) __threadfence();  // this CTA's partials before the counts that publish them
    const SegArgs& a = p.seg;
    for (uint32_t ci = 0; ci < chain_n; ++ci) {
        const uint32_t l = chains[ci] / a.R;
        unsigned last = 0;
        if (lane == 0) last = atomicAdd(&p.ladder_done[l], 1u) + 1u == a.R * shares ? 1u : 0u;
        if (!__shfl_sync(0xffffffffu, last, 0)) continue;
        __threadfence();
        const unsigned long long round = a.ctr->round, rec = a.ctr->rec;
        const bool keep = rec < a.ctr->capacity;
        exchange_ladder(l, a.R, round, rec, keep, p.n_ladders, p.cpk_of_chain, a.part, a.betas, p.holder,
                        const_cast<uint32_t*>(a.slot_of_chain), p.ladder_seed, p.records, p.swaps, E);
        __threadfence();  // every lane's writes before the count that ends the segment
        __syncwarp();
        if (lane == 0 && atomicAdd(&p.sched[2], 1u) + 1u == p.n_ladders)
            close_segment(const_cast<BatchCounters*>(a.ctr), round, rec, keep, a.sweeps);
    }
}

// KC: the cluster size; MINB: resident CTAs per SM the registers are capped
// for (1: 64 registers; 2: 32, with a few spills).
template <uint32_t KC, int MINB>
__global__ void __launch_bounds__(kPersistBlock, MINB) xy_batch_persistent(PersistArgs p)
{
    __shared__ SegShared sh;
    __shared__ uint32_t item_sh;
    __shared__ double E[kMaxRungs];  // the exchange's energies
    cg::cluster_group cl = cg::this_cluster();
    // big chains: the whole cluster, one band of rows per CTA
    for (;;) {
        if (cl.block_rank() == 0 && threadIdx.x == 0) item_sh = atomicAdd(&p.sched[0], 1u);
        cl.sync();
        const uint32_t it = *cl.map_shared_rank(&item_sh, 0);
        cl.sync();
        if (it >= p.n_big) break;
        const uint4 w = p.items[it];
        SegArgs a = p.seg;
        a.L = w.z;
        a.H = w.z / 2;
        a.half = w.z * w.z / 2;
        const uint32_t rows = w.z / KC, share = cl.block_rank();
        if constexpr (KC == 1) run_share<false>(a, sh, p.chains + w.x, 1, 0, rows, 0);  // the whole chain
        else run_share<true>(a, sh, p.chains + w.x, 1, share * rows, rows, share);
        complete_item(p, p.chains + w.x, 1, KC, E);
    }
    // packed smaller chains, one CTA each
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) item_sh = atomicAdd(&p.sched[1], 1u);
        __syncthreads();
        const uint32_t it = p.n_big + item_sh;
        if (it >= p.n_items) break;
        const uint4 w = p.items[it];
        SegArgs a = p.seg;
        a.L = w.z;
        a.H = w.z / 2;
        a.half = w.z * w.z / 2;
        run_share<false>(a, sh, p.chains + w.x, w.y, 0, w.z, 0);
        complete_item(p, p.chains + w.x, w.y, 1, E);
    }
}

// Random start: angle 2 pi u from key (chain_seed, 0, init tag, natural site id).
__global__ void xy_batch_randomize(float* theta, const unsigned long long* off, const uint32_t* Ls, uint32_t n_chains,
                                   const unsigned long long* chain_seed)
{
    const uint32_t c = blockIdx.y;
    if (c >= n_chains) return;
    const uint32_t L = Ls[c], n = L * L, half = n / 2;
    const uint64_t kb = key_base(key_seed(chain_seed[c], 0, kTagInit));
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        const uint32_t x = s % L, y = s / L;
        const uint32_t k = ((x + y) & 1u) * half + (s >> 1);
        theta[off[c] + k] = twice_u_f32(first_draw(kb, s)) * 3.14159265358979f;
    }
}

struct GroupCfg
{
    uint32_t cpc = 1, cpk = 1, block = 256;
};

std::mutex g_tune_mutex;
std::map<std::string, GroupCfg> g_tune_cache;
bool g_tune_file_loaded = false;

// The autotuner's file cache: when UMC_TUNE_CACHE names a file, its lines
// "<key> <chains per CTA> <CTAs per chain> <block>" are read once per
// process and every new tuning result is appended, so later processes on the
// same kind of GPU skip the timing runs.  The key holds the GPU name, the
// model and kernel, the lattice side, the chain count and the sweeps per
// exchange.  Call with g_tune_mutex held.
const char* tune_file() { return std::getenv("UMC_TUNE_CACHE"); }

void load_tune_file()
{
    if (g_tune_file_loaded) return;
    g_tune_file_loaded = true;
    const char* path = tune_file();
    if (!path || !*path) return;
    std::FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[512];
    unsigned cpc, cpk, block;
    while (std::fscanf(f, "%511s %u %u %u", key, &cpc, &cpk, &block) == 4) {
        // block 0 marks a persistent-kernel entry whose batch runs the grouped form
        const bool grouped_mark = block == 0 && std::strstr(key, "/xy_batch_persistent/");
        if (cpc >= 1 && cpc <= kMaxCpc && cpk >= 1 && cpk <= kMaxShares &&
            ((block >= 32 && block <= 1024 && block % 32 == 0) || grouped_mark))
            g_tune_cache[key] = GroupCfg{cpc, cpk, block};
    }
    std::fclose(f);
}

void store_tune_file(const std::string& key, const GroupCfg& c)
{
    const char* path = tune_file();
    if (!path || !*path) return;
    if (std::FILE* f = std::fopen(path, "a")) {
        std::fprintf(f, "%s %u %u %u\n", key.c_str(), c.cpc, c.cpk, c.block);
        std::fclose(f);
    }
}

}  // namespace
}  // namespace umc

// ============================================================== batch object

struct umc_batch
{
    umc_batch_desc desc{};
    uint32_t n_ladders = 0, R = 0, n_chains = 0;
    std::vector<uint32_t> L;  // per chain
    std::vector<unsigned long long> off, chain_seed, ladder_seed;
    std::vector<double> betas;
    struct Group
    {
        uint32_t L = 0;
        std::vector<uint32_t> chains;
        umc::GroupCfg cfg;
        umc::DevBuf chains_dev;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
    };
    std::vector<Group> groups;
    std::vector<uint32_t> cpk_of_chain;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t fork = nullptr;
    umc::DevBuf theta, off_dev, seeds_dev, lseeds_dev, betas_dev, holder_dev, slot_dev, cpk_dev, part, records, ctr,
        swaps, Ls_dev;
    uint64_t total_sites = 0;
    uint64_t max_records = 0;
    uint32_t sweeps_per_exchange = 10;
    cudaGraphExec_t graph = nullptr;
    uint64_t launches = 0;
    // the one-kernel segment (xy_batch_persistent): its items, per-chain
    // share counts and scheduler counters; on by default
    bool persistent = true;
    uint32_t p_kc = 4, p_minb = 1, p_big = 0, p_items = 0, p_grid = 0;
    std::vector<uint32_t> p_cpk;
    umc::DevBuf p_items_dev, p_chains_dev, p_cpk_dev, p_sched;
};

namespace umc {
namespace {

void batch_scope(const umc_batch* b) { cuda_check(cudaSetDevice(b->device), "cudaSetDevice"); }

SegArgs seg_args(umc_batch* b, umc_batch::Group& g, float* theta)
{
    SegArgs a{};
    a.theta = theta;
    a.off = b->off_dev.as<unsigned long long>();
    a.chains = g.chains_dev.as<uint32_t>();
    a.n_chains = uint32_t(g.chains.size());
    a.L = g.L;
    a.H = g.L / 2;
    a.half = g.L * g.L / 2;
    a.cpc = g.cfg.cpc;
    a.cpk = g.cfg.cpk;
    a.sweeps = b->sweeps_per_exchange;
    a.ctr = b->ctr.as<BatchCounters>();
    a.slot_of_chain = b->slot_dev.as<uint32_t>();
    a.betas = b->betas_dev.as<double>();
    a.R = b->R;
    a.chain_seed = b->seeds_dev.as<unsigned long long>();
    a.J = float(b->desc.coupling);
    a.width = float(b->desc.width);
    a.J64 = b->desc.coupling;
    a.err_per_beta = xy_metropolis_err(1.0, b->desc.coupling, 4);
    a.part = b->part.as<double>();
    return a;
}

// priority: a launch priority for the segment graph's kernel node (0: the
// stream's own).  Larger sides get higher priority, so the longest chains
// take SMs first and the short groups fill the rest.
void launch_segment(umc_batch* b, umc_batch::Group& g, const GroupCfg& cfg, float* theta, cudaStream_t st,
                    int priority = 0)
{
    SegArgs a = seg_args(b, g, theta);
    a.cpc = cfg.cpc;
    a.cpk = cfg.cpk;
    const uint32_t nc = uint32_t(g.chains.size());
    cudaLaunchConfig_t lc{};
    lc.blockDim = dim3(cfg.block);
    lc.dynamicSmemBytes = 0;
    lc.stream = st;
    cudaLaunchAttribute attr[2];
    unsigned n_attr = 0;
    if (priority != 0) {
        attr[n_attr].id = cudaLaunchAttributePriority;
        attr[n_attr].val.priority = priority;
        ++n_attr;
    }
    if (cfg.cpk > 1) {
        lc.gridDim = dim3(nc * cfg.cpk);
        attr[n_attr].id = cudaLaunchAttributeClusterDimension;
        attr[n_attr].val.clusterDim.x = cfg.cpk;
        attr[n_attr].val.clusterDim.y = 1;
        attr[n_attr].val.clusterDim.z = 1;
        ++n_attr;
        lc.attrs = attr;
        lc.numAttrs = n_attr;
        cuda_check(cudaLaunchKernelEx(&lc, xy_batch_segment<true>, a), "batch segment (cluster)");
    } else {
        lc.gridDim = dim3((nc + cfg.cpc - 1) / cfg.cpc);
        lc.attrs = attr;
        lc.numAttrs = n_attr;
        cuda_check(cudaLaunchKernelEx(&lc, xy_batch_segment<false>, a), "batch segment");
    }
    b->launches++;
}

// Candidate launch shapes for chains of side L.
std::vector<GroupCfg> candidates(uint32_t L, uint32_t n_chains)
{
    std::vector<GroupCfg> out;
    const uint32_t half = L * L / 2;
    for (uint32_t block : {256u, 512u, 1024u}) {
        for (uint32_t cpc = 1; cpc <= kMaxCpc && cpc <= n_chains; cpc *= 2) {
            if (cpc > 1 && cpc * half > 8u * block * 4u) break;  // keep a CTA's share moderate
            out.push_back({cpc, 1, block});
        }
        for (uint32_t cpk = 2; cpk <= kMaxShares; cpk *= 2)
            if (L % cpk == 0 && (L / cpk) >= 2 && half >= cpk * block) out.push_back({1, cpk, block});
    }
    return out;
}

// Times each candidate on a scratch copy of the group's chains (state untouched).
GroupCfg autotune(umc_batch* b, umc_batch::Group& g)
{
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, b->device), "device properties");
    std::string gpu = prop.name;
    for (char& ch : gpu)
        if (ch == ' ') ch = '_';
    const std::string key = gpu + "/xy_batch_segment/L" + std::to_string(g.L) + "/n" + std::to_string(g.chains.size()) +
                            "/s" + std::to_string(b->sweeps_per_exchange);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        load_tune_file();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) return it->second;
    }
    DevBuf scratch;
    scratch.alloc(b->theta.bytes, "autotune scratch");
    cuda_check(cudaMemcpyAsync(scratch.p, b->theta.p, b->theta.bytes, cudaMemcpyDeviceToDevice, b->stream), "autotune copy");
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    GroupCfg best;
    float best_ms = 1e30f;
    for (const GroupCfg& cfg : candidates(g.L, uint32_t(g.chains.size()))) {
        // warm once, then the fastest of three timings of two launches each,
        // so that one noisy timing does not pick the shape
        try {
            launch_segment(b, g, cfg, scratch.as<float>(), b->stream);
        } catch (const Error&) {
            cudaGetLastError();
            continue;
        }
        float ms = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            cuda_check(cudaEventRecord(e0, b->stream), "event");
            launch_segment(b, g, cfg, scratch.as<float>(), b->stream);
            launch_segment(b, g, cfg, scratch.as<float>(), b->stream);
            cuda_check(cudaEventRecord(e1, b->stream), "event");
            cuda_check(cudaEventSynchronize(e1), "autotune");
            float t = 0;
            cuda_check(cudaEventElapsedTime(&t, e0, e1), "autotune");
            ms = std::min(ms, t);
        }
        if (ms < best_ms) {
            best_ms = ms;
            best = cfg;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    scratch.free_();
    b->launches = 0;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    if (g_tune_cache.emplace(key, best).second) store_tune_file(key, best);
    return best;
}

// Work items of the one-kernel segment, largest first: a chain whose colour
// class holds at least 2 kPersistSites sites and whose rows split into KC
// bands of at least 2 rows is swept by a whole cluster; the others are
// packed, chains of one side together, into CTA items of up to kPersistSites
// sites per colour.
void build_persistent(umc_batch* b, uint32_t kc)
{
    std::vector<uint32_t> order(b->n_chains);
    for (uint32_t c = 0; c < b->n_chains; ++c) order[c] = c;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return b->L[x] > b->L[y]; });
    std::vector<uint4> items;
    std::vector<uint32_t> chains;
    b->p_cpk.assign(b->n_chains, 1);
    uint32_t n_big = 0;
    size_t q = 0;
    while (q < order.size() && [&] {
        const uint32_t L = b->L[order[q]];
        return uint64_t(L) * L / 2 >= 2ull * kPersistSites && L % (2 * kc) == 0;
    }()) {
        const uint32_t c = order[q++];
        items.push_back(make_uint4(uint32_t(chains.size()), 1u, b->L[c], kc));
        chains.push_back(c);
        b->p_cpk[c] = kc;
        ++n_big;
    }
    while (q < order.size()) {
        const uint32_t L = b->L[order[q]];
        const uint32_t per = L * L / 2;
        const uint32_t cpc = std::max<uint32_t>(1, std::min<uint32_t>(kMaxCpc, kPersistSites / per));
        const uint32_t first = uint32_t(chains.size());
        uint32_t n = 0;
        while (q < order.size() && n < cpc && b->L[order[q]] == L) {
            chains.push_back(order[q++]);
            ++n;
        }
        items.push_back(make_uint4(first, n, L, 1u));
    }
    b->p_kc = kc;
    b->p_big = n_big;
    b->p_items = uint32_t(items.size());
    b->p_items_dev.alloc(items.size() * sizeof(uint4), "persistent items");
    cuda_check(cudaMemcpy(b->p_items_dev.p, items.data(), items.size() * sizeof(uint4), cudaMemcpyHostToDevice), "items");
    b->p_chains_dev.alloc(chains.size() * 4, "persistent chains");
    cuda_check(cudaMemcpy(b->p_chains_dev.p, chains.data(), chains.size() * 4, cudaMemcpyHostToDevice), "chains");
    b->p_cpk_dev.alloc(b->n_chains * 4, "persistent shares");
    cuda_check(cudaMemcpy(b->p_cpk_dev.p, b->p_cpk.data(), b->n_chains * 4, cudaMemcpyHostToDevice), "shares");
    b->p_sched.alloc((3 + size_t(b->n_ladders)) * 4, "persistent scheduler");
    b->p_grid = 0;
}

// The six kernel variants by (cluster size, CTAs per SM).
const void* persistent_kernel(uint32_t kc, uint32_t minb)
{
    if (kc == 8) return minb == 2 ? reinterpret_cast<const void*>(&xy_batch_persistent<8, 2>)
                                  : reinterpret_cast<const void*>(&xy_batch_persistent<8, 1>);
    if (kc == 1) return minb == 2 ? reinterpret_cast<const void*>(&xy_batch_persistent<1, 2>)
                                  : reinterpret_cast<const void*>(&xy_batch_persistent<1, 1>);
    if (kc != 4) throw Error(UMC_ERR_UNSUPPORTED, "persistent batch: cluster size must be 1, 4 or 8");
    return minb == 2 ? reinterpret_cast<const void*>(&xy_batch_persistent<4, 2>)
                     : reinterpret_cast<const void*>(&xy_batch_persistent<4, 1>);
}

cudaLaunchConfig_t persistent_config(uint32_t kc, uint32_t grid, cudaStream_t st, cudaLaunchAttribute* attr)
{
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(grid);
    lc.blockDim = dim3(kPersistBlock);
    lc.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kc;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return lc;
}

// Resident clusters: the kernel never waits across clusters, so this only
// sizes the grid to what runs at once.
uint32_t persistent_grid(umc_batch* b, uint32_t kc, uint32_t minb)
{
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t lc = persistent_config(kc, kc, nullptr, attr);
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, persistent_kernel(kc, minb), &lc) != cudaSuccess || clusters <= 0) {
        cudaGetLastError();
        int sms = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device), "SM count");
        clusters = std::max(1, sms / int(kc));
    }
    return uint32_t(clusters) * kc;
}

void launch_persistent(umc_batch* b, cudaStream_t st)
{
    if (!b->p_grid) b->p_grid = persistent_grid(b, b->p_kc, b->p_minb);
    cuda_check(cudaMemsetAsync(b->p_sched.p, 0, b->p_sched.bytes, st), "reset scheduler");
    PersistArgs p{};
    umc_batch::Group g0;  // seg_args takes the per-group fields from a group; the kernel sets L per item
    g0.L = 2;
    p.seg = seg_args(b, g0, b->theta.as<float>());
    p.seg.chains = nullptr;
    p.seg.n_chains = 0;
    p.items = b->p_items_dev.as<uint4>();
    p.chains = b->p_chains_dev.as<uint32_t>();
    p.n_big = b->p_big;
    p.n_items = b->p_items;
    p.sched = b->p_sched.as<unsigned>();
    p.ladder_done = b->p_sched.as<unsigned>() + 3;
    p.cpk_of_chain = b->p_cpk_dev.as<uint32_t>();
    p.n_ladders = b->n_ladders;
    p.records = b->records.as<double>();
    p.holder = b->holder_dev.as<uint32_t>();
    p.ladder_seed = b->lseeds_dev.as<unsigned long long>();
    p.swaps = b->swaps.as<unsigned long long>();
    cudaLaunchAttribute attr[1];
    cudaLaunchConfig_t lc = persistent_config(b->p_kc, b->p_grid, st, attr);
    cudaError_t e;
    // the kernel variant from the one table that also sizes the grid
    void* args[] = {&p};
    e = cudaLaunchKernelExC(&lc, persistent_kernel(b->p_kc, b->p_minb), args);
    cuda_check(e, "persistent batch segment");
}

// Picks the cluster size of the one-kernel segment by timing two segments of
// each on the batch itself; every buffer a segment changes (field, holders,
// slots, counters, swap count) is copied aside first and put back after.
// The choice is cached in the process (and in UMC_TUNE_CACHE) per GPU, side
// multiset, chain count and sweeps per exchange.
void build_graph(umc_batch* b);

void autotune_persistent(umc_batch* b)
{
    cudaDeviceProp prop{};
    cuda_check(cudaGetDeviceProperties(&prop, b->device), "device properties");
    std::string gpu = prop.name;
    for (char& ch : gpu)
        if (ch == ' ') ch = '_';
    std::map<uint32_t, uint32_t> sides;
    for (uint32_t c = 0; c < b->n_chains; ++c) sides[b->L[c]]++;
    std::string key = gpu + "/xy_batch_persistent/s" + std::to_string(b->sweeps_per_exchange);
    for (auto& [L, n] : sides) key += "/L" + std::to_string(L) + "x" + std::to_string(n);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        load_tune_file();
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            build_persistent(b, it->second.cpk);
            b->p_minb = it->second.cpc;
            b->persistent = it->second.block != 0;
            return;
        }
    }
    DevBuf keep_theta, keep_small;
    keep_theta.alloc(b->theta.bytes, "tuning copy");
    const size_t hb = b->holder_dev.bytes, sb = b->slot_dev.bytes, cb = sizeof(BatchCounters);
    keep_small.alloc(hb + sb + cb + 8, "tuning copy");
    auto save = [&](bool back) {
        auto cp = [&](void* dst, void* src, size_t n) {
            cuda_check(cudaMemcpyAsync(back ? src : dst, back ? dst : src, n, cudaMemcpyDeviceToDevice, b->stream), "copy");
        };
        uint8_t* k = static_cast<uint8_t*>(keep_small.p);
        cp(keep_theta.p, b->theta.p, b->theta.bytes);
        cp(k, b->holder_dev.p, hb);
        cp(k + hb, b->slot_dev.p, sb);
        cp(k + hb + sb, b->ctr.p, cb);
        cp(k + hb + sb + cb, b->swaps.p, 8);
    };
    save(false);
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    uint32_t best = kPersistClusters[0], best_minb = 1;
    float best_ms = 1e30f;
    for (uint32_t cand = 0; cand < 6; ++cand) {
        const uint32_t kc = kPersistClusters[cand % 3u], minb = 1 + cand / 3u;
        build_persistent(b, kc);
        b->p_minb = minb;
        launch_persistent(b, b->stream);  // warm
        cuda_check(cudaEventRecord(e0, b->stream), "event");
        launch_persistent(b, b->stream);
        launch_persistent(b, b->stream);
        cuda_check(cudaEventRecord(e1, b->stream), "event");
        cuda_check(cudaEventSynchronize(e1), "tuning");
        float ms = 0;
        cuda_check(cudaEventElapsedTime(&ms, e0, e1), "tuning");
        save(true);
        if (ms < best_ms) {
            best_ms = ms;
            best = kc;
            best_minb = minb;
        }
    }
    // the grouped form (one kernel per side group plus the exchange, as one graph)
    b->persistent = false;
    build_graph(b);
    cuda_check(cudaGraphLaunch(b->graph, b->stream), "tuning");  // warm
    cuda_check(cudaEventRecord(e0, b->stream), "event");
    cuda_check(cudaGraphLaunch(b->graph, b->stream), "tuning");
    cuda_check(cudaGraphLaunch(b->graph, b->stream), "tuning");
    cuda_check(cudaEventRecord(e1, b->stream), "event");
    cuda_check(cudaEventSynchronize(e1), "tuning");
    float grouped_ms = 0;
    cuda_check(cudaEventElapsedTime(&grouped_ms, e0, e1), "tuning");
    save(true);
    cuda_check(cudaStreamSynchronize(b->stream), "tuning");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    build_persistent(b, best);
    b->p_minb = best_minb;
    b->persistent = best_ms < grouped_ms;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    // the chains-per-CTA field holds CTAs per SM here, the block field 0 when
    // the grouped form measured faster
    GroupCfg cfg{best_minb, best, b->persistent ? kPersistBlock : 0u};
    if (g_tune_cache.emplace(key, cfg).second) store_tune_file(key, cfg);
    b->launches = 0;
}

void build_graph(umc_batch* b)
{
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t graph;
    cuda_check(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    if (b->persistent) {
        launch_persistent(b, b->stream);
        cuda_check(cudaStreamEndCapture(b->stream, &graph), "end capture");
        cuda_check(cudaGraphInstantiate(&b->graph, graph, 0), "instantiate graph");
        cudaGraphDestroy(graph);
        return;
    }
    cuda_check(cudaEventRecord(b->fork, b->stream), "fork");
    const uint64_t launches = b->launches;  // captured, not launched: replays are counted
    int least = 0, greatest = 0;
    cuda_check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "priority range");
    for (auto& g : b->groups) {
        // rank of this group's side among the groups, largest first
        int rank = 0;
        for (const auto& o : b->groups) rank += o.L > g.L ? 1 : 0;
        const int prio = std::min(least, greatest + rank);
        cuda_check(cudaStreamWaitEvent(g.stream, b->fork, 0), "fork wait");
        launch_segment(b, g, g.cfg, b->theta.as<float>(), g.stream, prio == least ? 0 : prio);
        cuda_check(cudaEventRecord(g.done, g.stream), "join");
        cuda_check(cudaStreamWaitEvent(b->stream, g.done, 0), "join wait");
    }
    xy_batch_swap<<<1, std::min(b->n_ladders, kSwapWarps) * 32, 0, b->stream>>>(b->ctr.as<BatchCounters>(), b->n_ladders, b->R, b->cpk_dev.as<uint32_t>(),
                                             b->part.as<double>(), b->betas_dev.as<double>(), b->holder_dev.as<uint32_t>(),
                                             b->slot_dev.as<uint32_t>(), b->lseeds_dev.as<unsigned long long>(),
                                             b->records.as<double>(), b->swaps.as<unsigned long long>(),
                                             b->sweeps_per_exchange);
    cuda_check(cudaGetLastError(), "swap kernel");
    b->launches = launches;
    cuda_check(cudaStreamEndCapture(b->stream, &graph), "end capture");
    cuda_check(cudaGraphInstantiate(&b->graph, graph, cudaGraphInstantiateFlagUseNodePriority), "instantiate graph");
    cudaGraphDestroy(graph);
}

void create_batch(const umc_batch_desc* d, umc_batch* b)
{
    if (!d) throw Error(UMC_ERR_INVALID_ARGUMENT, "null descriptor");
    b->desc = *d;
    b->n_ladders = d->n_ladders;
    b->R = d->replicas;
    if (b->n_ladders == 0 || b->R == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "need at least one ladder and one replica");
    if (b->R > kMaxRungs) throw Error(UMC_ERR_UNSUPPORTED, "at most 64 replicas per ladder");
    if (!d->L || !d->betas) throw Error(UMC_ERR_INVALID_ARGUMENT, "null L or betas");
    if (!std::isfinite(d->coupling) || !std::isfinite(d->width)) throw Error(UMC_ERR_INVALID_ARGUMENT, "J and width must be finite");
    b->sweeps_per_exchange = d->sweeps_per_exchange ? d->sweeps_per_exchange : 10;
    b->n_chains = b->n_ladders * b->R;
    b->device = d->device;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(UMC_ERR_CUDA, "no CUDA device available");
    }
    if (b->device < 0 || b->device >= count) throw Error(UMC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    batch_scope(b);
    b->betas.assign(d->betas, d->betas + b->n_chains);
    for (double beta : b->betas)
        if (!std::isfinite(beta)) throw Error(UMC_ERR_INVALID_ARGUMENT, "betas must be finite");
    b->L.resize(b->n_chains);
    b->off.resize(b->n_chains);
    b->chain_seed.resize(b->n_chains);
    b->ladder_seed.resize(b->n_ladders);
    uint64_t acc = 0;
    std::map<uint32_t, std::vector<uint32_t>> by_L;
    for (uint32_t l = 0; l < b->n_ladders; ++l) {
        const uint64_t L = d->L[l];
        if (L < 2 || L % 2 || L > 4096) throw Error(UMC_ERR_INVALID_ARGUMENT, "ladder side L must be even, in [2, 4096]");
        // keys of the global ladder first_ladder + l and its global chains
        const uint64_t gl = uint64_t(d->first_ladder) + l;
        b->ladder_seed[l] = mix64(d->seed + 0xD1B54A32D192ED03ULL * (gl + 1));
        for (uint32_t k = 0; k < b->R; ++k) {
            const uint32_t c = l * b->R + k;
            b->L[c] = uint32_t(L);
            b->off[c] = acc;
            acc += L * L;
            b->chain_seed[c] = mix64(d->seed + kGolden * (gl * b->R + k + 1ull));
            by_L[uint32_t(L)].push_back(c);
        }
    }
    b->total_sites = acc;
    if (acc > (1ull << 34)) throw Error(UMC_ERR_OVERFLOW, "too many sites in the batch");
    if (d->stream) {
        b->stream = static_cast<cudaStream_t>(d->stream);
    } else {
        cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
        b->own_stream = true;
    }
    cuda_check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "event");
    b->max_records = d->max_records ? d->max_records : 1024;
    auto up = [&](DevBuf& buf, const void* p, size_t bytes, const char* what) {
        buf.alloc(bytes, what);
        cuda_check(cudaMemcpy(buf.p, p, bytes, cudaMemcpyHostToDevice), what);
    };
    b->theta.alloc(acc * sizeof(float), "batch field");
    cuda_check(cudaMemset(b->theta.p, 0, acc * sizeof(float)), "zero field");
    up(b->off_dev, b->off.data(), b->off.size() * 8, "offsets");
    up(b->seeds_dev, b->chain_seed.data(), b->chain_seed.size() * 8, "chain seeds");
    up(b->lseeds_dev, b->ladder_seed.data(), b->ladder_seed.size() * 8, "ladder seeds");
    up(b->betas_dev, b->betas.data(), b->betas.size() * 8, "betas");
    up(b->Ls_dev, b->L.data(), b->L.size() * 4, "sides");
    std::vector<uint32_t> holder(b->n_chains), slot(b->n_chains);
    for (uint32_t c = 0; c < b->n_chains; ++c) holder[c] = slot[c] = c % b->R;
    for (uint32_t c = 0; c < b->n_chains; ++c) holder[c] = c;  // slot k of ladder l held by chain l*R+k
    up(b->holder_dev, holder.data(), holder.size() * 4, "holders");
    up(b->slot_dev, slot.data(), slot.size() * 4, "slots");
    b->records.alloc(b->max_records * b->n_chains * kObs * sizeof(double), "batch records");
    b->swaps.alloc(8, "swap counter");
    cuda_check(cudaMemset(b->swaps.p, 0, 8), "swap counter");
    BatchCounters c0{};
    c0.capacity = b->max_records;
    up(b->ctr, &c0, sizeof c0, "counters");

    // groups and their launch shapes
    b->cpk_of_chain.assign(b->n_chains, 1);
    for (auto& [L, chains] : by_L) {
        b->groups.emplace_back();
        auto& g = b->groups.back();
        g.L = L;
        g.chains = chains;
        up(g.chains_dev, chains.data(), chains.size() * 4, "group chains");
        cuda_check(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking), "group stream");
        cuda_check(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming), "event");
    }
    // shares of the energy partials need the largest cpk first: tune, then size
    b->part.alloc(uint64_t(b->n_chains) * kMaxShares * 4 * sizeof(double), "partials");
    for (auto& g : b->groups) {
        g.cfg = autotune(b, g);
        for (uint32_t c : g.chains) b->cpk_of_chain[c] = g.cfg.cpk;
    }
    up(b->cpk_dev, b->cpk_of_chain.data(), b->cpk_of_chain.size() * 4, "cpk");
    cuda_check(cudaMemset(b->ctr.p, 0, sizeof(BatchCounters)), "counters");
    cuda_check(cudaMemcpy(&b->ctr.as<BatchCounters>()->capacity, &b->max_records, 8, cudaMemcpyHostToDevice), "capacity");
    autotune_persistent(b);
    build_graph(b);
}

void destroy_batch(umc_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (auto& g : b->groups) {
        if (g.stream) cudaStreamDestroy(g.stream);
        if (g.done) cudaEventDestroy(g.done);
        g.chains_dev.free_();
    }
    if (b->fork) cudaEventDestroy(b->fork);
    for (DevBuf* x : {&b->theta, &b->off_dev, &b->seeds_dev, &b->lseeds_dev, &b->betas_dev, &b->holder_dev, &b->slot_dev,
                      &b->cpk_dev, &b->part, &b->records, &b->ctr, &b->swaps, &b->Ls_dev})
        x->free_();
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

template <class F>
int bguard(F&& f)
{
    try {
        set_last_error("");
        f();
        return UMC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}

// chain-local natural order <-> two-colour order
void to_colour_major(const float* src, float* dst, uint32_t L)
{
    const uint32_t half = L * L / 2;
    for (uint32_t s = 0; s < L * L; ++s) {
        const uint32_t x = s % L, y = s / L;
        dst[((x + y) & 1u) * half + s / 2] = src[s];
    }
}

void from_colour_major(const float* src, float* dst, uint32_t L)
{
    const uint32_t half = L * L / 2;
    for (uint32_t s = 0; s < L * L; ++s) {
        const uint32_t x = s % L, y = s / L;
        dst[s] = src[((x + y) & 1u) * half + s / 2];
    }
}

}  // namespace
}  // namespace umc

using namespace umc;

extern "C" {

int umc_batch_create(const umc_batch_desc* desc, umc_batch** out)
{
    return bguard([&] {
        if (!out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        auto* b = new umc_batch;
        try {
            create_batch(desc, b);
        } catch (...) {
            destroy_batch(b);
            delete b;
            throw;
        }
        *out = b;
    });
}

int umc_batch_destroy(umc_batch* b)
{
    return bguard([&] {
        destroy_batch(b);
        delete b;
    });
}

int umc_batch_randomize(umc_batch* b, uint64_t seed)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        batch_scope(b);
        // per-chain init keys derive from the run seed and the chain index
        std::vector<unsigned long long> s(b->n_chains);
        const uint64_t g0 = uint64_t(b->desc.first_ladder) * b->R;  // global index of chain 0
        for (uint32_t c = 0; c < b->n_chains; ++c) s[c] = mix64(seed + kGolden * (g0 + c + 1ull));
        DevBuf sd;
        sd.alloc(s.size() * 8, "init seeds");
        cuda_check(cudaMemcpy(sd.p, s.data(), s.size() * 8, cudaMemcpyHostToDevice), "init seeds");
        const uint32_t maxL = *std::max_element(b->L.begin(), b->L.end());
        xy_batch_randomize<<<dim3((maxL * maxL + 255) / 256, b->n_chains), 256, 0, b->stream>>>(
            b->theta.as<float>(), b->off_dev.as<unsigned long long>(), b->Ls_dev.as<uint32_t>(), b->n_chains,
            sd.as<unsigned long long>());
        cuda_check(cudaGetLastError(), "randomize");
        cuda_check(cudaStreamSynchronize(b->stream), "randomize");
    });
}

int umc_batch_set_field(umc_batch* b, uint32_t chain, const float* theta)
{
    return bguard([&] {
        if (!b || !theta) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (chain >= b->n_chains) throw Error(UMC_ERR_OUT_OF_RANGE, "chain index out of range");
        batch_scope(b);
        const uint32_t L = b->L[chain];
        std::vector<float> tmp(size_t(L) * L);
        to_colour_major(theta, tmp.data(), L);
        for (float& v : tmp) v = wrap_angle(v);  // within the FP32 decisions' sincos domain
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(b->theta.as<float>() + b->off[chain], tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice),
                   "upload chain");
    });
}

int umc_batch_get_field(umc_batch* b, uint32_t chain, float* theta)
{
    return bguard([&] {
        if (!b || !theta) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (chain >= b->n_chains) throw Error(UMC_ERR_OUT_OF_RANGE, "chain index out of range");
        batch_scope(b);
        const uint32_t L = b->L[chain];
        std::vector<float> tmp(size_t(L) * L);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(tmp.data(), b->theta.as<float>() + b->off[chain], tmp.size() * 4, cudaMemcpyDeviceToHost),
                   "download chain");
        from_colour_major(tmp.data(), theta, L);
    });
}

int umc_batch_enqueue(umc_batch* b, uint64_t n_segments)
{
    return bguard([&] {
        NvtxRange range("umc_batch_enqueue");
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        batch_scope(b);
        for (uint64_t s = 0; s < n_segments; ++s) cuda_check(cudaGraphLaunch(b->graph, b->stream), "segment graph");
        b->launches += n_segments * (b->persistent ? 1 : b->groups.size() + 1);
    });
}

int umc_batch_fetch(umc_batch* b, double* records, uint64_t capacity, uint64_t* n_records)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        batch_scope(b);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        BatchCounters c{};
        cuda_check(cudaMemcpy(&c, b->ctr.p, sizeof c, cudaMemcpyDeviceToHost), "counters");
        if (c.status & kBatchErrRecords) {
            const unsigned int zero = 0;
            cuda_check(cudaMemcpy(&b->ctr.as<BatchCounters>()->status, &zero, 4, cudaMemcpyHostToDevice), "status");
            const unsigned long long z = 0;
            cuda_check(cudaMemcpy(&b->ctr.as<BatchCounters>()->rec, &z, 8, cudaMemcpyHostToDevice), "records");
            throw Error(UMC_ERR_STATE, "batch records overflowed; fetch more often or raise max_records");
        }
        if (records && c.rec > capacity) throw Error(UMC_ERR_INVALID_ARGUMENT, "record buffer too small");
        if (records && c.rec)
            cuda_check(cudaMemcpy(records, b->records.p, c.rec * b->n_chains * kObs * sizeof(double), cudaMemcpyDeviceToHost),
                       "records");
        if (n_records) *n_records = c.rec;
        const unsigned long long z = 0;
        cuda_check(cudaMemcpy(&b->ctr.as<BatchCounters>()->rec, &z, 8, cudaMemcpyHostToDevice), "reset records");
    });
}

int umc_batch_run(umc_batch* b, uint64_t n_segments, double* records)
{
    return bguard([&] {
        NvtxRange range("umc_batch_run");
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        uint64_t done = 0;
        {
            uint64_t got = 0;  // drop records queued before this call
            const int st = umc_batch_fetch(b, nullptr, 0, &got);
            if (st != UMC_OK) throw Error(st, umc_last_error());
        }
        while (done < n_segments) {
            const uint64_t m = std::min<uint64_t>(n_segments - done, b->max_records);
            int st = umc_batch_enqueue(b, m);
            if (st != UMC_OK) throw Error(st, umc_last_error());
            uint64_t got = 0;
            st = umc_batch_fetch(b, records ? records + done * b->n_chains * kObs : nullptr, m, &got);
            if (st != UMC_OK) throw Error(st, umc_last_error());
            done += m;
        }
    });
}

int umc_batch_counters(const umc_batch* b, uint64_t* sweeps, uint64_t* rounds, uint64_t* swaps_accepted)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        batch_scope(b);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        BatchCounters c{};
        cuda_check(cudaMemcpy(&c, b->ctr.p, sizeof c, cudaMemcpyDeviceToHost), "counters");
        unsigned long long sw = 0;
        cuda_check(cudaMemcpy(&sw, b->swaps.p, 8, cudaMemcpyDeviceToHost), "swaps");
        if (sweeps) *sweeps = c.sweep;
        if (rounds) *rounds = c.round;
        if (swaps_accepted) *swaps_accepted = sw;
    });
}

int umc_batch_temperature_map(const umc_batch* b, uint32_t* holder)
{
    return bguard([&] {
        if (!b || !holder) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        batch_scope(b);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(holder, b->holder_dev.p, b->n_chains * 4, cudaMemcpyDeviceToHost), "holders");
    });
}

int umc_batch_set_state(umc_batch* b, uint64_t sweeps, uint64_t rounds, uint64_t swaps_accepted, const uint32_t* holder)
{
    return bguard([&] {
        if (!b || !holder) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        batch_scope(b);
        // holder must permute each ladder's own chains over its slots
        std::vector<uint32_t> slot(b->n_chains, 0xFFFFFFFFu);
        for (uint32_t l = 0; l < b->n_ladders; ++l)
            for (uint32_t k = 0; k < b->R; ++k) {
                const uint32_t c = holder[l * b->R + k];
                if (c / b->R != l || c >= b->n_chains || slot[c] != 0xFFFFFFFFu)
                    throw Error(UMC_ERR_INVALID_ARGUMENT, "holder is not a permutation of each ladder's chains");
                slot[c] = k;
            }
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        BatchCounters ctr{};
        cuda_check(cudaMemcpy(&ctr, b->ctr.p, sizeof ctr, cudaMemcpyDeviceToHost), "counters");
        ctr.sweep = sweeps;
        ctr.round = rounds;
        cuda_check(cudaMemcpy(b->ctr.p, &ctr, sizeof ctr, cudaMemcpyHostToDevice), "counters");
        const unsigned long long sw = swaps_accepted;
        cuda_check(cudaMemcpy(b->swaps.p, &sw, 8, cudaMemcpyHostToDevice), "swaps");
        cuda_check(cudaMemcpy(b->holder_dev.p, holder, b->n_chains * 4, cudaMemcpyHostToDevice), "holders");
        cuda_check(cudaMemcpy(b->slot_dev.p, slot.data(), b->n_chains * 4, cudaMemcpyHostToDevice), "slots");
    });
}

int umc_batch_seeds(const umc_batch* b, uint64_t* chain_seeds, uint64_t* ladder_seeds)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        if (chain_seeds) std::copy(b->chain_seed.begin(), b->chain_seed.end(), chain_seeds);
        if (ladder_seeds) std::copy(b->ladder_seed.begin(), b->ladder_seed.end(), ladder_seeds);
    });
}

int umc_batch_config(const umc_batch* b, uint32_t L, uint32_t* chains_per_cta, uint32_t* ctas_per_chain, uint32_t* block)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        for (const auto& g : b->groups)
            if (g.L == L) {
                if (chains_per_cta) *chains_per_cta = g.cfg.cpc;
                if (ctas_per_chain) *ctas_per_chain = g.cfg.cpk;
                if (block) *block = g.cfg.block;
                return;
            }
        throw Error(UMC_ERR_OUT_OF_RANGE, "no ladder with that side");
    });
}

int umc_batch_set_persistent(umc_batch* b, int enable)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        batch_scope(b);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        b->persistent = enable != 0;
        build_graph(b);
    });
}

int umc_batch_set_persistent_config(umc_batch* b, uint32_t cluster, uint32_t ctas_per_sm)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        if (cluster != 1 && cluster != 4 && cluster != 8)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "cluster size must be 1, 4 or 8");
        if (ctas_per_sm != 1 && ctas_per_sm != 2) throw Error(UMC_ERR_INVALID_ARGUMENT, "CTAs per SM must be 1 or 2");
        batch_scope(b);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        build_persistent(b, cluster);
        b->p_minb = ctas_per_sm;
        b->persistent = true;
        build_graph(b);
    });
}

int umc_batch_persistent_info(const umc_batch* b, int* enabled, uint32_t* grid, uint32_t* big_items, uint32_t* items,
                              uint32_t* cluster, uint32_t* ctas_per_sm)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        if (enabled) *enabled = b->persistent ? 1 : 0;
        if (grid) *grid = b->p_grid;
        if (cluster) *cluster = b->p_kc;
        if (ctas_per_sm) *ctas_per_sm = b->p_minb;
        if (big_items) *big_items = b->p_big;
        if (items) *items = b->p_items;
    });
}

int umc_batch_sites(const umc_batch* b, uint64_t* total_sites, uint64_t* kernel_launches)
{
    return bguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null batch");
        if (total_sites) *total_sites = b->total_sites;
        if (kernel_launches) *kernel_launches = b->launches;
    });
}

void* umc_batch_stream(const umc_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

}  // extern "C"
