// umc_device.cuh -- device-side plumbing shared by the update kernels.
//
//  * DevCtl: per-chain control block in device memory (pass tickets, per-pass
//    observable totals, an error-status word).
//  * block_sum / finish_pass: deterministic FP64 reductions.  Every block
//    writes its partial sums; the last block to arrive (atomic ticket) adds the
//    partials in a fixed order, so observables are reproducible bit-for-bit
//    from run to run.  The final pass of a sweep also folds the per-pass totals
//    into the sweep's observable record.
//  * uf_find / uf_union: lock-free union-find over 32-bit labels with bounded
//    loops; a bound that runs out raises a status bit instead of spinning.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <umc/keyed_pcg.cuh>

namespace umc {

constexpr int kObs = 8;           // doubles per observable record
constexpr int kMaxPasses = 64;    // colour classes per sweep
constexpr int kBlock = 256;       // threads per block of the update kernels

// status bits raised on the device
constexpr unsigned kDevErrUnionFind = 1u;   // union-find bound exhausted
constexpr unsigned kDevErrGeometry = 2u;    // index outside a table
constexpr unsigned kDevErrRetry = 4u;       // proposal retry bound exhausted
constexpr unsigned kDevErrBarrier = 8u;     // grid barrier wait bound exhausted

// counter + generation of the bounded grid barrier (umc_fused.cuh)
// Grid barrier of a cooperative launch: count only grows within a launch
// (barrier k completes at k * gridDim arrivals); the last block to retire
// resets both words for the next launch.
struct GridBarrier
{
    unsigned int count;
    unsigned int done;
};

struct DevCtl
{
    unsigned int ticket[kMaxPasses];
    unsigned int status;
    unsigned int xcount;  // entries of the fused Wolff step's crossing-bond list
    GridBarrier bar;
    double pass_total[kMaxPasses][kObs];
};

// Where a pass kernel deposits its observable contributions.
struct PassOut
{
    DevCtl* ctl;
    double* partials;      // >= gridDim.x * kObs doubles
    double* record;        // kObs doubles of this sweep's record (used by the final pass)
    unsigned long long* size_slot;  // Wolff cluster size of this flip (or null)
    int pass;              // index of this pass within the sweep
    int n_passes;          // passes in the sweep (the n_passes indices ending at pass)
    int final_pass;        // 1 if this pass completes the sweep
};

template <int V>
__device__ __forceinline__ void warp_sum(double (&v)[V])
{
#pragma unroll
    for (int k = 0; k < V; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
}

// Sum over the block; the result is valid in thread 0.  All threads call it.
template <int V>
__device__ __forceinline__ void block_sum(double (&v)[V])
{
    __shared__ double sh[32][V];
    __syncthreads();
    warp_sum<V>(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < V; ++k) sh[w][k] = v[k];
    __syncthreads();
    if (w == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < V; ++k) v[k] = lane < nw ? sh[lane][k] : 0.0;
        warp_sum<V>(v);
    }
}

// Block reduction, then the last block folds all partials (fixed order).
template <int V>
__device__ void finish_pass(double (&v)[V], const PassOut& o)
{
    static_assert(V <= kObs, "too many observables");
    block_sum<V>(v);
    __shared__ unsigned int is_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < V; ++k) o.partials[blockIdx.x * kObs + k] = v[k];
        __threadfence();
        const unsigned int t = atomicAdd(&o.ctl->ticket[o.pass], 1u);
        is_last = (t == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double s[V];
#pragma unroll
    for (int k = 0; k < V; ++k) s[k] = 0.0;
    const volatile double* part = o.partials;
    for (unsigned int b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < V; ++k) s[k] += part[b * kObs + k];
    block_sum<V>(s);
    if (threadIdx.x == 0) {
        volatile double* tot = o.ctl->pass_total[o.pass];
#pragma unroll
        for (int k = 0; k < kObs; ++k) tot[k] = k < V ? s[k] : 0.0;
        o.ctl->ticket[o.pass] = 0u;
        if (o.final_pass && o.record) {
            double r[kObs];
#pragma unroll
            for (int k = 0; k < kObs; ++k) r[k] = 0.0;
            // the sweep's passes are the n_passes ending at this one
            for (int p = o.pass - o.n_passes + 1; p <= o.pass; ++p) {
                const volatile double* pt = o.ctl->pass_total[p];
#pragma unroll
                for (int k = 0; k < kObs; ++k) r[k] += pt[k];
            }
#pragma unroll
            for (int k = 0; k < kObs; ++k) o.record[k] = r[k];
        }
        __threadfence();
    }
}

// ----------------------------------------------------------------- union-find
// Roots are linked by a fixed pseudorandom priority (a bijective hash of the
// index): the lower-priority root goes under the higher one.  Linking by index
// instead builds chains as long as a row of merging tiles (T2->T1, T3->T2, ...
// when the unions run concurrently) and every later find walks them; random
// priorities give expected logarithmic depth (randomised linking, Goel,
// Khanna, Larkin & Tarjan 2014).  Labels only ever point to higher priority,
// so every find terminates within n steps; the bound turns a logic error into
// a status bit.  The components -- and so the Wolff clusters -- do not depend
// on the linking order.
__device__ __forceinline__ uint32_t uf_priority(uint32_t x) { return stream_id(x); }

__device__ __forceinline__ uint32_t uf_find(uint32_t* lab, uint32_t x, uint32_t bound, unsigned* status)
{
    volatile uint32_t* L = lab;
    for (uint32_t it = 0; it < bound; ++it) {
        const uint32_t p = L[x];
        if (p == x) return x;
        const uint32_t gp = L[p];
        if (gp != p) L[x] = gp;  // path halving: gp is a valid ancestor of x
        x = gp;
    }
    atomicOr(status, kDevErrUnionFind);
    return x;
}

// Two finds walked in lockstep (independent load chains overlap their
// latency); same path halving and bound as uf_find.
__device__ __forceinline__ void uf_find2(uint32_t* lab, uint32_t x0, uint32_t x1, uint32_t bound, unsigned* status,
                                         uint32_t& r0, uint32_t& r1)
{
    volatile uint32_t* L = lab;
    bool d0 = false, d1 = false;
    for (uint32_t it = 0; it < bound; ++it) {
        const uint32_t p0 = d0 ? x0 : L[x0];
        const uint32_t p1 = d1 ? x1 : L[x1];
        d0 = d0 || p0 == x0;
        d1 = d1 || p1 == x1;
        if (d0 && d1) {
            r0 = x0;
            r1 = x1;
            return;
        }
        const uint32_t g0 = d0 ? x0 : L[p0];
        const uint32_t g1 = d1 ? x1 : L[p1];
        if (!d0 && g0 != p0) L[x0] = g0;
        if (!d1 && g1 != p1) L[x1] = g1;
        if (!d0) x0 = g0;
        if (!d1) x1 = g1;
    }
    atomicOr(status, kDevErrUnionFind);
    r0 = x0;
    r1 = x1;
}

// The root of s (read only: every thread of the grid walks this same path)
// together with two path-halving finds, all three load chains in lockstep.
__device__ __forceinline__ void uf_find_with_root(uint32_t* lab, uint32_t s, uint32_t x0, uint32_t x1, uint32_t bound,
                                                  unsigned* status, uint32_t& rs, uint32_t& r0, uint32_t& r1)
{
    volatile uint32_t* L = lab;
    bool ds = false, d0 = false, d1 = false;
    for (uint32_t it = 0; it < bound; ++it) {
        const uint32_t ps = ds ? s : L[s];
        const uint32_t p0 = d0 ? x0 : L[x0];
        const uint32_t p1 = d1 ? x1 : L[x1];
        ds = ds || ps == s;
        d0 = d0 || p0 == x0;
        d1 = d1 || p1 == x1;
        if (ds && d0 && d1) {
            rs = s;
            r0 = x0;
            r1 = x1;
            return;
        }
        const uint32_t g0 = d0 ? x0 : L[p0];
        const uint32_t g1 = d1 ? x1 : L[p1];
        if (!d0 && g0 != p0) L[x0] = g0;
        if (!d1 && g1 != p1) L[x1] = g1;
        if (!ds) s = ps;
        if (!d0) x0 = g0;
        if (!d1) x1 = g1;
    }
    atomicOr(status, kDevErrUnionFind);
    rs = s;
    r0 = x0;
    r1 = x1;
}

__device__ __forceinline__ void uf_union(uint32_t* lab, uint32_t a, uint32_t b, uint32_t bound, unsigned* status)
{
    // both finds walked together: their load chains overlap
    uf_find2(lab, a, b, bound, status, a, b);
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (a == b) return;
        if (uf_priority(a) > uf_priority(b)) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        // link the lower-priority root under the higher-priority one
        const uint32_t old = atomicCAS(lab + a, a, b);
        if (old == a) return;
        uf_find2(lab, old, b, bound, status, a, b);
    }
    atomicOr(status, kDevErrUnionFind);
}

}  // namespace umc
