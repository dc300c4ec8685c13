// umc_fused.cuh -- one cooperative kernel per step on the regular lattices.
//
// On small lattices (64^3 fits in L2) a step is bounded by per-kernel fixed
// costs, not by work: five launches (Wolff tile labelling, merge, flip, two
// colour passes) each pay ramp-up, drain and a last-block reduction.  This
// kernel runs the same phases back to back inside one launch, separated by a
// grid barrier, with all blocks co-resident (cooperative launch):
//
//   A  Wolff: per tile, bond activation + shared-memory union-find  (optional)
//   B  Wolff: union of the activated tile-crossing bonds, compacted
//      into a list in A, on the global labels                       (optional)
//   C  Wolff: reflect the seed's cluster                             (optional)
//   D  Metropolis pass over colour class 0                           (optional)
//   E  Metropolis pass over colour class 1, FP64 observables folded  (optional)
//
// The per-site arithmetic is shared with the multi-kernel path (same device
// functions), so results are identical up to the order of the FP64 sums.
//
// The grid barrier is bounded: a block that waits longer than kBarrierSpins
// polls raises kDevErrBarrier and leaves; the others then run out at their own
// next barrier, so the kernel always terminates.  Data written before a
// barrier by another block is read with L2-coherent loads (ld.global.cg).
#pragma once

#include "umc_wolff_tiled.cuh"

namespace umc {

// polls: the first kBarrierHot back to back (a balanced phase ends within a
// few L2 round trips), then with a 64 ns sleep; the bound is ~0.3 s
constexpr unsigned kBarrierSpins = 1u << 22;
constexpr unsigned kBarrierHot = 256u;

__device__ __forceinline__ bool grid_barrier(GridBarrier* b, unsigned* status)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        __threadfence();
        // arrival; this barrier completes when count reaches the next
        // multiple of gridDim (one round trip, no generation word to update)
        const unsigned int old = atomicAdd(&b->count, 1u);
        const unsigned int target = (old / gridDim.x + 1u) * gridDim.x;
        volatile unsigned int* cnt = &b->count;
        unsigned int it = 0;
        while (*cnt < target) {
            if (++it > kBarrierSpins) {
                atomicOr(status, kDevErrBarrier);
                ok = 0;
                break;
            }
            if (it > kBarrierHot) __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

// Once per block after its last barrier: the last block to get here has seen
// every other block leave its polls, so it can reset the counter for the next
// launch (stream-ordered after this one).  A block that left on a barrier
// error does not retire; the host clears the control block on that error.
__device__ __forceinline__ void grid_barrier_retire(GridBarrier* b)
{
    if (threadIdx.x == 0 && atomicAdd(&b->done, 1u) == gridDim.x - 1) {
        b->count = 0u;
        b->done = 0u;
    }
}

struct FusedArgs
{
    WolffTileArgs w;  // Wolff phases (w.field is the field)
    GridBarrier* bar;
    uint32_t do_wolff, do_sweep;
    uint32_t H, hshift, yshift;
    uint64_t sweep_kbase;  // key base of this sweep's site streams
    float beta_metro;
    uint32_t proposal;  // kPropSphere / kPropRotation
    float delta;
    PassOut out;        // record of the sweep (pass index: dedicated slot)
    uint32_t* xlist;    // activated tile-crossing bonds, site * 4 + direction
    uint32_t xcap;      // its capacity (>= every + bond that can leave a tile)
    double beta_metro64;  // beta of the FP64 accept decisions
    float err_metro;      // vector_metropolis_err
};

template <int N>
__device__ __forceinline__ void fused_site(const FusedArgs& a, const StencilTopo& t, uint32_t k, double* acc)
{
    float* f = static_cast<float*>(a.w.field);
    const uint32_t n = a.w.n;
    float s[N], h[N];
#pragma unroll
    for (int c = 0; c < N; ++c) {
        s[c] = __ldcg(f + c * n + k);
        h[c] = 0.0f;
    }
    t.neighbours(k, [&](uint32_t j, bool) {
#pragma unroll
        for (int c = 0; c < N; ++c) h[c] += __ldcg(f + c * n + j);
    });
    KeyedPcg g = KeyedPcg::open(a.sweep_kbase, k);
    float cand[N];
    bool ok = true;
    if (a.proposal == kPropSphere) sphere_sample<N>(g, cand);
    else if constexpr (N >= 2) ok = local_rotation<N>(g, a.delta, s, cand);
    bool acc_ok = false;
    if (ok) {
        const float dE = -a.w.J * (vdot<N>(cand, h) - vdot<N>(s, h));
        acc_ok = metropolis_accept(g, -a.beta_metro * dE, a.err_metro, [&] {
            // the reference's sum over bonds, in FP64 on the FP32 state
            double d = 0.0;
            t.neighbours(k, [&](uint32_t j, bool) {
                double pj = 0.0, oj = 0.0;
#pragma unroll
                for (int c = 0; c < N; ++c) {
                    const double v = __ldcg(f + c * n + j);
                    pj += double(cand[c]) * v;
                    oj += double(s[c]) * v;
                }
                d += -a.w.J64 * (pj - oj);
            });
            return -a.beta_metro64 * d;
        });
    }
    if (acc_ok) {
#pragma unroll
        for (int c = 0; c < N; ++c) {
            s[c] = cand[c];
            f[c * n + k] = cand[c];
        }
    }
    // every bond joins the two classes: count it in the pass of class 1
    if (t.colour == 1u) acc[0] += double(-a.w.J * vdot<N>(s, h));
#pragma unroll
    for (int c = 0; c < N; ++c) acc[1 + c] += double(s[c]);
    acc[7] += acc_ok ? 1.0 : 0.0;
}

// MODEL = N >= 1 (VectorSpin<N>).  Phase A: one tile of TX*TY*TZ sites per
// block and iteration, SPT sites per thread (local ids tid + u * blockDim).
// Each thread first activates the bonds of all its sites (their loads and
// draws overlap), then does the shared-memory unions.
template <int MODEL, int TX, int TY, int TZ, int SPT>
__global__ void __launch_bounds__(TX * TY * TZ / SPT, 2 * SPT) hybrid_fused(FusedArgs a)
{
    constexpr int N = MODEL;
    constexpr int T = TX * TY * TZ;
    constexpr int BT = T / SPT;
    static_assert(T % SPT == 0, "sites per thread must divide the tile");
    __shared__ uint32_t lab[T];
    __shared__ float r_sh[4];
    __shared__ uint32_t seed_sh;
    __shared__ uint32_t xs_cnt, xs_base;
    const WolffTileArgs& w = a.w;
    unsigned* status = &w.ctl->status;
    const uint32_t tid = threadIdx.x;
    const uint32_t gtid = blockIdx.x * blockDim.x + tid, gsize = gridDim.x * blockDim.x;

    if (a.do_wolff) {
        KeyedPcg gax = KeyedPcg::open_key(w.seed, w.flip, kTagAxis, 0);
        if (tid == 0) {
            float r[N];
            sphere_sample<N>(gax, r);
            for (int c = 0; c < N; ++c) r_sh[c] = r[c];
            // seed site: next draw of the axis stream, colour-major -> natural
            const uint32_t ks = uint32_t(u_f64(gax.next()) * double(w.n));
            const uint32_t c = ks >= w.half ? 1u : 0u, rank = ks - c * w.half;
            uint32_t nat = 2 * rank;
            const uint32_t x = nat % w.Lx, rr = nat / w.Lx, y = rr % w.Ly, z = rr / w.Ly;
            if (((x + y + z) & 1u) != c) ++nat;
            seed_sh = nat;
            if (blockIdx.x == 0) *w.size_slot = 0ull;
        }
        // ---- A: tiles
        const uint32_t ntz = (w.Lz + TZ - 1) / TZ;
        const uint32_t ntiles = w.ntx * w.nty * ntz;
        const uint64_t kb = key_base(key_seed(w.seed, w.flip, kTagBond));
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            __syncthreads();
#pragma unroll
            for (int u = 0; u < SPT; ++u) lab[tid + u * BT] = tid + u * BT;
            __syncthreads();
            float r[N];
#pragma unroll
            for (int c = 0; c < N; ++c) r[c] = r_sh[c];
            const uint32_t bx = tile % w.ntx, byz = tile / w.ntx;
            const uint32_t by = byz % w.nty, bz = byz / w.nty;
            uint32_t nat[SPT], cross[SPT], inner[SPT], tjs[SPT][3];
            // bond activation of every site of this thread
#pragma unroll
            for (int u = 0; u < SPT; ++u) {
                const uint32_t lid = tid + u * BT;
                const uint32_t tx = lid % TX, ty = (lid / TX) % TY, tz = lid / (TX * TY);
                const uint32_t x = bx * TX + tx, y = by * TY + ty, z = bz * TZ + tz;
                cross[u] = 0;
                inner[u] = 0;
                nat[u] = 0xFFFFFFFFu;
                if (!(x < w.Lx && y < w.Ly && z < w.Lz)) continue;
                nat[u] = (z * w.Ly + y) * w.Lx + x;
                float si[N];
                load_spin<N>(w.field, w.n, colour_major(nat[u], x, y, z, w.half), si);
                uint32_t rank = 0;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    tjs[u][d] = 0;
                    const uint32_t L = d == 0 ? w.Lx : (d == 1 ? w.Ly : w.Lz);
                    if (L < 2) continue;
                    uint32_t xj = x, yj = y, zj = z;
                    if (d == 0) xj = x + 1 == w.Lx ? 0 : x + 1;
                    if (d == 1) yj = y + 1 == w.Ly ? 0 : y + 1;
                    if (d == 2) zj = z + 1 == w.Lz ? 0 : z + 1;
                    const uint32_t nj = (zj * w.Ly + yj) * w.Lx + xj;
                    float sj[N];
                    load_spin<N>(w.field, w.n, colour_major(nj, xj, yj, zj, w.half), sj);
                    const uint32_t k = first_draw(kb, nat[u] * w.ndir + rank);
                    ++rank;
                    if (!vector_bond_active<N>(w.J, w.beta, w.J64, w.beta64, w.err, si, sj, r, k)) continue;
                    if (xj / TX == bx && yj / TY == by && zj / TZ == bz) {
                        tjs[u][d] = ((zj - bz * TZ) * TY + (yj - by * TY)) * TX + (xj - bx * TX);
                        inner[u] |= 1u << d;
                    } else {
                        cross[u] |= 1u << d;
                    }
                }
            }
            // unions inside the tile
#pragma unroll
            for (int u = 0; u < SPT; ++u)
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if (inner[u] & (1u << d)) smem_union(lab, tid + u * BT, tjs[u][d], status);
            // compact this tile's activated crossing bonds into the global list:
            // one atomic per block, then each thread writes its bonds
            if (tid == 0) xs_cnt = 0;
            __syncthreads();
            uint32_t nc = 0;
#pragma unroll
            for (int u = 0; u < SPT; ++u) nc += __popc(cross[u]);
            const uint32_t off = nc ? atomicAdd(&xs_cnt, nc) : 0u;
            __syncthreads();
            if (tid == 0) xs_base = xs_cnt ? atomicAdd(&w.ctl->xcount, xs_cnt) : 0u;
            __syncthreads();
            uint32_t slot = xs_base + off;
#pragma unroll
            for (int u = 0; u < SPT; ++u) {
                if (nat[u] == 0xFFFFFFFFu) continue;
                const uint32_t root = smem_find(lab, tid + u * BT);
                const uint32_t rx = root % TX, ry = (root / TX) % TY, rz = root / (TX * TY);
                w.label[nat[u]] = ((bz * TZ + rz) * w.Ly + (by * TY + ry)) * w.Lx + (bx * TX + rx);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    if (!(cross[u] & (1u << d))) continue;
                    if (slot < a.xcap) a.xlist[slot] = nat[u] * 4u + uint32_t(d);
                    else atomicOr(status, kDevErrGeometry);
                    ++slot;
                }
            }
        }
        if (!grid_barrier(a.bar, status)) return;

        // ---- B: tile-crossing bonds, one list entry per thread
        const uint32_t xcount = min(__ldcg(&w.ctl->xcount), a.xcap);
        for (uint32_t i = gtid; i < xcount; i += gsize) {
            const uint32_t e = __ldcg(a.xlist + i);
            const uint32_t nat = e >> 2, d = e & 3u;
            const uint32_t x = nat % w.Lx, rr = nat / w.Lx, y = rr % w.Ly, z = rr / w.Ly;
            uint32_t xj = x, yj = y, zj = z;
            if (d == 0) xj = x + 1 == w.Lx ? 0 : x + 1;
            if (d == 1) yj = y + 1 == w.Ly ? 0 : y + 1;
            if (d == 2) zj = z + 1 == w.Lz ? 0 : z + 1;
            uf_union(w.label, nat, (zj * w.Ly + yj) * w.Lx + xj, w.n + 1, status);
        }
        if (!grid_barrier(a.bar, status)) return;

        // ---- C: flip the seed's cluster (the list is consumed: reset it)
        if (gtid == 0) w.ctl->xcount = 0u;
        {
            float r[N];
#pragma unroll
            for (int c = 0; c < N; ++c) r[c] = r_sh[c];
            const uint32_t seed = seed_sh;
            uint32_t root = 0xFFFFFFFFu;
            double cnt[1] = {0.0};
            float* f = static_cast<float*>(w.field);
            // two sites per thread and iteration, their finds walked together;
            // in the first iteration every thread also walks the seed's path
            // to its root (read only) in the same lockstep, so no thread waits
            // for one thread's find of the seed
            for (uint32_t n0 = gtid; n0 < w.n; n0 += 2 * gsize) {
                const uint32_t n1 = n0 + gsize;
                uint32_t r0, r1;
                if (root == 0xFFFFFFFFu) uf_find_with_root(w.label, seed, n0, n1 < w.n ? n1 : n0, w.n + 1, status, root, r0, r1);
                else uf_find2(w.label, n0, n1 < w.n ? n1 : n0, w.n + 1, status, r0, r1);
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const uint32_t nat = u ? n1 : n0;
                    if ((u ? r1 : r0) != root || nat >= w.n) continue;
                    cnt[0] += 1.0;
                    const uint32_t x = nat % w.Lx, rr = nat / w.Lx, y = rr % w.Ly, z = rr / w.Ly;
                    const uint32_t k = colour_major(nat, x, y, z, w.half);
                    float si[N];
#pragma unroll
                    for (int c = 0; c < N; ++c) si[c] = __ldcg(f + c * w.n + k);
                    reflect<N>(si, r);
#pragma unroll
                    for (int c = 0; c < N; ++c) f[c * w.n + k] = si[c];
                }
            }
            block_sum<1>(cnt);
            if (tid == 0 && cnt[0] > 0.0) atomicAdd(w.size_slot, (unsigned long long)cnt[0]);
        }
        if (a.do_sweep && !grid_barrier(a.bar, status)) return;
    }

    if (a.do_sweep) {
        double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
        StencilTopo t{a.H, w.Ly, w.Lz, w.half, 0u, w.Ly > 1 ? 1u : 0u, w.Lz > 1 ? 1u : 0u, a.hshift, a.yshift};
        // ---- D: colour class 0
        for (uint32_t q = gtid; q < w.half; q += gsize) fused_site<N>(a, t, q, acc);
        if (!grid_barrier(a.bar, status)) return;
        // ---- E: colour class 1, then the sweep's record
        t.colour = 1u;
        for (uint32_t q = gtid; q < w.n - w.half; q += gsize) fused_site<N>(a, t, w.half + q, acc);
        finish_pass<kObs>(acc, a.out);
    }
    grid_barrier_retire(a.bar);
}

}  // namespace umc
