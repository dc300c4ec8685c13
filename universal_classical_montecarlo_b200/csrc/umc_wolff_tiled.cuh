// umc_wolff_tiled.cuh -- Wolff flip on the regular lattices in three kernels:
//
//   wolff_tile_local   one block per lattice tile: decides every + bond of its
//                      sites (same keyed draw as the CSR path: edge id =
//                      site * n_dirs + direction rank, the square/cubic
//                      builders' edge order), unions the bonds inside the tile
//                      in shared memory, writes each site's tile root as its
//                      global label and flags bonds leaving the tile;
//   wolff_tile_merge   unions the flagged tile-crossing bonds on the global
//                      labels (shallow trees: every label is one hop from a
//                      tile root);
//   wolff_tile_flip    reflects every site whose root is the seed's root.
//
// Labels are natural site ids and are rewritten by every flip, so nothing has
// to be reset in between.  The cluster is the seed's connected component over
// activated bonds, exactly as in the CSR kernels (umc_spin_kernels.cuh) and in
// the reference's depth-first growth (driver.hpp:124-157).
#pragma once

#include "umc_spin_kernels.cuh"

namespace umc {

struct WolffTileArgs
{
    void* field;            // colour-major: component c of site k at field[c*n + k]
    uint32_t* label;        // n natural-order labels
    uint8_t* cross;         // n bit masks of activated tile-crossing + bonds
    uint32_t n, half;
    uint32_t Lx, Ly, Lz;
    uint32_t ntx, nty;      // tiles along x and y
    uint32_t ndir;          // directions with extent > 1
    uint64_t seed, flip;
    float J, beta;
    unsigned long long cw[2];
    DevCtl* ctl;
    unsigned long long* size_slot;
    double J64, beta64;  // VectorSpin: the coupling and beta of the FP64 decisions
    float err;           // VectorSpin: vector_wolff_err
};

__device__ __forceinline__ uint32_t colour_major(uint32_t nat, uint32_t x, uint32_t y, uint32_t z, uint32_t half)
{
    return ((x + y + z) & 1u) * half + (nat >> 1);
}

template <int MODEL>
__device__ __forceinline__ void load_spin(const void* field, uint32_t n, uint32_t k, float* s)
{
    if constexpr (MODEL == 0) {
        s[0] = float(static_cast<const int8_t*>(field)[k]);
    } else {
#pragma unroll
        for (int c = 0; c < MODEL; ++c) s[c] = static_cast<const float*>(field)[c * n + k];
    }
}

__device__ __forceinline__ uint32_t smem_find(uint32_t* lab, uint32_t x)
{
    volatile uint32_t* L = lab;
    for (int it = 0; it < 4096; ++it) {
        const uint32_t p = L[x];
        if (p == x) return x;
        const uint32_t gp = L[p];
        if (gp != p) L[x] = gp;
        x = gp;
    }
    return x;
}

__device__ __forceinline__ void smem_union(uint32_t* lab, uint32_t a, uint32_t b, unsigned* status)
{
    a = smem_find(lab, a);
    b = smem_find(lab, b);
    for (int it = 0; it < 1 << 16; ++it) {
        if (a == b) return;
        if (uf_priority(a) > uf_priority(b)) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicCAS(lab + a, a, b);
        if (old == a) return;
        a = smem_find(lab, old);
        b = smem_find(lab, b);
    }
    atomicOr(status, kDevErrUnionFind);
}

// (512 threads, 4 blocks): at most 32 registers; the out-of-line FP64
// activation test spills inside itself instead of widening the kernel.
template <int MODEL, int TX, int TY, int TZ>
__global__ void __launch_bounds__(TX * TY * TZ, 65536 / (32 * TX * TY * TZ)) wolff_tile_local(WolffTileArgs a)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    constexpr int T = TX * TY * TZ;
    __shared__ uint32_t lab[T];
    __shared__ float r_sh[4];
    const uint32_t tid = threadIdx.x;
    const uint32_t bx = blockIdx.x % a.ntx, byz = blockIdx.x / a.ntx;
    const uint32_t by = byz % a.nty, bz = byz / a.nty;
    const uint32_t tx = tid % TX, ty = (tid / TX) % TY, tz = tid / (TX * TY);
    const uint32_t x = bx * TX + tx, y = by * TY + ty, z = bz * TZ + tz;
    const bool valid = x < a.Lx && y < a.Ly && z < a.Lz;
    if (tid == 0) {
        KeyedPcg g = KeyedPcg::open_key(a.seed, a.flip, kTagAxis, 0);
        float r[N];
        if constexpr (MODEL == 0) r[0] = 1.0f;
        else sphere_sample<MODEL>(g, r);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
        if (blockIdx.x == 0) *a.size_slot = 0ull;
    }
    lab[tid] = tid;
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint64_t kb = key_base(key_seed(a.seed, a.flip, kTagBond));
    uint32_t cross = 0;
    uint32_t nat = 0;
    if (valid) {
        nat = (z * a.Ly + y) * a.Lx + x;
        float si[N];
        load_spin<MODEL>(a.field, a.n, colour_major(nat, x, y, z, a.half), si);
        uint32_t rank = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const uint32_t L = d == 0 ? a.Lx : (d == 1 ? a.Ly : a.Lz);
            if (L < 2) continue;
            uint32_t xj = x, yj = y, zj = z;
            if (d == 0) xj = x + 1 == a.Lx ? 0 : x + 1;
            if (d == 1) yj = y + 1 == a.Ly ? 0 : y + 1;
            if (d == 2) zj = z + 1 == a.Lz ? 0 : z + 1;
            const uint32_t nj = (zj * a.Ly + yj) * a.Lx + xj;
            float sj[N];
            load_spin<MODEL>(a.field, a.n, colour_major(nj, xj, yj, zj, a.half), sj);
            const uint32_t k = first_draw(kb, nat * a.ndir + rank);
            ++rank;
            bool on;
            if constexpr (MODEL == 0) on = ising_bond_active(a.cw, int(si[0]), int(sj[0]), k);
            else on = vector_bond_active<N>(a.J, a.beta, a.J64, a.beta64, a.err, si, sj, r, k);
            if (!on) continue;
            const bool same = xj / TX == bx && yj / TY == by && zj / TZ == bz;
            if (same) {
                const uint32_t tj = ((zj - bz * TZ) * TY + (yj - by * TY)) * TX + (xj - bx * TX);
                smem_union(lab, tid, tj, &a.ctl->status);
            } else {
                cross |= 1u << d;
            }
        }
    }
    __syncthreads();
    if (valid) {
        const uint32_t root = smem_find(lab, tid);
        const uint32_t rx = root % TX, ry = (root / TX) % TY, rz = root / (TX * TY);
        a.label[nat] = ((bz * TZ + rz) * a.Ly + (by * TY + ry)) * a.Lx + (bx * TX + rx);
        a.cross[nat] = uint8_t(cross);
    }
}

__global__ void __launch_bounds__(kBlock) wolff_tile_merge(WolffTileArgs a)
{
    for (uint32_t nat = blockIdx.x * blockDim.x + threadIdx.x; nat < a.n; nat += gridDim.x * blockDim.x) {
        const uint32_t cross = a.cross[nat];
        if (!cross) continue;
        const uint32_t x = nat % a.Lx, r = nat / a.Lx, y = r % a.Ly, z = r / a.Ly;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (!(cross & (1u << d))) continue;
            uint32_t xj = x, yj = y, zj = z;
            if (d == 0) xj = x + 1 == a.Lx ? 0 : x + 1;
            if (d == 1) yj = y + 1 == a.Ly ? 0 : y + 1;
            if (d == 2) zj = z + 1 == a.Lz ? 0 : z + 1;
            uf_union(a.label, nat, (zj * a.Ly + yj) * a.Lx + xj, a.n + 1, &a.ctl->status);
        }
    }
}

template <int MODEL>
__global__ void __launch_bounds__(kBlock) wolff_tile_flip(WolffTileArgs a)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    __shared__ float r_sh[4];
    __shared__ uint32_t root_sh;
    if (threadIdx.x == 0) {
        KeyedPcg g = KeyedPcg::open_key(a.seed, a.flip, kTagAxis, 0);
        float r[N];
        if constexpr (MODEL == 0) r[0] = 1.0f;
        else sphere_sample<MODEL>(g, r);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
        // the seed is drawn in colour-major order (driver.hpp:114-115 on the
        // relabelled lattice): map it back to its natural site id
        const uint32_t ks = uint32_t(u_f64(g.next()) * double(a.n));
        const uint32_t c = ks >= a.half ? 1u : 0u, rank = ks - c * a.half;
        uint32_t nat = 2 * rank;
        const uint32_t x = nat % a.Lx, rr = nat / a.Lx, y = rr % a.Ly, z = rr / a.Ly;
        if (((x + y + z) & 1u) != c) ++nat;
        root_sh = nat < a.n ? uf_find(a.label, nat, a.n + 1, &a.ctl->status) : 0xFFFFFFFFu;
    }
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint32_t root = root_sh;
    double cnt[1] = {0.0};
    for (uint32_t nat = blockIdx.x * blockDim.x + threadIdx.x; nat < a.n; nat += gridDim.x * blockDim.x) {
        if (uf_find(a.label, nat, a.n + 1, &a.ctl->status) != root) continue;
        cnt[0] += 1.0;
        const uint32_t x = nat % a.Lx, rr = nat / a.Lx, y = rr % a.Ly, z = rr / a.Ly;
        const uint32_t k = colour_major(nat, x, y, z, a.half);
        if constexpr (MODEL == 0) {
            int8_t* s = static_cast<int8_t*>(a.field);
            s[k] = int8_t(-s[k]);
        } else {
            float* f = static_cast<float*>(a.field);
            float si[N];
#pragma unroll
            for (int c = 0; c < N; ++c) si[c] = f[c * a.n + k];
            reflect<N>(si, r);
#pragma unroll
            for (int c = 0; c < N; ++c) f[c * a.n + k] = si[c];
        }
    }
    block_sum<1>(cnt);
    if (threadIdx.x == 0 && cnt[0] > 0.0) atomicAdd(a.size_slot, (unsigned long long)cnt[0]);
}

}  // namespace umc
