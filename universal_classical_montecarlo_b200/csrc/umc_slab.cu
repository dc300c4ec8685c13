// umc_slab.cu -- one lattice over several GPUs: slab domain decomposition of
// the regular-lattice Metropolis sweep (one process per GPU).
//
// The lattice Lx x Ly x Lz (Lz = 1 in 2D) is cut along its slowest axis of
// extent above 1 (z in 3D, y in 2D) into contiguous planes; a rank holds its
// planes [first, first + planes) plus one halo plane on each side, in natural
// order (x fastest), one array per component (component c of local site q at
// field[c * local_sites + q]).  A colour pass updates the rank's sites of one
// checkerboard colour; their neighbours of the other colour lie in the slab
// or its halos, which the caller refreshes from the neighbouring ranks between
// passes (the boundary planes only: torch.distributed send/recv over NCCL, or
// any copy).  Every site draws from the keyed stream of its GLOBAL colour-major
// index, and sums its neighbours in the order of the single-GPU stencil
// kernels (umc_spin_kernels.cuh StencilTopo), so the union of the ranks'
// updates is the single-GPU chain: bit for bit for Ising (integer thresholds),
// and to the same FP32 arithmetic for VectorSpin<N>.
//
// The reference has no decomposition (one chain per driver object,
// driver.hpp:17-68); the per-site rule is its Metropolis::sweep body
// (driver.hpp:34-42) with Ising::energy_diff_at (example/ising.hpp:46-56) or
// VectorSpin::energy_diff_at (example/vector_spin.hpp:50-60).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "umc_chain.hpp"
#include "umc_nvtx.hpp"
#include "umc_spin_kernels.cuh"

namespace umc {
namespace {

struct SlabArgs
{
    void* field;
    uint32_t Lx, Ly, Lz;
    uint32_t along_z;  // 1: planes are z planes (3D); 0: rows y (2D)
    uint32_t first, planes;
    uint32_t P;        // sites per plane
    uint32_t nloc;     // (planes + 2) * P
    uint32_t half;     // global sites / 2
    uint32_t colour;
    uint64_t kbase;
    float J, beta, delta;
    double J64, beta64;
    float err;
    const uint32_t* tm1;  // Ising: accept iff draw <= tm1[s h + D]
    int32_t D, Jint;
    PassOut out;
};

// Owned site q of the pass's colour -> its local index, its global
// colour-major index, and its neighbours' local indices in StencilTopo's
// order: the two same-row neighbours (x+1, x-1 when the site sits on an even
// x of its row's colour pattern, else x-1, x+1), then y-1, y+1, then z-1, z+1,
// each pair only where that extent exceeds 1.
struct SlabSite
{
    uint32_t li, k, deg;
    uint32_t nb[6];
};

__device__ __forceinline__ SlabSite slab_site(const SlabArgs& a, uint32_t q)
{
    const uint32_t H = a.Lx / 2;
    const uint32_t per_plane = a.P / 2;
    const uint32_t pl = q / per_plane, r = q - pl * per_plane;
    uint32_t x, y, z;
    if (a.along_z) {
        y = r / H;
        const uint32_t i = r - y * H;
        z = a.first + pl;
        x = 2 * i + ((y + z + a.colour) & 1u);
    } else {
        y = a.first + pl;
        z = 0;
        x = 2 * r + ((y + a.colour) & 1u);
    }
    SlabSite s;
    const uint32_t lp = pl + 1;  // local plane (0 and planes + 1 are the halos)
    const uint32_t inplane = a.along_z ? y * a.Lx : 0u;
    s.li = lp * a.P + inplane + x;
    const uint32_t g = (z * a.Ly + y) * a.Lx + x;
    s.k = a.colour * a.half + g / 2;
    const uint32_t xp = x + 1 == a.Lx ? 0u : x + 1, xm = x == 0 ? a.Lx - 1 : x - 1;
    const uint32_t row = lp * a.P + inplane;
    const bool even = ((x & 1u) == 0u);
    s.nb[0] = row + (even ? xp : xm);
    s.nb[1] = row + (even ? xm : xp);
    s.deg = 2;
    if (a.Ly > 1) {
        if (a.along_z) {
            const uint32_t ym = y == 0 ? a.Ly - 1 : y - 1, yp = y + 1 == a.Ly ? 0u : y + 1;
            s.nb[s.deg++] = lp * a.P + ym * a.Lx + x;
            s.nb[s.deg++] = lp * a.P + yp * a.Lx + x;
        } else {
            s.nb[s.deg++] = (lp - 1) * a.P + x;
            s.nb[s.deg++] = (lp + 1) * a.P + x;
        }
    }
    if (a.along_z && a.Lz > 1) {
        s.nb[s.deg++] = (lp - 1) * a.P + y * a.Lx + x;
        s.nb[s.deg++] = (lp + 1) * a.P + y * a.Lx + x;
    }
    return s;
}

template <int N>
__device__ __noinline__ double slab_log_ratio64(const SlabArgs& a, SlabSite st, SpinVal<N> cand, SpinVal<N> s)
{
    const float* f = static_cast<const float*>(a.field);
    double d = 0.0;
    for (uint32_t m = 0; m < st.deg; ++m) {
        double pj = 0.0, oj = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c) {
            const double v = f[c * a.nloc + st.nb[m]];
            pj += double(cand.v[c]) * v;
            oj += double(s.v[c]) * v;
        }
        d += -a.J64 * (pj - oj);
    }
    return -a.beta64 * d;
}

template <int N, int PROP>
__global__ void __launch_bounds__(kBlock, 4) slab_vector_pass(SlabArgs a)
{
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    float* f = static_cast<float*>(a.field);
    const uint32_t count = a.planes * (a.P / 2);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const SlabSite st = slab_site(a, q);
        float s[N], h[N];
#pragma unroll
        for (int c = 0; c < N; ++c) {
            s[c] = f[c * a.nloc + st.li];
            h[c] = 0.0f;
        }
        for (uint32_t m = 0; m < st.deg; ++m)
#pragma unroll
            for (int c = 0; c < N; ++c) h[c] += f[c * a.nloc + st.nb[m]];
        KeyedPcg g = KeyedPcg::open(a.kbase, st.k);
        float cand[N];
        bool ok = true;
        if constexpr (PROP == kPropSphere) sphere_sample<N>(g, cand);
        else ok = local_rotation<N>(g, a.delta, s, cand);
        bool acc_ok = false;
        if (ok) {
            const float dE = -a.J * (vdot<N>(cand, h) - vdot<N>(s, h));
            acc_ok = metropolis_accept(g, -a.beta * dE, a.err, [&] {
                SpinVal<N> cv, sv;
#pragma unroll
                for (int c = 0; c < N; ++c) {
                    cv.v[c] = cand[c];
                    sv.v[c] = s[c];
                }
                return slab_log_ratio64<N>(a, st, cv, sv);
            });
        }
        if (acc_ok) {
#pragma unroll
            for (int c = 0; c < N; ++c) {
                s[c] = cand[c];
                f[c * a.nloc + st.li] = cand[c];
            }
        }
        // every bond joins the two colours: count it in the colour-1 pass
        if (a.colour == 1u) acc[0] += double(-a.J * vdot<N>(s, h));
#pragma unroll
        for (int c = 0; c < N; ++c) acc[1 + c] += double(s[c]);
        acc[7] += acc_ok ? 1.0 : 0.0;
    }
    finish_pass<kObs>(acc, a.out);
}

// 2D Ising with the rows split by colour (local row r holds the class-0 sites
// of its row at r * Lx + [0, H), the class-1 sites at r * Lx + H + [0, H), in
// x order; row y's class-c sites sit at x = 2i + ((y + c) & 1)): the pass of
// ising_packed_pass (umc_spin_kernels.cuh) -- 16 sites of a row per thread,
// one 16-byte load of the own class and three of the other class (rows y-1,
// y, y+1, the outer two possibly halo rows), the 16 consecutive outputs of the
// stream of the vector's global colour-major index / 16 -- so each site takes
// the draw, the threshold and the update of the single-GPU pass.  Needs H a
// multiple of 16.
__global__ void __launch_bounds__(kBlock) slab_ising_row_pass(SlabArgs a)
{
    __shared__ uint32_t tm1[5];
    // the slab's table is indexed by s h + D (D = 4); this pass by (s h + 4) / 2
    if (threadIdx.x < 5) tm1[threadIdx.x] = a.tm1[2 * threadIdx.x];
    __syncthreads();
    int64_t e_acc = 0, m_acc = 0, n_acc = 0;
    int8_t* sp = static_cast<int8_t*>(a.field);
    const uint32_t H = a.Lx / 2, vpr = H >> 4;
    const uint32_t nvec = a.planes * vpr;
    const uint32_t oc = (1u - a.colour) * H, cc = a.colour * H;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < nvec; v += gridDim.x * blockDim.x) {
        const uint32_t pl = v / vpr, i0 = (v - pl * vpr) << 4;
        const uint32_t lr = pl + 1, gy = a.first + pl;  // local and global row
        const uint32_t p = (gy + a.colour) & 1u;
        int8_t* own = sp + size_t(lr) * a.Lx + cc;
        const int8_t* mid = sp + size_t(lr) * a.Lx + oc;
        const uint4 s4 = *reinterpret_cast<const uint4*>(own + i0);
        const uint4 m4 = *reinterpret_cast<const uint4*>(mid + i0);
        const uint4 u4 = *reinterpret_cast<const uint4*>(sp + size_t(lr + 1) * a.Lx + oc + i0);
        const uint4 d4 = *reinterpret_cast<const uint4*>(sp + size_t(lr - 1) * a.Lx + oc + i0);
        const uint32_t xe = p ? (i0 + 16 == H ? 0u : i0 + 16) : (i0 == 0 ? H - 1 : i0 - 1);
        const uint32_t extra = uint32_t(uint8_t(mid[xe]));
        const uint32_t sw[4] = {s4.x, s4.y, s4.z, s4.w};
        const uint32_t mw[4] = {m4.x, m4.y, m4.z, m4.w};
        const uint32_t uw[4] = {u4.x, u4.y, u4.z, u4.w};
        const uint32_t dw[4] = {d4.x, d4.y, d4.z, d4.w};
        uint32_t out[4];
        KeyedPcg rng = KeyedPcg::open(a.kbase, (a.colour * a.half + gy * H + i0) / kGroupSites);
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            // second horizontal neighbour: byte k-1 (p == 0) or k+1 (p == 1)
            const uint32_t h2 = p ? __byte_perm(mw[w], w == 3 ? extra : mw[w + 1], 0x4321)
                                  : __byte_perm(w == 0 ? (extra << 24) : mw[w - 1], mw[w], 0x6543);
            const uint32_t nd = down_bits(uw[w]) + down_bits(dw[w]) + down_bits(mw[w]) + down_bits(h2);
            const uint32_t di = down_bits(sw[w]);
            const uint32_t mask = di * 0xFFu;
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
            const int32_t sh = 16 - 2 * int32_t(byte_sum(nd)) - 8 * ndown + 4 * int32_t(byte_sum(nd & (dn * 0xFFu)));
            e_acc += sh;
        }
        *reinterpret_cast<uint4*>(own + i0) = make_uint4(out[0], out[1], out[2], out[3]);
    }
    // every bond joins the two classes: count it once, in the pass of class 1
    double v[kObs] = {a.colour == 1u ? double(-int64_t(a.Jint) * e_acc) : 0.0, double(m_acc), 0, 0, 0, 0, 0,
                      double(n_acc)};
    finish_pass<kObs>(v, a.out);
}

__global__ void __launch_bounds__(kBlock) slab_ising_pass(SlabArgs a)
{
    int64_t e_acc = 0, m_acc = 0, n_acc = 0;
    int8_t* sp = static_cast<int8_t*>(a.field);
    const uint32_t count = a.planes * (a.P / 2);
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        const SlabSite st = slab_site(a, q);
        int32_t h = 0;
        for (uint32_t m = 0; m < st.deg; ++m) h += sp[st.nb[m]];
        const int32_t s = sp[st.li];
        // one draw per site: output k % 16 of the stream of id k / 16, the
        // engine's Ising keying; integer thresholds make the decision exact
        const uint32_t r = group_draw(a.kbase, st.k);
        const bool flip = r <= a.tm1[s * h + a.D];
        const int32_t ns = flip ? -s : s;
        if (flip) sp[st.li] = int8_t(ns);
        if (a.colour == 1u) e_acc += ns * h;
        m_acc += ns;
        n_acc += flip;
    }
    double v[kObs] = {double(-int64_t(a.Jint) * e_acc), double(m_acc), 0, 0, 0, 0, 0, double(n_acc)};
    finish_pass<kObs>(v, a.out);
}

// ---------------------------------------------------------- Wolff across slabs
// One Wolff flip of the whole lattice: each rank decides the forward bonds of
// its owned sites (x+, y+, and z+ in 3D; the key of bond (site, direction) is
// the single-GPU one, natural site id * directions + direction rank), unions
// the ones inside its slab, and reports its boundary: the root of every site
// of its first and last owned planes and which last-plane sites have an
// activated bond into the next rank.  Every rank then merges all ranks'
// boundaries on the host in the same way and flips the local roots whose
// component holds the seed: the single-GPU flip's cluster.
struct SlabWolffArgs
{
    void* field;
    uint32_t Lx, Ly, Lz;
    uint32_t along_z;
    uint32_t first, planes, P, nloc, n, half;
    uint64_t seed, flip;
    float J, beta;
    double J64, beta64;
    float err;
    unsigned long long cw[2];
    uint32_t row_split;  // 2D Ising rows stored split by colour (slab_ising_row_pass)
    uint32_t* lab;   // per owned site (planes * P): union-find, then the root's global natural id
    uint8_t* up;     // per last-plane site: bond into the next plane activated
    DevCtl* ctl;
};

template <int MODEL>
__device__ __forceinline__ void slab_axis(const SlabWolffArgs& a, float* r, uint32_t* seed_nat)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    KeyedPcg g = KeyedPcg::open_key(a.seed, a.flip, kTagAxis, 0);
    if constexpr (MODEL == 0) r[0] = 1.0f;
    else sphere_sample<MODEL>(g, r);
    if (seed_nat) {
        // the seed in colour-major order (as the single-GPU flip draws it), as a natural id
        const uint32_t ks = uint32_t(u_f64(g.next()) * double(a.n));
        const uint32_t c = ks >= a.half ? 1u : 0u, rank = ks - c * a.half;
        uint32_t nat = 2 * rank;
        const uint32_t x = nat % a.Lx, rr = nat / a.Lx, y = rr % a.Ly, z = rr / a.Ly;
        if (((x + y + z) & 1u) != c) ++nat;
        *seed_nat = nat;
    }
    (void)N;
}

// Natural local index q (local plane * P + position) -> the storage index.
__device__ __forceinline__ uint32_t slab_store_index(const SlabWolffArgs& a, uint32_t q)
{
    if (!a.row_split) return q;
    const uint32_t lr = q / a.P, x = q - lr * a.P;
    return lr * a.P + ((x + a.first + lr - 1u) & 1u) * (a.P / 2) + x / 2;
}

template <int MODEL>
__device__ __forceinline__ void slab_load(const SlabWolffArgs& a, uint32_t q, float* s)
{
    if constexpr (MODEL == 0) s[0] = float(static_cast<const int8_t*>(a.field)[slab_store_index(a, q)]);
    else
#pragma unroll
        for (int c = 0; c < MODEL; ++c) s[c] = static_cast<const float*>(a.field)[c * a.nloc + q];
}

__global__ void slab_wolff_init(uint32_t* lab, uint32_t n_owned)
{
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < n_owned; o += gridDim.x * blockDim.x) lab[o] = o;
}

template <int MODEL>
__global__ void __launch_bounds__(kBlock) slab_wolff_bonds(SlabWolffArgs a)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    __shared__ float r_sh[4];
    if (threadIdx.x == 0) {
        float r[N];
        slab_axis<MODEL>(a, r, nullptr);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
    }
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint64_t kb = key_base(key_seed(a.seed, a.flip, kTagBond));
    const uint32_t n_owned = a.planes * a.P;
    const uint32_t ndir = 1u + (a.Ly > 1 ? 1u : 0u) + (a.Lz > 1 ? 1u : 0u);
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < n_owned; o += gridDim.x * blockDim.x) {
        const uint32_t lp = o / a.P, pos = o - lp * a.P;  // owned plane (0 = the first), position in it
        const uint32_t q = o + a.P;                        // local index (plane lp + 1)
        const uint32_t x = pos % a.Lx;
        const uint32_t gplane = a.first + lp;
        const uint32_t nat = gplane * a.P + pos;
        float si[N];
        slab_load<MODEL>(a, q, si);
        // neighbours in direction order x, y (3D only, in-plane), then the cut axis
        uint32_t nbq[3], nbo[3];
        bool cross[3];
        uint32_t nd = 0;
        {
            const uint32_t xj = x + 1 == a.Lx ? 0u : x + 1;
            const uint32_t pj = pos - x + xj;
            nbq[nd] = lp * a.P + pj + a.P;
            nbo[nd] = lp * a.P + pj;
            cross[nd++] = false;
        }
        if (a.along_z && a.Ly > 1) {
            const uint32_t y = pos / a.Lx;
            const uint32_t yj = y + 1 == a.Ly ? 0u : y + 1;
            const uint32_t pj = yj * a.Lx + x;
            nbq[nd] = lp * a.P + pj + a.P;
            nbo[nd] = lp * a.P + pj;
            cross[nd++] = false;
        }
        if (a.along_z ? a.Lz > 1 : a.Ly > 1) {
            nbq[nd] = q + a.P;  // the next plane: owned, or the halo after the last one
            nbo[nd] = o + a.P;
            cross[nd++] = lp + 1 == a.planes;
        }
        for (uint32_t d = 0; d < nd; ++d) {
            float sj[N];
            slab_load<MODEL>(a, nbq[d], sj);
            const uint32_t k = first_draw(kb, nat * ndir + d);
            bool on;
            if constexpr (MODEL == 0) on = ising_bond_active(a.cw, int(si[0]), int(sj[0]), k);
            else on = vector_bond_active<N>(a.J, a.beta, a.J64, a.beta64, a.err, si, sj, r, k);
            if (cross[d]) a.up[pos] = on ? 1 : 0;
            else if (on) uf_union(a.lab, o, nbo[d], n_owned + 1, &a.ctl->status);
        }
    }
}

// every owned site's label becomes its root's global natural id
__global__ void __launch_bounds__(kBlock) slab_wolff_roots(SlabWolffArgs a, uint32_t* glab)
{
    const uint32_t n_owned = a.planes * a.P;
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < n_owned; o += gridDim.x * blockDim.x) {
        const uint32_t root = uf_find(a.lab, o, n_owned + 1, &a.ctl->status);
        glab[o] = (a.first + root / a.P) * a.P + root % a.P;
    }
}

template <int MODEL>
__global__ void slab_wolff_seed(SlabWolffArgs a, uint32_t* seed_nat)
{
    float r[MODEL == 0 ? 1 : MODEL];
    slab_axis<MODEL>(a, r, seed_nat);
}

// slot[0] = the seed's natural id, slot[1] = its root where this slab owns
// it (else 0xFFFFFFFF): read back with the boundary, in the same copy batch.
template <int MODEL>
__global__ void slab_wolff_seed_root(SlabWolffArgs a, const uint32_t* glab, uint32_t* slot)
{
    float r[MODEL == 0 ? 1 : MODEL];
    uint32_t nat = 0;
    slab_axis<MODEL>(a, r, &nat);
    const uint32_t plane = nat / a.P;
    slot[0] = nat;
    slot[1] = plane >= a.first && plane - a.first < a.planes ? glab[nat - a.first * a.P] : 0xFFFFFFFFu;
}

// mark[root - first * P] = 1 for the roots to flip
__global__ void slab_wolff_mark(const uint32_t* roots, uint32_t n_roots, uint32_t base, uint8_t* mark)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_roots; i += gridDim.x * blockDim.x)
        mark[roots[i] - base] = 1;
}

template <int MODEL>
__global__ void __launch_bounds__(kBlock) slab_wolff_flip(SlabWolffArgs a, const uint32_t* glab, const uint8_t* mark,
                                                         unsigned long long* flipped)
{
    constexpr int N = MODEL == 0 ? 1 : MODEL;
    __shared__ float r_sh[4];
    if (threadIdx.x == 0) {
        float r[N];
        slab_axis<MODEL>(a, r, nullptr);
        for (int c = 0; c < N; ++c) r_sh[c] = r[c];
    }
    __syncthreads();
    float r[N];
#pragma unroll
    for (int c = 0; c < N; ++c) r[c] = r_sh[c];
    const uint32_t n_owned = a.planes * a.P, base = a.first * a.P;
    double cnt[1] = {0.0};
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < n_owned; o += gridDim.x * blockDim.x) {
        if (!mark[glab[o] - base]) continue;
        cnt[0] += 1.0;
        const uint32_t q = o + a.P;
        if constexpr (MODEL == 0) {
            int8_t* s = static_cast<int8_t*>(a.field);
            const uint32_t qi = slab_store_index(a, q);
            s[qi] = int8_t(-s[qi]);
        } else {
            float* f = static_cast<float*>(a.field);
            float si[N];
#pragma unroll
            for (int c = 0; c < N; ++c) si[c] = f[c * a.nloc + q];
            reflect<N>(si, r);
#pragma unroll
            for (int c = 0; c < N; ++c) f[c * a.nloc + q] = si[c];
        }
    }
    block_sum<1>(cnt);
    if (threadIdx.x == 0 && cnt[0] > 0.0) atomicAdd(flipped, (unsigned long long)cnt[0]);
}

}  // namespace
}  // namespace umc

using namespace umc;

struct umc_slab
{
    umc_slab_desc desc{};
    uint32_t P = 0, nloc = 0, half = 0, along_z = 0, deg = 0;
    int device = 0;
    uint32_t grid = 0;
    DevBuf ctl, partials, record, tm1;
    DevBuf w_lab, w_glab, w_up, w_mark, w_roots, w_slot;  // Wolff work buffers (first Wolff call)
    uint32_t row_split = 0;  // 2D Ising, Lx / 2 a multiple of 16: rows split by colour
    uint32_t seed_host[2] = {0, 0};  // seed site and its root of flip seed_flip, read with the boundary
    uint64_t seed_flip = 0;
    bool seed_valid = false;
    uint32_t row_grid = 0;
    std::vector<uint32_t> h_tm1;
    double tm1_beta = std::nan("");
    int32_t J_int = 0;
};

namespace {

template <class F>
int slab_guard(F&& f)
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

template <int N>
void launch_vector(const umc_slab* s, const SlabArgs& a, cudaStream_t st)
{
    if (s->desc.proposal == UMC_PROPOSAL_ROTATION) slab_vector_pass<N, kPropRotation><<<s->grid, kBlock, 0, st>>>(a);
    else slab_vector_pass<N, kPropSphere><<<s->grid, kBlock, 0, st>>>(a);
}

SlabWolffArgs wolff_args(umc_slab* s, void* field, double beta, uint64_t flip)
{
    const umc_slab_desc& d = s->desc;
    SlabWolffArgs a{};
    a.field = field;
    a.Lx = d.Lx;
    a.Ly = d.Ly;
    a.Lz = d.Lz;
    a.along_z = s->along_z;
    a.first = d.first_plane;
    a.planes = d.planes;
    a.P = s->P;
    a.nloc = s->nloc;
    a.n = uint32_t(uint64_t(d.Lx) * d.Ly * d.Lz);
    a.half = s->half;
    a.seed = d.seed;
    a.flip = flip;
    a.J = float(d.coupling);
    a.beta = float(beta);
    a.J64 = d.coupling;
    a.beta64 = beta;
    a.err = vector_wolff_err(beta, d.coupling, d.components);
    if (d.model == UMC_MODEL_ISING) ising_wolff_thresholds(s->J_int, beta, a.cw);
    const size_t n_owned = size_t(d.planes) * s->P;
    if (!s->w_lab.p) {
        s->w_lab.alloc(n_owned * 4, "slab Wolff labels");
        s->w_glab.alloc(n_owned * 4, "slab Wolff roots");
        s->w_up.alloc(s->P, "slab Wolff boundary bonds");
        s->w_mark.alloc(n_owned, "slab Wolff marks");
        s->w_roots.alloc((2 * size_t(s->P) + 1) * 4, "slab Wolff flip roots");
        s->w_slot.alloc(16, "slab Wolff slots");
    }
    a.row_split = s->row_split;
    a.lab = s->w_lab.as<uint32_t>();
    a.up = s->w_up.as<uint8_t>();
    a.ctl = s->ctl.as<DevCtl>();
    return a;
}

template <class F>
void by_model(const umc_slab* s, F&& f)
{
    if (s->desc.model == UMC_MODEL_ISING) return f(std::integral_constant<int, 0>{});
    switch (s->desc.components) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    default: return f(std::integral_constant<int, 4>{});
    }
}

}  // namespace

extern "C" {

int umc_slab_create(const umc_slab_desc* d, umc_slab** out)
{
    return slab_guard([&] {
        if (!d || !out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        const uint64_t Lx = d->Lx, Ly = d->Ly, Lz = d->Lz;
        if (Lx < 2 || Lx % 2 || Ly < 2 || Ly % 2 || (Lz != 1 && Lz % 2))
            throw Error(UMC_ERR_INVALID_ARGUMENT, "slabs need Lx and Ly even and at least 2, Lz 1 or even");
        if (Lx * Ly * Lz > 0xFFFFFFFFull) throw Error(UMC_ERR_OVERFLOW, "lattice exceeds uint32 sites");
        const uint64_t planes_total = Lz > 1 ? Lz : Ly;
        if (d->planes == 0 || uint64_t(d->first_plane) + d->planes > planes_total)
            throw Error(UMC_ERR_OUT_OF_RANGE, "slab planes outside the lattice");
        if (d->model == UMC_MODEL_ISING) {
            if (d->coupling != std::floor(d->coupling) || std::fabs(d->coupling) > 1e6)
                throw Error(UMC_ERR_INVALID_ARGUMENT, "Ising coupling J must be an integer");
            if (d->proposal != UMC_PROPOSAL_FLIP) throw Error(UMC_ERR_UNSUPPORTED, "Ising slabs use the Flip proposal");
        } else if (d->model == UMC_MODEL_VECTOR) {
            if (d->components < 1 || d->components > 4) throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin<N>: N must be 1..4");
            if (d->proposal != UMC_PROPOSAL_SPHERE && d->proposal != UMC_PROPOSAL_ROTATION)
                throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin slabs use UniformSphereN or LocalRotation");
        } else {
            throw Error(UMC_ERR_UNSUPPORTED, "slabs are provided for Ising and VectorSpin on square and cubic lattices");
        }
        auto s = std::make_unique<umc_slab>();
        s->desc = *d;
        s->along_z = Lz > 1 ? 1u : 0u;
        s->P = uint32_t(s->along_z ? Lx * Ly : Lx);
        const uint64_t nloc = (uint64_t(d->planes) + 2) * s->P;
        if (nloc > 0xFFFFFFFFull / 4) throw Error(UMC_ERR_OVERFLOW, "slab too large");
        s->nloc = uint32_t(nloc);
        s->half = uint32_t(Lx * Ly * Lz / 2);
        s->deg = 2 + (Ly > 1 ? 2 : 0) + (Lz > 1 ? 2 : 0);
        s->device = d->device;
        s->J_int = int32_t(d->coupling);
        cuda_check(cudaSetDevice(d->device), "cudaSetDevice");
        int sms = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d->device), "SM count");
        const uint64_t work = (uint64_t(d->planes) * s->P / 2 + kBlock - 1) / kBlock;
        s->grid = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(work, uint64_t(sms) * 8)));
        s->row_split = d->model == UMC_MODEL_ISING && !s->along_z && (Lx / 2) % 16 == 0 ? 1u : 0u;
        const uint64_t row_work = (uint64_t(d->planes) * (Lx / 2) / 16 + kBlock - 1) / kBlock;
        s->row_grid = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(row_work, s->grid)));
        s->ctl.alloc(sizeof(DevCtl), "slab control");
        cuda_check(cudaMemset(s->ctl.p, 0, sizeof(DevCtl)), "slab control");
        s->partials.alloc(size_t(s->grid) * kObs * sizeof(double), "slab partials");
        s->record.alloc(kObs * sizeof(double), "slab record");
        cuda_check(cudaMemset(s->record.p, 0, kObs * sizeof(double)), "slab record");
        *out = s.release();
    });
}

int umc_slab_destroy(umc_slab* s)
{
    return slab_guard([&] { delete s; });
}

uint64_t umc_slab_local_sites(const umc_slab* s) { return s ? s->nloc : 0; }

uint32_t umc_slab_row_split(const umc_slab* s) { return s ? s->row_split : 0u; }

int umc_slab_pass(umc_slab* s, void* field, double beta, uint64_t sweep, uint32_t colour, void* stream)
{
    return slab_guard([&] {
        NvtxRange range("umc_slab_pass");
        if (!s || !field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (colour > 1) throw Error(UMC_ERR_INVALID_ARGUMENT, "colour is 0 or 1");
        if (!std::isfinite(beta)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta must be finite");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const umc_slab_desc& d = s->desc;
        SlabArgs a{};
        a.field = field;
        a.Lx = d.Lx;
        a.Ly = d.Ly;
        a.Lz = d.Lz;
        a.along_z = s->along_z;
        a.first = d.first_plane;
        a.planes = d.planes;
        a.P = s->P;
        a.nloc = s->nloc;
        a.half = s->half;
        a.colour = colour;
        a.kbase = key_base(key_seed(d.seed, sweep, tag_site(0)));
        a.J = float(d.coupling);
        a.beta = float(beta);
        a.delta = float(d.width);
        a.J64 = d.coupling;
        a.beta64 = beta;
        a.out = PassOut{s->ctl.as<DevCtl>(), s->partials.as<double>(), s->record.as<double>(), nullptr, int(colour),
                        2, colour == 1 ? 1 : 0};
        if (d.model == UMC_MODEL_ISING) {
            if (!(s->tm1_beta == beta)) {
                s->h_tm1 = ising_metropolis_thresholds(s->J_int, beta, s->deg);
                if (!s->tm1.p) s->tm1.alloc(s->h_tm1.size() * 4, "slab thresholds");
                cuda_check(cudaMemcpyAsync(s->tm1.p, s->h_tm1.data(), s->h_tm1.size() * 4, cudaMemcpyHostToDevice, st),
                           "slab thresholds");
                cuda_check(cudaStreamSynchronize(st), "slab thresholds");
                s->tm1_beta = beta;
            }
            a.tm1 = s->tm1.as<uint32_t>();
            a.D = int32_t(s->deg);
            a.Jint = s->J_int;
            if (s->row_split) slab_ising_row_pass<<<s->row_grid, kBlock, 0, st>>>(a);
            else slab_ising_pass<<<s->grid, kBlock, 0, st>>>(a);
        } else {
            a.err = vector_metropolis_err(beta, d.coupling, d.components, s->deg);
            switch (d.components) {
            case 1: launch_vector<1>(s, a, st); break;
            case 2: launch_vector<2>(s, a, st); break;
            case 3: launch_vector<3>(s, a, st); break;
            default: launch_vector<4>(s, a, st); break;
            }
        }
        cuda_check(cudaGetLastError(), "slab pass");
    });
}

int umc_slab_record(umc_slab* s, double* out, void* stream)
{
    return slab_guard([&] {
        if (!s || !out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        cuda_check(cudaMemcpyAsync(out, s->record.p, kObs * sizeof(double), cudaMemcpyDeviceToHost, st), "slab record");
        cuda_check(cudaStreamSynchronize(st), "slab record");
        unsigned status = 0;
        cuda_check(cudaMemcpy(&status, &s->ctl.as<DevCtl>()->status, sizeof status, cudaMemcpyDeviceToHost),
                   "slab status");
        if (status) throw Error(UMC_ERR_DEVICE_TIMEOUT, "slab pass reported a device error");
    });
}

int umc_slab_wolff_local(umc_slab* s, void* field, double beta, uint64_t flip, void* stream)
{
    return slab_guard([&] {
        NvtxRange range("umc_slab_wolff_local");
        if (!s || !field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!std::isfinite(beta)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta must be finite");
        if (s->desc.model == UMC_MODEL_VECTOR && s->desc.components > 4)
            throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin<N>: N must be 1..4");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        SlabWolffArgs a = wolff_args(s, field, beta, flip);
        const uint32_t n_owned = s->desc.planes * s->P;
        slab_wolff_init<<<s->grid, kBlock, 0, st>>>(a.lab, n_owned);
        by_model(s, [&](auto m) { slab_wolff_bonds<decltype(m)::value><<<s->grid, kBlock, 0, st>>>(a); });
        slab_wolff_roots<<<s->grid, kBlock, 0, st>>>(a, s->w_glab.as<uint32_t>());
        by_model(s, [&](auto m) {
            slab_wolff_seed_root<decltype(m)::value><<<1, 1, 0, st>>>(a, s->w_glab.as<uint32_t>(), s->w_slot.as<uint32_t>());
        });
        cuda_check(cudaGetLastError(), "slab Wolff labels");
        s->seed_flip = flip;
        s->seed_valid = false;
    });
}

int umc_slab_wolff_boundary(umc_slab* s, uint32_t* first_roots, uint32_t* last_roots, uint8_t* last_up,
                            void* stream)
{
    return slab_guard([&] {
        if (!s || !first_roots || !last_roots || !last_up) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!s->w_glab.p) throw Error(UMC_ERR_STATE, "umc_slab_wolff_local has not run");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const uint32_t* g = s->w_glab.as<uint32_t>();
        const size_t P = s->P;
        cuda_check(cudaMemcpyAsync(first_roots, g, P * 4, cudaMemcpyDeviceToHost, st), "slab Wolff boundary");
        cuda_check(cudaMemcpyAsync(last_roots, g + size_t(s->desc.planes - 1) * P, P * 4, cudaMemcpyDeviceToHost, st),
                   "slab Wolff boundary");
        cuda_check(cudaMemcpyAsync(last_up, s->w_up.p, P, cudaMemcpyDeviceToHost, st), "slab Wolff boundary");
        // the seed and its root (umc_slab_wolff_local computed them) and the
        // status word ride in the same batch of copies: one synchronisation
        unsigned status = 0;
        cuda_check(cudaMemcpyAsync(s->seed_host, s->w_slot.p, 8, cudaMemcpyDeviceToHost, st), "slab Wolff seed");
        cuda_check(cudaMemcpyAsync(&status, &s->ctl.as<DevCtl>()->status, sizeof status, cudaMemcpyDeviceToHost, st),
                   "slab status");
        cuda_check(cudaStreamSynchronize(st), "slab Wolff boundary");
        if (status) throw Error(UMC_ERR_DEVICE_TIMEOUT, "slab Wolff labelling reported a device error");
        s->seed_valid = true;
    });
}

int umc_slab_wolff_seed(umc_slab* s, uint64_t flip, uint32_t* seed_nat, uint32_t* seed_root, void* stream)
{
    return slab_guard([&] {
        if (!s || !seed_nat || !seed_root) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (s->seed_valid && s->seed_flip == flip) {  // read back with the boundary
            *seed_nat = s->seed_host[0];
            *seed_root = s->seed_host[1];
            return;
        }
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        SlabWolffArgs a = wolff_args(s, nullptr, 1.0, flip);
        uint32_t* slot = s->w_slot.as<uint32_t>();
        by_model(s, [&](auto m) { slab_wolff_seed<decltype(m)::value><<<1, 1, 0, st>>>(a, slot); });
        cuda_check(cudaGetLastError(), "slab Wolff seed");
        cuda_check(cudaMemcpyAsync(seed_nat, slot, 4, cudaMemcpyDeviceToHost, st), "slab Wolff seed");
        cuda_check(cudaStreamSynchronize(st), "slab Wolff seed");
        *seed_root = 0xFFFFFFFFu;
        const uint64_t plane = *seed_nat / s->P;
        if (plane >= s->desc.first_plane && plane < uint64_t(s->desc.first_plane) + s->desc.planes) {
            if (!s->w_glab.p) throw Error(UMC_ERR_STATE, "umc_slab_wolff_local has not run");
            const size_t o = *seed_nat - size_t(s->desc.first_plane) * s->P;
            cuda_check(cudaMemcpy(seed_root, s->w_glab.as<uint32_t>() + o, 4, cudaMemcpyDeviceToHost), "slab Wolff seed");
        }
    });
}

int umc_slab_wolff_merge(uint32_t world, uint32_t plane_sites, const uint32_t* first_roots, const uint32_t* last_roots,
                         const uint8_t* last_up, uint32_t seed_root, uint32_t rank, const uint32_t* rank_roots_first,
                         const uint32_t* rank_roots_last, uint32_t rank_seed_root, uint32_t* roots, uint32_t* n_roots)
{
    return slab_guard([&] {
        if (!first_roots || !last_roots || !last_up || !rank_roots_first || !rank_roots_last || !roots || !n_roots)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (world == 0 || rank >= world) throw Error(UMC_ERR_INVALID_ARGUMENT, "rank outside the world");
        const size_t P = plane_sites;
        // union-find over the boundary labels (global natural ids of local roots)
        std::unordered_map<uint32_t, uint32_t> parent;
        auto find = [&](uint32_t x) {
            auto it = parent.find(x);
            while (it != parent.end() && it->second != x) {
                const uint32_t p = it->second;
                auto pit = parent.find(p);
                if (pit != parent.end() && pit->second != p) it->second = pit->second;  // path halving
                x = it->second;
                it = parent.find(x);
            }
            return x;
        };
        auto unite = [&](uint32_t a, uint32_t b) {
            parent.emplace(a, a);
            parent.emplace(b, b);
            a = find(a);
            b = find(b);
            if (a == b) return;
            if (a > b) std::swap(a, b);
            parent[b] = a;  // the smaller id is the root: the same on every rank
        };
        for (uint32_t r = 0; r < world; ++r) {
            const uint32_t nx = (r + 1) % world;
            for (size_t q = 0; q < P; ++q)
                if (last_up[r * P + q]) unite(last_roots[r * P + q], first_roots[nx * P + q]);
        }
        const uint32_t g = find(seed_root);
        std::vector<uint32_t> out;
        auto take = [&](uint32_t L) {
            if (find(L) == g) out.push_back(L);
        };
        for (size_t q = 0; q < P; ++q) {
            take(rank_roots_first[q]);
            take(rank_roots_last[q]);
        }
        if (rank_seed_root != 0xFFFFFFFFu) take(rank_seed_root);
        std::sort(out.begin(), out.end());
        out.erase(std::unique(out.begin(), out.end()), out.end());
        std::copy(out.begin(), out.end(), roots);
        *n_roots = uint32_t(out.size());
    });
}

int umc_slab_wolff_flip(umc_slab* s, void* field, uint64_t flip, const uint32_t* roots, uint32_t n_roots,
                        uint64_t* flipped, void* stream)
{
    return slab_guard([&] {
        NvtxRange range("umc_slab_wolff_flip");
        if (!s || !field || !flipped || (n_roots && !roots)) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!s->w_glab.p) throw Error(UMC_ERR_STATE, "umc_slab_wolff_local has not run");
        if (n_roots > 2 * s->P + 1) throw Error(UMC_ERR_INVALID_ARGUMENT, "more roots than the boundary holds");
        const uint32_t base = s->desc.first_plane * s->P, n_owned = s->desc.planes * s->P;
        for (uint32_t i = 0; i < n_roots; ++i)
            if (roots[i] < base || roots[i] - base >= n_owned) throw Error(UMC_ERR_OUT_OF_RANGE, "root outside the slab");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        SlabWolffArgs a = wolff_args(s, field, 1.0, flip);
        cuda_check(cudaMemsetAsync(s->w_mark.p, 0, n_owned, st), "slab Wolff marks");
        unsigned long long* count = reinterpret_cast<unsigned long long*>(s->w_slot.as<uint8_t>() + 8);
        cuda_check(cudaMemsetAsync(count, 0, 8, st), "slab Wolff count");
        if (n_roots) {
            cuda_check(cudaMemcpyAsync(s->w_roots.p, roots, size_t(n_roots) * 4, cudaMemcpyHostToDevice, st),
                       "slab Wolff roots");
            slab_wolff_mark<<<1, kBlock, 0, st>>>(s->w_roots.as<uint32_t>(), n_roots, base, s->w_mark.as<uint8_t>());
            by_model(s, [&](auto m) {
                slab_wolff_flip<decltype(m)::value><<<s->grid, kBlock, 0, st>>>(a, s->w_glab.as<uint32_t>(),
                                                                                  s->w_mark.as<uint8_t>(), count);
            });
        }
        cuda_check(cudaGetLastError(), "slab Wolff flip");
        unsigned long long c = 0;
        cuda_check(cudaMemcpyAsync(&c, count, 8, cudaMemcpyDeviceToHost, st), "slab Wolff count");
        cuda_check(cudaStreamSynchronize(st), "slab Wolff count");
        *flipped = c;
    });
}

}  // extern "C"
