// umc_gauge_kernels.cuh -- colour-pass Metropolis for U(1) and SU(N) links on a
// cell complex of plaquettes (arity 4, orientation U0 U1 U2^dag U3^dag).
//
// The reference recomputes every incident plaquette before and after the
// proposal (example/u1_gauge.hpp:35-52, example/sun_gauge.hpp:36-51).  Since
// the plaquette is linear in the link, here each incidence (cell, which)
// contributes a staple B so that ReTr(U_p) = ReTr(U B) (U(1): cos(theta + phi));
// the staple sum A is built once per link and reused by all hits:
//     dE = (beta / N) ReTr((U - U') A)            (SU(N))
//     dE = beta Re((e^{i theta} - e^{i theta'}) S) (U(1)).
// Every other occurrence of the link inside a cell keeps its old value, exactly
// as the reference's delta does (term/plaquette.hpp:34-47).
//
// Link storage: colour-major; U(1) one FP32 angle per link; SU(N) 2N^2 FP32
// components per link, component q of link k at f[q * n + k] (row-major,
// interleaved re/im), so a warp's loads of one component are contiguous.
#pragma once

#include "umc_device.cuh"
#include "umc_spin_kernels.cuh"

namespace umc {

// ------------------------------------------------------- complex N x N algebra
template <int N>
struct Mat
{
    float re[N * N];
    float im[N * N];
};

template <int N>
__device__ __forceinline__ void mat_load(Mat<N>& m, const float* f, uint32_t n, uint32_t k)
{
#pragma unroll
    for (int q = 0; q < N * N; ++q) {
        m.re[q] = f[(2 * q) * n + k];
        m.im[q] = f[(2 * q + 1) * n + k];
    }
}

template <int N>
__device__ __forceinline__ void mat_store(const Mat<N>& m, float* f, uint32_t n, uint32_t k)
{
#pragma unroll
    for (int q = 0; q < N * N; ++q) {
        f[(2 * q) * n + k] = m.re[q];
        f[(2 * q + 1) * n + k] = m.im[q];
    }
}

// r = op(a) op(b), op = identity or dagger (conjugate transpose)
template <int N, bool DA, bool DB>
__device__ __forceinline__ void mat_mul(const Mat<N>& a, const Mat<N>& b, Mat<N>& r)
{
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = 0; j < N; ++j) {
            float sr = 0.f, si = 0.f;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const int ia = DA ? k * N + i : i * N + k;
                const int ib = DB ? j * N + k : k * N + j;
                const float ar = a.re[ia], ai = DA ? -a.im[ia] : a.im[ia];
                const float br = b.re[ib], bi = DB ? -b.im[ib] : b.im[ib];
                sr = fmaf(ar, br, fmaf(-ai, bi, sr));
                si = fmaf(ar, bi, fmaf(ai, br, si));
            }
            r.re[i * N + j] = sr;
            r.im[i * N + j] = si;
        }
}

template <int N>
__device__ __forceinline__ void mat_add(Mat<N>& a, const Mat<N>& b)
{
#pragma unroll
    for (int q = 0; q < N * N; ++q) {
        a.re[q] += b.re[q];
        a.im[q] += b.im[q];
    }
}

template <int N>
__device__ __forceinline__ void mat_zero(Mat<N>& a)
{
#pragma unroll
    for (int q = 0; q < N * N; ++q) a.re[q] = a.im[q] = 0.f;
}

template <int N>
__device__ __forceinline__ void mat_identity(Mat<N>& a)
{
    mat_zero(a);
#pragma unroll
    for (int i = 0; i < N; ++i) a.re[i * N + i] = 1.f;
}

// Re Tr(a b)
template <int N>
__device__ __forceinline__ float re_tr_mul(const Mat<N>& a, const Mat<N>& b)
{
    float t = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int k = 0; k < N; ++k) t = fmaf(a.re[i * N + k], b.re[k * N + i], fmaf(-a.im[i * N + k], b.im[k * N + i], t));
    return t;
}

// sun_detail::norm (dof/sun.hpp:104-114): max row sum of |a_ij|
template <int N>
__device__ __forceinline__ float mat_norm(const Mat<N>& a)
{
    float n = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float row = 0.f;
#pragma unroll
        for (int j = 0; j < N; ++j) row += hypotf(a.re[i * N + j], a.im[i * N + j]);
        n = fmaxf(n, row);
    }
    return n;
}

// exp(A) for anti-Hermitian A by scaling and squaring plus a Taylor series,
// the method of sun_detail::expm (dof/sun.hpp:118-146) with an FP32 stopping
// threshold.
template <int N>
__device__ __forceinline__ void mat_expm(const Mat<N>& a, Mat<N>& result)
{
    float nrm = mat_norm<N>(a);
    int squarings = 0;
    while (nrm > 0.5f && squarings < 30) {
        nrm *= 0.5f;
        ++squarings;
    }
    const float scale = ldexpf(1.f, -squarings);
    Mat<N> b, term, tmp;
#pragma unroll
    for (int q = 0; q < N * N; ++q) {
        b.re[q] = a.re[q] * scale;
        b.im[q] = a.im[q] * scale;
    }
    mat_identity(result);
    mat_identity(term);
    for (int k = 1; k <= 30; ++k) {
        mat_mul<N, false, false>(term, b, tmp);
        const float inv = 1.f / float(k);
#pragma unroll
        for (int q = 0; q < N * N; ++q) {
            term.re[q] = tmp.re[q] * inv;
            term.im[q] = tmp.im[q] * inv;
        }
        mat_add(result, term);
        if (mat_norm<N>(term) < 1e-9f) break;
    }
    for (int k = 0; k < squarings; ++k) {
        mat_mul<N, false, false>(result, result, tmp);
        result = tmp;
    }
}

// exp(i X) for a traceless Hermitian X in closed form (the reference sums the
// Taylor series with scaling and squaring, dof/sun.hpp:118-146; both agree to
// FP32 rounding).  SU(2): X^2 = |q|^2 I, so exp(iX) = cos|q| I + i sin|q|/|q| X.
// SU(3): Cayley-Hamilton, exp(iX) = f0 I + f1 X + f2 X^2 with f_j from
// c0 = det X and c1 = tr X^2 / 2 (Morningstar & Peardon, Phys. Rev. D 69,
// 054501 (2004)), using f_j(-c0) = (-1)^j conj f_j(c0) so that the
// denominator 9u^2 - w^2 stays >= 2 c1.  Other N: the Taylor series.
template <int N>
__device__ __forceinline__ void su_exp_i(const Mat<N>& x, Mat<N>& e)
{
    if constexpr (N == 2) {
        const float q2 = x.re[0] * x.re[0] + x.re[1] * x.re[1] + x.im[1] * x.im[1];
        const float q = sqrtf(q2);
        float sn, cs;
        sincosf(q, &sn, &cs);
        const float sq = q > 1e-3f ? sn / q : 1.f - q2 * (1.f / 6.f);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            e.re[k] = (k == 0 || k == 3 ? cs : 0.f) - sq * x.im[k];
            e.im[k] = sq * x.re[k];
        }
    } else if constexpr (N == 3) {
        // X^2 of a Hermitian X is Hermitian: the diagonal is real and the
        // lower triangle is the conjugate of the upper one
        Mat<3> x2;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            float d = 0.f;
#pragma unroll
            for (int k = 0; k < 3; ++k) d = fmaf(x.re[i * 3 + k], x.re[i * 3 + k], fmaf(x.im[i * 3 + k], x.im[i * 3 + k], d));
            x2.re[i * 4] = d;
            x2.im[i * 4] = 0.f;
#pragma unroll
            for (int j = i + 1; j < 3; ++j) {
                // (X^2)_ij = sum_k x_ik conj(x_jk)
                float sr = 0.f, si = 0.f;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float ar = x.re[i * 3 + k], ai = x.im[i * 3 + k];
                    const float br = x.re[j * 3 + k], bi = x.im[j * 3 + k];
                    sr = fmaf(ar, br, fmaf(ai, bi, sr));
                    si = fmaf(ai, br, fmaf(-ar, bi, si));
                }
                x2.re[i * 3 + j] = sr;
                x2.im[i * 3 + j] = si;
                x2.re[j * 3 + i] = sr;
                x2.im[j * 3 + i] = -si;
            }
        }
        const float c1 = 0.5f * (x2.re[0] + x2.re[4] + x2.re[8]);
        // tr(X X^2) = 3 det X; both Hermitian, so the sum over i != j is twice
        // the real part over i < j
        float off = 0.f, tr3 = 0.f;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            tr3 = fmaf(x.re[i * 4], x2.re[i * 4], tr3);
#pragma unroll
            for (int j = i + 1; j < 3; ++j)
                off = fmaf(x.re[i * 3 + j], x2.re[i * 3 + j], fmaf(x.im[i * 3 + j], x2.im[i * 3 + j], off));
        }
        tr3 = fmaf(2.f, off, tr3);
        const float c0 = tr3 * (1.f / 3.f);
        float f0r, f0i, f1r, f1i, f2r, f2i;
        if (c1 <= 0.75f) {
            // |eigenvalues| <= sqrt(4 c1 / 3) <= 1: sum the series exp(iX) =
            // sum_k i^k X^k / k! with X^k = a_k I + b_k X + d_k X^2, reduced by
            // X^3 = c1 X + c0 I (Cayley-Hamilton): a' = c0 d, b' = a + c1 d,
            // d' = b.  Twelve terms leave < 1/13! = 1.6e-10; no transcendentals.
            constexpr double kInvFact[13] = {1.0, 1.0, 1.0 / 2, 1.0 / 6, 1.0 / 24, 1.0 / 120, 1.0 / 720, 1.0 / 5040,
                                             1.0 / 40320, 1.0 / 362880, 1.0 / 3628800, 1.0 / 39916800,
                                             1.0 / 479001600};
            float a = 1.f, b = 0.f, d = 0.f;
            f0r = 1.f;
            f0i = f1r = f1i = f2r = f2i = 0.f;
#pragma unroll
            for (int k = 1; k <= 12; ++k) {
                const float na = c0 * d, nb = fmaf(c1, d, a);
                d = b;
                a = na;
                b = nb;
                const float t = float(kInvFact[k]) * ((k & 2) ? -1.f : 1.f);  // i^k = +1, +i, -1, -i
                if (k & 1) {
                    f0i = fmaf(t, a, f0i);
                    f1i = fmaf(t, b, f1i);
                    f2i = fmaf(t, d, f2i);
                } else {
                    f0r = fmaf(t, a, f0r);
                    f1r = fmaf(t, b, f1r);
                    f2r = fmaf(t, d, f2r);
                }
            }
        } else {
            const bool neg = c0 < 0.f;
            // theta = acos(|c0| / c0_max), c0_max = 2 (c1 / 3)^(3/2)
            const float c13 = c1 * (1.f / 3.f);
            const float th = acosf(fminf(fabsf(c0) / (2.f * c13 * sqrtf(c13)), 1.f));
            float s3, c3;
            sincosf(th * (1.f / 3.f), &s3, &c3);
            const float u = sqrtf(c1 * (1.f / 3.f)) * c3, w = sqrtf(c1) * s3;
            const float w2 = w * w, u2 = u * u;
            float su, cu, sw, cw;
            sincosf(u, &su, &cu);
            sincosf(w, &sw, &cw);
            // sin 2u, cos 2u by the double-angle formulas
            const float s2u = 2.f * su * cu, c2u = fmaf(cu, cu, -su * su);
            const float xi = fabsf(w) < 0.05f ? 1.f - w2 * (1.f / 6.f) * (1.f - w2 * (1.f / 20.f) * (1.f - w2 * (1.f / 42.f)))
                                              : sw / w;
            // e^{-iu} = (cu, -su)
            auto emiu = [&](float ar, float ai, float& rr, float& ri) {  // e^{-iu} (ar + i ai)
                rr = cu * ar + su * ai;
                ri = cu * ai - su * ar;
            };
            float h0r, h0i, h1r, h1i, h2r, h2i, tr, ti;
            emiu(8.f * u2 * cw, 2.f * u * (3.f * u2 + w2) * xi, tr, ti);
            h0r = (u2 - w2) * c2u + tr;
            h0i = (u2 - w2) * s2u + ti;
            emiu(2.f * u * cw, -(3.f * u2 - w2) * xi, tr, ti);
            h1r = 2.f * u * c2u - tr;
            h1i = 2.f * u * s2u - ti;
            emiu(cw, 3.f * u * xi, tr, ti);
            h2r = c2u - tr;
            h2i = s2u - ti;
            const float id = 1.f / (9.f * u2 - w2);
            f0r = h0r * id;
            f0i = h0i * id;
            f1r = h1r * id;
            f1i = h1i * id;
            f2r = h2r * id;
            f2i = h2i * id;
            if (neg) {  // f_j(-c0) = (-1)^j conj f_j(c0)
                f0i = -f0i;
                f1r = -f1r;
                f2i = -f2i;
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            const float d = k % 4 == 0 ? 1.f : 0.f;
            e.re[k] = f0r * d + f1r * x.re[k] - f1i * x.im[k] + f2r * x2.re[k] - f2i * x2.im[k];
            e.im[k] = f0i * d + f1r * x.im[k] + f1i * x.re[k] + f2r * x2.im[k] + f2i * x2.re[k];
        }
    } else {
        Mat<N> a;
#pragma unroll
        for (int q = 0; q < N * N; ++q) {  // a = i x
            a.re[q] = -x.im[q];
            a.im[q] = x.re[q];
        }
        mat_expm<N>(a, e);
    }
}

// SUShift<N>::sample (dof/sun.hpp:163-204): traceless Hermitian X from N + N(N-1)
// keyed uniforms (diagonal first, then (a, b) per upper pair), U' = U exp(iX).
template <int N>
__device__ __forceinline__ void su_shift(KeyedPcg& g, float width, const Mat<N>& cur, Mat<N>& out)
{
    Mat<N> x;
    mat_zero(x);
    float tr = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const float d = width * sym_f32(g.next());
        x.re[i * N + i] = d;
        tr += d;
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int j = i + 1; j < N; ++j) {
            const float ar = width * sym_f32(g.next());
            const float br = width * sym_f32(g.next());
            x.re[i * N + j] = ar;
            x.im[i * N + j] = br;
            x.re[j * N + i] = ar;
            x.im[j * N + i] = -br;
        }
#pragma unroll
    for (int i = 0; i < N; ++i) x.re[i * N + i] -= tr / float(N);
    Mat<N> e;
    su_exp_i<N>(x, e);
    mat_mul<N, false, false>(cur, e, out);
}

// Projection back onto SU(N) after FP32 round-off: Gram-Schmidt on the rows;
// the last row of SU(3) is the conjugate cross product of the first two, the
// second row of SU(2) is (-conj(b), conj(a)).  Not in the reference, which
// keeps FP64 links and never reunitarises.
template <int N>
__device__ __forceinline__ void reunitarise(Mat<N>& u)
{
    float n0 = 0.f;
#pragma unroll
    for (int k = 0; k < N; ++k) n0 = fmaf(u.re[k], u.re[k], fmaf(u.im[k], u.im[k], n0));
    const float i0 = rsqrtf(n0);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        u.re[k] *= i0;
        u.im[k] *= i0;
    }
    if constexpr (N == 2) {
        u.re[2] = -u.re[1];
        u.im[2] = u.im[1];
        u.re[3] = u.re[0];
        u.im[3] = -u.im[0];
    } else if constexpr (N == 3) {
        // <r0, r1> = sum conj(r0_k) r1_k
        float pr = 0.f, pi = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            pr = fmaf(u.re[k], u.re[3 + k], fmaf(u.im[k], u.im[3 + k], pr));
            pi = fmaf(u.re[k], u.im[3 + k], fmaf(-u.im[k], u.re[3 + k], pi));
        }
        float n1 = 0.f;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u.re[3 + k] -= pr * u.re[k] - pi * u.im[k];
            u.im[3 + k] -= pr * u.im[k] + pi * u.re[k];
            n1 = fmaf(u.re[3 + k], u.re[3 + k], fmaf(u.im[3 + k], u.im[3 + k], n1));
        }
        const float i1 = rsqrtf(n1);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u.re[3 + k] *= i1;
            u.im[3 + k] *= i1;
        }
        // r2 = conj(r0 x r1)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int a = (k + 1) % 3, b = (k + 2) % 3;
            const float cr = (u.re[a] * u.re[3 + b] - u.im[a] * u.im[3 + b]) - (u.re[b] * u.re[3 + a] - u.im[b] * u.im[3 + a]);
            const float ci = (u.re[a] * u.im[3 + b] + u.im[a] * u.re[3 + b]) - (u.re[b] * u.im[3 + a] + u.im[b] * u.re[3 + a]);
            u.re[6 + k] = cr;
            u.im[6 + k] = -ci;
        }
    }
}

// ------------------------------------------------------------------ passes

// One colour class of links.  inc packs (cell << 2 | which); cells holds the
// four colour-major link ids of every cell.
struct GaugeArgs
{
    float* f;
    uint32_t n;  // links
    uint32_t first, count;
    const uint32_t* inc_off;
    const uint32_t* inc;
    const uint4* cells;
    uint64_t seed, sweep;
    uint32_t hits;
    float model_beta, driver_beta, width;
    PassOut out;
    double model_beta64, driver_beta64;  // the couplings of the FP64 decisions
    float err;                           // u1_metropolis_err / su_metropolis_err
    const uint32_t* gid;                 // key id of each link (null: its index), for a slab's local links
};

// Key base of hit h of this sweep (the same for every link): the first
// kHitKeys are computed once per block into shared memory.
constexpr uint32_t kHitKeys = 32;

__device__ __forceinline__ void hit_keys_init(uint64_t* keys, const GaugeArgs& a)
{
    for (uint32_t h = threadIdx.x; h < a.hits && h < kHitKeys; h += blockDim.x)
        keys[h] = key_base(key_seed(a.seed, a.sweep, tag_site(h)));
    __syncthreads();
}

__device__ __forceinline__ uint64_t hit_key(const uint64_t* keys, const GaugeArgs& a, uint32_t h)
{
    return h < kHitKeys ? keys[h] : key_base(key_seed(a.seed, a.sweep, tag_site(h)));
}

// model_beta sum over link k's cells of cos(theta_p) - cos(theta_p') for the
// link going from angle t to p, in FP64 on the FP32 angles; the plaquette angle
// theta0 + theta1 - theta2 - theta3 (dof/u1.hpp:18-21) is +-(theta_k + phi)
// with phi the sum of the cell's other three links.  Out of line and on plain
// pointers: it runs only for decisions the FP32 test cannot call.
static __device__ __noinline__ double u1_delta64(const float* f, const uint32_t* inc_off, const uint32_t* inc,
                                          const uint4* cells, uint32_t k, float t, float p, double model_beta)
{
    double d = 0.0;
    for (uint32_t e = inc_off[k]; e < inc_off[k + 1]; ++e) {
        const uint32_t w = inc[e];
        const uint4 c = cells[w >> 2];
        const double t0 = f[c.x], t1 = f[c.y], t2 = f[c.z], t3 = f[c.w];
        double phi;
        switch (w & 3u) {
        case 0: phi = t1 - t2 - t3; break;
        case 1: phi = t0 - t2 - t3; break;
        case 2: phi = t3 - t0 - t1; break;
        default: phi = t2 - t0 - t1; break;
        }
        d += model_beta * (cos(double(t) + phi) - cos(double(p) + phi));
    }
    return d;
}

// (kBlock, 5): at most 48 registers; the out-of-line FP64 decision spills
// inside itself instead of widening the kernel.
static __global__ void __launch_bounds__(kBlock, 5) u1_pass(GaugeArgs a)
{
    __shared__ uint64_t keys[kHitKeys];
    hit_keys_init(keys, a);
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < a.count; q += gridDim.x * blockDim.x) {
        const uint32_t k = a.first + q;
        const uint32_t kid = a.gid ? a.gid[k] : k;
        float Sr = 0.f, Si = 0.f;
        for (uint32_t e = a.inc_off[k]; e < a.inc_off[k + 1]; ++e) {
            const uint32_t w = a.inc[e];
            const uint4 c = a.cells[w >> 2];
            const float t0 = a.f[c.x], t1 = a.f[c.y], t2 = a.f[c.z], t3 = a.f[c.w];
            float phi;
            switch (w & 3u) {
            case 0: phi = t1 - t2 - t3; break;
            case 1: phi = t0 - t2 - t3; break;
            case 2: phi = t3 - t0 - t1; break;
            default: phi = t2 - t0 - t1; break;
            }
            float sn, cs;
            sincosf(phi, &sn, &cs);
            Sr += cs;
            Si += sn;
        }
        float th = a.f[k];
        float so, co;
        sincosf(th, &so, &co);
        uint32_t accepted = 0;
        for (uint32_t h = 0; h < a.hits; ++h) {
            KeyedPcg g = KeyedPcg::open(hit_key(keys, a, h), kid);
            const float p = u1_shift(g, a.width, th);
            float sp, cp;
            sincosf(p, &sp, &cp);
            // beta * sum_p (cos theta_p - cos theta_p')
            const float dE = a.model_beta * ((co - cp) * Sr - (so - sp) * Si);
            const bool ok = metropolis_accept(g, -a.driver_beta * dE, a.err, [&] {
                return -a.driver_beta64 * u1_delta64(a.f, a.inc_off, a.inc, a.cells, k, th, p, a.model_beta64);
            });
            if (ok) {
                th = p;
                co = cp;
                so = sp;
                ++accepted;
            }
        }
        if (accepted) a.f[k] = th;
        acc[7] += double(accepted);
    }
    finish_pass<kObs>(acc, a.out);
}

// The SU(N) accept test in FP32: u_f32(k) < __expf(log_p) (driver.hpp:39-40,
// monotone-equivalent to log u < log_p), the uniform drawn only when needed.
// Unlike the other passes there is no FP64 retake near the threshold: the
// FP32 ReTr(U A) of a staple of 2(d-1) products of three FP32 links is within
// about 1e-4 of its FP64 value in log_p at beta = 5.7, and the FP32 candidate
// U exp(iX) moves log_p by the same order against the FP64 reference's own
// candidate, so a retake (two FP64 staples per undecided hit) would cost
// much more than it brings: measured on a 24^4 lattice, 1.93 ms per 10-hit
// sweep against 0.82 ms.
__device__ __forceinline__ bool su_accept_f32(KeyedPcg& g, float log_p)
{
    if (log_p >= 0.0f) return true;
    return u_f32(g.next()) < __expf(log_p);
}

template <int N>
__global__ void __launch_bounds__(kBlock, 3) su_pass(GaugeArgs a)
{
    __shared__ uint64_t keys[kHitKeys];
    hit_keys_init(keys, a);
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < a.count; q += gridDim.x * blockDim.x) {
        const uint32_t k = a.first + q;
        const uint32_t kid = a.gid ? a.gid[k] : k;
        Mat<N> A, B, T, u0, u1;
        mat_zero(A);
        for (uint32_t e = a.inc_off[k]; e < a.inc_off[k + 1]; ++e) {
            const uint32_t w = a.inc[e];
            const uint4 c = a.cells[w >> 2];
            // ReTr(U0 U1 U2^dag U3^dag) = ReTr(U B) with U at position `which`
            switch (w & 3u) {
            case 0:  // B = U1 U2^dag U3^dag
                mat_load(u0, a.f, a.n, c.y);
                mat_load(u1, a.f, a.n, c.z);
                mat_mul<N, false, true>(u0, u1, T);
                mat_load(u0, a.f, a.n, c.w);
                mat_mul<N, false, true>(T, u0, B);
                break;
            case 1:  // B = U2^dag U3^dag U0
                mat_load(u0, a.f, a.n, c.z);
                mat_load(u1, a.f, a.n, c.w);
                mat_mul<N, true, true>(u0, u1, T);
                mat_load(u0, a.f, a.n, c.x);
                mat_mul<N, false, false>(T, u0, B);
                break;
            case 2:  // B = U1^dag U0^dag U3
                mat_load(u0, a.f, a.n, c.y);
                mat_load(u1, a.f, a.n, c.x);
                mat_mul<N, true, true>(u0, u1, T);
                mat_load(u0, a.f, a.n, c.w);
                mat_mul<N, false, false>(T, u0, B);
                break;
            default:  // B = U2 U1^dag U0^dag
                mat_load(u0, a.f, a.n, c.z);
                mat_load(u1, a.f, a.n, c.y);
                mat_mul<N, false, true>(u0, u1, T);
                mat_load(u0, a.f, a.n, c.x);
                mat_mul<N, false, true>(T, u0, B);
                break;
            }
            mat_add(A, B);
        }
        Mat<N> U, V;
        mat_load(U, a.f, a.n, k);
        float tr_old = re_tr_mul<N>(U, A);
        uint32_t accepted = 0;
        const float coef = a.model_beta / float(N);
        for (uint32_t h = 0; h < a.hits; ++h) {
            KeyedPcg g = KeyedPcg::open(hit_key(keys, a, h), kid);
            su_shift<N>(g, a.width, U, V);
            const float tr_new = re_tr_mul<N>(V, A);
            const float dE = coef * (tr_old - tr_new);
            // decided in FP32 (see su_accept_f32): an FP64 retake would not
            // bring the decision closer to the FP64 reference's, whose
            // candidate differs from this FP32 one by as much
            if (su_accept_f32(g, -a.driver_beta * dE)) {
                U = V;
                tr_old = tr_new;
                ++accepted;
            }
        }
        reunitarise<N>(U);
        mat_store(U, a.f, a.n, k);
        acc[7] += double(accepted);
    }
    finish_pass<kObs>(acc, a.out);
}

// ------------------------------------------------------------ observables
// Per cell: ReTr(U0 U1 U2^dag U3^dag)/N (dof/sun.hpp:78-84) or cos(theta_p)
// (dof/u1.hpp:18-21), reduced in FP64 into [S, <P>, Q].  Q (the 2D U(1)
// topological charge) sums remainder(theta_p, 2 pi) / 2 pi.
// n_cells cells summed; <P> normalised by n_norm (a slab sums its share of
// the lattice's cells).
template <int N>
__global__ void __launch_bounds__(kBlock) plaquette_sum(const float* f, uint32_t n, const uint4* cells,
                                                        uint32_t n_cells, uint64_t n_norm, float model_beta,
                                                        PassOut out)
{
    double acc[kObs] = {0, 0, 0, 0, 0, 0, 0, 0};
    const double inv_cells = 1.0 / double(n_norm);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_cells; c += gridDim.x * blockDim.x) {
        const uint4 q = cells[c];
        double P, theta_p = 0.0;
        if constexpr (N == 1) {
            const double t = double(f[q.x]) + double(f[q.y]) - double(f[q.z]) - double(f[q.w]);
            P = cos(t);
            theta_p = remainder(t, 6.283185307179586);
        } else {
            Mat<N> a, b, t1, t2;
            mat_load(a, f, n, q.x);
            mat_load(b, f, n, q.y);
            mat_mul<N, false, false>(a, b, t1);
            mat_load(a, f, n, q.z);
            mat_mul<N, false, true>(t1, a, t2);
            mat_load(a, f, n, q.w);
            // Re Tr(t2 a^dag) = sum_ij Re(t2_ij conj(a_ij))
            double tr = 0.0;
#pragma unroll
            for (int qq = 0; qq < N * N; ++qq) tr += double(t2.re[qq]) * a.re[qq] + double(t2.im[qq]) * a.im[qq];
            P = tr / N;
        }
        acc[0] += double(model_beta) * (1.0 - P);
        acc[1] += P * inv_cells;
        acc[2] += theta_p / 6.283185307179586;
    }
    finish_pass<kObs>(acc, out);
}

// ------------------------------------------------------- layout and starts

// host AoS (link-major, 2N^2 floats) <-> device colour-major SoA
static __global__ void gauge_scatter(const float* src, float* dst, uint32_t n, uint32_t comps, const uint32_t* position)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = position[i];
        for (uint32_t c = 0; c < comps; ++c) dst[uint64_t(c) * n + k] = src[uint64_t(i) * comps + c];
    }
}

static __global__ void gauge_gather(const float* src, float* dst, uint32_t n, uint32_t comps, const uint32_t* position)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = position[i];
        for (uint32_t c = 0; c < comps; ++c) dst[uint64_t(i) * comps + c] = src[uint64_t(c) * n + k];
    }
}

template <int N>
__global__ void gauge_identity(float* f, uint32_t n)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        Mat<N> u;
        mat_identity(u);
        mat_store(u, f, n, k);
    }
}

// Haar-random start (no reference counterpart; the reference's hot start applies
// SUShift repeatedly, test/su_check.cpp:51-60).  Link i (original index) draws
// 2N^2 normals from key (seed, 0, tag 3, i) by Box-Muller, orthonormalises the
// columns (Gram-Schmidt, i.e. QR with a positive diagonal: Haar on U(N),
// Mezzadri 2007) and divides by a root of the determinant to land in SU(N).
// U(1): theta = 2 pi u.
template <int N>
__global__ void gauge_haar(float* f, uint32_t n, uint64_t seed, const uint32_t* position)
{
    const uint64_t kb = key_base(key_seed(seed, 0, kTagInit));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = position[i];
        KeyedPcg g = KeyedPcg::open(kb, i);
        if constexpr (N == 1) {
            f[k] = twice_u_f32(g.next()) * 3.14159265358979f;
        } else {
            Mat<N> z;
#pragma unroll
            for (int q = 0; q < N * N; ++q) {
                // Box-Muller: u1 in (0, 1], u2 in [0, 1)
                const float u1 = (float(g.next()) + 1.0f) * 0x1.0p-32f;
                const float u2 = twice_u_f32(g.next());
                const float r = sqrtf(-2.f * logf(u1));
                float sn, cs;
                sincospif(u2, &sn, &cs);
                z.re[q] = r * cs * 0.70710678f;
                z.im[q] = r * sn * 0.70710678f;
            }
            // Gram-Schmidt on columns
#pragma unroll
            for (int j = 0; j < N; ++j) {
#pragma unroll
                for (int p = 0; p < j; ++p) {
                    float pr = 0.f, pi = 0.f;  // <col_p, col_j>
#pragma unroll
                    for (int r = 0; r < N; ++r) {
                        pr += z.re[r * N + p] * z.re[r * N + j] + z.im[r * N + p] * z.im[r * N + j];
                        pi += z.re[r * N + p] * z.im[r * N + j] - z.im[r * N + p] * z.re[r * N + j];
                    }
#pragma unroll
                    for (int r = 0; r < N; ++r) {
                        z.re[r * N + j] -= pr * z.re[r * N + p] - pi * z.im[r * N + p];
                        z.im[r * N + j] -= pr * z.im[r * N + p] + pi * z.re[r * N + p];
                    }
                }
                float nn = 0.f;
#pragma unroll
                for (int r = 0; r < N; ++r) nn += z.re[r * N + j] * z.re[r * N + j] + z.im[r * N + j] * z.im[r * N + j];
                const float inv = rsqrtf(nn);
#pragma unroll
                for (int r = 0; r < N; ++r) {
                    z.re[r * N + j] *= inv;
                    z.im[r * N + j] *= inv;
                }
            }
            // det of the unitary; multiply by det^(-1/N)
            float dr, di;
            if constexpr (N == 2) {
                dr = z.re[0] * z.re[3] - z.im[0] * z.im[3] - (z.re[1] * z.re[2] - z.im[1] * z.im[2]);
                di = z.re[0] * z.im[3] + z.im[0] * z.re[3] - (z.re[1] * z.im[2] + z.im[1] * z.re[2]);
            } else {
                dr = 0.f;
                di = 0.f;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int a = (c + 1) % 3, b = (c + 2) % 3;
                    // minor m = z[1][a] z[2][b] - z[1][b] z[2][a]
                    const float mr = (z.re[3 + a] * z.re[6 + b] - z.im[3 + a] * z.im[6 + b]) - (z.re[3 + b] * z.re[6 + a] - z.im[3 + b] * z.im[6 + a]);
                    const float mi = (z.re[3 + a] * z.im[6 + b] + z.im[3 + a] * z.re[6 + b]) - (z.re[3 + b] * z.im[6 + a] + z.im[3 + b] * z.re[6 + a]);
                    dr += z.re[c] * mr - z.im[c] * mi;
                    di += z.re[c] * mi + z.im[c] * mr;
                }
            }
            const float ph = -atan2f(di, dr) / float(N);
            float sn, cs;
            sincosf(ph, &sn, &cs);
#pragma unroll
            for (int q = 0; q < N * N; ++q) {
                const float re = z.re[q] * cs - z.im[q] * sn, im = z.re[q] * sn + z.im[q] * cs;
                z.re[q] = re;
                z.im[q] = im;
            }
            // classical Gram-Schmidt in FP32 loses orthogonality on badly
            // conditioned draws: project the result back onto SU(N)
            reunitarise<N>(z);
            mat_store(z, f, n, k);
        }
    }
}

}  // namespace umc
