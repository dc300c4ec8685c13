// umc_learn_kernels.cuh -- the learned U(1) proposal on sm_100a.
//
// A 3-64-64-16 ReLU network maps the staple of a link to a 4-component von
// Mises mixture over the link's new angle; the proposal is used only inside a
// Metropolis-Hastings step (dof/proposal.hpp:5-12, driver.hpp:29-42) whose dE
// is the plain model's, so the target distribution is unchanged.
//
//   x  = (cos a, sin a, |S|),  S = sum_p exp(i phi_p), cos theta_p = cos(theta + phi_p)
//   h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), o = h2 W3 + b3
//   component k: weight softmax(o[4k]), mean atan2(o[4k+2], o[4k+1]),
//                concentration clamp(softplus(o[4k+3]), 1e-4, 80)
//
// The three products run on the tensor cores (tcgen05.mma kind::f16, BF16
// operands, FP32 accumulators in TMEM) for tiles of 128 links, one link per
// thread: thread t owns row t of every tile, which is TMEM lane t, so a
// layer's epilogue (bias, ReLU, BF16) goes TMEM -> registers -> the next
// layer's shared-memory operand without any exchange between threads.
//
// Training (maximum likelihood on angles the plain sampler produced) runs the
// same forward, the loss head in FP32, the two data-gradient products
// (dH2 = dO W3^T, dH1 = dZ2 W2^T) and the weight gradients as two stacked
// M = 128 products over the samples of a tile, accumulated in TMEM over all
// the tiles a CTA processes:
//   [x^T; 1; 0]   (128 x 128) . [dZ1 | dZ2 | dO]  -> dW1, and db1|db2|db3 (ones row)
//   [h1^T; h2^T]  (128 x 128) . [dZ2 | dO]        -> dW2 and dW3 blocks
// A reduction kernel sums the per-CTA partials in a fixed order and applies
// Adam to the FP32 master parameters, then rewrites the BF16 operand image.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "umc_device.cuh"
#include <umc/keyed_pcg.cuh>
#include "umc_tc.cuh"

namespace umc {
namespace learn {

constexpr int kIn = 3, kH = 64, kOut = 16, kComp = 4;
constexpr int P_W1 = 0, P_B1 = 192, P_W2 = 256, P_B2 = 4352, P_W3 = 4416, P_B3 = 5440, kParams = 5456;
constexpr uint32_t kTile = 128;            // rows (links or samples) per tile = threads per CTA
constexpr uint32_t kTagLearned = 6;        // key tag of the learned update, id = link
constexpr float kKappaMin = 1e-4f, kKappaMax = 80.0f;
constexpr int kTries = 32;                 // Best-Fisher trials per proposal

// BF16 operand image (bytes), each block in the K-major layout of umc_tc.cuh;
// the forward operands and the FP32 biases come first so that the sampler
// stages only IMG_FWD_BYTES.
constexpr uint32_t IMG_B1 = 0;         // N 64 (h1 unit j)  x K 16 (input f, zero past 3)
constexpr uint32_t IMG_B2 = 2048;      // N 64 (h2 unit j)  x K 64 (h1 unit i)
constexpr uint32_t IMG_B3 = 10240;     // N 16 (output o)   x K 64 (h2 unit j)
constexpr uint32_t IMG_BIAS = 12288;   // b1[64], b2[64], b3[16] in FP32
constexpr uint32_t IMG_FWD_BYTES = IMG_BIAS + 144 * 4;
constexpr uint32_t IMG_B3T = 12928;    // N 64 (h2 unit j)  x K 16 (output o)
constexpr uint32_t IMG_B2T = 14976;    // N 64 (h1 unit i)  x K 64 (h2 unit j)
constexpr uint32_t IMG_BYTES = IMG_B2T + 8192;

// Tensor-memory columns.  The output layer reuses the first layer's columns
// (read out before the second product is issued), so a forward needs 128.
// The sampler's second layer also reuses them (64 columns per tile group);
// training keeps z2 / dH2 at column 64.
constexpr uint32_t TM_Z1 = 0, TM_Z2 = 64, TM_O = 0;     // forward (and dH1 / dH2)
constexpr uint32_t TM_G1 = 128, TM_G2 = 288;            // weight-gradient accumulators (144 + 80)
constexpr uint32_t kFwdCols = 64, kTrainCols = 512;
// tcgen05.alloc takes a power of two >= 32 columns
__host__ __device__ constexpr uint32_t alloc_cols(uint32_t c)
{
    uint32_t p = 32;
    while (p < c) p <<= 1;
    return p;
}
// Dynamic shared memory of the forward kernels is at least this, so that at
// most three of their CTAs (3 x 128 TMEM columns) share an SM.
constexpr uint32_t kFwdMinSmem = 58 * 1024;

// Status bits (shared with the chain engine's conventions).
constexpr unsigned kStatusTimeout = 16u;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// 16 values at columns k0 .. k0 + 15 of one row of an R-row operand.
__device__ __forceinline__ void store_row16(uint8_t* buf, uint32_t R, uint32_t row, uint32_t k0, const float* v)
{
    uint4 a, b;
    a.x = pack_bf16(v[0], v[1]);
    a.y = pack_bf16(v[2], v[3]);
    a.z = pack_bf16(v[4], v[5]);
    a.w = pack_bf16(v[6], v[7]);
    b.x = pack_bf16(v[8], v[9]);
    b.y = pack_bf16(v[10], v[11]);
    b.z = pack_bf16(v[12], v[13]);
    b.w = pack_bf16(v[14], v[15]);
    *reinterpret_cast<uint4*>(buf + tc::kmajor_offset(R, row, k0)) = a;
    *reinterpret_cast<uint4*>(buf + tc::kmajor_offset(R, row, k0 + 8)) = b;
}

// One element (row n, column k) of an R-row operand.
__device__ __forceinline__ void store_elem(uint8_t* buf, uint32_t R, uint32_t n, uint32_t k, float v)
{
    *reinterpret_cast<__nv_bfloat16*>(buf + tc::kmajor_offset(R, n, k)) = __float2bfloat16_rn(v);
}

// Builds the operand image from the FP32 master parameters.
__global__ void mlp_image(const float* __restrict__ P, uint8_t* __restrict__ img)
{
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    auto put = [&](uint32_t off, uint32_t R, uint32_t r, uint32_t k, float v) {
        *reinterpret_cast<__nv_bfloat16*>(img + off + tc::kmajor_offset(R, r, k)) = __float2bfloat16_rn(v);
    };
    if (e < 1024) {  // B1: r = j, k = f
        const uint32_t j = e >> 4, f = e & 15u;
        put(IMG_B1, 64, j, f, f < 3 ? P[P_W1 + f * 64 + j] : 0.0f);
    } else if (e < 5120) {  // B2: r = j, k = i ; B2T: r = i, k = j
        const uint32_t q = e - 1024, i = q >> 6, j = q & 63u;
        const float w = P[P_W2 + i * 64 + j];
        put(IMG_B2, 64, j, i, w);
        put(IMG_B2T, 64, i, j, w);
    } else if (e < 6144) {  // B3: r = o, k = j ; B3T: r = j, k = o
        const uint32_t q = e - 5120, j = q >> 4, o = q & 15u;
        const float w = P[P_W3 + j * 16 + o];
        put(IMG_B3, 16, o, j, w);
        put(IMG_B3T, 64, j, o, w);
    } else if (e < 6144 + 144) {
        const uint32_t q = e - 6144;
        const float b = q < 64 ? P[P_B1 + q] : (q < 128 ? P[P_B2 + q - 64] : P[P_B3 + q - 128]);
        reinterpret_cast<float*>(img + IMG_BIAS)[q] = b;
    }
}
constexpr uint32_t kImageThreads = 6144 + 144;

// Shared-memory context of one tile group: 128 threads (four consecutive
// warps, so TMEM lane quadrants 0..3) that process tiles together, with their
// own operand buffers, mbarrier, TMEM columns and named barrier.
struct Tile
{
    const uint8_t* img;  // operand image (shared by the CTA)
    uint8_t* X;          // 128 x 16 input operand
    uint8_t* H1;         // 128 x 64
    uint8_t* H2;         // 128 x 64 (may alias H1 in the sampler)
    uint64_t* mbar;
    uint32_t tmem;       // first TMEM column of the group
    uint32_t phase;
    uint32_t row;        // this thread's row, 0..127
    uint32_t bar;        // named barrier id of the group (1..15)
    uint32_t z2col;      // TMEM column of the second layer's accumulator
};

// Waits for the next MMA completion; records a timeout in *fail.
__device__ __forceinline__ void tile_wait(Tile& t, bool& fail)
{
    if (!tc::mbar_wait(t.mbar, t.phase)) fail = true;
    t.phase ^= 1u;
    tc::fence_after();
}

// Writers done with shared operands / readers done with TMEM -> MMA issue.
// Returns true (uniformly over the group) if any thread saw a timeout.
__device__ __forceinline__ bool tile_sync(const Tile& t, bool fail)
{
    tc::fence_async_smem();
    tc::fence_before();
    return tc::bar_or(t.bar, kTile, fail);
}

// Epilogue of a 64-wide layer: z (TMEM) + bias -> ReLU -> BF16 row of `dst`.
// Returns the ReLU mask (bit j set iff z_j > 0).
__device__ __forceinline__ uint64_t layer_epilogue(const Tile& t, uint32_t col, const float* bias, uint8_t* dst)
{
    uint64_t mask = 0;
    const uint32_t row = t.row;
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
        float v[16];
        tc::tmem_ld16(tc::tmem_lane_addr(t.tmem, col + 16 * c), v);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float z = v[i] + bias[16 * c + i];
            if (z > 0.0f) mask |= 1ull << (16 * c + i);
            v[i] = fmaxf(z, 0.0f);
        }
        store_row16(dst, kTile, row, 16 * c, v);
    }
    return mask;
}

// The same epilogue without the mask (sampler and forward): bias added in FP32,
// then BF16 rounding and ReLU on packed pairs (relu(bf16(z)) = bf16(relu(z))).
__device__ __forceinline__ void layer_epilogue_fast(const Tile& t, uint32_t col, const float* bias, uint8_t* dst)
{
    const __nv_bfloat162 zero = __float2bfloat162_rn(0.0f);
    const uint32_t row = t.row;
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c) {
        float v[16];
        tc::tmem_ld16(tc::tmem_lane_addr(t.tmem, col + 16 * c), v);
        tc::tmem_wait_ld();
        uint32_t w[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 b = reinterpret_cast<const float4*>(bias + 16 * c)[q];
            __nv_bfloat162 p0 = __hmax2(__floats2bfloat162_rn(v[4 * q] + b.x, v[4 * q + 1] + b.y), zero);
            __nv_bfloat162 p1 = __hmax2(__floats2bfloat162_rn(v[4 * q + 2] + b.z, v[4 * q + 3] + b.w), zero);
            w[2 * q] = *reinterpret_cast<uint32_t*>(&p0);
            w[2 * q + 1] = *reinterpret_cast<uint32_t*>(&p1);
        }
        *reinterpret_cast<uint4*>(dst + tc::kmajor_offset(kTile, row, 16 * c)) = make_uint4(w[0], w[1], w[2], w[3]);
        *reinterpret_cast<uint4*>(dst + tc::kmajor_offset(kTile, row, 16 * c + 8)) = make_uint4(w[4], w[5], w[6], w[7]);
    }
}

// Forward pass of one tile: x (this thread's row) -> o[16].  All 128 threads
// call it.  h1 goes to t.H1, h2 to t.H2; masks receive the ReLU masks.
// Returns true (uniformly) on a wait timeout.
__device__ bool tile_forward(Tile& t, const float x[3], float o[16], uint64_t* masks = nullptr)
{
    const uint32_t row = t.row;
    const uint32_t ximg = tc::smem_addr(t.img);
    const float* bias = reinterpret_cast<const float*>(t.img + IMG_BIAS);
    {
        float v[16] = {x[0], x[1], x[2], 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        store_row16(t.X, kTile, row, 0, v);
    }
    bool fail = false;
    if (tile_sync(t, false)) return true;
    if (row == 0) {
        tc::fence_after();
        tc::mma_bf16(t.tmem + TM_Z1, tc::operand_desc(tc::smem_addr(t.X), kTile, 0),
                     tc::operand_desc(ximg + IMG_B1, 64, 0), tc::idesc_bf16(128, 64), false);
        tc::mma_commit(t.mbar);
    }
    tile_wait(t, fail);
    uint64_t m1 = 0, m2 = 0;
    if (masks) m1 = layer_epilogue(t, TM_Z1, bias, t.H1);
    else layer_epilogue_fast(t, TM_Z1, bias, t.H1);
    if (tile_sync(t, fail)) return true;
    if (row == 0) {
        tc::fence_after();
        for (uint32_t s = 0; s < 4; ++s)
            tc::mma_bf16(t.tmem + t.z2col, tc::operand_desc(tc::smem_addr(t.H1), kTile, s),
                         tc::operand_desc(ximg + IMG_B2, 64, s), tc::idesc_bf16(128, 64), s > 0);
        tc::mma_commit(t.mbar);
    }
    tile_wait(t, fail);
    if (masks) m2 = layer_epilogue(t, t.z2col, bias + 64, t.H2);
    else layer_epilogue_fast(t, t.z2col, bias + 64, t.H2);
    if (tile_sync(t, fail)) return true;
    if (row == 0) {
        tc::fence_after();
        for (uint32_t s = 0; s < 4; ++s)
            tc::mma_bf16(t.tmem + TM_O, tc::operand_desc(tc::smem_addr(t.H2), kTile, s),
                         tc::operand_desc(ximg + IMG_B3, 16, s), tc::idesc_bf16(128, 16), s > 0);
        tc::mma_commit(t.mbar);
    }
    tile_wait(t, fail);
    tc::tmem_ld16(tc::tmem_lane_addr(t.tmem, TM_O), o);
    tc::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] += bias[128 + i];
    if (masks) {
        masks[0] = m1;
        masks[1] = m2;
    }
    return tile_sync(t, fail);
}

// ------------------------------------------------------------ mixture head

struct Mixture
{
    float w[kComp], mu[kComp], kappa[kComp], lw[kComp];  // lw = log w (FP32 inputs)
    double lwd[kComp];                                   // log w in FP64
};

__device__ __forceinline__ float softplus_f(float v) { return v > 20.0f ? v : log1pf(__expf(v)); }

__device__ __forceinline__ void mixture_of(const float o[16], Mixture& m)
{
    float mx = o[0];
#pragma unroll
    for (int k = 1; k < kComp; ++k) mx = fmaxf(mx, o[4 * k]);
    float z = 0.0f;
    float e[kComp];
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        e[k] = expf(o[4 * k] - mx);
        z += e[k];
    }
    const double lz = log(double(z));
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        m.w[k] = e[k] / z;
        m.lwd[k] = double(o[4 * k] - mx) - lz;
        m.mu[k] = atan2f(o[4 * k + 2], o[4 * k + 1]);
        m.kappa[k] = fminf(fmaxf(softplus_f(o[4 * k + 3]), kKappaMin), kKappaMax);
    }
}

// Component from one draw: smallest k with u < w_0 + ... + w_k.
__device__ __forceinline__ int pick_component(const Mixture& m, uint32_t d0)
{
    const float u = u_f32(d0);
    float c = 0.0f;
#pragma unroll
    for (int k = 0; k < kComp - 1; ++k) {
        c += m.w[k];
        if (u < c) return k;
    }
    return kComp - 1;
}

// One Best-Fisher trial (Best & Fisher 1979) around 0 with concentration kappa.
// Written with r - 1 = s + s^2 / (1 + sqrt(1 + s^2)), 1 - z = 2 sin^2(pi u1 / 2),
// 1 - f = (r - 1)(1 - z) / (r + z) and acos f = 2 asin(sqrt((1 - f) / 2)), so
// FP32 keeps full relative precision near the mode at large kappa.
__device__ __forceinline__ bool vm_trial(float kappa, uint32_t d1, uint32_t d2, uint32_t d3, float& angle)
{
    const float s = 0.5f / kappa;
    const float q = sqrtf(1.0f + s * s);
    const float rm1 = s + s * s / (1.0f + q);
    const float r = 1.0f + rm1;
    const float u1 = u_f32(d1), u2 = u_f32(d2);
    const float sh = sinpif(0.5f * u1);
    const float omz = 2.0f * sh * sh;
    const float z = cospif(u1);
    const float omf = rm1 * omz / (r + z);
    const float c = kappa * (rm1 + omf);
    if (c * (2.0f - c) - u2 > 0.0f || logf(c / u2) + 1.0f - c >= 0.0f) {
        const float a = 2.0f * asinf(fminf(sqrtf(0.5f * omf), 1.0f));
        angle = (d3 & 0x80000000u) ? a : -a;
        return true;
    }
    return false;
}

// log q(theta) of the mixture in FP64 (log-sum-exp over components).
__device__ __forceinline__ double mixture_logpdf(const Mixture& m, const double* li, double theta)
{
    double l[kComp], mx = -1e300;
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        l[k] = m.lwd[k] + double(m.kappa[k]) * cos(theta - double(m.mu[k])) - li[k];
        mx = fmax(mx, l[k]);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kComp; ++k) s += exp(l[k] - mx);
    return mx + log(s);
}

// NLL of target angle `th` and its gradient with respect to the 16 outputs (FP32).
__device__ __forceinline__ float head_loss_grad(const float o[16], float th, float dO[16])
{
    Mixture m;
    mixture_of(o, m);
    float l[kComp], mx = -1e30f;
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        const float kp = m.kappa[k];
        l[k] = float(m.lwd[k]) + kp * cosf(th - m.mu[k]) - logf(cyl_bessel_i0f(kp)) - 1.8378770664093453f;
        mx = fmaxf(mx, l[k]);
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kComp; ++k) s += expf(l[k] - mx);
    const float lse = mx + logf(s);
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        const float gam = expf(l[k] - lse);
        dO[4 * k] = m.w[k] - gam;
        const float u = o[4 * k + 1], v = o[4 * k + 2];
        const float rr = u * u + v * v;
        float sn, cs;
        sincosf(th - m.mu[k], &sn, &cs);
        const float dmu = -gam * m.kappa[k] * sn;
        dO[4 * k + 1] = rr > 0.0f ? dmu * (-v / rr) : 0.0f;
        dO[4 * k + 2] = rr > 0.0f ? dmu * (u / rr) : 0.0f;
        const float raw = softplus_f(o[4 * k + 3]);
        float dk = 0.0f;
        if (raw > kKappaMin && raw < kKappaMax) {
            const float kp = m.kappa[k];
            const float A = cyl_bessel_i1f(kp) / cyl_bessel_i0f(kp);
            const float sig = 1.0f / (1.0f + expf(-o[4 * k + 3]));
            dk = -gam * (cs - A) * sig;
        }
        dO[4 * k + 3] = dk;
    }
    return -lse;
}

// Features of a staple sum S = Sr + i Si.
__device__ __forceinline__ void staple_features(float Sr, float Si, float x[3])
{
    const float r = sqrtf(Sr * Sr + Si * Si);
    if (r > 0.0f) {
        x[0] = Sr / r;
        x[1] = Si / r;
    } else {
        x[0] = 1.0f;
        x[1] = 0.0f;
    }
    x[2] = r;
}

// ------------------------------------------------------------ 2D U(1) chains
//
// Chain layout: 2 L^2 FP32 angles in the colour-major order of the
// square-plaquette complex (links mu L^2 + y L + x): class 2 mu + ((x + y) & 1),
// then (y L + x) / 2.  Plaquette (x, y) has links
// [(0,x,y), (1,x+1,y), (0,x,y+1), (1,x,y)] and angle t0 + t1 - t2 - t3.

struct Lat2
{
    uint32_t L, Lh, half;
    __device__ __forceinline__ uint32_t idx(uint32_t mu, uint32_t x, uint32_t y) const
    {
        return (2u * mu + ((x + y) & 1u)) * half + y * Lh + (x >> 1);
    }
};

// Staple sum of the link at position q of colour class cls; the plaquette
// phases are formed exactly as the cell-complex U(1) pass forms them.
__device__ __forceinline__ void staple2(const float* th, const Lat2& g, uint32_t cls, uint32_t q, float& Sr,
                                        float& Si)
{
    const uint32_t mu = cls >> 1, p = cls & 1u;
    const uint32_t y = q / g.Lh, j = q - y * g.Lh;
    const uint32_t x = 2u * j + ((y + p) & 1u);
    const uint32_t L = g.L;
    const uint32_t xp = x + 1 == L ? 0u : x + 1, xm = x == 0 ? L - 1 : x - 1;
    const uint32_t yp = y + 1 == L ? 0u : y + 1, ym = y == 0 ? L - 1 : y - 1;
    float phA, phB;
    if (mu == 0) {
        phA = th[g.idx(1, xp, y)] - th[g.idx(0, x, yp)] - th[g.idx(1, x, y)];     // cell (x,y), slot 0
        phB = th[g.idx(1, x, ym)] - th[g.idx(0, x, ym)] - th[g.idx(1, xp, ym)];   // cell (x,y-1), slot 2
    } else {
        phA = th[g.idx(0, xm, y)] - th[g.idx(0, xm, yp)] - th[g.idx(1, xm, y)];   // cell (x-1,y), slot 1
        phB = th[g.idx(0, x, yp)] - th[g.idx(0, x, y)] - th[g.idx(1, xp, y)];     // cell (x,y), slot 3
    }
    float sA, cA, sB, cB;
    sincosf(phA, &sA, &cA);
    sincosf(phB, &sB, &cB);
    Sr = cA + cB;
    Si = sA + sB;
}

// model_beta sum over the link's two cells of cos(theta_p) - cos(theta_p') for
// the link going from t to p, in FP64 on the FP32 angles (the cells of staple2).
__device__ __noinline__ double u1_delta2_64(const float* th, const Lat2& g, uint32_t cls, uint32_t q, float t, float p,
                                            double model_beta)
{
    const uint32_t mu = cls >> 1, par = cls & 1u;
    const uint32_t y = q / g.Lh, j = q - y * g.Lh;
    const uint32_t x = 2u * j + ((y + par) & 1u);
    const uint32_t L = g.L;
    const uint32_t xp = x + 1 == L ? 0u : x + 1, xm = x == 0 ? L - 1 : x - 1;
    const uint32_t yp = y + 1 == L ? 0u : y + 1, ym = y == 0 ? L - 1 : y - 1;
    double phA, phB;
    if (mu == 0) {
        phA = double(th[g.idx(1, xp, y)]) - double(th[g.idx(0, x, yp)]) - double(th[g.idx(1, x, y)]);
        phB = double(th[g.idx(1, x, ym)]) - double(th[g.idx(0, x, ym)]) - double(th[g.idx(1, xp, ym)]);
    } else {
        phA = double(th[g.idx(0, xm, y)]) - double(th[g.idx(0, xm, yp)]) - double(th[g.idx(1, xm, y)]);
        phB = double(th[g.idx(0, x, yp)]) - double(th[g.idx(0, x, y)]) - double(th[g.idx(1, xp, y)]);
    }
    return model_beta * ((cos(double(t) + phA) - cos(double(p) + phA)) + (cos(double(t) + phB) - cos(double(p) + phB)));
}

struct U1BatchArgs
{
    float* theta;                         // n_chains x 2 L^2
    uint32_t n_chains, L;
    const unsigned long long* chain_seed;
    unsigned long long sweep0;
    uint32_t n_sweeps;
    float model_beta, driver_beta, width;
    const uint8_t* img;                   // learned: operand image; plain: unused
    double* records;                      // [sweep][chain][4]: S, P, Q, accepted
    unsigned long long rec_slot0;         // record slot of the first sweep
    unsigned long long rec_capacity;      // slots (sweeps) in the record buffer
    float* dump;                          // learned: outputs of chain 0, first sweep (2 L^2 x 16)
    unsigned int* status;
    double model_beta64, driver_beta64;   // plain: the couplings of the FP64 decisions
    float err;                            // plain: u1_metropolis_err(driver_beta, model_beta, 2)
};

// Per-sweep observables of the chain in shared memory (all threads call it).
__device__ __forceinline__ void chain_record(const U1BatchArgs& a, const float* th, const Lat2& g, uint32_t chain,
                                             uint32_t s, double accepted)
{
    double v[3] = {0.0, 0.0, accepted};
    const uint32_t L = g.L, L2 = L * L;
    for (uint32_t pp = threadIdx.x; pp < L2; pp += blockDim.x) {
        const uint32_t y = pp / L, x = pp - y * L;
        const uint32_t xp = x + 1 == L ? 0u : x + 1, yp = y + 1 == L ? 0u : y + 1;
        const float tp = th[g.idx(0, x, y)] + th[g.idx(1, xp, y)] - th[g.idx(0, x, yp)] - th[g.idx(1, x, y)];
        v[0] += double(cosf(tp));
        v[1] += double(remainderf(tp, 6.283185307179586f));
    }
    // the third entry is only thread-local counts: sum them too
    block_sum<3>(v);
    if (threadIdx.x == 0 && a.records) {
        const unsigned long long slot = a.rec_slot0 + s;
        if (slot < a.rec_capacity) {
            double* r = a.records + (slot * a.n_chains + chain) * 4;
            r[0] = double(a.model_beta) * (double(L2) - v[0]);
            r[1] = v[0] / double(L2);
            r[2] = v[1] / 6.283185307179586;
            r[3] = v[2];
        }
    }
}

// Mixture parameters as the sampler uses them: weights, log weights,
// concentrations and mean directions (cos mu, sin mu) = (u, v) / |(u, v)|
// ((1, 0) when u = v = 0, matching atan2(0, 0) = 0).
struct MixtureDir
{
    float w[kComp], lw[kComp], kappa[kComp], cu[kComp], su[kComp];
};

__device__ __forceinline__ void mixture_dir(const float o[16], MixtureDir& m)
{
    float mx = o[0];
#pragma unroll
    for (int k = 1; k < kComp; ++k) mx = fmaxf(mx, o[4 * k]);
    float z = 0.0f;
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        m.w[k] = expf(o[4 * k] - mx);
        z += m.w[k];
    }
    const float lz = logf(z), iz = 1.0f / z;
#pragma unroll
    for (int k = 0; k < kComp; ++k) {
        m.w[k] *= iz;
        m.lw[k] = (o[4 * k] - mx) - lz;
        m.kappa[k] = fminf(fmaxf(softplus_f(o[4 * k + 3]), kKappaMin), kKappaMax);
        const float u = o[4 * k + 1], v = o[4 * k + 2], rr = u * u + v * v;
        const float n = rr > 0.0f ? rsqrtf(rr) : 0.0f;
        m.cu[k] = rr > 0.0f ? u * n : 1.0f;
        m.su[k] = v * n;
    }
}

// The learned Metropolis-Hastings step of link k (colour-major) given the
// network outputs o and the staple sum: component by inverse CDF, Best-Fisher
// angle around mu = atan2(v, u), dE as the plain model computes it, and
//   log_p = -beta dE + log q(old) - log q(new)
// with log q(t) = logsumexp_k(log w_k - log I0(kappa_k) + kappa_k cos(t - mu_k))
// (the common log 2 pi cancels).  The per-component terms are FP32 -- their
// error, about kappa 1e-7, is the size of the FP32 angle quantisation of the
// proposal itself.  The accept test compares in FP32 with error bounds and
// forms log_p in FP64 only inside them.  Returns true if accepted.
__device__ __forceinline__ bool learned_update(const U1BatchArgs& a, float* th, uint32_t k, const float o[16],
                                               float Sr, float Si, uint64_t kbase)
{
    MixtureDir m;
    mixture_dir(o, m);
    KeyedPcg r = KeyedPcg::open(kbase, k);
    const float u0 = u_f32(r.next());
    int comp = kComp - 1;
    {
        // smallest kk with u0 < w_0 + ... + w_kk
        float c = 0.0f;
#pragma unroll
        for (int kk = 0; kk < kComp - 1; ++kk) {
            c += m.w[kk];
            if (comp == kComp - 1 && u0 < c) comp = kk;
        }
    }
    float kc = m.kappa[0], uc = o[1], vc = o[2];
#pragma unroll
    for (int kk = 1; kk < kComp; ++kk)
        if (comp == kk) {
            kc = m.kappa[kk];
            uc = o[4 * kk + 1];
            vc = o[4 * kk + 2];
        }
    float ang = 0.0f;
    bool moved = false;
    for (int tr = 0; tr < kTries && !moved; ++tr) {
        const uint32_t d1 = r.next(), d2 = r.next(), d3 = r.next();
        moved = vm_trial(kc, d1, d2, d3, ang);
    }
    if (!moved) return false;
    const float tcur = th[k];
    const float p = remainderf(atan2f(vc, uc) + ang, 6.283185307179586f);
    float so, co, sp, cp;
    sincosf(tcur, &so, &co);
    sincosf(p, &sp, &cp);
    const float dE = a.model_beta * ((co - cp) * Sr - (so - sp) * Si);
    float lo[kComp], ln[kComp], mo = -3.0e38f, mn = -3.0e38f;
#pragma unroll
    for (int kk = 0; kk < kComp; ++kk) {
        const float base = m.lw[kk] - logf(cyl_bessel_i0f(m.kappa[kk]));
        lo[kk] = base + m.kappa[kk] * (co * m.cu[kk] + so * m.su[kk]);
        ln[kk] = base + m.kappa[kk] * (cp * m.cu[kk] + sp * m.su[kk]);
        mo = fmaxf(mo, lo[kk]);
        mn = fmaxf(mn, ln[kk]);
    }
    float so_ = 0.0f, sn_ = 0.0f;
#pragma unroll
    for (int kk = 0; kk < kComp; ++kk) {
        so_ += expf(lo[kk] - mo);
        sn_ += expf(ln[kk] - mn);
    }
    // MH test: log_p = -beta dE + log q(old|new) - log q(new|old) in FP64, accept
    // iff log_p >= 0 or log u < log_p (driver.hpp:36-41).  The same comparisons
    // are made first in FP32 with error bounds far above FP32 round-off (2^-18
    // of the terms' magnitude for log_p, 2^-17 of |log u| + 1 for log u); only
    // a decision inside those bounds evaluates the FP64 expressions, so every
    // decision is the FP64 one.
    const float bdE = a.driver_beta * dE;
    const float lp = (-bdE + (mo - mn)) + (logf(so_) - logf(sn_));
    const float ep = ldexpf(4.0f + fabsf(mo) + fabsf(mn) + fabsf(bdE), -18);
    auto log_p64 = [&] {
        const double lr = (double(mo) - double(mn)) + log(double(so_) / double(sn_));
        return -double(a.driver_beta) * double(dE) + lr;
    };
    bool accept;
    if (lp >= ep) {
        accept = true;
    } else if (lp <= -ep) {
        const uint32_t kd = r.next();
        const float lu = logf(u_f32(kd));
        const float eu = ldexpf(1.0f + fabsf(lu), -17);
        if (lu + eu < lp - ep) accept = true;
        else if (lu - eu > lp + ep) accept = false;
        else accept = log(u_f64(kd)) < log_p64();
    } else {
        const double lp64 = log_p64();
        accept = lp64 >= 0.0 || log(u_f64(r.next())) < lp64;
    }
    if (accept) th[k] = p;
    return accept;
}

// Plain U1Shift Metropolis, one CTA per chain at a time, chain in shared memory.
__global__ void __launch_bounds__(256) u1_plain_batch(U1BatchArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    float* th = reinterpret_cast<float*>(smem);
    const Lat2 g{a.L, a.L / 2, a.L * a.L / 2};
    const uint32_t nl = 2 * a.L * a.L;
    for (uint32_t c = blockIdx.x; c < a.n_chains; c += gridDim.x) {
        float* gth = a.theta + size_t(c) * nl;
        for (uint32_t i = threadIdx.x; i < nl; i += blockDim.x) th[i] = gth[i];
        __syncthreads();
        for (uint32_t s = 0; s < a.n_sweeps; ++s) {
            const uint64_t kbase = key_base(key_seed(a.chain_seed[c], a.sweep0 + s, tag_site(0)));
            uint32_t acc = 0;
            for (uint32_t cls = 0; cls < 4; ++cls) {
                for (uint32_t q = threadIdx.x; q < g.half; q += blockDim.x) {
                    float Sr, Si;
                    staple2(th, g, cls, q, Sr, Si);
                    const uint32_t k = cls * g.half + q;
                    const float t = th[k];
                    float so, co;
                    sincosf(t, &so, &co);
                    KeyedPcg r = KeyedPcg::open(kbase, k);
                    const float p = u1_shift(r, a.width, t);
                    float sp, cp;
                    sincosf(p, &sp, &cp);
                    const float dE = a.model_beta * ((co - cp) * Sr - (so - sp) * Si);
                    const bool ok = metropolis_accept(r, -a.driver_beta * dE, a.err, [&] {
                        return -a.driver_beta64 * u1_delta2_64(th, g, cls, q, t, p, a.model_beta64);
                    });
                    if (ok) {
                        th[k] = p;
                        ++acc;
                    }
                }
                __syncthreads();
            }
            chain_record(a, th, g, c, s, double(acc));
        }
        for (uint32_t i = threadIdx.x; i < nl; i += blockDim.x) gth[i] = th[i];
        __syncthreads();
    }
}

// Shared-memory plan of the learned sampler and the forward kernel (bytes,
// 128-byte aligned blocks): the forward operand image, then per tile group an
// input operand X (128 x 16) and a hidden operand H (128 x 64), the group
// mbarriers and the TMEM address slot, then the chain's angles.  The total is
// padded so that the CTAs one SM can hold never ask for more than 512 TMEM
// columns between them.
// Tile groups of the learned sampler: 8 (1024 threads, 8 x 64 = 512 TMEM
// columns, two rounds of tiles per 2048-link colour class of a 64 x 64 chain)
// when the shared-memory plan fits, else 6 or 4 for larger chains.
constexpr uint32_t kGroupChoices[3] = {8, 6, 4};

struct LearnSmem
{
    uint32_t img, X, H, group_bytes, bar, field, total;
    __host__ __device__ static LearnSmem plan(uint32_t L, uint32_t groups)
    {
        LearnSmem p{};
        p.img = 0;
        p.X = (IMG_FWD_BYTES + 127u) & ~127u;
        p.group_bytes = kTile * 16 * 2 + kTile * 64 * 2;
        p.H = p.X + kTile * 16 * 2;
        p.bar = p.X + groups * p.group_bytes;
        p.field = p.bar + 128;
        p.total = p.field + 2u * L * L * 4u;
        const uint32_t per_sm = 512u / alloc_cols(groups * kFwdCols);  // CTAs whose TMEM fits one SM
        const uint32_t floor_bytes = 228u * 1024u / (per_sm + 1) + 1024u;
        if (p.total < floor_bytes) p.total = floor_bytes;
        return p;
    }
};

// Learned Metropolis-Hastings sweeps.  One CTA holds one chain at a time in
// shared memory; its G tile groups share each colour class's tiles, and
// the class passes are separated by CTA-wide barriers.
template <uint32_t G>
__global__ void __launch_bounds__(kTile * G, 1) u1_learned_batch(U1BatchArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const LearnSmem sp = LearnSmem::plan(a.L, G);
    uint8_t* img = smem + sp.img;
    float* th = reinterpret_cast<float*>(smem + sp.field);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + sp.bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + sp.bar + 64);
    const uint32_t t = threadIdx.x, grp = t / kTile;

    for (uint32_t i = t; i < IMG_FWD_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(img)[i] = reinterpret_cast<const uint4*>(a.img)[i];
    if (t == 0)
        for (uint32_t g = 0; g < G; ++g) tc::mbar_init(mbar + g, 1);
    if (t < 32) tc::tmem_alloc(tslot, alloc_cols(kFwdCols * G));
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    uint8_t* gx = smem + sp.X + grp * sp.group_bytes;
    Tile tl{img, gx, gx + kTile * 32, gx + kTile * 32, mbar + grp, *tslot + grp * kFwdCols, 0u, t % kTile, 1u + grp, 0u};

    const Lat2 g{a.L, a.L / 2, a.L * a.L / 2};
    const uint32_t nl = 2 * a.L * a.L;
    const uint32_t tiles = (g.half + kTile - 1) / kTile;
    bool failed = false;
    for (uint32_t c = blockIdx.x; c < a.n_chains && !failed; c += gridDim.x) {
        float* gth = a.theta + size_t(c) * nl;
        for (uint32_t i = t; i < nl; i += blockDim.x) th[i] = gth[i];
        __syncthreads();
        for (uint32_t s = 0; s < a.n_sweeps && !failed; ++s) {
            const uint64_t kbase = key_base(key_seed(a.chain_seed[c], a.sweep0 + s, kTagLearned));
            double acc = 0.0;
            for (uint32_t cls = 0; cls < 4; ++cls) {
                for (uint32_t tile = grp; tile < tiles; tile += G) {
                    const uint32_t q = tile * kTile + tl.row;
                    const bool valid = q < g.half;
                    float Sr = 1.0f, Si = 0.0f;
                    if (valid) staple2(th, g, cls, q, Sr, Si);
                    float x[3], o[16];
                    staple_features(Sr, Si, x);
                    if (tile_forward(tl, x, o)) {
                        failed = true;
                        break;
                    }
                    if (!valid) continue;
                    const uint32_t k = cls * g.half + q;
                    if (a.dump && c == 0 && s == 0)
                        for (int i = 0; i < 16; ++i) a.dump[size_t(k) * 16 + i] = o[i];
                    if (learned_update(a, th, k, o, Sr, Si, kbase)) acc += 1.0;
                }
                failed = __syncthreads_or(failed ? 1 : 0) != 0;
                if (failed) break;
            }
            if (!failed) chain_record(a, th, g, c, s, acc);
        }
        for (uint32_t i = t; i < nl; i += blockDim.x) gth[i] = th[i];
        __syncthreads();
    }
    if (failed && t == 0) atomicOr(a.status, kStatusTimeout);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t < 32) tc::tmem_dealloc(*tslot, alloc_cols(kFwdCols * G));
}

// ------------------------------------------------------------ forward (tests)

__global__ void __launch_bounds__(kTile) mlp_forward_kernel(const uint8_t* gimg, const float* x, uint32_t n,
                                                            float* out, unsigned int* status)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const LearnSmem sp = LearnSmem::plan(0, 1);
    uint8_t* img = smem + sp.img;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + sp.bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + sp.bar + 64);
    const uint32_t t = threadIdx.x;
    for (uint32_t i = t; i < IMG_FWD_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(img)[i] = reinterpret_cast<const uint4*>(gimg)[i];
    if (t == 0) tc::mbar_init(mbar, 1);
    if (t < 32) tc::tmem_alloc(tslot, kFwdCols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    Tile tl{img, smem + sp.X, smem + sp.H, smem + sp.H, mbar, *tslot, 0u, t, 1u, 0u};
    const uint32_t tiles = (n + kTile - 1) / kTile;
    bool failed = false;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t s = tile * kTile + t;
        float xi[3] = {0.0f, 0.0f, 0.0f}, o[16];
        if (s < n)
            for (int f = 0; f < 3; ++f) xi[f] = x[size_t(s) * 3 + f];
        if (tile_forward(tl, xi, o)) {
            failed = true;
            break;
        }
        if (s < n)
            for (int i = 0; i < 16; ++i) out[size_t(s) * 16 + i] = o[i];
    }
    if (failed && t == 0) atomicOr(status, kStatusTimeout);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t < 32) tc::tmem_dealloc(tl.tmem, kFwdCols);
}

// ------------------------------------------------------------------ training

struct TrainArgs
{
    const uint8_t* img;
    // explicit samples (x[n][3], theta[n]) ...
    const float* x;
    const float* target;
    // ... or samples drawn from stored configurations
    const float* configs;         // n_configs x 2 L^2 (colour-major)
    unsigned long long n_configs;
    uint32_t L;
    unsigned long long seed, step;
    uint32_t n;                   // samples in this step
    float* partial;               // gridDim.x x kParams
    double* partial_loss;         // gridDim.x
    unsigned int* status;
};

struct TrainSmem
{
    uint32_t img, X, H1, H2, DO, AG1, AG2, BG, bar, total;
    __host__ __device__ static TrainSmem plan()
    {
        TrainSmem p{};
        p.img = 0;
        p.X = (IMG_BYTES + 127u) & ~127u;
        p.H1 = p.X + kTile * 16 * 2;
        p.H2 = p.H1 + kTile * 64 * 2;
        p.DO = p.H2 + kTile * 64 * 2;
        p.AG1 = p.DO + kTile * 16 * 2;
        p.AG2 = p.AG1 + 128 * kTile * 2;
        p.BG = p.AG2 + 128 * kTile * 2;
        p.bar = p.BG + 144 * kTile * 2;
        p.total = p.bar + 128;
        return p;
    }
};

// One training sample: explicit, or a random link of a random stored
// configuration (key (seed, step, learn tag, sample)).
__device__ __forceinline__ void train_sample(const TrainArgs& a, uint32_t s, float x[3], float& th)
{
    if (a.x) {
        for (int f = 0; f < 3; ++f) x[f] = a.x[size_t(s) * 3 + f];
        th = a.target[s];
        return;
    }
    KeyedPcg r = KeyedPcg::open_key(a.seed, a.step, kTagLearn, s);
    const uint32_t nl = 2 * a.L * a.L;
    const unsigned long long cfg = (unsigned long long)((uint64_t(r.next()) * a.n_configs) >> 32);
    const uint32_t k = uint32_t((uint64_t(r.next()) * nl) >> 32);
    const Lat2 g{a.L, a.L / 2, a.L * a.L / 2};
    const float* c = a.configs + size_t(cfg) * nl;
    float Sr, Si;
    staple2(c, g, k / g.half, k % g.half, Sr, Si);
    staple_features(Sr, Si, x);
    th = c[k];
}

__global__ void __launch_bounds__(kTile) mlp_train_kernel(TrainArgs a)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const TrainSmem sp = TrainSmem::plan();
    uint8_t* img = smem + sp.img;
    uint8_t* AG1 = smem + sp.AG1;
    uint8_t* AG2 = smem + sp.AG2;
    uint8_t* BG = smem + sp.BG;
    uint8_t* DO = smem + sp.DO;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + sp.bar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + sp.bar + 64);
    const uint32_t t = threadIdx.x;

    for (uint32_t i = t; i < IMG_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(img)[i] = reinterpret_cast<const uint4*>(a.img)[i];
    // [x^T; 1; 0]: rows 3.. are constant (row 3 ones, the rest zero)
    for (uint32_t i = t; i < 128u * kTile; i += blockDim.x) {
        const uint32_t n = i / kTile, k = i % kTile;
        store_elem(AG1, 128, n, k, n == 3 ? 1.0f : 0.0f);
    }
    if (t == 0) tc::mbar_init(mbar, 1);
    if (t < 32) tc::tmem_alloc(tslot, kTrainCols);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    Tile tl{img, smem + sp.X, smem + sp.H1, smem + sp.H2, mbar, *tslot, 0u, t, 1u, TM_Z2};
    const uint32_t ximg = tc::smem_addr(img);

    const uint32_t tiles = (a.n + kTile - 1) / kTile;
    double loss = 0.0;
    bool failed = false, first = true;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t s = tile * kTile + t;
        const bool valid = s < a.n;
        float x[3] = {1.0f, 0.0f, 0.0f}, th = 0.0f;
        if (valid) train_sample(a, s, x, th);
        for (int f = 0; f < 3; ++f) store_elem(AG1, 128, f, t, valid ? x[f] : 0.0f);
        float o[16];
        uint64_t masks[2];
        if (tile_forward(tl, x, o, masks)) {
            failed = true;
            break;
        }
        // transposed activations for the weight gradients
        {
            const uint8_t* h1 = tl.H1;
            const uint8_t* h2 = tl.H2;
            for (uint32_t j = 0; j < 64; ++j) {
                const uint16_t v1 = *reinterpret_cast<const uint16_t*>(h1 + tc::kmajor_offset(kTile, t, j));
                const uint16_t v2 = *reinterpret_cast<const uint16_t*>(h2 + tc::kmajor_offset(kTile, t, j));
                *reinterpret_cast<uint16_t*>(AG2 + tc::kmajor_offset(128, j, t)) = valid ? v1 : 0;
                *reinterpret_cast<uint16_t*>(AG2 + tc::kmajor_offset(128, 64 + j, t)) = valid ? v2 : 0;
            }
        }
        float dO[16];
        if (valid) loss += double(head_loss_grad(o, th, dO));
        else
            for (int i = 0; i < 16; ++i) dO[i] = 0.0f;
        store_row16(DO, kTile, t, 0, dO);
        for (int i = 0; i < 16; ++i) store_elem(BG, 144, 128 + i, t, dO[i]);
        bool fail = false;
        if (tile_sync(tl, false)) {
            failed = true;
            break;
        }
        if (t == 0) {  // dH2 = dO W3^T
            tc::fence_after();
            tc::mma_bf16(tl.tmem + TM_Z2, tc::operand_desc(tc::smem_addr(DO), kTile, 0),
                         tc::operand_desc(ximg + IMG_B3T, 64, 0), tc::idesc_bf16(128, 64), false);
            tc::mma_commit(mbar);
        }
        tile_wait(tl, fail);
        for (uint32_t c = 0; c < 4; ++c) {  // dZ2 -> H1 (as A operand) and B rows 64..127
            float v[16];
            tc::tmem_ld16(tc::tmem_lane_addr(tl.tmem, TM_Z2 + 16 * c), v);
            tc::tmem_wait_ld();
            for (int i = 0; i < 16; ++i) {
                if (!((masks[1] >> (16 * c + i)) & 1ull)) v[i] = 0.0f;
                store_elem(BG, 144, 64 + 16 * c + i, t, v[i]);
            }
            store_row16(tl.H1, kTile, t, 16 * c, v);
        }
        if (tile_sync(tl, fail)) {
            failed = true;
            break;
        }
        if (t == 0) {  // dH1 = dZ2 W2^T
            tc::fence_after();
            for (uint32_t k = 0; k < 4; ++k)
                tc::mma_bf16(tl.tmem + TM_Z1, tc::operand_desc(tc::smem_addr(tl.H1), kTile, k),
                             tc::operand_desc(ximg + IMG_B2T, 64, k), tc::idesc_bf16(128, 64), k > 0);
            tc::mma_commit(mbar);
        }
        tile_wait(tl, fail);
        for (uint32_t c = 0; c < 4; ++c) {  // dZ1 -> B rows 0..63
            float v[16];
            tc::tmem_ld16(tc::tmem_lane_addr(tl.tmem, TM_Z1 + 16 * c), v);
            tc::tmem_wait_ld();
            for (int i = 0; i < 16; ++i)
                store_elem(BG, 144, 16 * c + i, t, ((masks[0] >> (16 * c + i)) & 1ull) ? v[i] : 0.0f);
        }
        if (tile_sync(tl, fail)) {
            failed = true;
            break;
        }
        if (t == 0) {  // weight gradients, accumulated over this CTA's tiles
            tc::fence_after();
            const uint32_t ag1 = tc::smem_addr(AG1), ag2 = tc::smem_addr(AG2), bg = tc::smem_addr(BG);
            for (uint32_t k = 0; k < kTile / 16; ++k)
                tc::mma_bf16(tl.tmem + TM_G1, tc::operand_desc(ag1, 128, k), tc::operand_desc(bg, 144, k),
                             tc::idesc_bf16(128, 144), !(first && k == 0));
            for (uint32_t k = 0; k < kTile / 16; ++k)
                tc::mma_bf16(tl.tmem + TM_G2, tc::operand_desc(ag2, 128, k), tc::operand_desc(bg, 144, k, 64),
                             tc::idesc_bf16(128, 80), !(first && k == 0));
            tc::mma_commit(mbar);
        }
        tile_wait(tl, fail);
        first = false;
        if (tile_sync(tl, fail)) {
            failed = true;
            break;
        }
    }
    // partial gradients of this CTA: row t of the accumulators
    float* pg = a.partial + size_t(blockIdx.x) * kParams;
    if (!failed) {
        for (uint32_t c = 0; c < 9; ++c) {
            float v[16];
            tc::tmem_ld16(tc::tmem_lane_addr(tl.tmem, TM_G1 + 16 * c), v);
            tc::tmem_wait_ld();
            for (int i = 0; i < 16; ++i) {
                const uint32_t col = 16 * c + i;
                const float g = first ? 0.0f : v[i];
                if (t < 3 && col < 64) pg[P_W1 + t * 64 + col] = g;
                if (t == 3) {
                    if (col < 64) pg[P_B1 + col] = g;
                    else if (col < 128) pg[P_B2 + col - 64] = g;
                    else pg[P_B3 + col - 128] = g;
                }
            }
        }
        for (uint32_t c = 0; c < 5; ++c) {
            float v[16];
            tc::tmem_ld16(tc::tmem_lane_addr(tl.tmem, TM_G2 + 16 * c), v);
            tc::tmem_wait_ld();
            for (int i = 0; i < 16; ++i) {
                const uint32_t col = 16 * c + i;
                const float g = first ? 0.0f : v[i];
                if (t < 64 && col < 64) pg[P_W2 + t * 64 + col] = g;
                if (t >= 64 && col >= 64) pg[P_W3 + (t - 64) * 16 + (col - 64)] = g;
            }
        }
    }
    double lv[1] = {loss};
    block_sum<1>(lv);
    if (t == 0) {
        a.partial_loss[blockIdx.x] = lv[0];
        if (failed) atomicOr(a.status, kStatusTimeout);
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (t < 32) tc::tmem_dealloc(tl.tmem, kTrainCols);
}

struct AdamArgs
{
    const float* partial;
    const double* partial_loss;
    uint32_t n_parts;
    uint32_t n;            // samples (the loss is their mean)
    float* params;
    float* m;
    float* v;
    float* grad_out;       // mean gradient (may be null)
    double* loss_out;      // mean loss (may be null)
    uint32_t apply;        // 0: only reduce
    float lr, b1, b2, eps;
    float c1, c2;          // 1 - b1^t, 1 - b2^t
};

// Fixed-order reduction of the partials, then Adam on the FP32 master values.
__global__ void mlp_reduce_adam(AdamArgs a)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0 && a.loss_out) {
        double s = 0.0;
        for (uint32_t c = 0; c < a.n_parts; ++c) s += a.partial_loss[c];
        *a.loss_out = s / double(a.n);
    }
    if (p >= uint32_t(kParams)) return;
    double s = 0.0;
    for (uint32_t c = 0; c < a.n_parts; ++c) s += double(a.partial[size_t(c) * kParams + p]);
    const float g = float(s / double(a.n));
    if (a.grad_out) a.grad_out[p] = g;
    if (!a.apply) return;
    const float m = a.b1 * a.m[p] + (1.0f - a.b1) * g;
    const float v = a.b2 * a.v[p] + (1.0f - a.b2) * g * g;
    a.m[p] = m;
    a.v[p] = v;
    a.params[p] -= a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
}

}  // namespace learn
}  // namespace umc
