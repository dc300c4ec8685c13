/*
 * umc_oracle_learn.c -- CPU oracle for the learned U(1) proposal (TEST INFRASTRUCTURE).
 *
 * The checker, not the product: a double-precision restatement of what the
 * GPU's learned-proposal kernels compute, so that tests can compare them.
 * Only tests/ and bench.py's CPU-baseline leg load it.
 *
 * The reference has no learned proposal.  What is fixed by the reference is
 * the contract this proposal plugs into: a Proposal supplies sample() and
 * log_ratio() = log q(old|new) - log q(new|old) (dof/proposal.hpp:5-12), and
 * the Metropolis driver accepts with min(1, exp(-beta dE + log_ratio))
 * (driver.hpp:29-42), dE from the model's energy_diff_at (here the U(1)
 * plaquette term, model/cell.hpp:64-78 with term/plaquette.hpp:34-47).
 * oracle/ref_harness.cpp drives that reference driver with this proposal, so
 * the composition below is pinned against the reference itself.
 *
 * Network (parameters packed as in ORC_MLP_* offsets, FP32 master values):
 *   x  = (cos a, sin a, |S|), S = sum over the link's plaquettes of
 *        exp(i phi_p) with cos(theta_p) = cos(theta + phi_p), a = arg S
 *   h1 = relu(x W1 + b1), h2 = relu(h1 W2 + b2), o = h2 W3 + b3   (3-64-64-16)
 *   component k: weight softmax(o[4k]), mean atan2(o[4k+2], o[4k+1]),
 *                concentration clamp(softplus(o[4k+3]), 1e-4, 80)
 * The GPU multiplies BF16 operands with FP32 accumulation; with emulate != 0
 * the oracle rounds the same operands to BF16 (round to nearest even) and
 * accumulates in FP64.
 *
 * Sampling: component by inverse CDF on one draw, then the von Mises sample of
 * Best & Fisher (1979, Appl. Statist. 28:152-157) with r = s + sqrt(1 + s^2),
 * s = 1/(2 kappa) (an algebraically equal form of their (1 + rho^2)/(2 rho)),
 * three draws per trial, at most ORC_VM_TRIES trials (a failed proposal keeps
 * the link; the failure probability does not depend on the current angle, so
 * detailed balance holds).  log I0 and I1/I0 are power series of the modified
 * Bessel functions (Abramowitz & Stegun 9.6.10).
 */
#include <math.h>
#include <string.h>

#include "umc_oracle.h"

#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------ Bessel */

/* I_nu(x) for nu in {0, 1}: sum_k (x/2)^(2k+nu) / (k! (k+nu)!).  All terms are
 * positive; for x <= 80 the largest term is below 1e35 and 200 terms reach the
 * double rounding level. */
static double bessel_i(int nu, double x)
{
    const double q = 0.25 * x * x;
    double term = nu ? 0.5 * x : 1.0;
    double sum = term;
    for (int k = 1; k < 400; ++k) {
        term *= q / ((double)k * (double)(k + nu));
        sum += term;
        if (term < sum * 1e-17) break;
    }
    return sum;
}

double orc_log_i0(double x) { return log(bessel_i(0, x)); }
double orc_i1_over_i0(double x) { return bessel_i(1, x) / bessel_i(0, x); }

/* ----------------------------------------------------------------- BF16 */

double orc_bf16(double v)
{
    float f = (float)v;
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return v; /* inf / nan unchanged */
    u += 0x7fffu + ((u >> 16) & 1u);
    u &= 0xffff0000u;
    memcpy(&f, &u, 4);
    return (double)f;
}

static double maybe_bf16(double v, int emulate) { return emulate ? orc_bf16(v) : v; }

/* ------------------------------------------------------------ the network */

void orc_u1_features(double Sr, double Si, double* x)
{
    const double r = sqrt(Sr * Sr + Si * Si);
    if (r > 0.0) {
        x[0] = Sr / r;
        x[1] = Si / r;
    } else {
        x[0] = 1.0;
        x[1] = 0.0;
    }
    x[2] = r;
}

/* Forward pass for one input; keeps the activations for the backward pass. */
static void mlp_forward_keep(const double* P, const double* x, int emulate, double* xb, double* z1,
                             double* h1, double* z2, double* h2, double* o)
{
    const int H = ORC_MLP_HIDDEN, O = ORC_MLP_OUT;
    const double* W1 = P + ORC_MLP_W1;
    const double* b1 = P + ORC_MLP_B1;
    const double* W2 = P + ORC_MLP_W2;
    const double* b2 = P + ORC_MLP_B2;
    const double* W3 = P + ORC_MLP_W3;
    const double* b3 = P + ORC_MLP_B3;
    for (int f = 0; f < ORC_MLP_IN; ++f) xb[f] = maybe_bf16(x[f], emulate);
    for (int j = 0; j < H; ++j) {
        double s = 0.0;
        for (int f = 0; f < ORC_MLP_IN; ++f) s += xb[f] * maybe_bf16(W1[f * H + j], emulate);
        z1[j] = s + b1[j];
        h1[j] = maybe_bf16(z1[j] > 0.0 ? z1[j] : 0.0, emulate);
    }
    for (int j = 0; j < H; ++j) {
        double s = 0.0;
        for (int i = 0; i < H; ++i) s += h1[i] * maybe_bf16(W2[i * H + j], emulate);
        z2[j] = s + b2[j];
        h2[j] = maybe_bf16(z2[j] > 0.0 ? z2[j] : 0.0, emulate);
    }
    for (int k = 0; k < O; ++k) {
        double s = 0.0;
        for (int j = 0; j < H; ++j) s += h2[j] * maybe_bf16(W3[j * O + k], emulate);
        o[k] = s + b3[k];
    }
}

void orc_mlp_forward(const double* P, uint64_t n, const double* x, int emulate, double* out)
{
    double xb[ORC_MLP_IN], z1[ORC_MLP_HIDDEN], h1[ORC_MLP_HIDDEN], z2[ORC_MLP_HIDDEN],
        h2[ORC_MLP_HIDDEN];
    for (uint64_t s = 0; s < n; ++s)
        mlp_forward_keep(P, x + 3 * s, emulate, xb, z1, h1, z2, h2, out + ORC_MLP_OUT * s);
}

/* ------------------------------------------------------ von Mises mixture */

static double softplus(double v) { return v > 20.0 ? v : log1p(exp(v)); }

void orc_vm_mixture(const double* o, double* w, double* mu, double* kappa, double* log_i0)
{
    const int K = ORC_VM_COMPONENTS;
    double mx = o[0];
    for (int k = 1; k < K; ++k)
        if (o[4 * k] > mx) mx = o[4 * k];
    double z = 0.0;
    for (int k = 0; k < K; ++k) {
        w[k] = exp(o[4 * k] - mx);
        z += w[k];
    }
    for (int k = 0; k < K; ++k) {
        w[k] /= z;
        mu[k] = atan2(o[4 * k + 2], o[4 * k + 1]);
        double kp = softplus(o[4 * k + 3]);
        if (kp < ORC_VM_KAPPA_MIN) kp = ORC_VM_KAPPA_MIN;
        if (kp > ORC_VM_KAPPA_MAX) kp = ORC_VM_KAPPA_MAX;
        kappa[k] = kp;
        if (log_i0) log_i0[k] = orc_log_i0(kp);
    }
}

double orc_vm_mixture_logpdf(const double* w, const double* mu, const double* kappa,
                             const double* log_i0, double theta)
{
    const int K = ORC_VM_COMPONENTS;
    double l[ORC_VM_COMPONENTS], mx = -INFINITY;
    for (int k = 0; k < K; ++k) {
        l[k] = log(w[k]) + kappa[k] * cos(theta - mu[k]) - log_i0[k] - log(2.0 * ORC_PI);
        if (l[k] > mx) mx = l[k];
    }
    double s = 0.0;
    for (int k = 0; k < K; ++k) s += exp(l[k] - mx);
    return mx + log(s);
}

/* Best-Fisher von Mises sample around 0 with concentration kappa, from the
 * open keyed stream; returns 0 when ORC_VM_TRIES trials all fail.  The uniform
 * draws are the GPU's FP32 values, u = k 2^-32 rounded to float. */
static double u32f(uint32_t k) { return (double)((float)k * 0x1.0p-32f); }

int orc_vm_trial(double kappa, uint32_t d1, uint32_t d2, uint32_t d3, double* angle)
{
    const double s = 0.5 / kappa;
    const double r = s + sqrt(1.0 + s * s);
    const double u1 = u32f(d1), u2 = u32f(d2);
    const double z = cos(ORC_PI * u1);
    const double f = (1.0 + r * z) / (r + z);
    const double c = kappa * (r - f);
    if (c * (2.0 - c) - u2 > 0.0 || log(c / u2) + 1.0 - c >= 0.0) {
        const double a = acos(f > 1.0 ? 1.0 : (f < -1.0 ? -1.0 : f));
        *angle = (d3 & 0x80000000u) ? a : -a;
        return 1;
    }
    return 0;
}

int orc_vm_sample(orc_pcg32* g, double kappa, double* angle)
{
    for (int t = 0; t < ORC_VM_TRIES; ++t) {
        const uint32_t d1 = orc_pcg32_next(g);
        const uint32_t d2 = orc_pcg32_next(g);
        const uint32_t d3 = orc_pcg32_next(g);
        if (orc_vm_trial(kappa, d1, d2, d3, angle)) return 1;
    }
    return 0;
}

/* Component choice: smallest k with u < w_0 + ... + w_k (last component if
 * rounding leaves u above the total). */
int orc_vm_pick(const double* w, uint32_t d0)
{
    const double u = u32f(d0);
    double c = 0.0;
    for (int k = 0; k < ORC_VM_COMPONENTS - 1; ++k) {
        c += w[k];
        if (u < c) return k;
    }
    return ORC_VM_COMPONENTS - 1;
}

int orc_vm_mixture_sample(orc_pcg32* g, const double* w, const double* mu, const double* kappa,
                          double* theta)
{
    const int k = orc_vm_pick(w, orc_pcg32_next(g));
    double a;
    if (!orc_vm_sample(g, kappa[k], &a)) return 0;
    *theta = remainder(mu[k] + a, 2.0 * ORC_PI);
    return 1;
}

/* --------------------------------------------------------- the loss / grad */

/* NLL of one target angle and its gradient with respect to the 16 outputs. */
static double head_loss_grad(const double* o, double theta, double* dout)
{
    const int K = ORC_VM_COMPONENTS;
    double w[ORC_VM_COMPONENTS], mu[ORC_VM_COMPONENTS], kp[ORC_VM_COMPONENTS], li[ORC_VM_COMPONENTS];
    orc_vm_mixture(o, w, mu, kp, li);
    double l[ORC_VM_COMPONENTS], mx = -INFINITY;
    for (int k = 0; k < K; ++k) {
        l[k] = log(w[k]) + kp[k] * cos(theta - mu[k]) - li[k] - log(2.0 * ORC_PI);
        if (l[k] > mx) mx = l[k];
    }
    double s = 0.0;
    for (int k = 0; k < K; ++k) s += exp(l[k] - mx);
    const double lse = mx + log(s);
    for (int k = 0; k < K; ++k) {
        const double gam = exp(l[k] - lse);
        /* d(-lse)/d logit_k = w_k - gamma_k */
        dout[4 * k] = w[k] - gam;
        /* d(-lse)/d mu_k = -gamma_k kappa_k sin(theta - mu_k); mu = atan2(v, u) */
        const double u = o[4 * k + 1], v = o[4 * k + 2];
        const double rr = u * u + v * v;
        const double dmu = -gam * kp[k] * sin(theta - mu[k]);
        dout[4 * k + 1] = rr > 0.0 ? dmu * (-v / rr) : 0.0;
        dout[4 * k + 2] = rr > 0.0 ? dmu * (u / rr) : 0.0;
        /* d(-lse)/d kappa_k = -gamma_k (cos(theta - mu_k) - I1/I0(kappa_k)) */
        const double raw = softplus(o[4 * k + 3]);
        double dk = 0.0;
        if (raw > ORC_VM_KAPPA_MIN && raw < ORC_VM_KAPPA_MAX) {
            const double sig = 1.0 / (1.0 + exp(-o[4 * k + 3]));
            dk = -gam * (cos(theta - mu[k]) - orc_i1_over_i0(kp[k])) * sig;
        }
        dout[4 * k + 3] = dk;
    }
    return -lse;
}

double orc_mlp_loss_grad(const double* P, uint64_t n, const double* x, const double* theta,
                         int emulate, double* grad)
{
    const int H = ORC_MLP_HIDDEN, O = ORC_MLP_OUT;
    const double* W2 = P + ORC_MLP_W2;
    const double* W3 = P + ORC_MLP_W3;
    if (grad) memset(grad, 0, sizeof(double) * ORC_MLP_PARAMS);
    double loss = 0.0;
    for (uint64_t s = 0; s < n; ++s) {
        double xb[ORC_MLP_IN], z1[64], h1[64], z2[64], h2[64], o[16], dout[16], dh2[64], dh1[64];
        mlp_forward_keep(P, x + 3 * s, emulate, xb, z1, h1, z2, h2, o);
        loss += head_loss_grad(o, theta[s], dout);
        if (!grad) continue;
        for (int k = 0; k < O; ++k) grad[ORC_MLP_B3 + k] += dout[k];
        for (int j = 0; j < H; ++j) {
            double a = 0.0;
            for (int k = 0; k < O; ++k) {
                grad[ORC_MLP_W3 + j * O + k] += h2[j] * dout[k];
                a += maybe_bf16(W3[j * O + k], emulate) * dout[k];
            }
            dh2[j] = z2[j] > 0.0 ? a : 0.0;
            grad[ORC_MLP_B2 + j] += dh2[j];
        }
        for (int i = 0; i < H; ++i) {
            double a = 0.0;
            for (int j = 0; j < H; ++j) {
                grad[ORC_MLP_W2 + i * H + j] += h1[i] * dh2[j];
                a += maybe_bf16(W2[i * H + j], emulate) * dh2[j];
            }
            dh1[i] = z1[i] > 0.0 ? a : 0.0;
            grad[ORC_MLP_B1 + i] += dh1[i];
        }
        for (int f = 0; f < ORC_MLP_IN; ++f)
            for (int j = 0; j < H; ++j) grad[ORC_MLP_W1 + f * H + j] += xb[f] * dh1[j];
    }
    const double inv = n ? 1.0 / (double)n : 0.0;
    if (grad)
        for (int p = 0; p < ORC_MLP_PARAMS; ++p) grad[p] *= inv;
    return loss * inv;
}

void orc_adam_step(uint64_t n, double* p, const double* g, double* m, double* v, uint64_t t,
                   double lr, double b1, double b2, double eps)
{
    const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
    for (uint64_t i = 0; i < n; ++i) {
        m[i] = b1 * m[i] + (1.0 - b1) * g[i];
        v[i] = b2 * v[i] + (1.0 - b2) * g[i] * g[i];
        p[i] -= lr * (m[i] / c1) / (sqrt(v[i] / c2) + eps);
    }
}

/* ------------------------------------------------- the learned U(1) update */

/* cos(theta_p) = cos(theta + phi) for the link at position `which` of cell q
 * (orientation theta_0 + theta_1 - theta_2 - theta_3, dof/u1.hpp plaquette). */
static double staple_phase(const double* th, const uint32_t* q, uint8_t which)
{
    const double t0 = th[q[0]], t1 = th[q[1]], t2 = th[q[2]], t3 = th[q[3]];
    switch (which) {
    case 0: return t1 - t2 - t3;
    case 1: return t0 - t2 - t3;
    case 2: return t3 - t0 - t1;
    default: return t2 - t0 - t1;
    }
}

void orc_u1_learned_metropolis(uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                               const uint64_t* inc_offset, const uint32_t* inc_cell,
                               const uint8_t* inc_which, const double* P, const double* given_out,
                               double model_beta, double driver_beta, uint64_t seed, uint64_t sweep0,
                               uint64_t n_sweeps, double* th, double* obs_out, double* margin_out,
                               double* out_dump, uint8_t* accepted)
{
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        const int last = k + 1 == n_sweeps;
        for (uint64_t i = 0; i < n_links; ++i) {
            double Sr = 0.0, Si = 0.0;
            for (uint64_t a = inc_offset[i]; a < inc_offset[i + 1]; ++a) {
                const double phi = staple_phase(th, cells + 4 * (uint64_t)inc_cell[a], inc_which[a]);
                Sr += cos(phi);
                Si += sin(phi);
            }
            double x[3], o[16];
            orc_u1_features(Sr, Si, x);
            if (given_out) memcpy(o, given_out + 16 * i, sizeof o);
            else orc_mlp_forward(P, 1, x, 1, o);
            if (out_dump && last) memcpy(out_dump + 16 * i, o, sizeof o);
            double w[4], mu[4], kp[4], li[4];
            orc_vm_mixture(o, w, mu, kp, li);
            orc_pcg32 g;
            orc_key_open(&g, seed, counter, ORC_TAG_LEARNED, (uint32_t)i);
            double p;
            int acc = 0;
            double margin = INFINITY;
            if (orc_vm_mixture_sample(&g, w, mu, kp, &p)) {
                /* dE exactly as the plain model computes it: per cell, before - after */
                double d = 0.0;
                for (uint64_t a = inc_offset[i]; a < inc_offset[i + 1]; ++a) {
                    const uint32_t* q = cells + 4 * (uint64_t)inc_cell[a];
                    double t[4] = {th[q[0]], th[q[1]], th[q[2]], th[q[3]]};
                    const double before = cos(t[0] + t[1] - t[2] - t[3]);
                    t[inc_which[a]] = p;
                    const double after = cos(t[0] + t[1] - t[2] - t[3]);
                    d += model_beta * (before - after);
                }
                const double lr = orc_vm_mixture_logpdf(w, mu, kp, li, th[i]) -
                                  orc_vm_mixture_logpdf(w, mu, kp, li, p);
                const double log_p = -driver_beta * d + lr;
                if (log_p >= 0.0) acc = 1;
                else {
                    const double lu = log(orc_pcg32_uni(&g));
                    margin = lu - log_p;
                    acc = lu < log_p;
                }
                if (acc) th[i] = p;
            }
            if (margin_out && last) margin_out[i] = margin;
            if (accepted && last) accepted[i] = (uint8_t)acc;
        }
        if (obs_out) {
            const double Pm = orc_u1_mean_plaquette(n_cells, cells, th);
            obs_out[3 * k + 0] = model_beta * (double)n_cells * (1.0 - Pm);
            obs_out[3 * k + 1] = Pm;
            obs_out[3 * k + 2] = orc_u1_topological_charge(n_cells, cells, th);
        }
    }
}
