/*
 * umc_oracle.h -- CPU oracle for the local-update hot path (TEST INFRASTRUCTURE).
 *
 * This is the checker, not the product.  It is a plain-C, double-precision
 * restatement of the reference library's algorithms (universal_monte_carlo:
 * rng.hpp, driver.hpp, lattice/, dof/, example/, model/, term/) driven by the
 * counter-keyed random stream the GPU path uses.  Only tests/, the package's
 * smoke check and bench.py's CPU-baseline leg may load it.
 *
 * Parity is pinned two ways: (1) against golden vectors produced by the
 * reference's own headers compiled into oracle/_ref (see ref_harness.cpp and
 * tests/golden/make_golden.py), and (2) live against oracle/_ref when that
 * library has been built.
 *
 * Conventions shared with the GPU path
 * ------------------------------------
 *  - Every random draw comes from a reference PCG32 (rng.hpp:8-44) constructed
 *    per key:  Pcg32(id_seed(key_seed(seed, counter, tag), id), 0),
 *      key_seed(s,c,t) = mix64(mix64(s ^ (t << 32)) + c * 0x9E3779B97F4A7C15)
 *      id_seed(k,id)   = mix64(k + (id + 1) * 0x9E3779B97F4A7C15)
 *      mix64           = splitmix64 finaliser (Steele, Lea, Flood 2014)
 *    and draws are consumed sequentially inside the key, exactly as the
 *    reference driver would consume them from one Pcg32.
 *  - counter = sweep index for Metropolis, flip index for Wolff.
 *  - id = colour-major site index (Metropolis), edge-list index (Wolff bond),
 *    0 (Wolff axis and seed draw), link index (gauge).
 *  - tag: UMC_TAG_SITE(h) for Metropolis hit h, UMC_TAG_BOND, UMC_TAG_AXIS ...
 *  - Sites are visited in index order (driver.hpp:34); callers pass tables
 *    that are already relabelled colour-major, so index order == colour order.
 */
#ifndef UMC_ORACLE_H
#define UMC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_TAG_BOND 1u
#define ORC_TAG_AXIS 2u
#define ORC_TAG_INIT 3u
#define ORC_TAG_SWAP 4u
#define ORC_TAG_SITE(h) (0x100u + (uint32_t)(h))

/* ---- RNG (rng.hpp:8-44) --------------------------------------------------- */
typedef struct {
    uint64_t state;
    uint64_t inc;
} orc_pcg32;

void     orc_pcg32_seed(orc_pcg32* g, uint64_t seed, uint64_t stream);
uint32_t orc_pcg32_next(orc_pcg32* g);
double   orc_pcg32_uni(orc_pcg32* g);
uint64_t orc_mix64(uint64_t z);
uint64_t orc_key_seed(uint64_t seed, uint64_t counter, uint32_t tag);
uint64_t orc_id_seed(uint64_t kseed, uint32_t id);
uint32_t orc_stream_id(uint32_t id); /* lowbias32: union-find linking priority */
void     orc_key_open(orc_pcg32* g, uint64_t seed, uint64_t counter, uint32_t tag, uint32_t id);
/* n raw 32-bit outputs of the keyed stream */
void     orc_key_draws(uint64_t seed, uint64_t counter, uint32_t tag, uint32_t id,
                       uint32_t n, uint32_t* out);
/* n raw outputs of a plain Pcg32(seed, stream) */
void     orc_pcg32_draws(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out);

/* ---- tables ------------------------------------------------------------------ */
/* Status codes mirror the reference builders' exceptions. */
#define ORC_OK 0
#define ORC_ERR_OUT_OF_RANGE -1   /* std::out_of_range   */
#define ORC_ERR_INVALID -2        /* std::invalid_argument */
#define ORC_ERR_OVERFLOW -3       /* std::overflow_error */

/* PairGraph CSR (lattice/pair_graph.hpp:49-83).  offset has n+1 entries; bonds
 * and slot_edge have offset[n] entries (call with bonds==NULL to size). */
int orc_pair_graph(uint64_t n, const uint32_t* ei, const uint32_t* ej, uint64_t m,
                   int symmetric, uint32_t* offset, uint32_t* bonds, uint32_t* slot_edge);
/* square_lattice edge list (lattice/square.hpp:15-38); returns edge count. */
int64_t orc_square_edges(uint64_t Lx, uint64_t Ly, uint32_t* ei, uint32_t* ej);
/* periodic cubic edge list, same conventions (+x,+y,+z per site, site=(z*Ly+y)*Lx+x). */
int64_t orc_cubic_edges(uint64_t Lx, uint64_t Ly, uint64_t Lz, uint32_t* ei, uint32_t* ej);
/* hypercubic_plaquettes cells (lattice/hypercubic.hpp:15-64): 6 L^4 x 4 site ids. */
int64_t orc_hypercubic_cells(uint64_t L, uint32_t* cells);
/* 2D periodic plaquettes, same orientation rule: links mu*L^2 + y*L + x. */
int64_t orc_square_plaquette_cells(uint64_t L, uint32_t* cells);
/* CellComplex incidence (lattice/cell_complex.hpp:36-63).  offset: n+1 entries. */
int orc_cell_incidence(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells,
                       uint64_t* offset, uint32_t* inc_cell, uint8_t* inc_which);
/* 1 if no two sites of one colour share a bond (symmetrised), else 0. */
int orc_check_colouring(uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                        const uint32_t* colour);
/* 1 if no two sites of one colour share a cell, else 0. */
int orc_check_cell_colouring(uint64_t n_sites, uint32_t arity, const uint32_t* cells,
                             uint64_t n_cells, const uint32_t* colour);

/* ---- Ising (example/ising.hpp) under Metropolis / Wolff (driver.hpp) ----------
 * spins: int8 in {-1,+1}, updated in place.  E_out / M_out: one entry per sweep
 * or flip (may be NULL); E = 0.5 * sum_i energy_at(i).  Metropolis draws one
 * uniform per site (Flip draws none): site i reads output i % ORC_GROUP_SITES of
 * the keyed stream of id i / ORC_GROUP_SITES. */
#define ORC_GROUP_SITES 16
void orc_ising_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, int32_t J,
                          double beta, uint64_t seed, uint64_t sweep0, uint64_t n_sweeps,
                          int8_t* spins, double* E_out, double* M_out);
void orc_ising_wolff(uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                     const uint32_t* slot_edge, int32_t J, double beta, uint64_t seed,
                     uint64_t flip0, uint64_t n_flips, int8_t* spins, uint64_t* sizes,
                     double* E_out, double* M_out);

/* ---- weighted Ising: the reference graph test's IsingGraph (test/graph_check.cpp:
 * 34-83) on a PairGraph<double>, c[a] the coupling of CSR slot a ---------------------
 * spins: doubles in {-1,+1}, updated in place.  Metropolis with the test's Flip:
 * site i's accept draw is the first output of its keyed stream (id i); margin_out
 * (may be NULL) as in orc_vector_metropolis.  Wolff with r = 1: the bond in slot a
 * draws from key[a].  E_out (may be NULL): 0.5 * sum_i energy_at(i) per sweep/flip. */
void orc_weighted_ising_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, const double* c,
                                   double beta, uint64_t seed, uint64_t sweep0, uint64_t n_sweeps, double* spins,
                                   double* E_out, double* margin_out);
void orc_weighted_ising_wolff(uint64_t n, const uint32_t* offset, const uint32_t* bonds, const uint32_t* key,
                              const double* c, double beta, uint64_t seed, uint64_t flip0, uint64_t n_flips,
                              double* spins, uint64_t* sizes, double* E_out);

/* ---- VectorSpin<N> (example/vector_spin.hpp) -------------------------------------
 * spins: n*N doubles.  proposal: 0 = UniformSphereN<N>, 1 = LocalRotation<N>{delta}.
 * obs_out (may be NULL): per sweep/flip, [E, M_0 .. M_{N-1}]  (stride N+1).
 * margin_out (may be NULL): per site of the LAST sweep, log(u) - log_p of the
 * accept test (+inf when log_p >= 0, i.e. accepted without a draw), and 0 when
 * the LocalRotation frame was ill-conditioned (|v - (v.u) u| < ORC_FRAME_TOL:
 * FP32 rounding of u, v grows by 1/|v - (v.u) u| in the candidate). */
#define ORC_PROP_SPHERE 0
#define ORC_PROP_ROTATION 1
#define ORC_FRAME_TOL 0.1
void orc_vector_metropolis(uint32_t N, uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                           double J, double beta, int proposal, double delta, uint64_t seed,
                           uint64_t sweep0, uint64_t n_sweeps, double* spins, double* obs_out,
                           double* margin_out);
void orc_vector_wolff(uint32_t N, uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                      const uint32_t* slot_edge, double J, double beta, uint64_t seed,
                      uint64_t flip0, uint64_t n_flips, double* spins, uint64_t* sizes,
                      double* obs_out, double* margin_out);
/* UniformSphereN<N> sample from the keyed stream (dof/vector.hpp:35-61). */
void orc_sphere_sample(uint32_t N, orc_pcg32* g, double* out);

/* ---- XY model on angles: PairModel<U1Dof, XY pair term> with U1Shift --------------
 * theta: n angles.  E = -J sum cos(theta_i - theta_j).  obs: [E, Mx, My]. */
void orc_xy_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, double J,
                       double beta, double width, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* theta, double* obs_out, double* margin_out);

/* ---- replica exchange (no reference counterpart) ------------------------------
 * One exchange round of a ladder of R replicas (temperature slots 0..R-1 with
 * inverse temperatures betas[k]).  holder[k] = chain currently at slot k,
 * energy[c] = energy of chain c.  Pairs (k, k+1) with k = parity, parity+2, ...
 * are proposed; the swap is accepted iff Delta >= 0 or log(u) < Delta with
 * Delta = (betas[k] - betas[k+1]) * (energy[holder[k]] - energy[holder[k+1]])
 * and u the first draw of key (seed, round, ORC_TAG_SWAP, k).  accepted[k]
 * (may be NULL) receives 1/0 per proposed pair.  Returns the number accepted. */
int orc_replica_exchange(uint32_t R, const double* betas, uint32_t* holder, const double* energy,
                         uint64_t seed, uint64_t round, uint32_t parity, uint8_t* accepted);

/* ---- U(1) gauge on a cell complex (example/u1_gauge.hpp, model/cell.hpp + term/plaquette.hpp)
 * theta: n_links angles.  model_beta multiplies the action, driver_beta the exponent.
 * hits: number of U1Shift hits per link (multi-hit; 1 = the reference sweep).
 * obs: per sweep [S, mean plaquette]. */
void orc_u1_metropolis(uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                       const uint64_t* inc_offset, const uint32_t* inc_cell,
                       const uint8_t* inc_which, double model_beta, double driver_beta,
                       double width, uint32_t hits, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* theta, double* obs_out, double* margin_out);
double orc_u1_mean_plaquette(uint64_t n_cells, const uint32_t* cells, const double* theta);
/* 2D topological charge Q = (1/2pi) sum_p remainder(theta_p, 2pi). */
double orc_u1_topological_charge(uint64_t n_cells, const uint32_t* cells, const double* theta);

/* ---- SU(N) gauge (example/sun_gauge.hpp, dof/sun.hpp) --------------------------------
 * links: n_links * N*N complex numbers as interleaved (re, im) doubles, row-major.
 * obs: per sweep [S, mean plaquette]. */
void orc_su_metropolis(uint32_t N, uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                       const uint64_t* inc_offset, const uint32_t* inc_cell,
                       const uint8_t* inc_which, double model_beta, double driver_beta,
                       double width, uint32_t hits, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* links, double* obs_out, double* margin_out);
double orc_su_mean_plaquette(uint32_t N, uint64_t n_cells, const uint32_t* cells,
                             const double* links);
/* SUShift<N>::sample on one link (dof/sun.hpp:163-204) from the keyed stream. */
void orc_su_shift(uint32_t N, double width, orc_pcg32* g, const double* cur, double* out);
/* sun_detail::expm (dof/sun.hpp:118-146). a, out: N*N interleaved complex. */
void orc_su_expm(uint32_t N, const double* a, double* out);
/* max_ij |(U^dagger U - I)_ij| (dof/sun.hpp:43-54). */
double orc_su_unitarity_error(uint32_t N, const double* u);

/* ---- learned U(1) proposal (umc_oracle_learn.c; no reference counterpart) -------
 * Parameters: FP32 master values packed W1[3][64], b1[64], W2[64][64], b2[64],
 * W3[64][16], b3[16] (row = input unit).  Outputs per link: 4 components x
 * (logit, u, v, pre-softplus concentration), mean = atan2(v, u). */
#define ORC_TAG_LEARN 5u   /* training minibatch selection */
#define ORC_TAG_LEARNED 6u /* learned Metropolis-Hastings update, id = link */
#define ORC_MLP_IN 3
#define ORC_MLP_HIDDEN 64
#define ORC_MLP_OUT 16
#define ORC_MLP_W1 0
#define ORC_MLP_B1 (ORC_MLP_W1 + ORC_MLP_IN * ORC_MLP_HIDDEN)
#define ORC_MLP_W2 (ORC_MLP_B1 + ORC_MLP_HIDDEN)
#define ORC_MLP_B2 (ORC_MLP_W2 + ORC_MLP_HIDDEN * ORC_MLP_HIDDEN)
#define ORC_MLP_W3 (ORC_MLP_B2 + ORC_MLP_HIDDEN)
#define ORC_MLP_B3 (ORC_MLP_W3 + ORC_MLP_HIDDEN * ORC_MLP_OUT)
#define ORC_MLP_PARAMS (ORC_MLP_B3 + ORC_MLP_OUT)
#define ORC_VM_COMPONENTS 4
#define ORC_VM_KAPPA_MIN 1e-4
#define ORC_VM_KAPPA_MAX 80.0
#define ORC_VM_TRIES 32

double orc_bf16(double v);
double orc_log_i0(double x);
double orc_i1_over_i0(double x);
/* x[3] = (cos a, sin a, |S|) of the staple sum S = Sr + i Si ((1, 0, 0) for S = 0). */
void orc_u1_features(double Sr, double Si, double* x);
/* out[n][16]; emulate != 0 rounds operands to BF16 as the tensor-core path does. */
void orc_mlp_forward(const double* params, uint64_t n, const double* x, int emulate, double* out);
/* Mixture parameters of one output row; log_i0 may be NULL. */
void orc_vm_mixture(const double* out16, double* w, double* mu, double* kappa, double* log_i0);
double orc_vm_mixture_logpdf(const double* w, const double* mu, const double* kappa,
                             const double* log_i0, double theta);
/* Best-Fisher sample around 0; returns 0 if every trial was rejected. */
int orc_vm_sample(orc_pcg32* g, double kappa, double* angle);
/* One Best-Fisher trial from three raw draws (d3's top bit picks the sign). */
int orc_vm_trial(double kappa, uint32_t d1, uint32_t d2, uint32_t d3, double* angle);
/* Component index from one raw draw: smallest k with u < w_0 + ... + w_k. */
int orc_vm_pick(const double* w, uint32_t d0);
int orc_vm_mixture_sample(orc_pcg32* g, const double* w, const double* mu, const double* kappa,
                          double* theta);
/* Mean negative log-likelihood of targets theta[n] under the mixture the network
 * gives for x[n][3]; grad (may be NULL) receives its gradient (ORC_MLP_PARAMS). */
double orc_mlp_loss_grad(const double* params, uint64_t n, const double* x, const double* theta,
                         int emulate, double* grad);
/* One Adam step (Kingma & Ba 2015) with bias correction at step t >= 1. */
void orc_adam_step(uint64_t n, double* p, const double* g, double* m, double* v, uint64_t t,
                   double lr, double b1, double b2, double eps);
/* Learned-proposal Metropolis-Hastings sweeps of U(1) links in index order
 * (tables relabelled colour-major by the caller).  given_out (n_links x 16, one
 * sweep only) replaces the network's outputs; out_dump receives the outputs of
 * the last sweep.  obs per sweep: [S, mean plaquette, Q].  margin_out: log u -
 * log_p of the accept test (+inf when accepted without a draw or no proposal). */
void orc_u1_learned_metropolis(uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                               const uint64_t* inc_offset, const uint32_t* inc_cell,
                               const uint8_t* inc_which, const double* params,
                               const double* given_out, double model_beta, double driver_beta,
                               uint64_t seed, uint64_t sweep0, uint64_t n_sweeps, double* theta,
                               double* obs_out, double* margin_out, double* out_dump,
                               uint8_t* accepted);

#ifdef __cplusplus
}
#endif
#endif
