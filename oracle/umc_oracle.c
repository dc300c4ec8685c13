/*
 * umc_oracle.c -- CPU oracle (TEST INFRASTRUCTURE; see umc_oracle.h).
 *
 * Double-precision restatement of the reference algorithms.  Every function
 * cites the reference file:line it follows.  Expressions are written in the
 * reference's evaluation order so that, built without FMA contraction, the
 * results agree bit-for-bit with the reference headers compiled in oracle/_ref.
 */
#include "umc_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ RNG */

/* Pcg32 constructor, rng.hpp:14-20: state=0, inc=(stream<<1)|1, advance, add
 * seed, advance. */
void orc_pcg32_seed(orc_pcg32* g, uint64_t seed, uint64_t stream)
{
    g->state = 0;
    g->inc = (stream << 1u) | 1u;
    (void)orc_pcg32_next(g);
    g->state += seed;
    (void)orc_pcg32_next(g);
}

/* Pcg32::next, rng.hpp:31-40 (XSH-RR output of the old state). */
uint32_t orc_pcg32_next(orc_pcg32* g)
{
    const uint64_t old = g->state;
    g->state = old * 6364136223846793005ULL + g->inc;
    const uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((32u - rot) & 31u));
}

/* Pcg32::uni, rng.hpp:24-27: k * 2^-32. */
double orc_pcg32_uni(orc_pcg32* g) { return orc_pcg32_next(g) * 0x1.0p-32; }

/* splitmix64 finaliser (Steele, Lea, Flood, OOPSLA 2014). */
uint64_t orc_mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return z;
}

uint64_t orc_key_seed(uint64_t seed, uint64_t counter, uint32_t tag)
{
    return orc_mix64(orc_mix64(seed ^ ((uint64_t)tag << 32)) + counter * 0x9E3779B97F4A7C15ULL);
}

/* lowbias32 integer hash (C. Wellons, 2018); every step is invertible.  The
 * GPU's union-find linking priority of a site. */
uint32_t orc_stream_id(uint32_t x)
{
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

uint64_t orc_id_seed(uint64_t kseed, uint32_t id)
{
    return orc_mix64(kseed + ((uint64_t)id + 1ULL) * 0x9E3779B97F4A7C15ULL);
}

void orc_key_open(orc_pcg32* g, uint64_t seed, uint64_t counter, uint32_t tag, uint32_t id)
{
    orc_pcg32_seed(g, orc_id_seed(orc_key_seed(seed, counter, tag), id), 0);
}

void orc_key_draws(uint64_t seed, uint64_t counter, uint32_t tag, uint32_t id, uint32_t n,
                   uint32_t* out)
{
    orc_pcg32 g;
    orc_key_open(&g, seed, counter, tag, id);
    for (uint32_t k = 0; k < n; ++k) out[k] = orc_pcg32_next(&g);
}

void orc_pcg32_draws(uint64_t seed, uint64_t stream, uint32_t n, uint32_t* out)
{
    orc_pcg32 g;
    orc_pcg32_seed(&g, seed, stream);
    for (uint32_t k = 0; k < n; ++k) out[k] = orc_pcg32_next(&g);
}

/* --------------------------------------------------------------------- tables */

/* PairGraph(n, edges, symmetric), lattice/pair_graph.hpp:49-83: degree count,
 * exclusive scan, scatter in edge-list order.  slot_edge records which input
 * edge produced each stored slot (the reference's Bond carries only j). */
int orc_pair_graph(uint64_t n, const uint32_t* ei, const uint32_t* ej, uint64_t m, int symmetric,
                   uint32_t* offset, uint32_t* bonds, uint32_t* slot_edge)
{
    if (n > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    uint64_t* degree = (uint64_t*)calloc(n + 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < m; ++e) {
        if (ei[e] >= n || ej[e] >= n) { free(degree); return ORC_ERR_OUT_OF_RANGE; }
        if (ei[e] == ej[e]) { free(degree); return ORC_ERR_INVALID; }
        ++degree[ei[e]];
        if (symmetric) ++degree[ej[e]];
    }
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        offset[i] = (uint32_t)total;
        total += degree[i];
        if (total > 0xFFFFFFFFull) { free(degree); return ORC_ERR_OVERFLOW; }
    }
    offset[n] = (uint32_t)total;
    if (bonds) {
        for (uint64_t i = 0; i < n; ++i) degree[i] = offset[i];  /* reuse as cursor */
        for (uint64_t e = 0; e < m; ++e) {
            const uint64_t a = degree[ei[e]]++;
            bonds[a] = ej[e];
            if (slot_edge) slot_edge[a] = (uint32_t)e;
            if (symmetric) {
                const uint64_t b = degree[ej[e]]++;
                bonds[b] = ei[e];
                if (slot_edge) slot_edge[b] = (uint32_t)e;
            }
        }
    }
    free(degree);
    return ORC_OK;
}

/* square_lattice, lattice/square.hpp:15-38: site y*Lx+x; per site a +x edge if
 * Lx>1, then a +y edge if Ly>1. */
int64_t orc_square_edges(uint64_t Lx, uint64_t Ly, uint32_t* ei, uint32_t* ej)
{
    if (Lx == 0 || Ly == 0) return ORC_ERR_INVALID;
    if (Lx * Ly > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    int64_t m = 0;
    for (uint64_t y = 0; y < Ly; ++y)
        for (uint64_t x = 0; x < Lx; ++x) {
            const uint32_t i = (uint32_t)(y * Lx + x);
            if (Lx > 1) {
                if (ei) { ei[m] = i; ej[m] = (uint32_t)(y * Lx + (x + 1) % Lx); }
                ++m;
            }
            if (Ly > 1) {
                if (ei) { ei[m] = i; ej[m] = (uint32_t)(((y + 1) % Ly) * Lx + x); }
                ++m;
            }
        }
    return m;
}

/* Periodic cubic lattice with the square_lattice conventions extended to 3D
 * (the reference ships no 3D builder). */
int64_t orc_cubic_edges(uint64_t Lx, uint64_t Ly, uint64_t Lz, uint32_t* ei, uint32_t* ej)
{
    if (Lx == 0 || Ly == 0 || Lz == 0) return ORC_ERR_INVALID;
    if (Lx * Ly * Lz > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    int64_t m = 0;
    for (uint64_t z = 0; z < Lz; ++z)
        for (uint64_t y = 0; y < Ly; ++y)
            for (uint64_t x = 0; x < Lx; ++x) {
                const uint32_t i = (uint32_t)((z * Ly + y) * Lx + x);
                if (Lx > 1) {
                    if (ei) { ei[m] = i; ej[m] = (uint32_t)((z * Ly + y) * Lx + (x + 1) % Lx); }
                    ++m;
                }
                if (Ly > 1) {
                    if (ei) { ei[m] = i; ej[m] = (uint32_t)((z * Ly + (y + 1) % Ly) * Lx + x); }
                    ++m;
                }
                if (Lz > 1) {
                    if (ei) { ei[m] = i; ej[m] = (uint32_t)((((z + 1) % Lz) * Ly + y) * Lx + x); }
                    ++m;
                }
            }
    return m;
}

/* hypercubic_plaquettes, lattice/hypercubic.hpp:15-64: links mu*L^4 +
 * ((t*L+z)*L+y)*L+x, plaquette (mu<nu) = [U_mu(c), U_nu(c+mu), U_mu(c+nu), U_nu(c)]
 * with c = {t,z,y,x} and direction mu stepping coordinate c[mu]. */
int64_t orc_hypercubic_cells(uint64_t L, uint32_t* cells)
{
    if (L == 0) return ORC_ERR_INVALID;
    const uint64_t L4 = L * L * L * L;
    if (4 * L4 > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    int64_t m = 0;
    for (uint64_t mu = 0; mu < 4; ++mu)
        for (uint64_t nu = mu + 1; nu < 4; ++nu)
            for (uint64_t t = 0; t < L; ++t)
                for (uint64_t z = 0; z < L; ++z)
                    for (uint64_t y = 0; y < L; ++y)
                        for (uint64_t x = 0; x < L; ++x) {
                            uint64_t c[4] = {t, z, y, x}, cm[4], cn[4];
                            memcpy(cm, c, sizeof c);
                            memcpy(cn, c, sizeof c);
                            cm[mu] = (cm[mu] + 1) % L;
                            cn[nu] = (cn[nu] + 1) % L;
#define ORC_IDX(d, v) ((d) * L4 + (((v)[0] * L + (v)[1]) * L + (v)[2]) * L + (v)[3])
                            if (cells) {
                                cells[4 * m + 0] = (uint32_t)ORC_IDX(mu, c);
                                cells[4 * m + 1] = (uint32_t)ORC_IDX(nu, cm);
                                cells[4 * m + 2] = (uint32_t)ORC_IDX(mu, cn);
                                cells[4 * m + 3] = (uint32_t)ORC_IDX(nu, c);
                            }
#undef ORC_IDX
                            ++m;
                        }
    return m;
}

/* Two-dimensional analogue of hypercubic_plaquettes (no reference builder):
 * links mu*L^2 + y*L + x with mu=0 stepping x and mu=1 stepping y; one
 * plaquette per site, [U_0(c), U_1(c+x), U_0(c+y), U_1(c)]. */
int64_t orc_square_plaquette_cells(uint64_t L, uint32_t* cells)
{
    if (L == 0) return ORC_ERR_INVALID;
    const uint64_t L2 = L * L;
    if (2 * L2 > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    int64_t m = 0;
    for (uint64_t y = 0; y < L; ++y)
        for (uint64_t x = 0; x < L; ++x) {
            if (cells) {
                cells[4 * m + 0] = (uint32_t)(0 * L2 + y * L + x);
                cells[4 * m + 1] = (uint32_t)(1 * L2 + y * L + (x + 1) % L);
                cells[4 * m + 2] = (uint32_t)(0 * L2 + ((y + 1) % L) * L + x);
                cells[4 * m + 3] = (uint32_t)(1 * L2 + y * L + x);
            }
            ++m;
        }
    return m;
}

/* CellComplex constructor, lattice/cell_complex.hpp:36-63. */
int orc_cell_incidence(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells,
                       uint64_t* offset, uint32_t* inc_cell, uint8_t* inc_which)
{
    if (n_sites > 0xFFFFFFFFull || n_cells > 0xFFFFFFFFull) return ORC_ERR_OVERFLOW;
    memset(offset, 0, (n_sites + 1) * sizeof(uint64_t));
    for (uint64_t c = 0; c < n_cells; ++c)
        for (uint32_t k = 0; k < arity; ++k) {
            const uint32_t s = cells[c * arity + k];
            if (s >= n_sites) return ORC_ERR_OUT_OF_RANGE;
            ++offset[s + 1];
        }
    for (uint64_t i = 0; i < n_sites; ++i) offset[i + 1] += offset[i];
    if (inc_cell) {
        uint64_t* cursor = (uint64_t*)malloc((n_sites + 1) * sizeof(uint64_t));
        memcpy(cursor, offset, (n_sites + 1) * sizeof(uint64_t));
        for (uint64_t c = 0; c < n_cells; ++c)
            for (uint32_t k = 0; k < arity; ++k) {
                const uint32_t s = cells[c * arity + k];
                const uint64_t a = cursor[s]++;
                inc_cell[a] = (uint32_t)c;
                inc_which[a] = (uint8_t)k;
            }
        free(cursor);
    }
    return ORC_OK;
}

int orc_check_colouring(uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                        const uint32_t* colour)
{
    for (uint64_t i = 0; i < n; ++i)
        for (uint32_t a = offset[i]; a < offset[i + 1]; ++a)
            if (colour[bonds[a]] == colour[i]) return 0;
    return 1;
}

int orc_check_cell_colouring(uint64_t n_sites, uint32_t arity, const uint32_t* cells,
                             uint64_t n_cells, const uint32_t* colour)
{
    (void)n_sites;
    for (uint64_t c = 0; c < n_cells; ++c)
        for (uint32_t a = 0; a < arity; ++a)
            for (uint32_t b = a + 1; b < arity; ++b) {
                const uint32_t sa = cells[c * arity + a], sb = cells[c * arity + b];
                if (sa != sb && colour[sa] == colour[sb]) return 0;
            }
    return 1;
}

/* ----------------------------------------------------------------------- Ising */

/* Ising::energy_at, example/ising.hpp:35-43. */
static int32_t ising_energy_at(const uint32_t* offset, const uint32_t* bonds, int32_t J,
                               const int8_t* s, uint64_t i)
{
    int32_t e = 0;
    for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) e += -J * ((int32_t)s[i] * (int32_t)s[bonds[a]]);
    return e;
}

static void ising_observe(uint64_t n, const uint32_t* offset, const uint32_t* bonds, int32_t J,
                          const int8_t* s, double* E, double* M)
{
    double e = 0.0, m = 0.0;
    for (uint64_t i = 0; i < n; ++i) {
        e += (double)ising_energy_at(offset, bonds, J, s, i);
        m += (double)s[i];
    }
    if (E) *E = 0.5 * e;
    if (M) *M = m;
}

/* Metropolis::sweep (driver.hpp:29-43) over Ising (example/ising.hpp:46-56)
 * with Flip (dof/ising.hpp:27-38). */
void orc_ising_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, int32_t J,
                          double beta, uint64_t seed, uint64_t sweep0, uint64_t n_sweeps,
                          int8_t* s, double* E_out, double* M_out)
{
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n; ++i) {
            /* one draw per site: output i % 16 of the stream of id i / 16 */
            orc_pcg32 g;
            orc_key_open(&g, seed, counter, ORC_TAG_SITE(0), (uint32_t)(i / ORC_GROUP_SITES));
            for (uint64_t q = 0; q < i % ORC_GROUP_SITES; ++q) orc_pcg32_next(&g);
            const int8_t old = s[i];
            const int8_t p = (int8_t)(-old);
            int32_t d = 0;
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const int8_t sj = s[bonds[a]];
                d += -J * ((int32_t)p * sj - (int32_t)old * sj);
            }
            const double dE = (double)d;
            const double log_p = -beta * dE + 0.0;
            if (log_p >= 0.0 || log(orc_pcg32_uni(&g)) < log_p) s[i] = p;
        }
        ising_observe(n, offset, bonds, J, s, E_out ? E_out + k : NULL, M_out ? M_out + k : NULL);
    }
}

/* Wolff::flip (driver.hpp:104-162) with FixedAxis (dof/ising.hpp:41-49) and
 * Ising::energy_diff_bond (example/ising.hpp:59-65). */
void orc_ising_wolff(uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                     const uint32_t* slot_edge, int32_t J, double beta, uint64_t seed,
                     uint64_t flip0, uint64_t n_flips, int8_t* s, uint64_t* sizes, double* E_out,
                     double* M_out)
{
    char* in_cluster = (char*)malloc(n ? n : 1);
    uint64_t* stack = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    for (uint64_t f = 0; f < n_flips; ++f) {
        const uint64_t counter = flip0 + f;
        orc_pcg32 g;
        orc_key_open(&g, seed, counter, ORC_TAG_AXIS, 0);
        const int8_t r = 1;
        memset(in_cluster, 0, n);
        const uint64_t seed_site = (uint64_t)(orc_pcg32_uni(&g) * (double)n);
        in_cluster[seed_site] = 1;
        stack[0] = seed_site;
        uint64_t top = 1, cluster = 0;
        while (top > 0) {
            const uint64_t i = stack[--top];
            ++cluster;
            const int8_t si = s[i];
            const int8_t dot = (int8_t)(si * r);
            const int8_t prop = (int8_t)(si - 2 * dot * r);
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const uint32_t j = bonds[a];
                if (in_cluster[j]) continue;
                const int8_t t = s[j];
                const int8_t d = (int8_t)(t * r);
                const int8_t nb = (int8_t)(t - 2 * d * r);
                const int32_t de = -J * ((int32_t)nb * si - (int32_t)t * si);
                const double dE = (double)de;
                orc_pcg32 gb;
                orc_key_open(&gb, seed, counter, ORC_TAG_BOND, slot_edge[a]);
                if (orc_pcg32_uni(&gb) < 1.0 - exp(-beta * dE)) {
                    in_cluster[j] = 1;
                    stack[top++] = j;
                }
            }
            s[i] = prop;
        }
        if (sizes) sizes[f] = cluster;
        ising_observe(n, offset, bonds, J, s, E_out ? E_out + f : NULL, M_out ? M_out + f : NULL);
    }
    free(in_cluster);
    free(stack);
}

/* ------------------------------------------------- weighted Ising (bond payload)
 * The reference graph test's IsingGraph (test/graph_check.cpp:34-83): double
 * spins, coupling c[a] carried by CSR slot a (PairGraph<double>'s Bond::c).  */

static double wising_energy_at(const uint32_t* offset, const uint32_t* bonds, const double* c, const double* s,
                               uint64_t i)
{
    double e = 0.0; /* IsingGraph::energy_at, test/graph_check.cpp:47-54 */
    for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) e += -c[a] * s[i] * s[bonds[a]];
    return e;
}

static double wising_half_energy(uint64_t n, const uint32_t* offset, const uint32_t* bonds, const double* c,
                                 const double* s)
{
    double e = 0.0;
    for (uint64_t i = 0; i < n; ++i) e += wising_energy_at(offset, bonds, c, s, i);
    return 0.5 * e;
}

/* Metropolis::sweep (driver.hpp:29-43) over IsingGraph with the test's Flip
 * (test/graph_check.cpp:15-24): site i opens its own keyed stream (id i), the
 * accept test takes its first output. */
void orc_weighted_ising_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, const double* c,
                                   double beta, uint64_t seed, uint64_t sweep0, uint64_t n_sweeps, double* s,
                                   double* E_out, double* margin_out)
{
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n; ++i) {
            orc_pcg32 g;
            orc_key_open(&g, seed, counter, ORC_TAG_SITE(0), (uint32_t)i);
            const double p = s[i] > 0.0 ? -1.0 : 1.0;
            double d = 0.0; /* IsingGraph::energy_diff_at, test/graph_check.cpp:58-65 */
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) d += -c[a] * (p - s[i]) * s[bonds[a]];
            const double log_p = -beta * d + 0.0;
            int accept;
            double margin = INFINITY;
            if (log_p >= 0.0) accept = 1;
            else {
                const double lu = log(orc_pcg32_uni(&g));
                margin = lu - log_p;
                accept = lu < log_p;
            }
            if (margin_out && k + 1 == n_sweeps) margin_out[i] = margin;
            if (accept) s[i] = p;
        }
        if (E_out) E_out[k] = wising_half_energy(n, offset, bonds, c, s);
    }
}

/* Wolff::flip (driver.hpp:104-162) over IsingGraph with the fixed axis r = 1
 * (test/graph_check.cpp:27-32) and IsingGraph::energy_diff_bond (:67-70); the
 * uniform of the bond in slot a is keyed by key[a]. */
void orc_weighted_ising_wolff(uint64_t n, const uint32_t* offset, const uint32_t* bonds, const uint32_t* key,
                              const double* c, double beta, uint64_t seed, uint64_t flip0, uint64_t n_flips,
                              double* s, uint64_t* sizes, double* E_out)
{
    char* in_cluster = (char*)malloc(n ? n : 1);
    uint64_t* stack = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    for (uint64_t f = 0; f < n_flips; ++f) {
        const uint64_t counter = flip0 + f;
        orc_pcg32 g;
        orc_key_open(&g, seed, counter, ORC_TAG_AXIS, 0);
        const double r = 1.0;
        memset(in_cluster, 0, n);
        const uint64_t seed_site = (uint64_t)(orc_pcg32_uni(&g) * (double)n);
        in_cluster[seed_site] = 1;
        stack[0] = seed_site;
        uint64_t top = 1, cluster = 0;
        while (top > 0) {
            const uint64_t i = stack[--top];
            ++cluster;
            const double si = s[i];
            const double prop = si - 2.0 * (si * r) * r;
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const uint32_t j = bonds[a];
                if (in_cluster[j]) continue;
                const double t = s[j];
                const double nb = t - 2.0 * (t * r) * r;
                const double dE = -c[a] * (nb - s[j]) * si;
                orc_pcg32 gb;
                orc_key_open(&gb, seed, counter, ORC_TAG_BOND, key[a]);
                if (orc_pcg32_uni(&gb) < 1.0 - exp(-beta * dE)) {
                    in_cluster[j] = 1;
                    stack[top++] = j;
                }
            }
            s[i] = prop;
        }
        if (sizes) sizes[f] = cluster;
        if (E_out) E_out[f] = wising_half_energy(n, offset, bonds, c, s);
    }
    free(in_cluster);
    free(stack);
}

/* ------------------------------------------------------------------ VectorSpin */

static const double ORC_PI = 3.141592653589793238462643383279502884;

/* dot<N>, dof/vector.hpp:23-31. */
static double vdot(uint32_t N, const double* a, const double* b)
{
    double s = 0.0;
    for (uint32_t k = 0; k < N; ++k) s += a[k] * b[k];
    return s;
}

/* UniformSphereN<N, double>::sample, dof/vector.hpp:35-61 (recursive height
 * method: N==1 sign, N==2 angle, N>=3 uniform height then recurse). */
void orc_sphere_sample(uint32_t N, orc_pcg32* g, double* out)
{
    if (N == 1) {
        out[0] = orc_pcg32_uni(g) < 0.5 ? -1.0 : 1.0;
    } else if (N == 2) {
        const double phi = 2.0 * ORC_PI * orc_pcg32_uni(g);
        out[0] = cos(phi);
        out[1] = sin(phi);
    } else {
        const double z = 2.0 * orc_pcg32_uni(g) - 1.0;
        const double r = sqrt(1.0 - z * z);
        orc_sphere_sample(N - 1, g, out);
        for (uint32_t k = 0; k < N - 1; ++k) out[k] *= r;
        out[N - 1] = z;
    }
}

/* LocalRotation<N, double>::sample, dof/vector.hpp:70-122.  Returns |v - (v.u) u|
 * of the accepted frame: rounding of u and v (FP32 on the GPU) is amplified by
 * its inverse in the normalised second axis. */
static double local_rotation(uint32_t N, double delta, orc_pcg32* g, const double* cur, double* out)
{
    double u[8] = {0}, v[8] = {0}, frame = 0.0;
    orc_sphere_sample(N, g, u);
    const double eps = 64.0 * 2.220446049250313080847263336181640625e-16;
    for (;;) {
        orc_sphere_sample(N, g, v);
        double proj = 0;
        for (uint32_t k = 0; k < N; ++k) proj += v[k] * u[k];
        double r2 = 0;
        for (uint32_t k = 0; k < N; ++k) {
            v[k] -= proj * u[k];
            r2 += v[k] * v[k];
        }
        if (r2 > eps) {
            const double inv = 1.0 / sqrt(r2);
            for (uint32_t k = 0; k < N; ++k) v[k] *= inv;
            frame = sqrt(r2);
            break;
        }
    }
    const double th = delta * (2.0 * orc_pcg32_uni(g) - 1.0);
    const double c = cos(th);
    const double sn = sin(th);
    double cu = 0, cv = 0;
    for (uint32_t k = 0; k < N; ++k) {
        cu += u[k] * cur[k];
        cv += v[k] * cur[k];
    }
    for (uint32_t k = 0; k < N; ++k)
        out[k] = cur[k] + (c - 1.0) * (cu * u[k] + cv * v[k]) + sn * (cu * v[k] - cv * u[k]);
    return frame;
}

/* VectorSpin<N>::energy_at, example/vector_spin.hpp:39-47. */
static void vector_observe(uint32_t N, uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                           double J, const double* s, double* obs)
{
    double e = 0.0;
    double m[8] = {0};
    for (uint64_t i = 0; i < n; ++i) {
        const double* si = s + i * N;
        double ei = 0.0;
        for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) ei += -J * vdot(N, si, s + (uint64_t)bonds[a] * N);
        e += ei;
        for (uint32_t k = 0; k < N; ++k) m[k] += si[k];
    }
    obs[0] = 0.5 * e;
    for (uint32_t k = 0; k < N; ++k) obs[1 + k] = m[k];
}

/* Metropolis::sweep (driver.hpp:29-43) over VectorSpin<N>::energy_diff_at
 * (example/vector_spin.hpp:50-60). */
void orc_vector_metropolis(uint32_t N, uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                           double J, double beta, int proposal, double delta, uint64_t seed,
                           uint64_t sweep0, uint64_t n_sweeps, double* s, double* obs_out,
                           double* margin_out)
{
    double cand[8];
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n; ++i) {
            orc_pcg32 g;
            orc_key_open(&g, seed, counter, ORC_TAG_SITE(0), (uint32_t)i);
            double* cur = s + i * N;
            double frame = 1.0;
            if (proposal == ORC_PROP_SPHERE) orc_sphere_sample(N, &g, cand);
            else frame = local_rotation(N, delta, &g, cur, cand);
            double d = 0.0;
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const double* sj = s + (uint64_t)bonds[a] * N;
                d += -J * (vdot(N, cand, sj) - vdot(N, cur, sj));
            }
            const double log_p = -beta * d + 0.0;
            int accept;
            double margin = INFINITY;
            if (log_p >= 0.0) accept = 1;
            else {
                const double lu = log(orc_pcg32_uni(&g));
                margin = lu - log_p;
                accept = lu < log_p;
            }
            /* an ill-conditioned rotation frame makes the candidate itself
             * precision-sensitive: report it like a near-threshold decision */
            if (frame < ORC_FRAME_TOL) margin = 0.0;
            if (margin_out && k + 1 == n_sweeps) margin_out[i] = margin;
            if (accept) memcpy(cur, cand, N * sizeof(double));
        }
        if (obs_out) vector_observe(N, n, offset, bonds, J, s, obs_out + k * (N + 1));
    }
}

/* Wolff::flip (driver.hpp:104-162) with a UniformSphereN<N> axis and
 * VectorSpin<N>::energy_diff_bond (example/vector_spin.hpp:63-69).
 * margin_out: per flip, min over tested bonds of |u - p| (closeness of the
 * nearest activation decision to its threshold). */
void orc_vector_wolff(uint32_t N, uint64_t n, const uint32_t* offset, const uint32_t* bonds,
                      const uint32_t* slot_edge, double J, double beta, uint64_t seed,
                      uint64_t flip0, uint64_t n_flips, double* s, uint64_t* sizes,
                      double* obs_out, double* margin_out)
{
    char* in_cluster = (char*)malloc(n ? n : 1);
    uint64_t* stack = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    double r[8], prop[8], nb[8];
    for (uint64_t f = 0; f < n_flips; ++f) {
        const uint64_t counter = flip0 + f;
        orc_pcg32 g;
        orc_key_open(&g, seed, counter, ORC_TAG_AXIS, 0);
        orc_sphere_sample(N, &g, r);
        memset(in_cluster, 0, n);
        const uint64_t seed_site = (uint64_t)(orc_pcg32_uni(&g) * (double)n);
        in_cluster[seed_site] = 1;
        stack[0] = seed_site;
        uint64_t top = 1, cluster = 0;
        double min_margin = INFINITY;
        while (top > 0) {
            const uint64_t i = stack[--top];
            ++cluster;
            const double* si = s + i * N;
            double dot = 0;
            for (uint32_t k = 0; k < N; ++k) dot += si[k] * r[k];
            for (uint32_t k = 0; k < N; ++k) prop[k] = si[k] - 2.0 * dot * r[k];
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const uint32_t j = bonds[a];
                if (in_cluster[j]) continue;
                const double* t = s + (uint64_t)j * N;
                double d = 0;
                for (uint32_t k = 0; k < N; ++k) d += t[k] * r[k];
                for (uint32_t k = 0; k < N; ++k) nb[k] = t[k] - 2.0 * d * r[k];
                const double dE = -J * (vdot(N, nb, si) - vdot(N, t, si));
                orc_pcg32 gb;
                orc_key_open(&gb, seed, counter, ORC_TAG_BOND, slot_edge[a]);
                const double u = orc_pcg32_uni(&gb);
                const double p = 1.0 - exp(-beta * dE);
                if (p > 0.0 && fabs(u - p) < min_margin) min_margin = fabs(u - p);
                if (u < p) {
                    in_cluster[j] = 1;
                    stack[top++] = j;
                }
            }
            memcpy(s + i * N, prop, N * sizeof(double));
        }
        if (sizes) sizes[f] = cluster;
        if (margin_out) margin_out[f] = min_margin;
        if (obs_out) vector_observe(N, n, offset, bonds, J, s, obs_out + f * (N + 1));
    }
    free(in_cluster);
    free(stack);
}

/* ------------------------------------------------------------------ XY angles */

/* U1Shift::sample, dof/u1.hpp:35-50: theta + width*(2u-1), wrapped by
 * remainder(., 2 pi) into [-pi, pi]. */
static double u1_shift(double width, orc_pcg32* g, double cur)
{
    const double two_pi = 2.0 * ORC_PI;
    const double shift = width * (2.0 * orc_pcg32_uni(g) - 1.0);
    return remainder(cur + shift, two_pi);
}

/* PairModel::energy_diff_at (model/pair.hpp:53-64) with the pair term
 * E = -J cos(theta_i - theta_j) (a user CellTerm of arity 2), driven by
 * Metropolis::sweep (driver.hpp:29-43) and U1Shift. */
void orc_xy_metropolis(uint64_t n, const uint32_t* offset, const uint32_t* bonds, double J,
                       double beta, double width, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* th, double* obs_out, double* margin_out)
{
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n; ++i) {
            orc_pcg32 g;
            orc_key_open(&g, seed, counter, ORC_TAG_SITE(0), (uint32_t)i);
            const double old = th[i];
            const double p = u1_shift(width, &g, old);
            double d = 0.0;
            for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) {
                const double fixed = th[bonds[a]];
                d += -J * (cos(p - fixed) - cos(old - fixed));
            }
            const double log_p = -beta * d + 0.0;
            int accept;
            double margin = INFINITY;
            if (log_p >= 0.0) accept = 1;
            else {
                const double lu = log(orc_pcg32_uni(&g));
                margin = lu - log_p;
                accept = lu < log_p;
            }
            if (margin_out && k + 1 == n_sweeps) margin_out[i] = margin;
            if (accept) th[i] = p;
        }
        if (obs_out) {
            double e = 0.0, mx = 0.0, my = 0.0;
            for (uint64_t i = 0; i < n; ++i) {
                double ei = 0.0; /* PairModel::energy_at, model/pair.hpp:40-50 */
                for (uint32_t a = offset[i]; a < offset[i + 1]; ++a) ei += -J * cos(th[i] - th[bonds[a]]);
                e += ei;
                mx += cos(th[i]);
                my += sin(th[i]);
            }
            obs_out[3 * k + 0] = 0.5 * e;
            obs_out[3 * k + 1] = mx;
            obs_out[3 * k + 2] = my;
        }
    }
}

/* ------------------------------------------------------- replica exchange */

/* Parallel tempering swap between neighbouring temperature slots (project-
 * defined; the reference has none): detailed balance for the joint ensemble
 * with acceptance min(1, exp((beta_k - beta_{k+1}) (E_k - E_{k+1}))). */
int orc_replica_exchange(uint32_t R, const double* betas, uint32_t* holder, const double* energy,
                         uint64_t seed, uint64_t round, uint32_t parity, uint8_t* accepted)
{
    int n = 0;
    for (uint32_t k = parity; k + 1 < R; k += 2) {
        const uint32_t a = holder[k], b = holder[k + 1];
        const double delta = (betas[k] - betas[k + 1]) * (energy[a] - energy[b]);
        orc_pcg32 g;
        orc_key_open(&g, seed, round, ORC_TAG_SWAP, k);
        const int acc = delta >= 0.0 || log(orc_pcg32_uni(&g)) < delta;
        if (accepted) accepted[k] = (uint8_t)acc;
        if (acc) {
            holder[k] = b;
            holder[k + 1] = a;
            ++n;
        }
    }
    return n;
}

/* --------------------------------------------------------------------- U(1) */

/* plaquette(t0..t3), dof/u1.hpp:18-21. */
static double u1_plaq(double t0, double t1, double t2, double t3) { return cos(t0 + t1 - t2 - t3); }

double orc_u1_mean_plaquette(uint64_t n_cells, const uint32_t* cells, const double* th)
{
    double sum = 0.0;
    for (uint64_t c = 0; c < n_cells; ++c) {
        const uint32_t* q = cells + 4 * c;
        sum += u1_plaq(th[q[0]], th[q[1]], th[q[2]], th[q[3]]);
    }
    return sum / (double)n_cells;
}

double orc_u1_topological_charge(uint64_t n_cells, const uint32_t* cells, const double* th)
{
    double q = 0.0;
    for (uint64_t c = 0; c < n_cells; ++c) {
        const uint32_t* p = cells + 4 * c;
        q += remainder(th[p[0]] + th[p[1]] - th[p[2]] - th[p[3]], 2.0 * ORC_PI);
    }
    return q / (2.0 * ORC_PI);
}

/* CellModel::energy_diff_at (model/cell.hpp:64-78) with U1PlaquetteTerm::delta
 * (term/plaquette.hpp:34-47); identical arithmetic to U1Gauge::energy_diff_at
 * (example/u1_gauge.hpp:35-52).  hits > 1 repeats the Metropolis step on each
 * link with fresh keyed draws (tag ORC_TAG_SITE(h)). */
void orc_u1_metropolis(uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                       const uint64_t* inc_offset, const uint32_t* inc_cell,
                       const uint8_t* inc_which, double model_beta, double driver_beta,
                       double width, uint32_t hits, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* th, double* obs_out, double* margin_out)
{
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n_links; ++i) {
            for (uint32_t h = 0; h < hits; ++h) {
                orc_pcg32 g;
                orc_key_open(&g, seed, counter, ORC_TAG_SITE(h), (uint32_t)i);
                const double p = u1_shift(width, &g, th[i]);
                double d = 0.0;
                for (uint64_t a = inc_offset[i]; a < inc_offset[i + 1]; ++a) {
                    const uint32_t* q = cells + 4 * (uint64_t)inc_cell[a];
                    double t[4] = {th[q[0]], th[q[1]], th[q[2]], th[q[3]]};
                    const double before = u1_plaq(t[0], t[1], t[2], t[3]);
                    t[inc_which[a]] = p;
                    const double after = u1_plaq(t[0], t[1], t[2], t[3]);
                    d += model_beta * (before - after);
                }
                const double log_p = -driver_beta * d + 0.0;
                int accept;
                double margin = INFINITY;
                if (log_p >= 0.0) accept = 1;
                else {
                    const double lu = log(orc_pcg32_uni(&g));
                    margin = lu - log_p;
                    accept = lu < log_p;
                }
                if (margin_out && k + 1 == n_sweeps) {
                    if (h == 0 || fabs(margin) < fabs(margin_out[i])) margin_out[i] = margin;
                }
                if (accept) th[i] = p;
            }
        }
        (void)n_cells;
        if (obs_out) {
            const double P = orc_u1_mean_plaquette(n_cells, cells, th);
            obs_out[2 * k + 0] = model_beta * (double)n_cells * (1.0 - P);
            obs_out[2 * k + 1] = P;
        }
    }
}

/* -------------------------------------------------------------------- SU(N) */

typedef double _Complex cplx;

/* SULink operator*, dof/sun.hpp:65-75 (and sun_detail::mul :91-102). */
static void su_mul(uint32_t N, const cplx* a, const cplx* b, cplx* r)
{
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = 0; j < N; ++j) {
            double sr = 0.0, si = 0.0;
            for (uint32_t k = 0; k < N; ++k) {
                const double ar = creal(a[i * N + k]), ai = cimag(a[i * N + k]);
                const double br = creal(b[k * N + j]), bi = cimag(b[k * N + j]);
                sr += ar * br - ai * bi;
                si += ar * bi + ai * br;
            }
            r[i * N + j] = CMPLX(sr, si);
        }
}

/* SULink::dagger, dof/sun.hpp:34-41. */
static void su_dagger(uint32_t N, const cplx* a, cplx* r)
{
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = 0; j < N; ++j) r[i * N + j] = conj(a[j * N + i]);
}

/* plaquette(U0,U1,U2,U3) = ReTr(((U0 U1) U2^dag) U3^dag)/N, dof/sun.hpp:78-84. */
static double su_plaq(uint32_t N, const cplx* u0, const cplx* u1, const cplx* u2, const cplx* u3)
{
    cplx a[16], b[16], d[16];
    su_mul(N, u0, u1, a);
    su_dagger(N, u2, d);
    su_mul(N, a, d, b);
    su_dagger(N, u3, d);
    su_mul(N, b, d, a);
    double t = 0.0;
    for (uint32_t i = 0; i < N; ++i) t += creal(a[i * N + i]);
    return t / (double)N;
}

/* sun_detail::norm, dof/sun.hpp:104-114 (max row sum of |a_ij|). */
static double su_norm(uint32_t N, const cplx* a)
{
    double n = 0.0;
    for (uint32_t i = 0; i < N; ++i) {
        double row = 0.0;
        for (uint32_t j = 0; j < N; ++j) row += cabs(a[i * N + j]);
        if (row > n) n = row;
    }
    return n;
}

/* sun_detail::expm, dof/sun.hpp:118-146. */
static void su_expm_c(uint32_t N, const cplx* a, cplx* out)
{
    double n = su_norm(N, a);
    int squarings = 0;
    while (n > 0.5) {
        n *= 0.5;
        ++squarings;
    }
    const double scale = ldexp(1.0, -squarings);
    cplx b[16], result[16], term[16], tmp[16];
    for (uint32_t k = 0; k < N * N; ++k) b[k] = CMPLX(creal(a[k]) * scale, cimag(a[k]) * scale);
    for (uint32_t k = 0; k < N * N; ++k) result[k] = term[k] = 0.0;
    for (uint32_t i = 0; i < N; ++i) result[i * N + i] = term[i * N + i] = 1.0;
    for (uint32_t k = 1; k <= 30; ++k) {
        su_mul(N, term, b, tmp);
        for (uint32_t q = 0; q < N * N; ++q) term[q] = CMPLX(creal(tmp[q]) / (double)k, cimag(tmp[q]) / (double)k);
        for (uint32_t q = 0; q < N * N; ++q) result[q] = CMPLX(creal(result[q]) + creal(term[q]), cimag(result[q]) + cimag(term[q]));
        if (su_norm(N, term) < 1e-16) break;
    }
    for (int k = 0; k < squarings; ++k) {
        su_mul(N, result, result, tmp);
        memcpy(result, tmp, sizeof(cplx) * N * N);
    }
    memcpy(out, result, sizeof(cplx) * N * N);
}

void orc_su_expm(uint32_t N, const double* a, double* out)
{
    cplx ac[16], oc[16];
    for (uint32_t k = 0; k < N * N; ++k) ac[k] = CMPLX(a[2 * k], a[2 * k + 1]);
    su_expm_c(N, ac, oc);
    for (uint32_t k = 0; k < N * N; ++k) {
        out[2 * k] = creal(oc[k]);
        out[2 * k + 1] = cimag(oc[k]);
    }
}

/* SUShift<N>::sample, dof/sun.hpp:163-204: traceless Hermitian X from N + N(N-1)
 * uniforms (diagonal first, then (a,b) per upper pair), U' = U exp(iX). */
static void su_shift_c(uint32_t N, double width, orc_pcg32* g, const cplx* cur, cplx* out)
{
    cplx x[16], a[16], e[16];
    for (uint32_t k = 0; k < N * N; ++k) x[k] = 0.0;
    double tr = 0.0;
    for (uint32_t i = 0; i < N; ++i) {
        const double d = width * (2.0 * orc_pcg32_uni(g) - 1.0);
        x[i * N + i] = CMPLX(d, 0.0);
        tr += d;
    }
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = i + 1; j < N; ++j) {
            const double ar = width * (2.0 * orc_pcg32_uni(g) - 1.0);
            const double br = width * (2.0 * orc_pcg32_uni(g) - 1.0);
            x[i * N + j] = CMPLX(ar, br);
            x[j * N + i] = CMPLX(ar, -br);
        }
    for (uint32_t i = 0; i < N; ++i) x[i * N + i] = CMPLX(creal(x[i * N + i]) - tr / (double)N, cimag(x[i * N + i]));
    for (uint32_t k = 0; k < N * N; ++k) a[k] = CMPLX(-cimag(x[k]), creal(x[k]));
    su_expm_c(N, a, e);
    su_mul(N, cur, e, out);
}

void orc_su_shift(uint32_t N, double width, orc_pcg32* g, const double* cur, double* out)
{
    cplx c[16], o[16];
    for (uint32_t k = 0; k < N * N; ++k) c[k] = CMPLX(cur[2 * k], cur[2 * k + 1]);
    su_shift_c(N, width, g, c, o);
    for (uint32_t k = 0; k < N * N; ++k) {
        out[2 * k] = creal(o[k]);
        out[2 * k + 1] = cimag(o[k]);
    }
}

/* SULink::unitarity_error, dof/sun.hpp:43-54. */
double orc_su_unitarity_error(uint32_t N, const double* u)
{
    cplx c[16], d[16], p[16];
    for (uint32_t k = 0; k < N * N; ++k) c[k] = CMPLX(u[2 * k], u[2 * k + 1]);
    su_dagger(N, c, d);
    su_mul(N, d, c, p);
    double e = 0.0;
    for (uint32_t i = 0; i < N; ++i)
        for (uint32_t j = 0; j < N; ++j) {
            const double v = cabs(p[i * N + j] - (i == j ? 1.0 : 0.0));
            if (v > e) e = v;
        }
    return e;
}

static const cplx* su_at(uint32_t N, const cplx* links, uint64_t i) { return links + i * N * N; }

double orc_su_mean_plaquette(uint32_t N, uint64_t n_cells, const uint32_t* cells, const double* links)
{
    const cplx* l = (const cplx*)links;
    double sum = 0.0;
    for (uint64_t c = 0; c < n_cells; ++c) {
        const uint32_t* q = cells + 4 * c;
        sum += su_plaq(N, su_at(N, l, q[0]), su_at(N, l, q[1]), su_at(N, l, q[2]), su_at(N, l, q[3]));
    }
    return sum / (double)n_cells;
}

/* SUGauge<N>::energy_diff_at (example/sun_gauge.hpp:36-51), same arithmetic as
 * CellModel + SUPlaquetteTerm::delta (term/sun_plaquette.hpp:37-46), driven by
 * Metropolis::sweep (driver.hpp:29-43) with SUShift<N>, hits per link. */
void orc_su_metropolis(uint32_t N, uint64_t n_links, const uint32_t* cells, uint64_t n_cells,
                       const uint64_t* inc_offset, const uint32_t* inc_cell,
                       const uint8_t* inc_which, double model_beta, double driver_beta,
                       double width, uint32_t hits, uint64_t seed, uint64_t sweep0,
                       uint64_t n_sweeps, double* links, double* obs_out, double* margin_out)
{
    cplx* l = (cplx*)links;
    cplx cand[16];
    for (uint64_t k = 0; k < n_sweeps; ++k) {
        const uint64_t counter = sweep0 + k;
        for (uint64_t i = 0; i < n_links; ++i) {
            for (uint32_t h = 0; h < hits; ++h) {
                orc_pcg32 g;
                orc_key_open(&g, seed, counter, ORC_TAG_SITE(h), (uint32_t)i);
                su_shift_c(N, width, &g, su_at(N, l, i), cand);
                double d = 0.0;
                for (uint64_t a = inc_offset[i]; a < inc_offset[i + 1]; ++a) {
                    const uint32_t* q = cells + 4 * (uint64_t)inc_cell[a];
                    const cplx* p[4] = {su_at(N, l, q[0]), su_at(N, l, q[1]), su_at(N, l, q[2]), su_at(N, l, q[3])};
                    const double before = su_plaq(N, p[0], p[1], p[2], p[3]);
                    p[inc_which[a]] = cand;
                    const double after = su_plaq(N, p[0], p[1], p[2], p[3]);
                    d += model_beta * (before - after);
                }
                const double log_p = -driver_beta * d + 0.0;
                int accept;
                double margin = INFINITY;
                if (log_p >= 0.0) accept = 1;
                else {
                    const double lu = log(orc_pcg32_uni(&g));
                    margin = lu - log_p;
                    accept = lu < log_p;
                }
                if (margin_out && k + 1 == n_sweeps) {
                    if (h == 0 || fabs(margin) < fabs(margin_out[i])) margin_out[i] = margin;
                }
                if (accept) memcpy(l + i * N * N, cand, sizeof(cplx) * N * N);
            }
        }
        if (obs_out) {
            const double P = orc_su_mean_plaquette(N, n_cells, cells, links);
            obs_out[2 * k + 0] = model_beta * (double)n_cells * (1.0 - P);
            obs_out[2 * k + 1] = P;
        }
    }
}
