// umc_tables.cpp -- topology tables (host side) and the table part of the C ABI.
//
// PairGraph and CellComplex are rebuilt with the reference's construction order
// (lattice/pair_graph.hpp:49-83, lattice/cell_complex.hpp:36-63) so that row
// order, duplicates and error behaviour match.  On top of that every table gets
// a colouring and a colour-major relabelling: sites of one colour never share a
// bond (or a cell), so a whole colour class is updated by one kernel pass, and
// the reference driver visiting relabelled sites in index order (driver.hpp:34)
// performs exactly the same sequence of updates.

#include "umc_tables.hpp"

#include <algorithm>
#include <memory>
#include <cstring>
#include <limits>
#include <new>

namespace umc {

namespace {
thread_local std::string g_last_error;

constexpr uint64_t kMax32 = std::numeric_limits<uint32_t>::max();

// Colour-major positions from a colour assignment: classes in colour order,
// sites ascending inside a class.
void finish_colouring(Colouring& col)
{
    const uint64_t n = col.colour.size();
    col.class_start.assign(col.n_colours + 1, 0);
    for (uint64_t i = 0; i < n; ++i) ++col.class_start[col.colour[i] + 1];
    for (uint32_t c = 0; c < col.n_colours; ++c) col.class_start[c + 1] += col.class_start[c];
    std::vector<uint64_t> cursor(col.class_start.begin(), col.class_start.end() - 1);
    col.position.assign(n, 0);
    col.order.assign(n, 0);
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t p = cursor[col.colour[i]]++;
        col.position[i] = uint32_t(p);
        col.order[p] = uint32_t(i);
    }
}

// Two-colouring by breadth-first search when the graph is bipartite (site 0,
// and the first site of every further component, get colour 0); otherwise a
// greedy colouring in index order (smallest colour unused by any neighbour).
Colouring colour_graph(uint64_t n, const std::vector<uint32_t>& off, const std::vector<uint32_t>& adj)
{
    Colouring col;
    col.colour.assign(n, 0xFFFFFFFFu);
    bool bipartite = true;
    std::vector<uint32_t> queue;
    queue.reserve(n);
    for (uint64_t s = 0; s < n && bipartite; ++s) {
        if (col.colour[s] != 0xFFFFFFFFu) continue;
        col.colour[s] = 0;
        queue.clear();
        queue.push_back(uint32_t(s));
        for (size_t q = 0; q < queue.size() && bipartite; ++q) {
            const uint32_t i = queue[q];
            for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
                const uint32_t j = adj[a];
                if (col.colour[j] == 0xFFFFFFFFu) {
                    col.colour[j] = 1u - col.colour[i];
                    queue.push_back(j);
                } else if (col.colour[j] == col.colour[i]) {
                    bipartite = false;
                    break;
                }
            }
        }
    }
    if (bipartite) {
        col.n_colours = 1;
        for (uint64_t i = 0; i < n; ++i) col.n_colours = std::max(col.n_colours, col.colour[i] + 1);
    } else {
        col.colour.assign(n, 0xFFFFFFFFu);
        col.n_colours = 0;
        std::vector<uint64_t> stamp;
        for (uint64_t i = 0; i < n; ++i) {
            for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
                const uint32_t c = col.colour[adj[a]];
                if (c == 0xFFFFFFFFu) continue;
                if (c >= stamp.size()) stamp.resize(c + 1, ~uint64_t(0));
                stamp[c] = i;
            }
            uint32_t c = 0;
            while (c < stamp.size() && stamp[c] == i) ++c;
            col.colour[i] = c;
            col.n_colours = std::max(col.n_colours, c + 1);
        }
    }
    if (n == 0) col.n_colours = 0;
    finish_colouring(col);
    return col;
}

}  // namespace

void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
const char* last_error() { return g_last_error.c_str(); }

namespace {
// Fills g's tables from an edge list (lattice/pair_graph.hpp:49-83: same
// checks, same exceptions); g->kind and g->dims must already be set.
void fill_graph(umc_graph* g, uint64_t n, const uint32_t* ei, const uint32_t* ej, uint64_t m, bool symmetric)
{
    if (n > kMax32) throw Error(UMC_ERR_OVERFLOW, "PairGraph: site count exceeds uint32_t");
    if (m && (!ei || !ej)) throw Error(UMC_ERR_INVALID_ARGUMENT, "PairGraph: null edge arrays");
    std::vector<uint64_t> degree(n, 0);
    for (uint64_t e = 0; e < m; ++e) {
        if (ei[e] >= n || ej[e] >= n) throw Error(UMC_ERR_OUT_OF_RANGE, "PairGraph: edge endpoint out of range");
        if (ei[e] == ej[e]) throw Error(UMC_ERR_INVALID_ARGUMENT, "PairGraph: self-loop");
        ++degree[ei[e]];
        if (symmetric) ++degree[ej[e]];
    }
    g->n = n;
    g->symmetric = symmetric;
    g->max_degree = 0;
    g->ei.assign(ei, ei + m);
    g->ej.assign(ej, ej + m);
    g->offset.assign(n + 1, 0);
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        g->offset[i] = uint32_t(total);
        total += degree[i];
        if (total > kMax32) throw Error(UMC_ERR_OVERFLOW, "PairGraph: bond count exceeds uint32_t");
        g->max_degree = std::max<uint32_t>(g->max_degree, uint32_t(degree[i]));
    }
    if (n) g->offset[n] = uint32_t(total);
    g->bonds.assign(total, 0);
    g->slot_edge.assign(total, 0);
    {
        std::vector<uint64_t> pos(g->offset.begin(), g->offset.begin() + n);
        for (uint64_t e = 0; e < m; ++e) {
            const uint64_t a = pos[ei[e]]++;
            g->bonds[a] = ej[e];
            g->slot_edge[a] = uint32_t(e);
            if (symmetric) {
                const uint64_t b = pos[ej[e]]++;
                g->bonds[b] = ei[e];
                g->slot_edge[b] = uint32_t(e);
            }
        }
    }

    // Conflict graph for the colouring: the CSR itself when symmetric, else
    // its symmetrisation.
    if (symmetric) {
        g->col = colour_graph(n, g->offset, g->bonds);
    } else {
        std::vector<uint32_t> soff(n + 1, 0), sadj;
        for (uint64_t e = 0; e < m; ++e) {
            ++soff[ei[e] + 1];
            ++soff[ej[e] + 1];
        }
        for (uint64_t i = 0; i < n; ++i) soff[i + 1] += soff[i];
        sadj.assign(soff[n], 0);
        std::vector<uint32_t> pos(soff.begin(), soff.end() - 1);
        for (uint64_t e = 0; e < m; ++e) {
            sadj[pos[ei[e]]++] = ej[e];
            sadj[pos[ej[e]]++] = ei[e];
        }
        g->col = colour_graph(n, soff, sadj);
    }

    // Colour-major CSR: row k is the row of site order[k], targets relabelled.
    g->c_offset.assign(n + 1, 0);
    g->c_bonds.assign(total, 0);
    g->c_slot_edge.assign(total, 0);
    uint64_t acc = 0;
    for (uint64_t k = 0; k < n; ++k) {
        const uint32_t i = g->col.order[k];
        g->c_offset[k] = uint32_t(acc);
        for (uint32_t a = g->offset[i]; a < g->offset[i + 1]; ++a) {
            g->c_bonds[acc] = g->col.position[g->bonds[a]];
            g->c_slot_edge[acc] = g->slot_edge[a];
            ++acc;
        }
    }
    if (n) g->c_offset[n] = uint32_t(acc);

    // The regular-lattice kernels reproduce this graph exactly when every
    // extent is 1 or even (x even >= 2): then the two-colouring is
    // (x + y + z) & 1 and colour-major index = colour * n/2 + site/2.
    if (g->kind == Lattice::Square || g->kind == Lattice::Cubic) {
        const uint64_t Lx = g->dims[0], Ly = g->dims[1], Lz = g->dims[2];
        bool ok = Lx >= 2 && Lx % 2 == 0 && (Ly == 1 || Ly % 2 == 0) && (Lz == 1 || Lz % 2 == 0);
        if (ok && g->col.n_colours == 2) {
            for (uint64_t s = 0; s < n && ok; ++s) {
                const uint64_t x = s % Lx, y = (s / Lx) % Ly, z = s / (Lx * Ly);
                const uint32_t c = uint32_t((x + y + z) & 1);
                ok = g->col.colour[s] == c && g->col.position[s] == c * (n / 2) + s / 2;
            }
        } else {
            ok = false;
        }
        g->stencil = ok;
    }
    g->materialized = true;
}

// Edge list of the periodic square / cubic builders (lattice/square.hpp:27-35,
// extended to z): per site a +x, +y, +z edge when that extent exceeds 1.
void lattice_edges(uint64_t Lx, uint64_t Ly, uint64_t Lz, std::vector<uint32_t>& ei, std::vector<uint32_t>& ej)
{
    const uint64_t n = Lx * Ly * Lz;
    ei.clear();
    ej.clear();
    ei.reserve(3 * n);
    ej.reserve(3 * n);
    for (uint64_t z = 0; z < Lz; ++z)
        for (uint64_t y = 0; y < Ly; ++y)
            for (uint64_t x = 0; x < Lx; ++x) {
                const uint32_t i = uint32_t((z * Ly + y) * Lx + x);
                if (Lx > 1) { ei.push_back(i); ej.push_back(uint32_t((z * Ly + y) * Lx + (x + 1) % Lx)); }
                if (Ly > 1) { ei.push_back(i); ej.push_back(uint32_t((z * Ly + (y + 1) % Ly) * Lx + x)); }
                if (Lz > 1) { ei.push_back(i); ej.push_back(uint32_t((((z + 1) % Lz) * Ly + y) * Lx + x)); }
            }
}

// A regular lattice whose kernels need no table: keep n, extents, degree and
// the two colour classes; the tables are built on first request.
umc_graph* make_regular(Lattice kind, uint64_t Lx, uint64_t Ly, uint64_t Lz)
{
    const uint64_t n = Lx * Ly * Lz;
    const uint64_t ndir = (Lx > 1) + (Ly > 1) + (Lz > 1);
    if (2 * ndir * n > kMax32) throw Error(UMC_ERR_OVERFLOW, "PairGraph: bond count exceeds uint32_t");
    const bool closed = Lx >= 2 && Lx % 2 == 0 && (Ly == 1 || Ly % 2 == 0) && (Lz == 1 || Lz % 2 == 0);
    auto* g = new umc_graph;
    g->kind = kind;
    g->dims[0] = Lx;
    g->dims[1] = Ly;
    g->dims[2] = Lz;
    if (!closed) {
        std::vector<uint32_t> ei, ej;
        lattice_edges(Lx, Ly, Lz, ei, ej);
        try {
            fill_graph(g, n, ei.data(), ej.data(), ei.size(), true);
        } catch (...) {
            delete g;
            throw;
        }
        return g;
    }
    g->n = n;
    g->symmetric = true;
    g->max_degree = uint32_t(2 * ndir);
    g->col.n_colours = 2;
    g->col.class_start = {0, n / 2, n};
    g->stencil = true;
    g->materialized = false;
    return g;
}
}  // namespace

umc_graph* make_graph(uint64_t n, const uint32_t* ei, const uint32_t* ej, uint64_t m, bool symmetric,
                      Lattice kind, const uint64_t dims[3])
{
    auto* g = new umc_graph;
    g->kind = kind;
    if (dims) std::memcpy(g->dims, dims, sizeof g->dims);
    try {
        fill_graph(g, n, ei, ej, m, symmetric);
    } catch (...) {
        delete g;
        throw;
    }
    return g;
}

void materialize(const umc_graph* cg)
{
    if (cg->materialized) return;
    auto* g = const_cast<umc_graph*>(cg);  // the lazy tables are a cache of the extents
    std::vector<uint32_t> ei, ej;
    lattice_edges(g->dims[0], g->dims[1], g->dims[2], ei, ej);
    fill_graph(g, g->n, ei.data(), ej.data(), ei.size(), true);
}

umc_graph* make_square(uint64_t Lx, uint64_t Ly)
{
    // lattice/square.hpp:15-38
    if (Lx == 0 || Ly == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "square_lattice: Lx and Ly must be positive");
    if (Lx > std::numeric_limits<uint64_t>::max() / Ly) throw Error(UMC_ERR_OVERFLOW, "square_lattice: site count overflows size_t");
    if (Lx * Ly > kMax32) throw Error(UMC_ERR_OVERFLOW, "square_lattice: site count exceeds uint32_t");
    return make_regular(Lattice::Square, Lx, Ly, 1);
}

umc_graph* make_cubic(uint64_t Lx, uint64_t Ly, uint64_t Lz)
{
    if (Lx == 0 || Ly == 0 || Lz == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "cubic_lattice: extents must be positive");
    if (Lx > kMax32 || Ly > kMax32 || Lz > kMax32 || Lx * Ly > kMax32 || Lx * Ly * Lz > kMax32)
        throw Error(UMC_ERR_OVERFLOW, "cubic_lattice: site count exceeds uint32_t");
    return make_regular(Lattice::Cubic, Lx, Ly, Lz);
}

umc_cells* make_cells(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells,
                      Lattice kind, uint64_t L, uint32_t dim)
{
    // lattice/cell_complex.hpp:36-63
    if (arity < 1 || arity > 255) throw Error(UMC_ERR_INVALID_ARGUMENT, "CellComplex arity must fit uint8_t");
    if (n_sites > kMax32 || n_cells > kMax32) throw Error(UMC_ERR_OVERFLOW, "CellComplex: too many sites or cells");
    if (n_cells && !cells) throw Error(UMC_ERR_INVALID_ARGUMENT, "CellComplex: null cell array");
    auto* cc = new umc_cells;
    cc->n_sites = n_sites;
    cc->arity = arity;
    cc->kind = kind;
    cc->L = L;
    cc->dim = dim;
    cc->cells.assign(cells, cells + n_cells * arity);
    cc->inc_offset.assign(n_sites + 1, 0);
    for (uint64_t q = 0; q < n_cells * arity; ++q) {
        if (cells[q] >= n_sites) {
            delete cc;
            throw Error(UMC_ERR_OUT_OF_RANGE, "CellComplex: site out of range");
        }
        ++cc->inc_offset[cells[q] + 1];
    }
    for (uint64_t i = 0; i < n_sites; ++i) {
        cc->max_incident = std::max<uint32_t>(cc->max_incident, uint32_t(cc->inc_offset[i + 1]));
        cc->inc_offset[i + 1] += cc->inc_offset[i];
    }
    cc->inc_cell.assign(n_cells * arity, 0);
    cc->inc_which.assign(n_cells * arity, 0);
    {
        std::vector<uint64_t> cursor(cc->inc_offset.begin(), cc->inc_offset.end() - 1);
        for (uint64_t c = 0; c < n_cells; ++c)
            for (uint32_t k = 0; k < arity; ++k) {
                const uint64_t a = cursor[cells[c * arity + k]]++;
                cc->inc_cell[a] = uint32_t(c);
                cc->inc_which[a] = uint8_t(k);
            }
    }

    // Colouring: closed form (direction, parity) for the even periodic
    // plaquette complexes, greedy over shared cells otherwise.
    Colouring& col = cc->col;
    const bool closed = (kind == Lattice::Hypercubic || kind == Lattice::SquarePlaquettes) && L >= 2 && L % 2 == 0;
    if (closed) {
        uint64_t V = 1;
        for (uint32_t d = 0; d < dim; ++d) V *= L;
        col.n_colours = 2 * dim;
        col.colour.assign(n_sites, 0);
        for (uint64_t i = 0; i < n_sites; ++i) {
            const uint64_t mu = i / V, s = i % V;
            uint64_t par = 0, r = s;
            for (uint32_t d = 0; d < dim; ++d) {
                par += r % L;
                r /= L;
            }
            col.colour[i] = uint32_t(2 * mu + (par & 1));
        }
        finish_colouring(col);
        cc->stencil = true;
        for (uint64_t i = 0; i < n_sites && cc->stencil; ++i)
            cc->stencil = col.position[i] == col.colour[i] * (V / 2) + (i % V) / 2;
    } else {
        col.colour.assign(n_sites, 0xFFFFFFFFu);
        col.n_colours = 0;
        std::vector<uint64_t> stamp;
        for (uint64_t i = 0; i < n_sites; ++i) {
            for (uint64_t a = cc->inc_offset[i]; a < cc->inc_offset[i + 1]; ++a) {
                const uint32_t* cl = &cc->cells[uint64_t(cc->inc_cell[a]) * arity];
                for (uint32_t k = 0; k < arity; ++k) {
                    if (cl[k] == i) continue;
                    const uint32_t c = col.colour[cl[k]];
                    if (c == 0xFFFFFFFFu) continue;
                    if (c >= stamp.size()) stamp.resize(c + 1, ~uint64_t(0));
                    stamp[c] = i;
                }
            }
            uint32_t c = 0;
            while (c < stamp.size() && stamp[c] == i) ++c;
            col.colour[i] = c;
            col.n_colours = std::max(col.n_colours, c + 1);
        }
        if (n_sites == 0) col.n_colours = 0;
        finish_colouring(col);
    }

    // Colour-major copy: same cell order, relabelled link ids; incidence row k
    // is the row of link order[k] (cells ascending, as in the original).
    cc->c_cells.resize(cc->cells.size());
    for (uint64_t q = 0; q < cc->cells.size(); ++q) cc->c_cells[q] = col.position[cc->cells[q]];
    cc->c_inc_offset.assign(n_sites + 1, 0);
    cc->c_inc_cell.assign(cc->inc_cell.size(), 0);
    cc->c_inc_which.assign(cc->inc_which.size(), 0);
    uint64_t acc = 0;
    for (uint64_t k = 0; k < n_sites; ++k) {
        const uint32_t i = col.order[k];
        cc->c_inc_offset[k] = acc;
        for (uint64_t a = cc->inc_offset[i]; a < cc->inc_offset[i + 1]; ++a) {
            cc->c_inc_cell[acc] = cc->inc_cell[a];
            cc->c_inc_which[acc] = cc->inc_which[a];
            ++acc;
        }
    }
    cc->c_inc_offset[n_sites] = acc;
    return cc;
}

umc_cells* make_hypercubic(uint64_t L)
{
    // lattice/hypercubic.hpp:15-64
    if (L == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "hypercubic_plaquettes: L must be positive");
    if (L > 0xFFFF) throw Error(UMC_ERR_OVERFLOW, "hypercubic_plaquettes: site count does not fit uint32_t");
    const uint64_t L4 = L * L * L * L;
    if (4 * L4 > kMax32) throw Error(UMC_ERR_OVERFLOW, "hypercubic_plaquettes: site count does not fit uint32_t");
    std::vector<uint32_t> cells;
    cells.reserve(24 * L4);
    auto index = [L, L4](uint64_t mu, const uint64_t* c) {
        return uint32_t(mu * L4 + (((c[0] * L + c[1]) * L + c[2]) * L + c[3]));
    };
    for (uint64_t mu = 0; mu < 4; ++mu)
        for (uint64_t nu = mu + 1; nu < 4; ++nu)
            for (uint64_t t = 0; t < L; ++t)
                for (uint64_t z = 0; z < L; ++z)
                    for (uint64_t y = 0; y < L; ++y)
                        for (uint64_t x = 0; x < L; ++x) {
                            const uint64_t c[4] = {t, z, y, x};
                            uint64_t cm[4] = {t, z, y, x}, cn[4] = {t, z, y, x};
                            cm[mu] = (cm[mu] + 1) % L;
                            cn[nu] = (cn[nu] + 1) % L;
                            cells.push_back(index(mu, c));
                            cells.push_back(index(nu, cm));
                            cells.push_back(index(mu, cn));
                            cells.push_back(index(nu, c));
                        }
    return make_cells(4 * L4, 4, cells.data(), 6 * L4, Lattice::Hypercubic, L, 4);
}

umc_cells* make_square_plaquettes(uint64_t L)
{
    if (L == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "square_plaquettes: L must be positive");
    if (2 * L * L > kMax32) throw Error(UMC_ERR_OVERFLOW, "square_plaquettes: link count does not fit uint32_t");
    const uint64_t L2 = L * L;
    std::vector<uint32_t> cells;
    cells.reserve(4 * L2);
    for (uint64_t y = 0; y < L; ++y)
        for (uint64_t x = 0; x < L; ++x) {
            cells.push_back(uint32_t(y * L + x));
            cells.push_back(uint32_t(L2 + y * L + (x + 1) % L));
            cells.push_back(uint32_t(((y + 1) % L) * L + x));
            cells.push_back(uint32_t(L2 + y * L + x));
        }
    return make_cells(2 * L2, 4, cells.data(), L2, Lattice::SquarePlaquettes, L, 2);
}

}  // namespace umc

// ============================================================== C ABI: tables

namespace {
template <class F>
int guarded(F&& f)
{
    try {
        umc::set_last_error("");
        f();
        return UMC_OK;
    } catch (const umc::Error& e) {
        umc::set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        umc::set_last_error("out of host memory");
        return UMC_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        umc::set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}

void fill_colouring(const umc::Colouring& col, uint32_t* n_colours, uint32_t* colour, uint32_t* position)
{
    if (n_colours) *n_colours = col.n_colours;
    if (colour) std::copy(col.colour.begin(), col.colour.end(), colour);
    if (position) std::copy(col.position.begin(), col.position.end(), position);
}
}  // namespace

extern "C" {

const char* umc_last_error(void) { return umc::last_error(); }
int umc_abi_version(void) { return UMC_ABI_VERSION; }

int umc_graph_create(uint64_t n_sites, const uint32_t* edge_i, const uint32_t* edge_j, uint64_t n_edges,
                     int symmetric, umc_graph** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_graph(n_sites, edge_i, edge_j, n_edges, symmetric != 0, umc::Lattice::Generic, nullptr);
    });
}

int umc_graph_create_payload(uint64_t n_sites, const uint32_t* edge_i, const uint32_t* edge_j, uint64_t n_edges,
                             int symmetric, const void* payload, uint32_t payload_bytes, umc_graph** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        if (payload_bytes == 0 || payload_bytes > UMC_MAX_PAYLOAD_BYTES)
            throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "PairGraph: payload size must be 1 to 256 bytes");
        if (n_edges && !payload) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "PairGraph: null payload array");
        std::unique_ptr<umc_graph> g(
            umc::make_graph(n_sites, edge_i, edge_j, n_edges, symmetric != 0, umc::Lattice::Generic, nullptr));
        const auto* p = static_cast<const uint8_t*>(payload);
        g->payload_bytes = payload_bytes;
        g->payload.assign(p, p + n_edges * payload_bytes);
        *out = g.release();
    });
}

uint32_t umc_graph_payload_bytes(const umc_graph* g) { return g ? g->payload_bytes : 0u; }

int umc_graph_payloads(const umc_graph* g, void* out)
{
    return guarded([&] {
        if (!g) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null graph");
        if (!g->payload_bytes) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "graph has no payload (NoPayload)");
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output");
        auto* o = static_cast<uint8_t*>(out);
        const size_t b = g->payload_bytes;
        for (size_t a = 0; a < g->slot_edge.size(); ++a)
            std::memcpy(o + a * b, g->payload.data() + size_t(g->slot_edge[a]) * b, b);
    });
}

int umc_graph_slot_edges(const umc_graph* g, uint32_t* out)
{
    return guarded([&] {
        if (!g || !out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        umc::materialize(g);
        std::copy(g->slot_edge.begin(), g->slot_edge.end(), out);
    });
}

int umc_graph_square(uint64_t Lx, uint64_t Ly, umc_graph** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_square(Lx, Ly);
    });
}

int umc_graph_cubic(uint64_t Lx, uint64_t Ly, uint64_t Lz, umc_graph** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_cubic(Lx, Ly, Lz);
    });
}

void umc_graph_destroy(umc_graph* g) { delete g; }
uint64_t umc_graph_sites(const umc_graph* g) { return g ? g->n : 0; }
uint64_t umc_graph_slots(const umc_graph* g)
{
    if (!g) return 0;
    return g->materialized ? g->bonds.size() : g->n * g->max_degree;
}

int umc_graph_csr(const umc_graph* g, uint32_t* offset, uint32_t* bonds)
{
    return guarded([&] {
        if (!g) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null graph");
        umc::materialize(g);
        if (offset) std::copy(g->offset.begin(), g->offset.end(), offset);
        if (bonds) std::copy(g->bonds.begin(), g->bonds.end(), bonds);
    });
}

int umc_graph_colouring(const umc_graph* g, uint32_t* n_colours, uint32_t* colour, uint32_t* position)
{
    return guarded([&] {
        if (!g) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null graph");
        umc::materialize(g);
        fill_colouring(g->col, n_colours, colour, position);
    });
}

int umc_cells_create(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells, umc_cells** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_cells(n_sites, arity, cells, n_cells, umc::Lattice::Generic, 0, 0);
    });
}

int umc_cells_hypercubic(uint64_t L, umc_cells** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_hypercubic(L);
    });
}

int umc_cells_square_plaquettes(uint64_t L, umc_cells** out)
{
    return guarded([&] {
        if (!out) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = umc::make_square_plaquettes(L);
    });
}

void umc_cells_destroy(umc_cells* c) { delete c; }
uint64_t umc_cells_sites(const umc_cells* c) { return c ? c->n_sites : 0; }
uint64_t umc_cells_count(const umc_cells* c) { return c ? c->n_cells() : 0; }
uint32_t umc_cells_arity(const umc_cells* c) { return c ? c->arity : 0; }

int umc_cells_table(const umc_cells* c, uint32_t* cells)
{
    return guarded([&] {
        if (!c) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null cells");
        if (cells) std::copy(c->cells.begin(), c->cells.end(), cells);
    });
}

int umc_cells_incidence(const umc_cells* c, uint64_t* offset, uint32_t* inc_cell, uint8_t* inc_which)
{
    return guarded([&] {
        if (!c) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null cells");
        if (offset) std::copy(c->inc_offset.begin(), c->inc_offset.end(), offset);
        if (inc_cell) std::copy(c->inc_cell.begin(), c->inc_cell.end(), inc_cell);
        if (inc_which) std::copy(c->inc_which.begin(), c->inc_which.end(), inc_which);
    });
}

int umc_cells_colouring(const umc_cells* c, uint32_t* n_colours, uint32_t* colour, uint32_t* position)
{
    return guarded([&] {
        if (!c) throw umc::Error(UMC_ERR_INVALID_ARGUMENT, "null cells");
        fill_colouring(c->col, n_colours, colour, position);
    });
}

}  // extern "C"
