// umc_tables.hpp -- host-side topology tables and their colour-major relabelling.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/umc_b200.h"

namespace umc {

// A failure that crosses the C ABI as a status code plus a message.
struct Error : std::runtime_error
{
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const char* msg);

enum class Lattice : int { Generic = 0, Square = 1, Cubic = 2, Hypercubic = 3, SquarePlaquettes = 4 };

// A partition of sites into classes of mutually independent updates.
struct Colouring
{
    uint32_t n_colours = 0;
    std::vector<uint32_t> colour;       // site -> colour
    std::vector<uint32_t> position;     // site -> colour-major index
    std::vector<uint32_t> order;        // colour-major index -> site
    std::vector<uint64_t> class_start;  // n_colours + 1 offsets into colour-major order
};

}  // namespace umc

// PairGraph (lattice/pair_graph.hpp:29-107) plus what the device passes need.
struct umc_graph
{
    uint64_t n = 0;
    bool symmetric = true;
    std::vector<uint32_t> ei, ej;                    // edge list as given
    std::vector<uint32_t> offset, bonds, slot_edge;  // reference-order CSR
    umc::Lattice kind = umc::Lattice::Generic;
    uint64_t dims[3] = {1, 1, 1};
    umc::Colouring col;
    std::vector<uint32_t> c_offset, c_bonds, c_slot_edge;  // colour-major CSR
    uint32_t max_degree = 0;
    // true when the regular-lattice stencil kernels reproduce this graph exactly
    bool stencil = false;
    // regular lattices keep only their extents until a table is asked for
    // (edge list, CSR, colouring arrays); n, degree and the colour classes are
    // known in closed form
    bool materialized = true;
    // PairGraph<P>'s per-bond payload (lattice/pair_graph.hpp:36-41): one
    // payload_bytes record per input edge, copied into both directed slots
    // (slot a carries payload[slot_edge[a]]); payload_bytes 0 = NoPayload
    uint32_t payload_bytes = 0;
    std::vector<uint8_t> payload;
};

// CellComplex<A> (lattice/cell_complex.hpp:21-87) plus the colour-major copy.
struct umc_cells
{
    uint64_t n_sites = 0;
    uint32_t arity = 0;
    std::vector<uint32_t> cells;  // n_cells * arity
    std::vector<uint64_t> inc_offset;
    std::vector<uint32_t> inc_cell;
    std::vector<uint8_t> inc_which;
    umc::Lattice kind = umc::Lattice::Generic;
    uint64_t L = 0;
    uint32_t dim = 0;
    umc::Colouring col;
    std::vector<uint32_t> c_cells;  // cells with colour-major link ids
    std::vector<uint64_t> c_inc_offset;
    std::vector<uint32_t> c_inc_cell;
    std::vector<uint8_t> c_inc_which;
    uint32_t max_incident = 0;
    bool stencil = false;
    uint64_t n_cells() const { return arity ? cells.size() / arity : 0; }
};

namespace umc {

umc_graph* make_graph(uint64_t n, const uint32_t* ei, const uint32_t* ej, uint64_t m, bool symmetric,
                      Lattice kind, const uint64_t dims[3]);
umc_graph* make_square(uint64_t Lx, uint64_t Ly);
umc_graph* make_cubic(uint64_t Lx, uint64_t Ly, uint64_t Lz);
// Builds the edge list, CSR and colouring of a lazily created regular lattice.
void materialize(const umc_graph* g);
umc_cells* make_cells(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells,
                      Lattice kind, uint64_t L, uint32_t dim);
umc_cells* make_hypercubic(uint64_t L);
umc_cells* make_square_plaquettes(uint64_t L);

}  // namespace umc
