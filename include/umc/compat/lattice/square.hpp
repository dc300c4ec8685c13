// The reference's <lattice/square.hpp> on the engine: square_lattice.
#pragma once

#include <umc/compat/engine.hpp>
#include <lattice/pair_graph.hpp>

using umc::gpu::square_lattice;
