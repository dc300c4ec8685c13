// The reference's <example/ising.hpp> on the engine: Ising.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/ising.hpp>
#include <lattice/pair_graph.hpp>

using umc::gpu::Ising;
