// The reference's <example/vector_spin.hpp> on the engine: VectorSpin, XY, Heisenberg.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/vector.hpp>
#include <lattice/pair_graph.hpp>

using umc::gpu::VectorSpin;
using umc::gpu::XY;
using umc::gpu::Heisenberg;
