// The reference's <model/pair.hpp> on the engine: PairModel.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>
#include <lattice/pair_graph.hpp>
#include <term/cell.hpp>

using umc::gpu::PairModel;
