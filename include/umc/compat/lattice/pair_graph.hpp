// The reference's <lattice/pair_graph.hpp> on the engine: Bond, NoPayload, PairGraph, PairGraphLike.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::Bond;
using umc::gpu::NoPayload;
using umc::gpu::PairGraph;
using umc::gpu::PairGraphLike;
