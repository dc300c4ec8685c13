// The reference's <lattice/cell_complex.hpp> on the engine: Cell, CellComplex, CellComplexLike.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::Cell;
using umc::gpu::CellComplex;
using umc::gpu::CellComplexLike;
