// The reference's <model/cell.hpp> on the engine: CellModel.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>
#include <lattice/cell_complex.hpp>
#include <term/cell.hpp>

using umc::gpu::CellModel;
