// The reference's <term/cell.hpp> on the engine: CellTerm.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>

using umc::gpu::CellTerm;
