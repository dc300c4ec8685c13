// The reference's <term/heisenberg.hpp> on the engine: HeisenbergTerm.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/vector.hpp>
#include <term/cell.hpp>

using umc::gpu::HeisenbergTerm;
