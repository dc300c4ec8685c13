// The reference's <term/plaquette.hpp> on the engine: U1PlaquetteTerm.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/u1.hpp>
#include <term/cell.hpp>

using umc::gpu::U1PlaquetteTerm;
