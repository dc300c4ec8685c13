// The reference's <term/sun_plaquette.hpp> on the engine: SUPlaquetteTerm.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/sun.hpp>
#include <term/cell.hpp>

using umc::gpu::SUPlaquetteTerm;
