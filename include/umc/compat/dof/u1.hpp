// The reference's <dof/u1.hpp> on the engine: U1Link, U1Dof, U1Shift, plaquette.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>

using umc::gpu::U1Link;
using umc::gpu::U1Dof;
using umc::gpu::U1Shift;
using umc::gpu::plaquette;
