// The reference's <dof/dof.hpp> on the engine: Dof.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::Dof;
