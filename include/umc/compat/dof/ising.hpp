// The reference's <dof/ising.hpp> on the engine: IsingSpin, IsingDof, dot, Flip, FixedAxis.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>

using umc::gpu::IsingSpin;
using umc::gpu::IsingDof;
using umc::gpu::dot;
using umc::gpu::Flip;
using umc::gpu::FixedAxis;
