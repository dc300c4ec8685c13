// The reference's <dof/vector.hpp> on the engine: VectorDof, dot, UniformSphereN, LocalRotation.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>

using umc::gpu::VectorDof;
using umc::gpu::dot;
using umc::gpu::UniformSphereN;
using umc::gpu::LocalRotation;
