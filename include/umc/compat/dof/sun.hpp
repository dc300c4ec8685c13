// The reference's <dof/sun.hpp> on the engine: SULink, SUDof, SUShift, plaquette.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/dof.hpp>

using umc::gpu::SULink;
using umc::gpu::SUDof;
using umc::gpu::SUShift;
using umc::gpu::plaquette;
namespace sun_detail = umc::gpu::sun_detail;
