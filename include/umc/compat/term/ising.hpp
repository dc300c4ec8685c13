// The reference's <term/ising.hpp> on the engine: IsingTerm.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/ising.hpp>
#include <term/cell.hpp>

using umc::gpu::IsingTerm;
