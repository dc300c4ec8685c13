// The reference's <dof/proposal.hpp> on the engine: Proposal.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::Proposal;
