// The reference's <driver.hpp> on the engine: Metropolis, Wolff, WolffModel.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/proposal.hpp>
#include <model.hpp>

using umc::gpu::Metropolis;
using umc::gpu::Wolff;
using umc::gpu::WolffModel;
