// The reference's <model.hpp> on the engine: ModelLike, EnergyModel.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::ModelLike;
using umc::gpu::EnergyModel;
