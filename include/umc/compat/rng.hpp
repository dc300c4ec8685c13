// The reference's <rng.hpp> on the engine: Pcg32.
#pragma once

#include <umc/compat/engine.hpp>

using umc::gpu::Pcg32;
