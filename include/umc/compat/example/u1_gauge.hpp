// The reference's <example/u1_gauge.hpp> on the engine: U1Gauge.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/u1.hpp>
#include <lattice/cell_complex.hpp>
#include <lattice/hypercubic.hpp>

using umc::gpu::U1Gauge;
