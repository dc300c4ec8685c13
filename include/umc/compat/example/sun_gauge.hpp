// The reference's <example/sun_gauge.hpp> on the engine: SUGauge, SU2Gauge, SU3Gauge.
#pragma once

#include <umc/compat/engine.hpp>
#include <dof/sun.hpp>
#include <lattice/cell_complex.hpp>
#include <lattice/hypercubic.hpp>

using umc::gpu::SUGauge;
using umc::gpu::SU2Gauge;
using umc::gpu::SU3Gauge;
