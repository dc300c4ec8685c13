// The reference's <lattice/hypercubic.hpp> on the engine: hypercubic_plaquettes.
#pragma once

#include <umc/compat/engine.hpp>
#include <lattice/cell_complex.hpp>

using umc::gpu::hypercubic_plaquettes;
