// umc/compat: headers at the reference library's own include paths
// (driver.hpp, model.hpp, rng.hpp, dof/, example/, lattice/, model/, term/),
// each bringing the names its reference header declares into the global
// namespace, so that a reference program compiles unchanged against the
// engine's facade:
//     g++ -std=c++23 -I<repo>/include -I<repo>/include/umc/compat prog.cpp
//         -L<repo>/universal_classical_montecarlo_b200 -lumc_b200
// This header is the facade itself (namespace umc::gpu) with no global names.
#pragma once

#include <umc/driver.hpp>
#include <umc/lattice.hpp>

#if defined(__CUDACC__)
#include <umc/device_facade.cuh>  // user-written terms on the device (nvcc builds)
#endif
