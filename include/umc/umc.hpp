// umc/umc.hpp -- C++23 facade of the B200 engine with the reference library's
// names (universal_monte_carlo: rng.hpp, driver.hpp, model.hpp, lattice/,
// dof/, example/).  Everything lives in namespace umc::gpu; unless
// UMC_NO_GLOBAL_NAMES is defined the names are also brought into the global
// namespace, as the reference declares them, so reference-style programs
// compile after swapping their includes for this one.  Link with
// libumc_b200.so.
#pragma once

#include "detail.hpp"
#include "dof.hpp"
#include "driver.hpp"
#include "generic.hpp"
#include "lattice.hpp"
#include "models.hpp"
#include "rng.hpp"

#if defined(__CUDACC__)
#include "device_facade.cuh"  // user-written terms on the device (nvcc builds)
#endif

#ifndef UMC_NO_GLOBAL_NAMES
using umc::gpu::Bond;
using umc::gpu::Cell;
using umc::gpu::CellComplex;
using umc::gpu::CellComplexLike;
using umc::gpu::CellModel;
using umc::gpu::CellTerm;
using umc::gpu::cubic_lattice;
using umc::gpu::Dof;
using umc::gpu::EnergyModel;
using umc::gpu::FixedAxis;
using umc::gpu::Flip;
using umc::gpu::Heisenberg;
using umc::gpu::HeisenbergTerm;
using umc::gpu::Hits;
using umc::gpu::hypercubic_plaquettes;
using umc::gpu::Ising;
using umc::gpu::IsingDof;
using umc::gpu::IsingSpin;
using umc::gpu::IsingTerm;
using umc::gpu::LocalRotation;
using umc::gpu::Metropolis;
using umc::gpu::ModelLike;
using umc::gpu::NoPayload;
using umc::gpu::PairGraph;
using umc::gpu::PairGraphLike;
using umc::gpu::PairModel;
using umc::gpu::Pcg32;
using umc::gpu::plaquette;
using umc::gpu::Proposal;
using umc::gpu::square_lattice;
using umc::gpu::square_plaquettes;
using umc::gpu::SUDof;
using umc::gpu::SU2Gauge;
using umc::gpu::SU3Gauge;
using umc::gpu::SUGauge;
using umc::gpu::SULink;
using umc::gpu::SUPlaquetteTerm;
using umc::gpu::SUShift;
using umc::gpu::U1Dof;
using umc::gpu::U1Gauge;
using umc::gpu::U1Link;
using umc::gpu::U1PlaquetteTerm;
using umc::gpu::U1Shift;
using umc::gpu::UniformSphereN;
using umc::gpu::VectorDof;
using umc::gpu::VectorSpin;
using umc::gpu::Wolff;
using umc::gpu::WolffModel;
using umc::gpu::XY;
#endif
