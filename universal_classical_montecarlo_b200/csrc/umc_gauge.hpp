// umc_gauge.hpp -- gauge-model half of the chain (U(1) and SU(N) links on a
// cell complex): configuration, field transfer and the colour-pass sweep.
#pragma once

struct umc_chain;

namespace umc {

void gauge_configure(umc_chain* c);
void gauge_cold_start(umc_chain* c);
void gauge_release(umc_chain* c);
void gauge_set_field(umc_chain* c, const void* host_field);
void gauge_get_field(umc_chain* c, void* host_field);
void gauge_randomize(umc_chain* c, unsigned long long seed);
void gauge_sweep(umc_chain* c, double beta, double* record);
void gauge_observe(umc_chain* c, double* record);

}  // namespace umc
