// umc_gauge.cu -- placeholder: gauge models are not built yet.
#include "umc_chain.hpp"
#include "umc_gauge.hpp"

namespace umc {
[[noreturn]] static void nyi() { throw Error(UMC_ERR_UNSUPPORTED, "gauge models are not available in this build"); }
void gauge_configure(umc_chain*) { nyi(); }
void gauge_cold_start(umc_chain*) { nyi(); }
void gauge_release(umc_chain*) {}
void gauge_set_field(umc_chain*, const void*) { nyi(); }
void gauge_get_field(umc_chain*, void*) { nyi(); }
void gauge_randomize(umc_chain*, unsigned long long) { nyi(); }
void gauge_sweep(umc_chain*, double, double*) { nyi(); }
void gauge_observe(umc_chain*, double*) { nyi(); }
}  // namespace umc
