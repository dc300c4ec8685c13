// umc_nvtx.hpp -- NVTX ranges around the C ABI's run calls and every kernel
// launch, so a profiler timeline (Nsight Systems, ncu's NVTX filters) shows
// which sample()/run() call and which pass each kernel belongs to.  NVTX v3 is
// header-only: with no tool attached a range costs one well-predicted branch.
#pragma once

#include <nvtx3/nvToolsExt.h>

namespace umc {

struct NvtxRange
{
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Names of the kernel kinds of umc_chain_kernel_stats (UMC_KERNEL_*).
inline const char* kernel_kind_name(int kind)
{
    static const char* const names[] = {"metropolis pass", "wolff union", "wolff flip", "observe",
                                        "gauge pass",      "batch",       "learned",    "other",
                                        "wolff merge",     "fused step"};
    return kind >= 0 && kind < int(sizeof names / sizeof names[0]) ? names[kind] : "kernel";
}

}  // namespace umc
