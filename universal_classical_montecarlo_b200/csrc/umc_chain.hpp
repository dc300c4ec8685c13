// umc_chain.hpp -- the device chain behind the C ABI's umc_chain handle.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "umc_device.cuh"
#include "umc_tables.hpp"

namespace umc {

void cuda_check(cudaError_t e, const char* what);

// Device buffer owned by a chain (freed on destruction).
struct DevBuf
{
    void* p = nullptr;
    size_t bytes = 0;
    void alloc(size_t b, const char* what);
    void free_();
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Ising acceptance thresholds: accept iff draw <= tm1[s*h + D] where the
// reference would accept iff log_p >= 0 || log(k 2^-32) < log_p with
// log_p = -beta * (2 J s h) + 0.0 (driver.hpp:39-40, example/ising.hpp:46-56).
std::vector<uint32_t> ising_metropolis_thresholds(int32_t J, double beta, uint32_t D);
// Wolff-Ising: activate iff draw < cw[s_i s_j > 0] where the reference
// activates iff k 2^-32 < 1 - exp(-beta * dE) (driver.hpp:151), dE = 2 J s_i s_j.
void ising_wolff_thresholds(int32_t J, double beta, unsigned long long cw[2]);

}  // namespace umc

struct umc_chain
{
    umc_chain_desc desc{};
    int model = 0;
    int N = 1;               // components (VectorSpin<N>, SU(N))
    uint64_t n = 0;          // sites or links
    uint32_t n_colours = 0;
    std::vector<uint64_t> class_start;
    bool stencil = false;
    uint64_t dims[3] = {1, 1, 1};
    bool packed_ising = false;
    bool symmetric = true;
    uint32_t max_degree = 0;
    int32_t J_int = 0;
    float J = 1.0f;

    // host copies kept for lazy uploads
    std::vector<uint32_t> h_off, h_adj, h_slot, h_position;
    // cell-complex models
    uint64_t n_cells = 0;
    uint32_t max_incident = 0;
    uint32_t cell_dim = 0;
    uint64_t L = 0;
    std::vector<uint32_t> h_cells;
    std::vector<uint64_t> h_inc_off;
    std::vector<uint32_t> h_inc_cell;
    std::vector<uint8_t> h_inc_which;

    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    umc::DevBuf field, staging, off, adj, slot, position, lab0, lab1, xlist;
    umc::DevBuf cells, inc_off, inc_cell, inc_which;
    umc::DevBuf partials, ctl, records, sizes, tm1;
    size_t field_bytes = 0;
    size_t elem_bytes = 0;
    uint32_t comps = 1;  // scalars per site in the host layout
    uint32_t max_grid = 0;

    uint64_t max_records = 4096;
    // pinned host image of [status | records | sizes]: a fetch is one round
    // trip (three async copies, one stream synchronisation)
    void* host_stage = nullptr;
    size_t host_stage_bytes = 0;
    cudaEvent_t upload_done = nullptr;  // set_field waits on the copy, not the scatter
    bool stream_records = false;        // copy each record to host_stage as it is written
    uint64_t streamed = 0;              // records [0, streamed) already in host_stage
    cudaStream_t rec_stream = nullptr;  // those copies, off the chain's stream
    cudaEvent_t rec_ready[2] = {nullptr, nullptr};
    int rec_next = 0;
    // umc_chain_upload_async: copy stream, two staging buffers and their events
    cudaStream_t up_stream = nullptr;
    umc::DevBuf up_staging[2];
    cudaEvent_t up_copied[2] = {nullptr, nullptr}, up_consumed[2] = {nullptr, nullptr};
    int up_next = 0;
    uint64_t rec_pending = 0;
    bool rec_overflow = false;
    uint64_t sweeps = 0, flips = 0;
    int lab_cur = 0;  // which Wolff label buffer is the identity
    uint64_t wolff_flips_done = 0;
    double wolff_size_sum = 0.0;

    double tm1_beta = 0.0;
    bool tm1_valid = false;
    std::vector<uint32_t> h_tm1;
    double cw_beta = 0.0;
    bool cw_valid = false;
    unsigned long long cw[2] = {0, 0};

    // one cooperative kernel per step on regular lattices (umc_fused.cuh)
    bool fused = true;
    int fused_grid = -1;  // co-resident blocks; 0 = cooperative launch unavailable

    // learned proposal (U(1) only)
    void* learned = nullptr;

    // kernel accounting
    bool timing = false;
    uint64_t launches[UMC_KERNEL_KINDS] = {};
    double device_ms[UMC_KERNEL_KINDS] = {};
    struct Timed
    {
        int kind;
        cudaEvent_t a, b;
    };
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> event_pool;
};

namespace umc {
// Bracket one kernel launch: counts it and, with timing on, records events.
struct LaunchScope
{
    umc_chain* c;
    int kind;
    cudaEvent_t a = nullptr;
    LaunchScope(umc_chain* chain, int k);
    ~LaunchScope();
};
void collect_kernel_times(umc_chain* c);
}  // namespace umc
