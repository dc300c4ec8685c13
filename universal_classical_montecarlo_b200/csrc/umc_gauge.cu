// umc_gauge.cu -- gauge models on a plaquette complex: U(1) angles and SU(N)
// links (example/u1_gauge.hpp, example/sun_gauge.hpp, or CellModel with
// U1PlaquetteTerm / SUPlaquetteTerm, model/cell.hpp).
//
// A sweep is one kernel per colour class of links (no two links of a class
// share a plaquette), each link taking `hits` Metropolis steps against a staple
// built once, followed by one FP64 reduction of the plaquettes into the sweep's
// record [S, <P>, Q, ..., accepted].

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "umc_chain.hpp"
#include "umc_gauge.hpp"
#include "umc_gauge_kernels.cuh"

namespace umc {

namespace {

uint32_t ggrid(const umc_chain* c, uint64_t work)
{
    const uint64_t b = (work + kBlock - 1) / kBlock;
    return uint32_t(b < 1 ? 1 : (b > c->max_grid ? c->max_grid : b));
}

void gcheck(const char* what) { cuda_check(cudaGetLastError(), what); }

}  // namespace

void gauge_configure(umc_chain* c)
{
    const umc_cells* cc = c->desc.cells;
    if (!cc) throw Error(UMC_ERR_INVALID_ARGUMENT, "gauge models need a cell complex");
    if (cc->arity != 4) throw Error(UMC_ERR_UNSUPPORTED, "gauge models need plaquettes (arity 4)");
    if (c->model == UMC_MODEL_U1) {
        if (c->desc.proposal != UMC_PROPOSAL_U1SHIFT) throw Error(UMC_ERR_UNSUPPORTED, "U(1) takes U1Shift");
        c->N = 1;
        c->comps = 1;
    } else {
        if (c->N != 2 && c->N != 3) throw Error(UMC_ERR_UNSUPPORTED, "SU(N) is provided for N = 2 and 3");
        if (c->desc.proposal != UMC_PROPOSAL_SUSHIFT) throw Error(UMC_ERR_UNSUPPORTED, "SU(N) takes SUShift");
        c->comps = uint32_t(2 * c->N * c->N);
    }
    if (!std::isfinite(c->desc.coupling)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta must be finite");
    c->n = cc->n_sites;
    c->n_colours = cc->col.n_colours;
    if (c->n_colours + 1 > uint32_t(kMaxPasses - 1))
        throw Error(UMC_ERR_UNSUPPORTED, "cell complex needs more colour classes than the engine supports");
    c->class_start = cc->col.class_start;
    c->h_position = cc->col.position;
    c->n_cells = cc->n_cells();
    if (c->n_cells >= (1ull << 30)) throw Error(UMC_ERR_OVERFLOW, "too many cells for the packed incidence");
    c->h_cells = cc->c_cells;
    c->h_inc_off.assign(cc->c_inc_offset.begin(), cc->c_inc_offset.end());
    c->h_inc_cell.resize(cc->c_inc_cell.size());
    for (size_t e = 0; e < cc->c_inc_cell.size(); ++e) c->h_inc_cell[e] = (cc->c_inc_cell[e] << 2) | cc->c_inc_which[e];
    if (!c->h_inc_off.empty() && c->h_inc_off.back() > 0xFFFFFFFFull) throw Error(UMC_ERR_OVERFLOW, "incidence count exceeds uint32");
    c->max_incident = 0;
    for (size_t k = 0; k + 1 < c->h_inc_off.size(); ++k)
        c->max_incident = std::max<uint32_t>(c->max_incident, uint32_t(c->h_inc_off[k + 1] - c->h_inc_off[k]));
    c->J = float(c->desc.coupling);
    c->elem_bytes = 4;
    c->stencil = false;
}

void gauge_cold_start(umc_chain* c)
{
    std::vector<uint32_t> off32(c->h_inc_off.begin(), c->h_inc_off.end());
    auto up = [&](DevBuf& b, const void* p, size_t bytes, const char* what) {
        b.alloc(bytes, what);
        if (bytes) cuda_check(cudaMemcpyAsync(b.p, p, bytes, cudaMemcpyHostToDevice, c->stream), what);
    };
    up(c->cells, c->h_cells.data(), c->h_cells.size() * 4, "upload cells");
    up(c->inc_off, off32.data(), off32.size() * 4, "upload incidence offsets");
    up(c->inc_cell, c->h_inc_cell.data(), c->h_inc_cell.size() * 4, "upload incidence");
    up(c->position, c->h_position.data(), c->h_position.size() * 4, "upload positions");
    cuda_check(cudaStreamSynchronize(c->stream), "upload gauge tables");
    if (c->model == UMC_MODEL_U1) {
        cuda_check(cudaMemsetAsync(c->field.p, 0, c->field_bytes, c->stream), "cold start");
    } else {
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        if (c->N == 2) gauge_identity<2><<<ggrid(c, c->n), kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n));
        else gauge_identity<3><<<ggrid(c, c->n), kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n));
    }
    gcheck("gauge cold start");
}

void gauge_release(umc_chain*) {}

void gauge_set_field(umc_chain* c, const void* host_field)
{
    if (!c->staging.p) c->staging.alloc(c->field_bytes, "staging");
    cuda_check(cudaMemcpyAsync(c->staging.p, host_field, c->field_bytes, cudaMemcpyHostToDevice, c->stream), "upload field");
    {
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        gauge_scatter<<<ggrid(c, c->n), kBlock, 0, c->stream>>>(c->staging.as<float>(), c->field.as<float>(), uint32_t(c->n),
                                                                 c->comps, c->position.as<uint32_t>());
    }
    gcheck("scatter links");
    cuda_check(cudaStreamSynchronize(c->stream), "upload field");
}

void gauge_get_field(umc_chain* c, void* host_field)
{
    if (!c->staging.p) c->staging.alloc(c->field_bytes, "staging");
    {
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        gauge_gather<<<ggrid(c, c->n), kBlock, 0, c->stream>>>(c->field.as<float>(), c->staging.as<float>(), uint32_t(c->n),
                                                                c->comps, c->position.as<uint32_t>());
    }
    gcheck("gather links");
    cuda_check(cudaMemcpyAsync(host_field, c->staging.p, c->field_bytes, cudaMemcpyDeviceToHost, c->stream), "download field");
    cuda_check(cudaStreamSynchronize(c->stream), "download field");
}

void gauge_randomize(umc_chain* c, unsigned long long seed)
{
    const uint32_t g = ggrid(c, c->n);
    {
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        switch (c->N) {
        case 1: gauge_haar<1><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), seed, c->position.as<uint32_t>()); break;
        case 2: gauge_haar<2><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), seed, c->position.as<uint32_t>()); break;
        default: gauge_haar<3><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), seed, c->position.as<uint32_t>()); break;
        }
    }
    gcheck("Haar start");
    cuda_check(cudaStreamSynchronize(c->stream), "Haar start");
}

namespace {
void plaquettes(umc_chain* c, double* record, int pass, int n_passes)
{
    const PassOut o{c->ctl.as<DevCtl>(), c->partials.as<double>(), record, nullptr, pass, n_passes, 1};
    const uint32_t g = ggrid(c, c->n_cells);
    LaunchScope ls(c, UMC_KERNEL_OBSERVE);
    const uint4* cells = c->cells.as<uint4>();
    switch (c->N) {
    case 1: plaquette_sum<1><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), cells, uint32_t(c->n_cells), c->n_cells, c->J, o); break;
    case 2: plaquette_sum<2><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), cells, uint32_t(c->n_cells), c->n_cells, c->J, o); break;
    default: plaquette_sum<3><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), uint32_t(c->n), cells, uint32_t(c->n_cells), c->n_cells, c->J, o); break;
    }
    gcheck("plaquette reduction");
}
}  // namespace

void gauge_sweep(umc_chain* c, double beta, double* record)
{
    GaugeArgs a{};
    a.f = c->field.as<float>();
    a.n = uint32_t(c->n);
    a.inc_off = c->inc_off.as<uint32_t>();
    a.inc = c->inc_cell.as<uint32_t>();
    a.cells = c->cells.as<uint4>();
    a.seed = c->desc.seed;
    a.sweep = c->sweeps;
    a.hits = c->desc.hits;
    a.model_beta = c->J;
    a.driver_beta = float(beta);
    a.width = float(c->desc.width);
    a.model_beta64 = c->desc.coupling;
    a.driver_beta64 = beta;
    a.err = c->N == 1 ? u1_metropolis_err(beta, c->desc.coupling, c->max_incident) : 0.0f;  // SU(N): FP32 test
    const int np = int(c->n_colours) + 1;
    for (uint32_t p = 0; p < c->n_colours; ++p) {
        a.first = uint32_t(c->class_start[p]);
        a.count = uint32_t(c->class_start[p + 1] - c->class_start[p]);
        a.out = PassOut{c->ctl.as<DevCtl>(), c->partials.as<double>(), nullptr, nullptr, int(p), np, 0};
        const uint32_t g = ggrid(c, a.count);
        LaunchScope ls(c, UMC_KERNEL_GAUGE);
        switch (c->N) {
        case 1: u1_pass<<<g, kBlock, 0, c->stream>>>(a); break;
        case 2: su_pass<2><<<g, kBlock, 0, c->stream>>>(a); break;
        default: su_pass<3><<<g, kBlock, 0, c->stream>>>(a); break;
        }
        gcheck("gauge colour pass");
    }
    plaquettes(c, record, int(c->n_colours), np);
    c->sweeps++;
}

void gauge_observe(umc_chain* c, double* record) { plaquettes(c, record, kMaxPasses - 1, 1); }

}  // namespace umc
