// umc_gslab.cu -- one gauge lattice over several GPUs: the U(1) and SU(N)
// link sweeps of a plaquette complex split over ranks (one process per GPU).
//
// The caller assigns every link to a rank.  A rank keeps its owned links and
// the halo links that the plaquettes of its owned links touch.  Local links
// are numbered as the single-GPU chain numbers them -- its colour-major order
// (colour classes in turn) restricted to the owned links, then the halo links
// in the same order -- and each local link carries its global colour-major
// index, whose key it draws from.  Each owned link's incidence list keeps the
// single-GPU order of its plaquettes, so the staple sums round the same way.
// The colour pass is the single-GPU kernel itself (u1_pass, su_pass<N>) on
// the local tables; between passes the caller moves the links of the class
// just updated to the ranks that hold them as halo (umc_gslab_pack on the
// owner, umc_gslab_unpack on the holder; NCCL send/recv or any copy).  The
// union of the ranks' updates is then the single-GPU chain, bit for bit.
//
// The reference has no decomposition (one chain per driver object,
// driver.hpp:17-68); the per-link rule is its Metropolis::sweep body
// (driver.hpp:34-42) with the plaquette terms of term/plaquette.hpp and
// term/sun_plaquette.hpp and the proposals of dof/u1.hpp and dof/sun.hpp.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "umc_chain.hpp"
#include "umc_gauge_kernels.cuh"
#include "umc_nvtx.hpp"

namespace umc {
namespace {

// buf[q * m + j] = f[q * n + idx[j]] for the comps planes
__global__ void gslab_pack(const float* f, uint32_t n, uint32_t comps, const uint32_t* idx, uint32_t m, float* buf)
{
    const uint64_t total = uint64_t(m) * comps;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t q = uint32_t(t / m), j = uint32_t(t % m);
        buf[t] = f[uint64_t(q) * n + idx[j]];
    }
}

__global__ void gslab_unpack(float* f, uint32_t n, uint32_t comps, const uint32_t* idx, uint32_t m, const float* buf)
{
    const uint64_t total = uint64_t(m) * comps;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t < total; t += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t q = uint32_t(t / m), j = uint32_t(t % m);
        f[uint64_t(q) * n + idx[j]] = buf[t];
    }
}

// The local tables of rank r under a link -> rank assignment (colour-major
// link indices throughout).
struct LocalPlan
{
    std::vector<uint32_t> links;  // local -> global colour-major index: owned, then halo
    uint32_t n_owned = 0;
};

LocalPlan plan_for(const umc_cells* cc, const std::vector<uint32_t>& owner_cm, uint32_t r)
{
    LocalPlan p;
    const uint64_t n = cc->n_sites;
    std::vector<uint8_t> in(n, 0);
    for (uint64_t k = 0; k < n; ++k)
        if (owner_cm[k] == r) {
            p.links.push_back(uint32_t(k));
            in[k] = 1;
        }
    p.n_owned = uint32_t(p.links.size());
    std::vector<uint32_t> halo;
    for (uint32_t i = 0; i < p.n_owned; ++i) {
        const uint32_t k = p.links[i];
        for (uint64_t e = cc->c_inc_offset[k]; e < cc->c_inc_offset[k + 1]; ++e) {
            const uint32_t* c = cc->c_cells.data() + 4ull * cc->c_inc_cell[e];
            for (int j = 0; j < 4; ++j)
                if (!in[c[j]]) {
                    in[c[j]] = 2;
                    halo.push_back(c[j]);
                }
        }
    }
    std::sort(halo.begin(), halo.end());
    p.links.insert(p.links.end(), halo.begin(), halo.end());
    return p;
}

}  // namespace
}  // namespace umc

using namespace umc;

struct umc_gslab
{
    umc_gslab_desc desc{};
    uint32_t N = 1, comps = 1, n_local = 0, n_owned = 0, n_classes = 0, max_incident = 0, grid = 0;
    uint64_t n_cells_global = 0;
    uint32_t n_assigned = 0;  // cells whose first link this rank owns (the record's share)
    int device = 0;
    std::vector<uint32_t> class_first, class_count;  // owned local ranges per colour class
    std::vector<uint32_t> local_ref;                 // reference link id per local link
    // exchange lists per (peer, class): offsets into the flat index arrays
    std::vector<uint32_t> send_off, recv_off;
    DevBuf d_gid, d_inc_off, d_inc, d_cells, d_send, d_recv;
    DevBuf ctl, partials, record;
};

namespace {

template <class F>
int gslab_guard(F&& f)
{
    try {
        set_last_error("");
        f();
        return UMC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}

template <class T>
void upload(DevBuf& b, const std::vector<T>& v, const char* what)
{
    b.alloc(std::max<size_t>(1, v.size()) * sizeof(T), what);
    if (!v.empty()) cuda_check(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), what);
}

uint32_t grid_for(const umc_gslab* s, uint64_t work)
{
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device), "SM count");
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((work + kBlock - 1) / kBlock, uint64_t(sms) * 8)));
}

void build(umc_gslab* s)
{
    const umc_gslab_desc& d = s->desc;
    const umc_cells* cc = d.cells;
    const uint64_t n = cc->n_sites;
    const uint32_t r = d.rank;
    const Colouring& col = cc->col;
    s->n_classes = col.n_colours;
    if (s->n_classes + 1 > uint32_t(kMaxPasses - 1))
        throw Error(UMC_ERR_UNSUPPORTED, "cell complex needs more colour classes than the engine supports");
    std::vector<uint32_t> owner_cm(n);
    for (uint64_t k = 0; k < n; ++k) {
        const uint32_t o = d.owner[col.order[k]];
        if (o >= d.world) throw Error(UMC_ERR_OUT_OF_RANGE, "owner rank outside the world");
        owner_cm[k] = o;
    }
    const LocalPlan me = plan_for(cc, owner_cm, r);
    s->n_owned = me.n_owned;
    s->n_local = uint32_t(me.links.size());
    std::vector<uint32_t> local_of(n, 0xFFFFFFFFu);
    for (uint32_t i = 0; i < s->n_local; ++i) local_of[me.links[i]] = i;
    s->local_ref.resize(s->n_local);
    for (uint32_t i = 0; i < s->n_local; ++i) s->local_ref[i] = col.order[me.links[i]];
    // owned links are in colour-major order, so each class is one range
    s->class_first.assign(s->n_classes, 0);
    s->class_count.assign(s->n_classes, 0);
    for (uint32_t c = 0, i = 0; c < s->n_classes; ++c) {
        s->class_first[c] = i;
        while (i < s->n_owned && me.links[i] < col.class_start[c + 1]) ++i;
        s->class_count[c] = i - s->class_first[c];
    }
    // cells incident to owned links: the ones whose first link is owned
    // (this rank's share of the record) first, then the rest
    const uint64_t n_cells = cc->n_cells();
    s->n_cells_global = n_cells;
    std::vector<uint32_t> cell_local(n_cells, 0xFFFFFFFFu);
    std::vector<uint32_t> assigned, other;
    for (uint32_t i = 0; i < s->n_owned; ++i)
        for (uint64_t e = cc->c_inc_offset[me.links[i]]; e < cc->c_inc_offset[me.links[i] + 1]; ++e) {
            const uint32_t w = cc->c_inc_cell[e];
            if (cell_local[w] != 0xFFFFFFFFu) continue;
            cell_local[w] = 0;
            (owner_cm[cc->c_cells[4ull * w]] == r ? assigned : other).push_back(w);
        }
    std::sort(assigned.begin(), assigned.end());
    std::sort(other.begin(), other.end());
    s->n_assigned = uint32_t(assigned.size());
    std::vector<uint32_t> cells_global(assigned);
    cells_global.insert(cells_global.end(), other.begin(), other.end());
    std::vector<uint32_t> cells4(4 * cells_global.size());
    for (size_t j = 0; j < cells_global.size(); ++j) {
        cell_local[cells_global[j]] = uint32_t(j);
        for (int q = 0; q < 4; ++q) cells4[4 * j + q] = local_of[cc->c_cells[4ull * cells_global[j] + q]];
    }
    // incidence of the owned links, in the single-GPU order
    std::vector<uint32_t> inc_off(s->n_owned + 1, 0), inc;
    s->max_incident = 0;
    for (uint64_t k = 0; k < n; ++k)
        s->max_incident = std::max<uint32_t>(s->max_incident, uint32_t(cc->c_inc_offset[k + 1] - cc->c_inc_offset[k]));
    for (uint32_t i = 0; i < s->n_owned; ++i) {
        const uint32_t k = me.links[i];
        for (uint64_t e = cc->c_inc_offset[k]; e < cc->c_inc_offset[k + 1]; ++e)
            inc.push_back((cell_local[cc->c_inc_cell[e]] << 2) | cc->c_inc_which[e]);
        inc_off[i + 1] = uint32_t(inc.size());
    }
    // exchange lists per (peer, class), both sides sorted by global index
    auto class_of = [&](uint32_t k) {
        return uint32_t(std::upper_bound(col.class_start.begin(), col.class_start.end(), uint64_t(k)) -
                        col.class_start.begin()) - 1;
    };
    std::vector<std::vector<uint32_t>> sends(size_t(d.world) * s->n_classes), recvs(sends.size());
    for (uint32_t p = 0; p < d.world; ++p) {
        if (p == r) continue;
        const LocalPlan other_plan = plan_for(cc, owner_cm, p);
        for (size_t i = other_plan.n_owned; i < other_plan.links.size(); ++i) {
            const uint32_t k = other_plan.links[i];
            if (owner_cm[k] == r) sends[size_t(p) * s->n_classes + class_of(k)].push_back(local_of[k]);
        }
        for (uint32_t i = s->n_owned; i < s->n_local; ++i) {
            const uint32_t k = me.links[i];
            if (owner_cm[k] == p) recvs[size_t(p) * s->n_classes + class_of(k)].push_back(i);
        }
    }
    std::vector<uint32_t> send_flat, recv_flat;
    s->send_off.assign(sends.size() + 1, 0);
    s->recv_off.assign(sends.size() + 1, 0);
    for (size_t q = 0; q < sends.size(); ++q) {
        send_flat.insert(send_flat.end(), sends[q].begin(), sends[q].end());
        recv_flat.insert(recv_flat.end(), recvs[q].begin(), recvs[q].end());
        s->send_off[q + 1] = uint32_t(send_flat.size());
        s->recv_off[q + 1] = uint32_t(recv_flat.size());
    }
    upload(s->d_gid, me.links, "gauge slab keys");
    upload(s->d_inc_off, inc_off, "gauge slab incidence");
    upload(s->d_inc, inc, "gauge slab incidence");
    upload(s->d_cells, cells4, "gauge slab cells");
    upload(s->d_send, send_flat, "gauge slab send lists");
    upload(s->d_recv, recv_flat, "gauge slab receive lists");
    s->grid = grid_for(s, std::max<uint64_t>(s->n_owned, s->n_assigned));
    s->ctl.alloc(sizeof(DevCtl), "gauge slab control");
    cuda_check(cudaMemset(s->ctl.p, 0, sizeof(DevCtl)), "gauge slab control");
    s->partials.alloc(size_t(s->grid) * kObs * sizeof(double), "gauge slab partials");
    s->record.alloc(kObs * sizeof(double), "gauge slab record");
    cuda_check(cudaMemset(s->record.p, 0, kObs * sizeof(double)), "gauge slab record");
}

}  // namespace

extern "C" {

int umc_gslab_create(const umc_gslab_desc* d, umc_gslab** out)
{
    return gslab_guard([&] {
        if (!d || !out || !d->cells || !d->owner) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (d->cells->arity != 4) throw Error(UMC_ERR_UNSUPPORTED, "gauge slabs need plaquettes (arity 4)");
        if (d->world == 0 || d->rank >= d->world) throw Error(UMC_ERR_INVALID_ARGUMENT, "rank outside the world");
        if (d->hits == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "hits must be at least 1");
        if (!std::isfinite(d->coupling) || !std::isfinite(d->width))
            throw Error(UMC_ERR_INVALID_ARGUMENT, "beta and width must be finite");
        if (d->cells->n_sites > 0xFFFFFFFFull / 4) throw Error(UMC_ERR_OVERFLOW, "too many links");
        if (d->cells->n_cells() >= (1ull << 30)) throw Error(UMC_ERR_OVERFLOW, "too many cells for the packed incidence");
        auto s = std::make_unique<umc_gslab>();
        s->desc = *d;
        if (d->model == UMC_MODEL_U1) {
            s->N = 1;
            s->comps = 1;
        } else if (d->model == UMC_MODEL_SU) {
            if (d->N != 2 && d->N != 3) throw Error(UMC_ERR_UNSUPPORTED, "SU(N) is provided for N = 2 and 3");
            s->N = uint32_t(d->N);
            s->comps = 2 * s->N * s->N;
        } else {
            throw Error(UMC_ERR_UNSUPPORTED, "gauge slabs are provided for U(1) and SU(N)");
        }
        s->device = d->device;
        cuda_check(cudaSetDevice(d->device), "cudaSetDevice");
        build(s.get());
        s->desc.owner = nullptr;  // read once, not kept
        *out = s.release();
    });
}

int umc_gslab_destroy(umc_gslab* s)
{
    return gslab_guard([&] { delete s; });
}

int umc_gslab_info(const umc_gslab* s, uint32_t* n_local, uint32_t* n_owned, uint32_t* n_classes, uint32_t* comps)
{
    return gslab_guard([&] {
        if (!s) throw Error(UMC_ERR_INVALID_ARGUMENT, "null gauge slab");
        if (n_local) *n_local = s->n_local;
        if (n_owned) *n_owned = s->n_owned;
        if (n_classes) *n_classes = s->n_classes;
        if (comps) *comps = s->comps;
    });
}

int umc_gslab_local_links(const umc_gslab* s, uint32_t* ref_ids)
{
    return gslab_guard([&] {
        if (!s || !ref_ids) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        std::copy(s->local_ref.begin(), s->local_ref.end(), ref_ids);
    });
}

int umc_gslab_exchange_counts(const umc_gslab* s, uint32_t peer, uint32_t colour, uint32_t* n_send, uint32_t* n_recv)
{
    return gslab_guard([&] {
        if (!s) throw Error(UMC_ERR_INVALID_ARGUMENT, "null gauge slab");
        if (peer >= s->desc.world || colour >= s->n_classes) throw Error(UMC_ERR_OUT_OF_RANGE, "peer or class out of range");
        const size_t q = size_t(peer) * s->n_classes + colour;
        if (n_send) *n_send = s->send_off[q + 1] - s->send_off[q];
        if (n_recv) *n_recv = s->recv_off[q + 1] - s->recv_off[q];
    });
}

int umc_gslab_pack(umc_gslab* s, const float* field, uint32_t peer, uint32_t colour, float* buf, void* stream)
{
    return gslab_guard([&] {
        if (!s || !field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (peer >= s->desc.world || colour >= s->n_classes) throw Error(UMC_ERR_OUT_OF_RANGE, "peer or class out of range");
        const size_t q = size_t(peer) * s->n_classes + colour;
        const uint32_t m = s->send_off[q + 1] - s->send_off[q];
        if (!m) return;
        if (!buf) throw Error(UMC_ERR_INVALID_ARGUMENT, "null buffer");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        const uint32_t g = grid_for(s, uint64_t(m) * s->comps);
        gslab_pack<<<g, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(field, s->n_local, s->comps,
                                                                         s->d_send.as<uint32_t>() + s->send_off[q], m, buf);
        cuda_check(cudaGetLastError(), "gauge slab pack");
    });
}

int umc_gslab_unpack(umc_gslab* s, float* field, uint32_t peer, uint32_t colour, const float* buf, void* stream)
{
    return gslab_guard([&] {
        if (!s || !field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (peer >= s->desc.world || colour >= s->n_classes) throw Error(UMC_ERR_OUT_OF_RANGE, "peer or class out of range");
        const size_t q = size_t(peer) * s->n_classes + colour;
        const uint32_t m = s->recv_off[q + 1] - s->recv_off[q];
        if (!m) return;
        if (!buf) throw Error(UMC_ERR_INVALID_ARGUMENT, "null buffer");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        const uint32_t g = grid_for(s, uint64_t(m) * s->comps);
        gslab_unpack<<<g, kBlock, 0, static_cast<cudaStream_t>(stream)>>>(field, s->n_local, s->comps,
                                                                           s->d_recv.as<uint32_t>() + s->recv_off[q], m, buf);
        cuda_check(cudaGetLastError(), "gauge slab unpack");
    });
}

int umc_gslab_pass(umc_gslab* s, float* field, double beta, uint64_t sweep, uint32_t colour, void* stream)
{
    return gslab_guard([&] {
        NvtxRange range("umc_gslab_pass");
        if (!s || !field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (colour >= s->n_classes) throw Error(UMC_ERR_OUT_OF_RANGE, "colour class out of range");
        if (!std::isfinite(beta)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta must be finite");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const umc_gslab_desc& d = s->desc;
        GaugeArgs a{};
        a.f = field;
        a.n = s->n_local;
        a.first = s->class_first[colour];
        a.count = s->class_count[colour];
        a.inc_off = s->d_inc_off.as<uint32_t>();
        a.inc = s->d_inc.as<uint32_t>();
        a.cells = s->d_cells.as<uint4>();
        a.seed = d.seed;
        a.sweep = sweep;
        a.hits = d.hits;
        a.model_beta = float(d.coupling);
        a.driver_beta = float(beta);
        a.width = float(d.width);
        a.model_beta64 = d.coupling;
        a.driver_beta64 = beta;
        a.err = s->N == 1 ? u1_metropolis_err(beta, d.coupling, s->max_incident) : 0.0f;  // SU(N): FP32 test
        a.gid = s->d_gid.as<uint32_t>();
        const int np = int(s->n_classes) + 1;
        a.out = PassOut{s->ctl.as<DevCtl>(), s->partials.as<double>(), nullptr, nullptr, int(colour), np, 0};
        switch (s->N) {
        case 1: u1_pass<<<s->grid, kBlock, 0, st>>>(a); break;
        case 2: su_pass<2><<<s->grid, kBlock, 0, st>>>(a); break;
        default: su_pass<3><<<s->grid, kBlock, 0, st>>>(a); break;
        }
        cuda_check(cudaGetLastError(), "gauge slab pass");
    });
}

int umc_gslab_record(umc_gslab* s, const float* field, double* out, void* stream)
{
    return gslab_guard([&] {
        if (!s || !field || !out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        cuda_check(cudaSetDevice(s->device), "cudaSetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int np = int(s->n_classes) + 1;
        const PassOut o{s->ctl.as<DevCtl>(), s->partials.as<double>(), s->record.as<double>(), nullptr,
                        int(s->n_classes), np, 1};
        const uint4* cells = s->d_cells.as<uint4>();
        const float J = float(s->desc.coupling);
        switch (s->N) {
        case 1: plaquette_sum<1><<<s->grid, kBlock, 0, st>>>(field, s->n_local, cells, s->n_assigned, s->n_cells_global, J, o); break;
        case 2: plaquette_sum<2><<<s->grid, kBlock, 0, st>>>(field, s->n_local, cells, s->n_assigned, s->n_cells_global, J, o); break;
        default: plaquette_sum<3><<<s->grid, kBlock, 0, st>>>(field, s->n_local, cells, s->n_assigned, s->n_cells_global, J, o); break;
        }
        cuda_check(cudaGetLastError(), "gauge slab plaquettes");
        cuda_check(cudaMemcpyAsync(out, s->record.p, kObs * sizeof(double), cudaMemcpyDeviceToHost, st), "gauge slab record");
        cuda_check(cudaStreamSynchronize(st), "gauge slab record");
        unsigned status = 0;
        cuda_check(cudaMemcpy(&status, &s->ctl.as<DevCtl>()->status, sizeof status, cudaMemcpyDeviceToHost),
                   "gauge slab status");
        if (status) throw Error(UMC_ERR_DEVICE_TIMEOUT, "gauge slab pass reported a device error");
    });
}

}  // extern "C"
