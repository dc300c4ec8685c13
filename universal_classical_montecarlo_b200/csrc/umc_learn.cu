// umc_learn.cu -- batched 2D U(1) chains (plain U1Shift or the learned
// proposal) and the proposal network's training, behind the C ABI
// (umc_u1batch_*, umc_mlp_*).
//
// The reference has neither batching nor learned proposals.  A chain here is
// the reference's U(1) plaquette model (model/cell.hpp:64-78 with
// term/plaquette.hpp:34-47) on the 2D periodic plaquette complex, driven by
// the Metropolis rule of driver.hpp:29-42: with the plain proposal (U1Shift,
// dof/u1.hpp:36-52) chain c replays the single-chain U(1) sweep with seed
// chain_seed[c]; with the learned proposal the update is the same rule with a
// non-zero log_ratio (dof/proposal.hpp:5-12).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "umc_nvtx.hpp"
#include "umc_chain.hpp"
#include "umc_spin_kernels.cuh"
#include "umc_learn_kernels.cuh"

using umc::DevBuf;
using umc::Error;
using umc::cuda_check;

struct umc_mlp
{
    umc_mlp_desc desc{};
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DevBuf params, m, v, img, partial, partial_loss, status, grad, loss, xbuf, tbuf, obuf, configs;
    uint64_t steps = 0;
    uint64_t n_configs = 0;
    uint32_t n_sm = 0;
    uint64_t launches = 0;
};

struct umc_u1batch
{
    umc_u1batch_desc desc{};
    uint32_t n_chains = 0, L = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    DevBuf theta, seeds, records, status, dump;
    std::vector<unsigned long long> chain_seed;
    uint64_t sweeps = 0;
    uint64_t max_records = 0, rec_pending = 0;
    bool rec_overflow = false;
    int plain_grid = 0, learned_grid = 0;
    uint32_t groups = 0;  // tile groups of the learned kernel (learn::kGroupChoices)
    uint64_t launches = 0;
};

namespace umc {
namespace {

template <class F>
int lguard(F&& f)
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

void scope(int device) { cuda_check(cudaSetDevice(device), "cudaSetDevice"); }

void check_status(DevBuf& st, cudaStream_t s)
{
    unsigned int v = 0;
    cuda_check(cudaMemcpyAsync(&v, st.p, 4, cudaMemcpyDeviceToHost, s), "status");
    cuda_check(cudaStreamSynchronize(s), "sync");
    if (v) {
        cuda_check(cudaMemsetAsync(st.p, 0, 4, s), "status reset");
        cuda_check(cudaStreamSynchronize(s), "sync");
        throw Error(UMC_ERR_DEVICE_TIMEOUT, "tensor-core wait exceeded its iteration limit");
    }
}

// chain-local natural link order (mu L^2 + y L + x) <-> colour-major
uint32_t colour_index(uint32_t L, uint32_t link)
{
    const uint32_t L2 = L * L, mu = link / L2, s = link % L2, y = s / L, x = s % L;
    return (2 * mu + ((x + y) & 1u)) * (L2 / 2) + s / 2;
}

void upload_image(umc_mlp* n)
{
    learn::mlp_image<<<(learn::kImageThreads + 255) / 256, 256, 0, n->stream>>>(n->params.as<float>(),
                                                                              n->img.as<uint8_t>());
    cuda_check(cudaGetLastError(), "operand image");
    ++n->launches;
}

// He-style start from the seed: W ~ N(0, 2 / fan_in) (W3: 1 / fan_in), b ~ N(0, 0.01).
std::vector<float> initial_params(uint64_t seed)
{
    std::vector<float> P(learn::kParams);
    KeyedPcg g = KeyedPcg::open_key(seed, 0, kTagInit, 0xFFFFFFFFu);
    auto normal = [&]() {
        const double u1 = (double(g.next()) + 1.0) * 0x1.0p-32, u2 = double(g.next()) * 0x1.0p-32;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (int i = 0; i < learn::kParams; ++i) {
        double sd;
        if (i < learn::P_B1) sd = std::sqrt(2.0 / 3.0);
        else if (i < learn::P_W2) sd = 0.1;
        else if (i < learn::P_B2) sd = std::sqrt(2.0 / 64.0);
        else if (i < learn::P_W3) sd = 0.1;
        else if (i < learn::P_B3) sd = std::sqrt(1.0 / 64.0);
        else sd = 0.1;
        P[i] = float(sd * normal());
    }
    return P;
}

int resident_grid(const void* kernel, int threads, size_t smem, int device)
{
    int per_sm = 0, n_sm = 0;
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem), "occupancy");
    cuda_check(cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device), "SM count");
    return std::max(1, per_sm) * n_sm;
}

void enqueue_sweeps(umc_u1batch* b, uint64_t n_sweeps, const umc_mlp* net, float* dump)
{
    if (net && net->device != b->device) throw Error(UMC_ERR_INVALID_ARGUMENT, "network lives on another device");
    learn::U1BatchArgs a{};
    a.theta = b->theta.as<float>();
    a.n_chains = b->n_chains;
    a.L = b->L;
    a.chain_seed = b->seeds.as<unsigned long long>();
    a.model_beta = float(b->desc.beta);
    a.driver_beta = 1.0f;
    a.model_beta64 = b->desc.beta;
    a.driver_beta64 = 1.0;
    a.err = u1_metropolis_err(1.0, b->desc.beta, 2);
    a.width = float(b->desc.width);
    a.img = net ? net->img.as<uint8_t>() : nullptr;
    a.records = b->records.as<double>();
    a.rec_capacity = b->max_records;
    a.dump = dump;
    a.status = b->status.as<unsigned int>();
    // one launch per block of sweeps that fits the record buffer
    uint64_t done = 0;
    while (done < n_sweeps) {
        uint64_t chunk = n_sweeps - done;
        if (chunk > 1u << 20) chunk = 1u << 20;
        a.sweep0 = b->sweeps;
        a.n_sweeps = uint32_t(chunk);
        a.rec_slot0 = b->rec_pending;
        if (net) {
            const learn::LearnSmem sp = learn::LearnSmem::plan(b->L, b->groups);
            const int grid = std::min<int>(b->learned_grid, b->n_chains);
            switch (b->groups) {
            case 8: learn::u1_learned_batch<8><<<grid, learn::kTile * 8, sp.total, b->stream>>>(a); break;
            case 6: learn::u1_learned_batch<6><<<grid, learn::kTile * 6, sp.total, b->stream>>>(a); break;
            default: learn::u1_learned_batch<4><<<grid, learn::kTile * 4, sp.total, b->stream>>>(a); break;
            }
        } else {
            const size_t smem = size_t(2) * b->L * b->L * 4;
            learn::u1_plain_batch<<<std::min<int>(b->plain_grid, b->n_chains), 256, smem, b->stream>>>(a);
        }
        cuda_check(cudaGetLastError(), "U(1) batch sweeps");
        ++b->launches;
        b->sweeps += chunk;
        if (b->rec_pending + chunk > b->max_records) b->rec_overflow = true;
        b->rec_pending = std::min<uint64_t>(b->rec_pending + chunk, b->max_records);
        a.dump = nullptr;
        done += chunk;
    }
}

}  // namespace
}  // namespace umc

using namespace umc;

extern "C" {

// ================================================================== network

int umc_mlp_create(const umc_mlp_desc* d, umc_mlp** out)
{
    return lguard([&] {
        if (!d || !out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        auto* n = new umc_mlp;
        try {
            n->desc = *d;
            n->device = d->device;
            scope(n->device);
            if (d->stream) n->stream = static_cast<cudaStream_t>(d->stream);
            else {
                cuda_check(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking), "stream");
                n->own_stream = true;
            }
            int sms = 0;
            cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, n->device), "SM count");
            n->n_sm = uint32_t(sms);
            const size_t P = learn::kParams * 4;
            n->params.alloc(P, "parameters");
            n->m.alloc(P, "Adam m");
            n->v.alloc(P, "Adam v");
            n->grad.alloc(P, "gradient");
            n->img.alloc(learn::IMG_BYTES, "operand image");
            n->partial.alloc(size_t(n->n_sm) * P, "gradient partials");
            n->partial_loss.alloc(size_t(n->n_sm) * 8, "loss partials");
            n->status.alloc(4, "status");
            n->loss.alloc(8, "loss");
            cuda_check(cudaMemsetAsync(n->status.p, 0, 4, n->stream), "status");
            cuda_check(cudaMemsetAsync(n->img.p, 0, learn::IMG_BYTES, n->stream), "image");
            cuda_check(cudaMemsetAsync(n->m.p, 0, P, n->stream), "Adam m");
            cuda_check(cudaMemsetAsync(n->v.p, 0, P, n->stream), "Adam v");
            const auto P0 = initial_params(d->seed);
            cuda_check(cudaMemcpyAsync(n->params.p, P0.data(), P, cudaMemcpyHostToDevice, n->stream), "params");
            if (d->max_configs) {
                if (d->L < 4 || d->L % 2) throw Error(UMC_ERR_INVALID_ARGUMENT, "dataset lattice side must be even, >= 4");
                n->configs.alloc(size_t(d->max_configs) * 2 * d->L * d->L * 4, "configurations");
            }
            const size_t tsm = learn::TrainSmem::plan().total;
            cuda_check(cudaFuncSetAttribute(learn::mlp_train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(tsm)),
                       "train smem");
            const size_t fsm = learn::LearnSmem::plan(0, 1).total;
            cuda_check(cudaFuncSetAttribute(learn::mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(fsm)),
                       "forward smem");
            upload_image(n);
            cuda_check(cudaStreamSynchronize(n->stream), "create");
        } catch (...) {
            if (n->own_stream && n->stream) cudaStreamDestroy(n->stream);
            delete n;
            throw;
        }
        *out = n;
    });
}

int umc_mlp_destroy(umc_mlp* n)
{
    return lguard([&] {
        if (!n) return;
        scope(n->device);
        cudaStreamSynchronize(n->stream);
        if (n->own_stream) cudaStreamDestroy(n->stream);
        delete n;
    });
}

int umc_mlp_set_params(umc_mlp* n, const float* P)
{
    return lguard([&] {
        if (!n || !P) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(n->device);
        cuda_check(cudaMemcpyAsync(n->params.p, P, learn::kParams * 4, cudaMemcpyHostToDevice, n->stream), "params");
        cuda_check(cudaMemsetAsync(n->m.p, 0, learn::kParams * 4, n->stream), "Adam m");
        cuda_check(cudaMemsetAsync(n->v.p, 0, learn::kParams * 4, n->stream), "Adam v");
        n->steps = 0;
        upload_image(n);
        cuda_check(cudaStreamSynchronize(n->stream), "set params");
    });
}

int umc_mlp_get_params(umc_mlp* n, float* P)
{
    return lguard([&] {
        if (!n || !P) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(n->device);
        cuda_check(cudaMemcpyAsync(P, n->params.p, learn::kParams * 4, cudaMemcpyDeviceToHost, n->stream), "params");
        cuda_check(cudaStreamSynchronize(n->stream), "get params");
    });
}

int umc_mlp_forward(umc_mlp* n, const float* x, uint64_t count, float* out)
{
    return lguard([&] {
        if (!n || (count && (!x || !out))) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (count > (1u << 30)) throw Error(UMC_ERR_INVALID_ARGUMENT, "too many inputs");
        if (!count) return;
        scope(n->device);
        n->xbuf.alloc(count * 3 * 4, "inputs");
        n->obuf.alloc(count * 16 * 4, "outputs");
        cuda_check(cudaMemcpyAsync(n->xbuf.p, x, count * 12, cudaMemcpyHostToDevice, n->stream), "inputs");
        const uint32_t tiles = uint32_t((count + learn::kTile - 1) / learn::kTile);
        const size_t fsm = learn::LearnSmem::plan(0, 1).total;
        learn::mlp_forward_kernel<<<std::min<uint32_t>(tiles, 3 * n->n_sm), learn::kTile, fsm, n->stream>>>(
            n->img.as<uint8_t>(), n->xbuf.as<float>(), uint32_t(count), n->obuf.as<float>(),
            n->status.as<unsigned int>());
        cuda_check(cudaGetLastError(), "forward");
        ++n->launches;
        cuda_check(cudaMemcpyAsync(out, n->obuf.p, count * 64, cudaMemcpyDeviceToHost, n->stream), "outputs");
        check_status(n->status, n->stream);
    });
}

namespace {
// One pass of the training kernel plus the reduction (and Adam when lr > 0).
void train_pass(umc_mlp* n, const learn::TrainArgs& base, uint32_t count, double lr, bool apply, double* loss_dev)
{
    learn::TrainArgs a = base;
    a.img = n->img.as<uint8_t>();
    a.n = count;
    a.partial = n->partial.as<float>();
    a.partial_loss = n->partial_loss.as<double>();
    a.status = n->status.as<unsigned int>();
    const uint32_t tiles = (count + learn::kTile - 1) / learn::kTile;
    const uint32_t grid = std::min<uint32_t>(tiles, n->n_sm);
    learn::mlp_train_kernel<<<grid, learn::kTile, learn::TrainSmem::plan().total, n->stream>>>(a);
    cuda_check(cudaGetLastError(), "train kernel");
    learn::AdamArgs r{};
    r.partial = n->partial.as<float>();
    r.partial_loss = n->partial_loss.as<double>();
    r.n_parts = grid;
    r.n = count;
    r.params = n->params.as<float>();
    r.m = n->m.as<float>();
    r.v = n->v.as<float>();
    r.grad_out = n->grad.as<float>();
    r.loss_out = loss_dev;
    r.apply = apply ? 1u : 0u;
    if (apply) {
        const uint64_t t = n->steps + 1;
        r.lr = float(lr);
        r.b1 = 0.9f;
        r.b2 = 0.999f;
        r.eps = 1e-8f;
        r.c1 = float(1.0 - std::pow(0.9, double(t)));
        r.c2 = float(1.0 - std::pow(0.999, double(t)));
    }
    learn::mlp_reduce_adam<<<(learn::kParams + 255) / 256, 256, 0, n->stream>>>(r);
    cuda_check(cudaGetLastError(), "reduce");
    n->launches += 2;
    if (apply) {
        ++n->steps;
        upload_image(n);
    }
}
}  // namespace

int umc_mlp_loss_grad(umc_mlp* n, const float* x, const float* theta, uint64_t count, double* loss, float* grad)
{
    return lguard([&] {
        if (!n || !x || !theta || !count) throw Error(UMC_ERR_INVALID_ARGUMENT, "null or empty argument");
        if (count > (1u << 30)) throw Error(UMC_ERR_INVALID_ARGUMENT, "too many samples");
        scope(n->device);
        n->xbuf.alloc(count * 12, "inputs");
        n->tbuf.alloc(count * 4, "targets");
        cuda_check(cudaMemcpyAsync(n->xbuf.p, x, count * 12, cudaMemcpyHostToDevice, n->stream), "inputs");
        cuda_check(cudaMemcpyAsync(n->tbuf.p, theta, count * 4, cudaMemcpyHostToDevice, n->stream), "targets");
        learn::TrainArgs a{};
        a.x = n->xbuf.as<float>();
        a.target = n->tbuf.as<float>();
        train_pass(n, a, uint32_t(count), 0.0, false, n->loss.as<double>());
        if (grad)
            cuda_check(cudaMemcpyAsync(grad, n->grad.p, learn::kParams * 4, cudaMemcpyDeviceToHost, n->stream), "grad");
        if (loss) cuda_check(cudaMemcpyAsync(loss, n->loss.p, 8, cudaMemcpyDeviceToHost, n->stream), "loss");
        check_status(n->status, n->stream);
    });
}

int umc_mlp_apply_gradient(umc_mlp* n, const float* grad, double lr)
{
    return lguard([&] {
        if (!n || !grad) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(n->device);
        cuda_check(cudaMemcpyAsync(n->partial.p, grad, learn::kParams * 4, cudaMemcpyHostToDevice, n->stream),
                   "gradient");
        learn::AdamArgs r{};
        r.partial = n->partial.as<float>();
        r.partial_loss = n->partial_loss.as<double>();
        r.n_parts = 1;
        r.n = 1;
        r.params = n->params.as<float>();
        r.m = n->m.as<float>();
        r.v = n->v.as<float>();
        r.apply = 1;
        const uint64_t t = n->steps + 1;
        r.lr = float(lr);
        r.b1 = 0.9f;
        r.b2 = 0.999f;
        r.eps = 1e-8f;
        r.c1 = float(1.0 - std::pow(0.9, double(t)));
        r.c2 = float(1.0 - std::pow(0.999, double(t)));
        learn::mlp_reduce_adam<<<(learn::kParams + 255) / 256, 256, 0, n->stream>>>(r);
        cuda_check(cudaGetLastError(), "Adam");
        ++n->steps;
        ++n->launches;
        upload_image(n);
        cuda_check(cudaStreamSynchronize(n->stream), "Adam");
    });
}

int umc_mlp_add_configs(umc_mlp* n, umc_u1batch* b)
{
    return lguard([&] {
        if (!n || !b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!n->configs.p) throw Error(UMC_ERR_STATE, "network was created without a dataset");
        if (b->L != n->desc.L) throw Error(UMC_ERR_INVALID_ARGUMENT, "lattice side differs from the dataset's");
        if (b->device != n->device) throw Error(UMC_ERR_INVALID_ARGUMENT, "batch lives on another device");
        if (n->n_configs + b->n_chains > n->desc.max_configs) throw Error(UMC_ERR_OUT_OF_RANGE, "dataset is full");
        scope(n->device);
        const size_t per = size_t(2) * b->L * b->L * 4;
        cuda_check(cudaStreamSynchronize(b->stream), "batch");
        cuda_check(cudaMemcpyAsync(n->configs.as<uint8_t>() + n->n_configs * per, b->theta.p, per * b->n_chains,
                                   cudaMemcpyDeviceToDevice, n->stream),
                   "configurations");
        cuda_check(cudaStreamSynchronize(n->stream), "configurations");
        n->n_configs += b->n_chains;
    });
}

int umc_mlp_configs(const umc_mlp* n, uint64_t* count)
{
    return lguard([&] {
        if (!n || !count) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        *count = n->n_configs;
    });
}

int umc_mlp_clear_configs(umc_mlp* n)
{
    return lguard([&] {
        if (!n) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        n->n_configs = 0;
    });
}

int umc_mlp_train(umc_mlp* n, uint64_t steps, uint32_t batch, double lr, double* losses)
{
    return lguard([&] {
        NvtxRange range("umc_mlp_train");
        if (!n) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!n->n_configs) throw Error(UMC_ERR_STATE, "no training configurations");
        if (batch == 0 || batch > (1u << 24)) throw Error(UMC_ERR_INVALID_ARGUMENT, "batch out of range");
        if (!(lr > 0.0)) throw Error(UMC_ERR_INVALID_ARGUMENT, "learning rate must be positive");
        scope(n->device);
        DevBuf lbuf;
        lbuf.alloc(std::max<uint64_t>(steps, 1) * 8, "losses");
        for (uint64_t s = 0; s < steps; ++s) {
            learn::TrainArgs a{};
            a.configs = n->configs.as<float>();
            a.n_configs = n->n_configs;
            a.L = n->desc.L;
            a.seed = n->desc.seed;
            a.step = n->steps;
            train_pass(n, a, batch, lr, true, lbuf.as<double>() + s);
        }
        if (losses && steps)
            cuda_check(cudaMemcpyAsync(losses, lbuf.p, steps * 8, cudaMemcpyDeviceToHost, n->stream), "losses");
        check_status(n->status, n->stream);
    });
}

int umc_mlp_counters(const umc_mlp* n, uint64_t* steps, uint64_t* launches)
{
    return lguard([&] {
        if (!n) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (steps) *steps = n->steps;
        if (launches) *launches = n->launches;
    });
}

// ============================================================ U(1) batches

int umc_u1batch_create(const umc_u1batch_desc* d, umc_u1batch** out)
{
    return lguard([&] {
        if (!d || !out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        if (d->n_chains == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "no chains");
        if (d->L < 4 || d->L % 2 || d->L > 96) throw Error(UMC_ERR_UNSUPPORTED, "lattice side must be even, 4..96");
        auto* b = new umc_u1batch;
        try {
            b->desc = *d;
            b->n_chains = d->n_chains;
            b->L = d->L;
            b->device = d->device;
            scope(b->device);
            if (d->stream) b->stream = static_cast<cudaStream_t>(d->stream);
            else {
                cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
                b->own_stream = true;
            }
            const size_t per = size_t(2) * b->L * b->L;
            b->theta.alloc(per * b->n_chains * 4, "angles");
            cuda_check(cudaMemsetAsync(b->theta.p, 0, per * b->n_chains * 4, b->stream), "cold start");
            b->chain_seed.resize(b->n_chains);
            for (uint32_t c = 0; c < b->n_chains; ++c)
                b->chain_seed[c] = mix64(d->seed + kGolden * (uint64_t(d->first_chain) + c + 1ull));
            b->seeds.alloc(b->n_chains * 8, "seeds");
            cuda_check(cudaMemcpyAsync(b->seeds.p, b->chain_seed.data(), b->n_chains * 8, cudaMemcpyHostToDevice,
                                       b->stream),
                       "seeds");
            b->max_records = d->max_records ? d->max_records : 1024;
            b->records.alloc(b->max_records * b->n_chains * 4 * 8, "records");
            b->status.alloc(4, "status");
            cuda_check(cudaMemsetAsync(b->status.p, 0, 4, b->stream), "status");
            // the most tile groups whose shared-memory plan fits one CTA
            int smem_max = 0;
            cuda_check(cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device),
                       "shared memory limit");
            b->groups = 0;
            for (uint32_t gch : learn::kGroupChoices)
                if (!b->groups && learn::LearnSmem::plan(b->L, gch).total <= uint32_t(smem_max)) b->groups = gch;
            if (!b->groups) throw Error(UMC_ERR_UNSUPPORTED, "chain too large for the learned sampler's shared memory");
            const learn::LearnSmem sp = learn::LearnSmem::plan(b->L, b->groups);
            const void* lk = b->groups == 8   ? reinterpret_cast<const void*>(learn::u1_learned_batch<8>)
                             : b->groups == 6 ? reinterpret_cast<const void*>(learn::u1_learned_batch<6>)
                                              : reinterpret_cast<const void*>(learn::u1_learned_batch<4>);
            cuda_check(cudaFuncSetAttribute(lk, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sp.total)),
                       "learned smem");
            const size_t psm = per * 4;
            cuda_check(cudaFuncSetAttribute(learn::u1_plain_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            int(psm)),
                       "plain smem");
            b->learned_grid = resident_grid(lk, int(learn::kTile * b->groups), sp.total, b->device);
            b->plain_grid = resident_grid(reinterpret_cast<const void*>(learn::u1_plain_batch), 256, psm, b->device);
            cuda_check(cudaStreamSynchronize(b->stream), "create");
        } catch (...) {
            if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
            delete b;
            throw;
        }
        *out = b;
    });
}

int umc_u1batch_destroy(umc_u1batch* b)
{
    return lguard([&] {
        if (!b) return;
        scope(b->device);
        cudaStreamSynchronize(b->stream);
        if (b->own_stream) cudaStreamDestroy(b->stream);
        delete b;
    });
}

int umc_u1batch_randomize(umc_u1batch* b, uint64_t seed)
{
    return lguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(b->device);
        // hot start on the host from keyed draws: angle pi (2u - 1) of
        // (mix64(seed + golden (c + 1)), 0, init tag, natural link id)
        const uint32_t nl = 2 * b->L * b->L;
        std::vector<float> h(size_t(nl) * b->n_chains);
        for (uint32_t c = 0; c < b->n_chains; ++c) {
            const uint64_t kb =
                key_base(key_seed(mix64(seed + kGolden * (uint64_t(b->desc.first_chain) + c + 1ull)), 0, kTagInit));
            for (uint32_t i = 0; i < nl; ++i) {
                KeyedPcg g = KeyedPcg::open(kb, i);
                h[size_t(c) * nl + colour_index(b->L, i)] = 3.14159265358979f * sym_f32(g.next());
            }
        }
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(b->theta.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice), "hot start");
    });
}

int umc_u1batch_set_field(umc_u1batch* b, uint32_t chain, const float* theta)
{
    return lguard([&] {
        if (!b || !theta) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (chain >= b->n_chains) throw Error(UMC_ERR_OUT_OF_RANGE, "chain index out of range");
        scope(b->device);
        const uint32_t nl = 2 * b->L * b->L;
        std::vector<float> h(nl);
        for (uint32_t i = 0; i < nl; ++i) h[colour_index(b->L, i)] = theta[i];
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(b->theta.as<float>() + size_t(chain) * nl, h.data(), nl * 4, cudaMemcpyHostToDevice),
                   "upload chain");
    });
}

int umc_u1batch_get_field(umc_u1batch* b, uint32_t chain, float* theta)
{
    return lguard([&] {
        if (!b || !theta) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (chain >= b->n_chains) throw Error(UMC_ERR_OUT_OF_RANGE, "chain index out of range");
        scope(b->device);
        const uint32_t nl = 2 * b->L * b->L;
        std::vector<float> h(nl);
        cuda_check(cudaStreamSynchronize(b->stream), "sync");
        cuda_check(cudaMemcpy(h.data(), b->theta.as<float>() + size_t(chain) * nl, nl * 4, cudaMemcpyDeviceToHost),
                   "download chain");
        for (uint32_t i = 0; i < nl; ++i) theta[i] = h[colour_index(b->L, i)];
    });
}

int umc_u1batch_enqueue(umc_u1batch* b, uint64_t n_sweeps, const umc_mlp* net)
{
    return lguard([&] {
        NvtxRange range("umc_u1batch_enqueue");
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(b->device);
        enqueue_sweeps(b, n_sweeps, net, nullptr);
    });
}

int umc_u1batch_fetch(umc_u1batch* b, double* records, uint64_t max_sweeps, uint64_t* n_sweeps)
{
    return lguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(b->device);
        check_status(b->status, b->stream);
        const uint64_t n = std::min(b->rec_pending, max_sweeps);
        if (records && n)
            cuda_check(cudaMemcpy(records, b->records.p, n * b->n_chains * 32, cudaMemcpyDeviceToHost), "records");
        if (n_sweeps) *n_sweeps = n;
        const bool over = b->rec_overflow;
        b->rec_pending = 0;
        b->rec_overflow = false;
        if (over) throw Error(UMC_ERR_STATE, "record buffer overflowed: records past max_records were dropped");
    });
}

int umc_u1batch_run(umc_u1batch* b, uint64_t n_sweeps, const umc_mlp* net, double* records)
{
    return lguard([&] {
        NvtxRange range("umc_u1batch_run");
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (records && n_sweeps > b->max_records) throw Error(UMC_ERR_INVALID_ARGUMENT, "more sweeps than record slots");
        scope(b->device);
        if (b->rec_pending) throw Error(UMC_ERR_STATE, "unfetched records pending");
        enqueue_sweeps(b, n_sweeps, net, nullptr);
        check_status(b->status, b->stream);
        if (records && n_sweeps)
            cuda_check(cudaMemcpy(records, b->records.p, n_sweeps * b->n_chains * 32, cudaMemcpyDeviceToHost), "records");
        b->rec_pending = 0;
        b->rec_overflow = false;
    });
}

int umc_u1batch_run_dump(umc_u1batch* b, const umc_mlp* net, float* outputs)
{
    return lguard([&] {
        if (!b || !net || !outputs) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        scope(b->device);
        if (b->rec_pending) throw Error(UMC_ERR_STATE, "unfetched records pending");
        const size_t nl = size_t(2) * b->L * b->L;
        b->dump.alloc(nl * 64, "network outputs");
        cuda_check(cudaMemsetAsync(b->dump.p, 0, nl * 64, b->stream), "dump");
        enqueue_sweeps(b, 1, net, b->dump.as<float>());
        check_status(b->status, b->stream);
        std::vector<float> h(nl * 16);
        cuda_check(cudaMemcpy(h.data(), b->dump.p, nl * 64, cudaMemcpyDeviceToHost), "outputs");
        for (uint32_t i = 0; i < nl; ++i)
            std::memcpy(outputs + size_t(i) * 16, h.data() + size_t(colour_index(b->L, i)) * 16, 64);
        b->rec_pending = 0;
        b->rec_overflow = false;
    });
}

int umc_u1batch_counters(const umc_u1batch* b, uint64_t* sweeps, uint64_t* launches)
{
    return lguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (sweeps) *sweeps = b->sweeps;
        if (launches) *launches = b->launches;
    });
}

int umc_u1batch_set_counter(umc_u1batch* b, uint64_t sweeps)
{
    return lguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        b->sweeps = sweeps;
    });
}

int umc_u1batch_seeds(const umc_u1batch* b, uint64_t* seeds)
{
    return lguard([&] {
        if (!b || !seeds) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        for (uint32_t c = 0; c < b->n_chains; ++c) seeds[c] = b->chain_seed[c];
    });
}

int umc_u1batch_config(const umc_u1batch* b, uint32_t* plain_grid, uint32_t* learned_grid)
{
    return lguard([&] {
        if (!b) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (plain_grid) *plain_grid = uint32_t(b->plain_grid);
        if (learned_grid) *learned_grid = uint32_t(b->learned_grid);
    });
}

void* umc_u1batch_stream(const umc_u1batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }
void* umc_mlp_stream(const umc_mlp* n) { return n ? static_cast<void*>(n->stream) : nullptr; }

}  // extern "C"
