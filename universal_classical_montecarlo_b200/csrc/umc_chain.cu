// umc_chain.cu -- device chains: creation, field transfer, the Metropolis /
// Wolff schedules, observable records, and the chain part of the C ABI.
//
// A Metropolis sweep (driver.hpp:29-43) is one kernel per colour class; the
// last block of the last class folds the sweep's observables into a record.
// A Wolff flip (driver.hpp:104-162) is a bond-activation + union-find kernel
// followed by a flip kernel.  All launches go to the chain's stream; the
// blocking entry points synchronise once at the end and read the device
// status word, so bounded device-side waits surface as UMC_ERR_DEVICE_TIMEOUT.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <limits>
#include <new>

#include "umc_chain.hpp"
#include "umc_gauge.hpp"
#include "umc_spin_kernels.cuh"
#include "umc_fused.cuh"
#include "umc_nvtx.hpp"
#include "umc_wolff_tiled.cuh"

namespace umc {

void cuda_check(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return;
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) throw Error(UMC_ERR_OUT_OF_MEMORY, m);
    throw Error(UMC_ERR_CUDA, m);
}

void DevBuf::alloc(size_t b, const char* what)
{
    free_();
    if (b == 0) b = 16;
    cuda_check(cudaMalloc(&p, b), what);
    bytes = b;
}

void DevBuf::free_()
{
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

std::vector<uint32_t> ising_metropolis_thresholds(int32_t J, double beta, uint32_t D)
{
    std::vector<uint32_t> t(2 * size_t(D) + 1);
    for (int64_t m = -int64_t(D); m <= int64_t(D); ++m) {
        const int32_t dEi = int32_t(2 * int64_t(J) * m);
        const double dE = double(dEi);
        const double log_p = -beta * dE + 0.0;
        uint32_t tm1;
        if (log_p >= 0.0) {
            tm1 = 0xFFFFFFFFu;
        } else {
            // largest k with log(k 2^-32) < log_p; k = 0 always qualifies
            uint64_t lo = 0, hi = uint64_t(1) << 32;
            while (hi - lo > 1) {
                const uint64_t mid = (lo + hi) / 2;
                if (std::log(double(mid) * 0x1.0p-32) < log_p) lo = mid;
                else hi = mid;
            }
            tm1 = uint32_t(lo);
        }
        t[size_t(m + D)] = tm1;
    }
    return t;
}

void ising_wolff_thresholds(int32_t J, double beta, unsigned long long cw[2])
{
    for (int b = 0; b < 2; ++b) {
        const int32_t ss = b ? 1 : -1;
        const int32_t dEi = -J * ((-ss) - ss);  // energy_diff_bond with nb = -s_j
        const double p = 1.0 - std::exp(-beta * double(dEi));
        if (!(p > 0.0)) {
            cw[b] = 0;
            continue;
        }
        uint64_t lo = 0, hi = uint64_t(1) << 32;  // k = 0 qualifies since 0 < p
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) / 2;
            if (double(uint32_t(mid)) * 0x1.0p-32 < p) lo = mid;
            else hi = mid;
        }
        cw[b] = lo + 1;
    }
}


LaunchScope::LaunchScope(umc_chain* chain, int k) : c(chain), kind(k)
{
    nvtxRangePushA(kernel_kind_name(k));
    c->launches[k]++;
    if (!c->timing) return;
    if (c->event_pool.size() < 2) {
        for (int q = 0; q < 64; ++q) {
            cudaEvent_t e;
            cuda_check(cudaEventCreate(&e), "cudaEventCreate");
            c->event_pool.push_back(e);
        }
    }
    a = c->event_pool.back();
    c->event_pool.pop_back();
    cuda_check(cudaEventRecord(a, c->stream), "cudaEventRecord");
}

LaunchScope::~LaunchScope()
{
    nvtxRangePop();
    if (!a) return;
    cudaEvent_t b = c->event_pool.back();
    c->event_pool.pop_back();
    cudaEventRecord(b, c->stream);
    c->timed.push_back({kind, a, b});
    // bound the number of outstanding event pairs
    if (c->timed.size() >= 4096) {
        try {
            collect_kernel_times(c);
        } catch (...) {
        }
    }
}

void collect_kernel_times(umc_chain* c)
{
    if (c->timed.empty()) return;
    cuda_check(cudaStreamSynchronize(c->stream), "synchronise for kernel times");
    for (auto& t : c->timed) {
        float ms = 0.f;
        cuda_check(cudaEventElapsedTime(&ms, t.a, t.b), "cudaEventElapsedTime");
        c->device_ms[t.kind] += ms;
        c->event_pool.push_back(t.a);
        c->event_pool.push_back(t.b);
    }
    c->timed.clear();
}

namespace {

bool fused_step(umc_chain* c, double beta, bool wolff, bool sweep, double* rec, unsigned long long* size_slot);

uint32_t grid_for(const umc_chain* c, uint64_t work)
{
    const uint64_t b = (work + kBlock - 1) / kBlock;
    return uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(b, c->max_grid)));
}

void device_scope(const umc_chain* c) { cuda_check(cudaSetDevice(c->device), "cudaSetDevice"); }

void launch_check(const char* what) { cuda_check(cudaGetLastError(), what); }

template <class T>
void upload(DevBuf& b, const std::vector<T>& v, cudaStream_t s, const char* what)
{
    b.alloc(v.size() * sizeof(T), what);
    if (!v.empty()) cuda_check(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s), what);
}

Placement placement(const umc_chain* c)
{
    Placement pl{};
    if (c->stencil) {
        pl.position = nullptr;
        pl.Lx = uint32_t(c->dims[0]);
        pl.Ly = uint32_t(c->dims[1]);
        pl.half = uint32_t(c->n / 2);
    } else {
        pl.position = c->position.as<uint32_t>();
        pl.Lx = pl.Ly = 1;
        pl.half = 0;
    }
    return pl;
}

bool is_spin(const umc_chain* c)
{
    return c->model == UMC_MODEL_ISING || c->model == UMC_MODEL_VECTOR || c->model == UMC_MODEL_XY_ANGLE;
}

void ensure_csr(umc_chain* c)
{
    if (c->off.p) return;
    if (c->h_off.empty() && c->n > 0) {
        // regular lattice created without tables: build them from the extents
        umc_graph* g = make_cubic(c->dims[0], c->dims[1], c->dims[2]);
        materialize(g);
        c->h_off = g->c_offset;
        c->h_adj = g->c_bonds;
        c->h_slot = g->c_slot_edge;
        delete g;
    }
    upload(c->off, c->h_off, c->stream, "upload CSR offsets");
    upload(c->adj, c->h_adj, c->stream, "upload CSR bonds");
    upload(c->slot, c->h_slot, c->stream, "upload CSR edge ids");
}

void ensure_labels(umc_chain* c)
{
    if (c->lab0.p) return;
    c->lab0.alloc(c->n * 4, "Wolff labels");
    c->lab1.alloc(c->n * 4, "Wolff labels");
    const uint32_t g = grid_for(c, c->n);
    LaunchScope ls(c, UMC_KERNEL_OTHER);
    iota_u32<<<g, kBlock, 0, c->stream>>>(c->lab0.as<uint32_t>(), uint32_t(c->n));
    iota_u32<<<g, kBlock, 0, c->stream>>>(c->lab1.as<uint32_t>(), uint32_t(c->n));
    c->launches[UMC_KERNEL_OTHER]++;
    launch_check("iota labels");
}

// Next free record slot on the device (records are fetched in order).
uint64_t next_record(umc_chain* c)
{
    if (c->rec_pending >= c->max_records) c->rec_overflow = true;
    return (c->rec_pending++) % c->max_records;
}

double* record_ptr(umc_chain* c, uint64_t r) { return c->records.as<double>() + r * kObs; }
unsigned long long* size_ptr(umc_chain* c, uint64_t r) { return c->sizes.as<unsigned long long>() + r; }

template <class Topo>
void launch_ising_generic(umc_chain* c, IsingArgs a, Topo t)
{
    const size_t smem = (2 * size_t(a.D) + 1) * sizeof(uint32_t);
    LaunchScope ls(c, UMC_KERNEL_METROPOLIS);
    ising_pass<Topo><<<grid_for(c, a.count), kBlock, smem, c->stream>>>(a, t);
}

template <int N, class Topo>
void launch_vector(umc_chain* c, const VecArgs& a, Topo t)
{
    const uint32_t g = grid_for(c, a.count);
    LaunchScope ls(c, UMC_KERNEL_METROPOLIS);
    if (c->desc.proposal == UMC_PROPOSAL_ROTATION) vector_pass<N, kPropRotation, Topo><<<g, kBlock, 0, c->stream>>>(a, t);
    else vector_pass<N, kPropSphere, Topo><<<g, kBlock, 0, c->stream>>>(a, t);
}

template <class Topo>
void launch_vector_n(umc_chain* c, const VecArgs& a, Topo t)
{
    switch (c->N) {
    case 1: launch_vector<1>(c, a, t); break;
    case 2: launch_vector<2>(c, a, t); break;
    case 3: launch_vector<3>(c, a, t); break;
    case 4: launch_vector<4>(c, a, t); break;
    default: throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin<N>: N must be 1..4");
    }
}

template <class Topo>
void spin_pass(umc_chain* c, uint32_t p, double beta, uint64_t kbase, const PassOut& o, Topo t)
{
    const uint32_t first = uint32_t(c->class_start[p]);
    const uint32_t count = uint32_t(c->class_start[p + 1] - c->class_start[p]);
    if (c->model == UMC_MODEL_ISING) {
        IsingArgs a{c->field.as<int8_t>(), first, count, kbase, c->tm1.as<uint32_t>(), c->max_degree, c->J_int, o};
        launch_ising_generic(c, a, t);
    } else if (c->model == UMC_MODEL_VECTOR) {
        VecArgs a{c->field.as<float>(), uint32_t(c->n), first, count, kbase, c->J, float(beta), float(c->desc.width), o,
                  c->desc.coupling, beta, vector_metropolis_err(beta, c->desc.coupling, c->N, c->max_degree)};
        launch_vector_n(c, a, t);
    } else {
        XYArgs a{c->field.as<float>(), first, count, kbase, c->J, float(beta), float(c->desc.width), o,
                 c->desc.coupling, beta, xy_metropolis_err(beta, c->desc.coupling, c->max_degree)};
        LaunchScope ls(c, UMC_KERNEL_METROPOLIS);
        xy_pass<Topo><<<grid_for(c, count), kBlock, 0, c->stream>>>(a, t);
    }
}

void ensure_ising_tables(umc_chain* c, double beta)
{
    if (c->model != UMC_MODEL_ISING) return;
    if (c->tm1_valid && c->tm1_beta == beta) return;
    c->h_tm1 = ising_metropolis_thresholds(c->J_int, beta, c->max_degree);
    if (!c->tm1.p || c->tm1.bytes < c->h_tm1.size() * 4) c->tm1.alloc(c->h_tm1.size() * 4, "Ising thresholds");
    cuda_check(cudaMemcpyAsync(c->tm1.p, c->h_tm1.data(), c->h_tm1.size() * 4, cudaMemcpyHostToDevice, c->stream),
               "upload Ising thresholds");
    // the pageable source must stay alive until the copy ran
    cuda_check(cudaStreamSynchronize(c->stream), "upload Ising thresholds");
    c->tm1_beta = beta;
    c->tm1_valid = true;
}

void observe_into(umc_chain* c, double* rec, unsigned long long* size_slot)
{
    ensure_csr(c);
    const PassOut o{c->ctl.as<DevCtl>(), c->partials.as<double>(), rec, nullptr, kMaxPasses - 1, 1, 1};
    const uint32_t g = grid_for(c, c->n);
    LaunchScope ls(c, UMC_KERNEL_OBSERVE);
    switch (c->model) {
    case UMC_MODEL_ISING:
        observe_csr<0><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot);
        break;
    case UMC_MODEL_XY_ANGLE:
        observe_csr<-1><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot);
        break;
    case UMC_MODEL_VECTOR:
        switch (c->N) {
        case 1: observe_csr<1><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot); break;
        case 2: observe_csr<2><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot); break;
        case 3: observe_csr<3><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot); break;
        case 4: observe_csr<4><<<g, kBlock, 0, c->stream>>>(c->field.p, uint32_t(c->n), c->off.as<uint32_t>(), c->adj.as<uint32_t>(), c->J, o, size_slot); break;
        }
        break;
    }
    launch_check("observe");
}

// One Metropolis sweep of a spin model: one kernel per colour class.
void spin_sweep(umc_chain* c, double beta, double* rec)
{
    if (fused_step(c, beta, false, true, rec, nullptr)) return;
    ensure_ising_tables(c, beta);
    const uint64_t kbase = key_base(key_seed(c->desc.seed, c->sweeps, tag_site(0)));
    const bool fused = c->symmetric;
    for (uint32_t p = 0; p < c->n_colours; ++p) {
        const bool last = p + 1 == c->n_colours;
        const PassOut o{c->ctl.as<DevCtl>(), c->partials.as<double>(), fused ? rec : nullptr, nullptr,
                        int(p), int(c->n_colours), last ? 1 : 0};
        uint32_t tm[5] = {0, 0, 0, 0, 0};
        if (c->packed_ising)
            for (int t = 0; t < 5; ++t) tm[t] = c->h_tm1[size_t(int(c->max_degree) + 2 * t - 4)];
        const uint32_t vpr = uint32_t(c->dims[0] / 2 / 16);
        const bool fast = c->packed_ising && tm[0] == 0xFFFFFFFFu && tm[1] == 0xFFFFFFFFu && tm[2] == 0xFFFFFFFFu &&
                          tm[4] <= tm[3] && vpr < (1u << 15) && c->n / 2 / 16 < (uint64_t(1) << 25);
        if (fast) {
            IsingFastArgs a{};
            a.spins = c->field.as<int8_t>();
            a.H = uint32_t(c->dims[0] / 2);
            a.Ly = uint32_t(c->dims[1]);
            a.half = uint32_t(c->n / 2);
            a.colour = p;
            a.vpr = vpr;
            a.vmagic = ((uint64_t(1) << 40) / vpr) + 1;
            a.kbase = kbase;
            a.T3 = tm[3];
            a.T4 = tm[4];
            a.J = c->J_int;
            for (int b = 0; b < 4; ++b) {
                a.m1[b] = 2u << (8 * b);
                a.m2[b] = 0u - (4u << (8 * b));
            }
            a.out = o;
            const uint32_t g = grid_for(c, c->n / 2 / 16);
            LaunchScope ls(c, UMC_KERNEL_METROPOLIS);
            if (p == 1) ising_fast_pass<true><<<g, kBlock, 0, c->stream>>>(a);
            else ising_fast_pass<false><<<g, kBlock, 0, c->stream>>>(a);
        } else if (c->packed_ising) {
            IsingPackedArgs a{};
            a.spins = c->field.as<int8_t>();
            a.H = uint32_t(c->dims[0] / 2);
            a.Ly = uint32_t(c->dims[1]);
            a.half = uint32_t(c->n / 2);
            a.colour = p;
            a.kbase = kbase;
            for (int t = 0; t < 5; ++t) a.tm1[t] = tm[t];
            a.J = c->J_int;
            a.out = o;
            const uint32_t g = grid_for(c, c->n / 2 / 16);
            LaunchScope ls(c, UMC_KERNEL_METROPOLIS);
            ising_packed_pass<<<g, kBlock, 0, c->stream>>>(a);
        } else if (c->stencil) {
            StencilTopo t{uint32_t(c->dims[0] / 2), uint32_t(c->dims[1]), uint32_t(c->dims[2]), uint32_t(c->n / 2), p,
                          c->dims[1] > 1 ? 1u : 0u, c->dims[2] > 1 ? 1u : 0u, 0xFFu, 0xFFu};
            const uint64_t H = c->dims[0] / 2, Ly = c->dims[1];
            if ((H & (H - 1)) == 0 && (Ly & (Ly - 1)) == 0) {
                t.hshift = uint32_t(__builtin_ctzll(H));
                t.yshift = uint32_t(__builtin_ctzll(Ly));
            }
            spin_pass(c, p, beta, kbase, o, t);
        } else {
            CsrTopo t{c->off.as<uint32_t>(), c->adj.as<uint32_t>(), uint32_t(c->class_start[p])};
            spin_pass(c, p, beta, kbase, o, t);
        }
        launch_check("Metropolis colour pass");
    }
    if (!fused && rec) observe_into(c, rec, nullptr);
    c->sweeps++;
}

template <int MODEL, int TX, int TY, int TZ>
void launch_tiled(umc_chain* c, WolffTileArgs& t)
{
    t.ntx = uint32_t((t.Lx + TX - 1) / TX);
    t.nty = uint32_t((t.Ly + TY - 1) / TY);
    const uint32_t ntz = uint32_t((t.Lz + TZ - 1) / TZ);
    {
        LaunchScope ls(c, UMC_KERNEL_WOLFF_UNION);
        wolff_tile_local<MODEL, TX, TY, TZ><<<t.ntx * t.nty * ntz, TX * TY * TZ, 0, c->stream>>>(t);
    }
    const uint32_t g = grid_for(c, c->n);
    {
        LaunchScope ls(c, UMC_KERNEL_WOLFF_MERGE);
        wolff_tile_merge<<<g, kBlock, 0, c->stream>>>(t);
    }
    {
        LaunchScope ls(c, UMC_KERNEL_WOLFF_FLIP);
        wolff_tile_flip<MODEL><<<g, kBlock, 0, c->stream>>>(t);
    }
}

template <int MODEL>
void launch_tiled_dims(umc_chain* c, WolffTileArgs& t)
{
    if (t.Lz > 1) launch_tiled<MODEL, 8, 8, 8>(c, t);
    else launch_tiled<MODEL, 32, 16, 1>(c, t);
}

// Wolff flip on a regular lattice: tiled union-find (umc_wolff_tiled.cuh).
void stencil_flip(umc_chain* c, double beta, unsigned long long* size_slot)
{
    if (!c->lab0.p) {
        c->lab0.alloc(c->n * 4, "Wolff labels");
        c->lab1.alloc(c->n, "Wolff crossing bonds");
    }
    WolffTileArgs t{};
    t.field = c->field.p;
    t.label = c->lab0.as<uint32_t>();
    t.cross = c->lab1.as<uint8_t>();
    t.n = uint32_t(c->n);
    t.half = uint32_t(c->n / 2);
    t.Lx = uint32_t(c->dims[0]);
    t.Ly = uint32_t(c->dims[1]);
    t.Lz = uint32_t(c->dims[2]);
    t.ndir = (t.Lx > 1) + (t.Ly > 1) + (t.Lz > 1);
    t.seed = c->desc.seed;
    t.flip = c->flips;
    t.J = c->J;
    t.beta = float(beta);
    t.J64 = c->desc.coupling;
    t.beta64 = beta;
    t.err = vector_wolff_err(beta, c->desc.coupling, c->N);
    if (c->model == UMC_MODEL_ISING) {
        if (!c->cw_valid || c->cw_beta != beta) {
            ising_wolff_thresholds(c->J_int, beta, c->cw);
            c->cw_beta = beta;
            c->cw_valid = true;
        }
        t.cw[0] = c->cw[0];
        t.cw[1] = c->cw[1];
    }
    t.ctl = c->ctl.as<DevCtl>();
    t.size_slot = size_slot;
    switch (c->model == UMC_MODEL_ISING ? 0 : c->N) {
    case 0: launch_tiled_dims<0>(c, t); break;
    case 1: launch_tiled_dims<1>(c, t); break;
    case 2: launch_tiled_dims<2>(c, t); break;
    case 3: launch_tiled_dims<3>(c, t); break;
    default: launch_tiled_dims<4>(c, t); break;
    }
    launch_check("Wolff flip (tiled)");
}

// Fused step on a regular lattice (umc_fused.cuh): returns false when the
// chain does not qualify or cooperative launch is unavailable, in which case
// the caller runs the multi-kernel path.
template <int N, int TX, int TY, int TZ, int SPT>
bool launch_fused_t(umc_chain* c, FusedArgs& a)
{
    auto kern = hybrid_fused<N, TX, TY, TZ, SPT>;
    constexpr int T = TX * TY * TZ / SPT;  // threads per block
    if (c->fused_grid < 0) {
        int coop = 0, nb = 0, sms = 0;
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, T, 0) != cudaSuccess) {
            cudaGetLastError();
            nb = 0;
        }
        c->fused_grid = coop ? std::min<int>(nb * sms, int(c->max_grid)) : 0;
    }
    if (c->fused_grid <= 0) return false;
    a.w.ntx = uint32_t((a.w.Lx + TX - 1) / TX);
    a.w.nty = uint32_t((a.w.Ly + TY - 1) / TY);
    void* args[] = {&a};
    LaunchScope ls(c, UMC_KERNEL_FUSED);
    const cudaError_t e = cudaLaunchCooperativeKernel(reinterpret_cast<void*>(kern), dim3(c->fused_grid), dim3(T), args, 0,
                                                      c->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->fused_grid = 0;
        c->launches[UMC_KERNEL_FUSED]--;
        return false;
    }
    return true;
}

// Bound on the + bonds that can leave a TX x TY x TZ tile: in direction d
// only the sites of the last plane of each tile, ceil(L_d / T_d) planes of
// n / L_d sites.
uint64_t crossing_capacity(const umc_chain* c, uint32_t TX, uint32_t TY, uint32_t TZ)
{
    const uint64_t T[3] = {TX, TY, TZ};
    uint64_t cap = 0;
    for (int d = 0; d < 3; ++d) {
        const uint64_t L = c->dims[d];
        if (L < 2) continue;
        cap += (L + T[d] - 1) / T[d] * (c->n / L);
    }
    return cap;
}

template <int N>
bool launch_fused_n(umc_chain* c, FusedArgs& a)
{
    const bool three = a.w.Lz > 1;
    const uint64_t cap = three ? crossing_capacity(c, 8, 8, 8) : crossing_capacity(c, 32, 16, 1);
    if (a.do_wolff) {
        if (c->n >= (uint64_t(1) << 30)) return false;  // list entries are site * 4 + direction
        if (c->xlist.bytes < cap * 4) c->xlist.alloc(cap * 4, "Wolff crossing-bond list");
        a.xlist = c->xlist.as<uint32_t>();
        a.xcap = uint32_t(cap);
    }
    if (three) return launch_fused_t<N, 8, 8, 8, 2>(c, a);
    return launch_fused_t<N, 32, 16, 1, 2>(c, a);
}

bool fused_step(umc_chain* c, double beta, bool wolff, bool sweep, double* rec, unsigned long long* size_slot)
{
    if (!c->fused || !c->stencil || c->model != UMC_MODEL_VECTOR) return false;
    if (wolff && c->desc.wolff_axis != UMC_AXIS_SPHERE) return false;
    if (sweep && c->desc.proposal != UMC_PROPOSAL_SPHERE && c->desc.proposal != UMC_PROPOSAL_ROTATION) return false;
    if (c->dims[0] / 2 > 0xFFFFFFFFull) return false;
    if (wolff && !c->lab0.p) {
        c->lab0.alloc(c->n * 4, "Wolff labels");
        c->lab1.alloc(c->n, "Wolff crossing bonds");
    }
    FusedArgs a{};
    WolffTileArgs& t = a.w;
    t.field = c->field.p;
    t.label = c->lab0.as<uint32_t>();
    t.cross = c->lab1.as<uint8_t>();
    t.n = uint32_t(c->n);
    t.half = uint32_t(c->n / 2);
    t.Lx = uint32_t(c->dims[0]);
    t.Ly = uint32_t(c->dims[1]);
    t.Lz = uint32_t(c->dims[2]);
    t.ndir = (t.Lx > 1) + (t.Ly > 1) + (t.Lz > 1);
    t.seed = c->desc.seed;
    t.flip = c->flips;
    t.J = c->J;
    t.beta = float(beta);
    t.J64 = c->desc.coupling;
    t.beta64 = beta;
    t.err = vector_wolff_err(beta, c->desc.coupling, c->N);
    t.ctl = c->ctl.as<DevCtl>();
    t.size_slot = size_slot;
    a.bar = &c->ctl.as<DevCtl>()->bar;
    a.do_wolff = wolff ? 1u : 0u;
    a.do_sweep = sweep ? 1u : 0u;
    a.H = uint32_t(c->dims[0] / 2);
    a.hshift = a.yshift = 0xFFu;
    const uint64_t H = c->dims[0] / 2, Ly = c->dims[1];
    if ((H & (H - 1)) == 0 && (Ly & (Ly - 1)) == 0) {
        a.hshift = uint32_t(__builtin_ctzll(H));
        a.yshift = uint32_t(__builtin_ctzll(Ly));
    }
    a.sweep_kbase = key_base(key_seed(c->desc.seed, c->sweeps, tag_site(0)));
    a.beta_metro = float(beta);
    a.beta_metro64 = beta;
    a.err_metro = vector_metropolis_err(beta, c->desc.coupling, c->N, c->max_degree);
    a.proposal = c->desc.proposal == UMC_PROPOSAL_ROTATION ? kPropRotation : kPropSphere;
    a.delta = float(c->desc.width);
    a.out = PassOut{c->ctl.as<DevCtl>(), c->partials.as<double>(), sweep ? rec : nullptr, nullptr, kMaxPasses - 2, 1, 1};
    bool ok = false;
    switch (c->N) {
    case 1: ok = launch_fused_n<1>(c, a); break;
    case 2: ok = launch_fused_n<2>(c, a); break;
    case 3: ok = launch_fused_n<3>(c, a); break;
    default: ok = launch_fused_n<4>(c, a); break;
    }
    if (!ok) return false;
    if (wolff) c->flips++;
    if (sweep) c->sweeps++;
    return true;
}

// One Wolff flip of a spin model.
void spin_flip(umc_chain* c, double beta, double* rec, unsigned long long* size_slot)
{
    if (c->model == UMC_MODEL_XY_ANGLE || c->desc.wolff_axis == UMC_AXIS_NONE)
        throw Error(UMC_ERR_UNSUPPORTED, "Wolff needs a reflection axis (FixedAxis for Ising, UniformSphereN for VectorSpin)");
    if (!c->symmetric) throw Error(UMC_ERR_UNSUPPORTED, "Wolff needs a symmetric graph");
    if (c->stencil) {
        if (!fused_step(c, beta, true, false, nullptr, size_slot)) {
            stencil_flip(c, beta, size_slot);
            c->flips++;
        }
        if (rec) observe_into(c, rec, size_slot);
        return;
    }
    ensure_csr(c);
    ensure_labels(c);
    WolffArgs a{};
    a.field = c->field.p;
    a.n = uint32_t(c->n);
    a.off = c->off.as<uint32_t>();
    a.adj = c->adj.as<uint32_t>();
    a.slot = c->slot.as<uint32_t>();
    // labels of this flip (identity on entry) and of the next one (reset here)
    uint32_t* cur = (c->lab_cur ? c->lab1 : c->lab0).as<uint32_t>();
    uint32_t* nxt = (c->lab_cur ? c->lab0 : c->lab1).as<uint32_t>();
    a.lab = cur;
    a.lab_next = nxt;
    a.seed = c->desc.seed;
    a.flip = c->flips;
    a.J = c->J;
    a.beta = float(beta);
    a.J64 = c->desc.coupling;
    a.beta64 = beta;
    a.err = vector_wolff_err(beta, c->desc.coupling, c->N);
    if (c->model == UMC_MODEL_ISING) {
        if (!c->cw_valid || c->cw_beta != beta) {
            ising_wolff_thresholds(c->J_int, beta, c->cw);
            c->cw_beta = beta;
            c->cw_valid = true;
        }
        a.cw[0] = c->cw[0];
        a.cw[1] = c->cw[1];
    }
    a.ctl = c->ctl.as<DevCtl>();
    a.size_slot = size_slot;
    const uint32_t g = grid_for(c, c->n);
    const int model = c->model == UMC_MODEL_ISING ? 0 : c->N;
    {
        LaunchScope ls(c, UMC_KERNEL_WOLFF_UNION);
        switch (model) {
        case 0: wolff_union<0><<<g, kBlock, 0, c->stream>>>(a); break;
        case 1: wolff_union<1><<<g, kBlock, 0, c->stream>>>(a); break;
        case 2: wolff_union<2><<<g, kBlock, 0, c->stream>>>(a); break;
        case 3: wolff_union<3><<<g, kBlock, 0, c->stream>>>(a); break;
        case 4: wolff_union<4><<<g, kBlock, 0, c->stream>>>(a); break;
        }
    }
    {
        LaunchScope ls(c, UMC_KERNEL_WOLFF_FLIP);
        switch (model) {
        case 0: wolff_flip<0><<<g, kBlock, 0, c->stream>>>(a); break;
        case 1: wolff_flip<1><<<g, kBlock, 0, c->stream>>>(a); break;
        case 2: wolff_flip<2><<<g, kBlock, 0, c->stream>>>(a); break;
        case 3: wolff_flip<3><<<g, kBlock, 0, c->stream>>>(a); break;
        case 4: wolff_flip<4><<<g, kBlock, 0, c->stream>>>(a); break;
        }
    }
    launch_check("Wolff flip");
    c->lab_cur ^= 1;
    if (rec) observe_into(c, rec, size_slot);
    c->flips++;
}

void raise_status(umc_chain* c, unsigned int st)
{
    if (st) {
        // tickets and the barrier may be mid-count after an aborted kernel
        cuda_check(cudaMemset(c->ctl.p, 0, sizeof(DevCtl)), "clear control block");
        std::string m = "device-side bound exhausted:";
        if (st & kDevErrUnionFind) m += " union-find";
        if (st & kDevErrGeometry) m += " geometry";
        if (st & kDevErrRetry) m += " proposal-retry";
        if (st & kDevErrBarrier) m += " grid-barrier";
        throw Error(UMC_ERR_DEVICE_TIMEOUT, m);
    }
}

void check_status(umc_chain* c)
{
    unsigned int st = 0;
    cuda_check(cudaMemcpyAsync(&st, &c->ctl.as<DevCtl>()->status, sizeof st, cudaMemcpyDeviceToHost, c->stream), "read status");
    cuda_check(cudaStreamSynchronize(c->stream), "synchronise chain");
    raise_status(c, st);
}

// The chain's pinned host image [status | records | sizes].
struct Stage
{
    unsigned int* status;
    double* rec;
    unsigned long long* sz;
};

Stage host_stage(umc_chain* c)
{
    const size_t need = 16 + size_t(c->max_records) * (kObs * sizeof(double) + sizeof(unsigned long long));
    if (c->host_stage_bytes < need) {
        cuda_check(cudaStreamSynchronize(c->stream), "synchronise chain");
        if (c->rec_stream) cuda_check(cudaStreamSynchronize(c->rec_stream), "synchronise record copies");
        if (c->host_stage) cudaFreeHost(c->host_stage);
        c->host_stage = nullptr;
        c->host_stage_bytes = 0;
        c->streamed = 0;
        cuda_check(cudaHostAlloc(&c->host_stage, need, cudaHostAllocDefault), "pinned record stage");
        c->host_stage_bytes = need;
    }
    uint8_t* stage = static_cast<uint8_t*>(c->host_stage);
    return {reinterpret_cast<unsigned int*>(stage), reinterpret_cast<double*>(stage + 16),
            reinterpret_cast<unsigned long long*>(stage + 16 + size_t(c->max_records) * kObs * sizeof(double))};
}

// After the unit that writes ring slot r has been enqueued: with record
// streaming on, its record and size go to the pinned stage right behind it.
void record_done(umc_chain* c, uint64_t r)
{
    if (!c->stream_records || c->rec_overflow || r != c->streamed) return;
    const Stage h = host_stage(c);
    if (!c->rec_stream) {
        cuda_check(cudaStreamCreateWithFlags(&c->rec_stream, cudaStreamNonBlocking), "record stream");
        for (auto& e : c->rec_ready) cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "record event");
    }
    // the copies run on their own stream once the step has written slot r, so
    // the next step's work on the chain's stream does not queue behind them
    cudaEvent_t e = c->rec_ready[c->rec_next];
    c->rec_next ^= 1;
    cuda_check(cudaEventRecord(e, c->stream), "stream record");
    cuda_check(cudaStreamWaitEvent(c->rec_stream, e, 0), "stream record");
    cuda_check(cudaMemcpyAsync(h.rec + r * kObs, c->records.as<double>() + r * kObs, kObs * sizeof(double),
                               cudaMemcpyDeviceToHost, c->rec_stream), "stream record");
    cuda_check(cudaMemcpyAsync(h.sz + r, c->sizes.as<unsigned long long>() + r, sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, c->rec_stream), "stream record");
    c->streamed = r + 1;
}

// Status word, pending records and cluster sizes in one round trip: async
// copies into the chain's pinned stage (only the records not streamed there
// already), one synchronisation, then host copies.
void fetch(umc_chain* c, double* records, uint64_t* sizes, uint64_t capacity, uint64_t* n_out)
{
    const uint64_t pend = c->rec_overflow ? 0 : c->rec_pending;
    const Stage h = host_stage(c);
    unsigned int* st = h.status;
    double* rec = h.rec;
    unsigned long long* sz = h.sz;
    const uint64_t from = std::min(c->streamed, pend);
    c->streamed = 0;
    cuda_check(cudaMemcpyAsync(st, &c->ctl.as<DevCtl>()->status, sizeof *st, cudaMemcpyDeviceToHost, c->stream), "read status");
    if (pend > from) {
        cuda_check(cudaMemcpyAsync(rec + from * kObs, c->records.as<double>() + from * kObs,
                                   (pend - from) * kObs * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                   "fetch records");
        cuda_check(cudaMemcpyAsync(sz + from, c->sizes.as<unsigned long long>() + from,
                                   (pend - from) * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream),
                   "fetch sizes");
    }
    cuda_check(cudaStreamSynchronize(c->stream), "synchronise chain");
    if (c->rec_stream) cuda_check(cudaStreamSynchronize(c->rec_stream), "synchronise record copies");
    raise_status(c, *st);
    if (c->rec_overflow) {
        c->rec_overflow = false;
        c->rec_pending = 0;
        throw Error(UMC_ERR_STATE, "observable records overflowed the device ring; fetch more often or raise max_records");
    }
    const uint64_t n = c->rec_pending;
    if ((records || sizes) && n > capacity) throw Error(UMC_ERR_INVALID_ARGUMENT, "record buffer too small");
    if (records && n) std::memcpy(records, rec, n * kObs * sizeof(double));
    if (sizes)
        for (uint64_t k = 0; k < n; ++k) sizes[k] = sz[k];
    if (n_out) *n_out = n;
    c->rec_pending = 0;
}

// --------------------------------------------------------------- creation

// Which proposal / axis a model accepts (the reference enforces this through
// the Proposal concept's value type, dof/proposal.hpp:8-12).
void validate_proposal(umc_chain* c, int32_t proposal, double width, uint32_t hits)
{
    if (!std::isfinite(width)) throw Error(UMC_ERR_INVALID_ARGUMENT, "proposal width must be finite");
    if (hits == 0 || hits > 0xFF00) throw Error(UMC_ERR_INVALID_ARGUMENT, "hits must be in [1, 65280]");
    switch (c->model) {
    case UMC_MODEL_ISING:
        if (proposal != 0 && proposal != UMC_PROPOSAL_FLIP) throw Error(UMC_ERR_UNSUPPORTED, "Ising takes the Flip proposal");
        break;
    case UMC_MODEL_VECTOR:
        if (c->N < 1 || c->N > 4) throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin<N>: N must be 1..4");
        if (proposal != UMC_PROPOSAL_SPHERE && proposal != UMC_PROPOSAL_ROTATION)
            throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin takes UniformSphereN or LocalRotation");
        if (proposal == UMC_PROPOSAL_ROTATION && c->N < 2) throw Error(UMC_ERR_UNSUPPORTED, "LocalRotation needs N >= 2");
        break;
    case UMC_MODEL_XY_ANGLE:
    case UMC_MODEL_U1:
        if (proposal != UMC_PROPOSAL_U1SHIFT) throw Error(UMC_ERR_UNSUPPORTED, "angle models take U1Shift");
        break;
    case UMC_MODEL_SU:
        if (proposal != UMC_PROPOSAL_SUSHIFT) throw Error(UMC_ERR_UNSUPPORTED, "SU(N) takes SUShift");
        break;
    }
    if (hits != 1 && c->model != UMC_MODEL_U1 && c->model != UMC_MODEL_SU)
        throw Error(UMC_ERR_UNSUPPORTED, "multi-hit is provided for the gauge models");
}

void validate_axis(umc_chain* c, int32_t axis)
{
    if (axis == UMC_AXIS_NONE) return;
    if (c->model == UMC_MODEL_ISING && axis == UMC_AXIS_FIXED) return;
    if (c->model == UMC_MODEL_VECTOR && axis == UMC_AXIS_SPHERE) return;
    throw Error(UMC_ERR_UNSUPPORTED, "Wolff axis: FixedAxis for Ising, UniformSphereN for VectorSpin");
}

void create_chain(const umc_chain_desc* d, umc_chain* c)
{
    if (!d) throw Error(UMC_ERR_INVALID_ARGUMENT, "null descriptor");
    c->desc = *d;
    c->model = d->model;
    c->N = d->components <= 0 ? 1 : d->components;
    c->device = d->device;
    c->max_records = d->max_records ? d->max_records : 4096;
    if (c->desc.hits == 0) c->desc.hits = 1;
    if (c->desc.proposal == 0 && c->model == UMC_MODEL_ISING) c->desc.proposal = UMC_PROPOSAL_FLIP;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        throw Error(UMC_ERR_CUDA, "no CUDA device available");
    }
    if (c->device < 0 || c->device >= count) throw Error(UMC_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    cuda_check(cudaSetDevice(c->device), "cudaSetDevice");
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device), "SM count");
    c->max_grid = uint32_t(sms) * 8;

    if (is_spin(c)) {
        const umc_graph* g = d->graph;
        if (!g) throw Error(UMC_ERR_INVALID_ARGUMENT, "spin models need a graph");
        if (g->payload_bytes)
            throw Error(UMC_ERR_UNSUPPORTED,
                        "the built-in spin models take a graph without bond payloads, as the reference's Ising and "
                        "VectorSpin take PairGraph<>; a weighted model is a user model (umc/device.cuh BondTables)");
        c->n = g->n;
        c->symmetric = g->symmetric;
        c->n_colours = g->col.n_colours;
        c->class_start = g->col.class_start;
        c->stencil = g->stencil;
        std::memcpy(c->dims, g->dims, sizeof c->dims);
        c->max_degree = g->max_degree;
        if (g->materialized) {
            c->h_off = g->c_offset;
            c->h_adj = g->c_bonds;
            c->h_slot = g->c_slot_edge;
            c->h_position = g->col.position;
        }
        if (c->n_colours > uint32_t(kMaxPasses - 1))
            throw Error(UMC_ERR_UNSUPPORTED, "graph needs more colour classes than the engine supports (63)");
        validate_proposal(c, c->desc.proposal, c->desc.width, c->desc.hits);
        validate_axis(c, c->desc.wolff_axis);
        if (c->model == UMC_MODEL_ISING) {
            if (d->coupling != std::floor(d->coupling) || std::fabs(d->coupling) > 1e6)
                throw Error(UMC_ERR_INVALID_ARGUMENT, "Ising coupling J must be an integer (example/ising.hpp:18)");
            if (c->max_degree > 4096) throw Error(UMC_ERR_UNSUPPORTED, "Ising degree above 4096");
            c->J_int = int32_t(d->coupling);
            c->J = float(c->J_int);
            c->elem_bytes = 1;
            c->comps = 1;
            c->packed_ising = c->stencil && c->dims[2] == 1 && c->dims[1] >= 2 && (c->dims[0] / 2) % 16 == 0;
        } else if (c->model == UMC_MODEL_VECTOR) {
            c->J = float(d->coupling);
            c->elem_bytes = 4;
            c->comps = uint32_t(c->N);
        } else {
            c->J = float(d->coupling);
            c->elem_bytes = 4;
            c->comps = 1;
        }
    } else if (c->model == UMC_MODEL_U1 || c->model == UMC_MODEL_SU) {
        gauge_configure(c);
    } else {
        throw Error(UMC_ERR_INVALID_ARGUMENT, "unknown model");
    }
    if (c->n > 0xFFFFFFFFull) throw Error(UMC_ERR_OVERFLOW, "site count exceeds uint32_t");

    if (d->stream) {
        c->stream = static_cast<cudaStream_t>(d->stream);
    } else {
        cuda_check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        c->own_stream = true;
    }
    c->field_bytes = size_t(c->n) * c->comps * c->elem_bytes;
    c->field.alloc(c->field_bytes, "field");
    c->partials.alloc(size_t(c->max_grid) * kObs * sizeof(double), "partials");
    c->ctl.alloc(sizeof(DevCtl), "control block");
    cuda_check(cudaMemsetAsync(c->ctl.p, 0, sizeof(DevCtl), c->stream), "clear control block");
    c->records.alloc(c->max_records * kObs * sizeof(double), "records");
    c->sizes.alloc(c->max_records * sizeof(unsigned long long), "cluster sizes");
    cuda_check(cudaMemsetAsync(c->sizes.p, 0, c->max_records * sizeof(unsigned long long), c->stream), "clear sizes");
    if (!c->stencil && is_spin(c)) upload(c->position, c->h_position, c->stream, "upload positions");
    if (!c->stencil && is_spin(c)) ensure_csr(c);

    // cold start, as the reference constructors do
    if (c->model == UMC_MODEL_ISING) {
        cuda_check(cudaMemsetAsync(c->field.p, 1, c->field_bytes, c->stream), "cold start");
    } else if (c->model == UMC_MODEL_VECTOR) {
        cuda_check(cudaMemsetAsync(c->field.p, 0, c->field_bytes, c->stream), "cold start");
        std::vector<float> ones(c->n, 1.0f);
        cuda_check(cudaMemcpyAsync(c->field.as<float>() + (c->N - 1) * c->n, ones.data(), c->n * 4, cudaMemcpyHostToDevice, c->stream),
                   "cold start");
        cuda_check(cudaStreamSynchronize(c->stream), "cold start");
    } else if (c->model == UMC_MODEL_XY_ANGLE) {
        cuda_check(cudaMemsetAsync(c->field.p, 0, c->field_bytes, c->stream), "cold start");
    } else {
        gauge_cold_start(c);
    }
    cuda_check(cudaStreamSynchronize(c->stream), "chain creation");
}

void destroy_chain(umc_chain* c)
{
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->up_stream) cudaStreamSynchronize(c->up_stream);
    if (c->rec_stream) cudaStreamSynchronize(c->rec_stream);
    gauge_release(c);
    for (auto& t : c->timed) {
        cudaEventDestroy(t.a);
        cudaEventDestroy(t.b);
    }
    for (cudaEvent_t e : c->event_pool) cudaEventDestroy(e);
    if (c->upload_done) cudaEventDestroy(c->upload_done);
    for (int q = 0; q < 2; ++q) {
        if (c->up_copied[q]) cudaEventDestroy(c->up_copied[q]);
        if (c->up_consumed[q]) cudaEventDestroy(c->up_consumed[q]);
        c->up_staging[q].free_();
    }
    if (c->up_stream) cudaStreamDestroy(c->up_stream);
    if (c->rec_stream) cudaStreamDestroy(c->rec_stream);
    for (auto& e : c->rec_ready)
        if (e) cudaEventDestroy(e);
    if (c->host_stage) cudaFreeHost(c->host_stage);
    c->host_stage = nullptr;
    for (DevBuf* b : {&c->field, &c->staging, &c->off, &c->adj, &c->slot, &c->position, &c->lab0, &c->lab1, &c->xlist, &c->cells,
                      &c->inc_off, &c->inc_cell, &c->inc_which, &c->partials, &c->ctl, &c->records, &c->sizes, &c->tm1})
        b->free_();
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
}

template <class F>
int guarded(F&& f)
{
    try {
        set_last_error("");
        f();
        return UMC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("out of host memory");
        return UMC_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}

void check_beta(double beta)
{
    if (!std::isfinite(beta)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta must be finite");
}

void enqueue_sweeps(umc_chain* c, double beta, uint64_t n)
{
    check_beta(beta);
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t r = next_record(c);
        if (is_spin(c)) spin_sweep(c, beta, record_ptr(c, r));
        else gauge_sweep(c, beta, record_ptr(c, r));
        record_done(c, r);
    }
}

void enqueue_flips(umc_chain* c, double beta, uint64_t n, bool obs)
{
    check_beta(beta);
    if (!is_spin(c)) throw Error(UMC_ERR_UNSUPPORTED, "Wolff is defined for spin models only (driver.hpp:73-84)");
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t r = next_record(c);
        spin_flip(c, beta, obs ? record_ptr(c, r) : nullptr, size_ptr(c, r));
        record_done(c, r);
    }
}

void enqueue_hybrid(umc_chain* c, double beta, uint64_t n)
{
    check_beta(beta);
    if (!is_spin(c)) throw Error(UMC_ERR_UNSUPPORTED, "Wolff is defined for spin models only (driver.hpp:73-84)");
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t r = next_record(c);
        if (!fused_step(c, beta, true, true, record_ptr(c, r), size_ptr(c, r))) {
            spin_flip(c, beta, nullptr, size_ptr(c, r));
            spin_sweep(c, beta, record_ptr(c, r));
        }
        record_done(c, r);
    }
}

// Runs n units in chunks that fit the record ring, copying records out.
template <class Enq>
void run_chunked(umc_chain* c, uint64_t n, double* records, uint64_t* sizes, bool count_flips, Enq&& enq)
{
    if (c->rec_pending) fetch(c, nullptr, nullptr, 0, nullptr);  // drop stale records
    uint64_t done = 0;
    while (done < n) {
        const uint64_t m = std::min<uint64_t>(n - done, c->max_records);
        enq(m);
        std::vector<uint64_t> sz(m);
        uint64_t got = 0;
        fetch(c, records ? records + done * kObs : nullptr, sz.data(), m, &got);
        if (sizes) std::copy(sz.begin(), sz.end(), sizes + done);
        if (count_flips)
            for (uint64_t s : sz) {
                c->wolff_flips_done++;
                c->wolff_size_sum += double(s);
            }
        done += m;
    }
}

}  // namespace
// Self-test of the bounded grid barrier: a grid of two blocks of which only
// the first arrives, so the count never reaches gridDim and that block runs
// into kBarrierSpins.
static __global__ void barrier_selftest(GridBarrier* b, unsigned* status)
{
    if (blockIdx.x == 0) grid_barrier(b, status);
}

}  // namespace umc

using namespace umc;

extern "C" {

int umc_selftest_barrier_timeout(int32_t device, uint32_t* status_bits)
{
    return guarded([&] {
        cuda_check(cudaSetDevice(device), "cudaSetDevice");
        struct Cells
        {
            GridBarrier bar;
            unsigned status;
        };
        DevBuf buf;
        buf.alloc(sizeof(Cells), "self-test barrier");
        const Cells init{{0u, 0u}, 0u};
        cuda_check(cudaMemcpy(buf.p, &init, sizeof init, cudaMemcpyHostToDevice), "self-test set-up");
        Cells* d = buf.as<Cells>();
        barrier_selftest<<<2, 32>>>(&d->bar, &d->status);
        cuda_check(cudaGetLastError(), "self-test launch");
        Cells got{};
        cuda_check(cudaMemcpy(&got, buf.p, sizeof got, cudaMemcpyDeviceToHost), "self-test result");
        // the context still answers: a trivial operation after the timed-out kernel
        cuda_check(cudaMemset(buf.p, 0, sizeof(Cells)), "context check");
        cuda_check(cudaDeviceSynchronize(), "context check");
        if (status_bits) *status_bits = got.status;
        if (got.status & kDevErrBarrier)
            throw Error(UMC_ERR_DEVICE_TIMEOUT, "grid barrier wait bound exhausted (self-test)");
    });
}

int umc_device_count(int* count)
{
    return guarded([&] {
        if (!count) throw Error(UMC_ERR_INVALID_ARGUMENT, "null count");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

int umc_chain_create(const umc_chain_desc* desc, umc_chain** out)
{
    return guarded([&] {
        if (!out) throw Error(UMC_ERR_INVALID_ARGUMENT, "null output handle");
        *out = nullptr;
        auto* c = new umc_chain;
        try {
            create_chain(desc, c);
        } catch (...) {
            destroy_chain(c);
            delete c;
            throw;
        }
        *out = c;
    });
}

int umc_chain_destroy(umc_chain* c)
{
    return guarded([&] {
        destroy_chain(c);
        delete c;
    });
}

int umc_chain_set_field(umc_chain* c, const void* host_field)
{
    return guarded([&] {
        if (!c || !host_field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        device_scope(c);
        if (!is_spin(c)) {
            gauge_set_field(c, host_field);
            return;
        }
        if (!c->staging.p) c->staging.alloc(c->field_bytes, "staging");
        if (!c->upload_done) cuda_check(cudaEventCreateWithFlags(&c->upload_done, cudaEventDisableTiming), "upload event");
        cuda_check(cudaMemcpyAsync(c->staging.p, host_field, c->field_bytes, cudaMemcpyHostToDevice, c->stream), "upload field");
        cuda_check(cudaEventRecord(c->upload_done, c->stream), "upload field");
        const uint32_t g = grid_for(c, c->n);
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        if (c->elem_bytes == 1)
            scatter_field<int8_t><<<g, kBlock, 0, c->stream>>>(c->staging.as<int8_t>(), c->field.as<int8_t>(), uint32_t(c->n), 1, placement(c), false);
        else
            scatter_field<float><<<g, kBlock, 0, c->stream>>>(c->staging.as<float>(), c->field.as<float>(), uint32_t(c->n), c->comps, placement(c),
                                                               c->model == UMC_MODEL_XY_ANGLE);
        launch_check("scatter field");
        // the caller's buffer is free once the copy has landed; the scatter
        // is stream-ordered before any later work on the chain
        cuda_check(cudaEventSynchronize(c->upload_done), "upload field");
    });
}

namespace {
// Checkpoint image: this header, then the field in the reference's data()
// layout.  Fixed-width fields, little-endian as the host writes them.
// Version 1 ended after wolff_axis (88 bytes); version 2 appends the Wolff
// statistics behind mean_cluster_size (flips done and the sum of their sizes).
struct CheckpointHeader
{
    char magic[8];  // "UMCCHK01"
    uint32_t version;
    int32_t model;
    int32_t components;
    uint32_t hits;
    uint64_t n;
    uint64_t field_bytes;
    uint64_t seed, sweeps, flips;
    double coupling, width;
    int32_t proposal, wolff_axis;
    uint64_t wolff_flips_done;  // version 2
    double wolff_size_sum;      // version 2
};
constexpr size_t kCheckpointHeaderV1 = 88;
static_assert(offsetof(CheckpointHeader, wolff_flips_done) == kCheckpointHeaderV1, "checkpoint v1 layout");
static_assert(sizeof(CheckpointHeader) == 104, "checkpoint header layout");
constexpr uint32_t kCheckpointVersion = 2;
constexpr char kCheckpointMagic[8] = {'U', 'M', 'C', 'C', 'H', 'K', '0', '1'};

uint64_t host_field_bytes(const umc_chain* c) { return c->n * c->comps * c->elem_bytes; }
}  // namespace

int umc_chain_checkpoint_bytes(const umc_chain* c, uint64_t* bytes)
{
    return guarded([&] {
        if (!c || !bytes) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        *bytes = sizeof(CheckpointHeader) + host_field_bytes(c);
    });
}

int umc_chain_checkpoint(umc_chain* c, void* buffer, uint64_t capacity)
{
    return guarded([&] {
        if (!c || !buffer) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        const uint64_t fb = host_field_bytes(c);
        if (capacity < sizeof(CheckpointHeader) + fb)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint buffer too small (see umc_chain_checkpoint_bytes)");
        CheckpointHeader h{};
        std::memcpy(h.magic, kCheckpointMagic, 8);
        h.version = kCheckpointVersion;
        h.model = c->model;
        h.components = c->N;
        h.hits = c->desc.hits;
        h.n = c->n;
        h.field_bytes = fb;
        h.seed = c->desc.seed;
        h.sweeps = c->sweeps;
        h.flips = c->flips;
        h.coupling = c->desc.coupling;
        h.width = c->desc.width;
        h.proposal = c->desc.proposal;
        h.wolff_axis = c->desc.wolff_axis;
        h.wolff_flips_done = c->wolff_flips_done;
        h.wolff_size_sum = c->wolff_size_sum;
        uint8_t* out = static_cast<uint8_t*>(buffer);
        const int st = umc_chain_get_field(c, out + sizeof h);
        if (st != UMC_OK) throw Error(st, umc_last_error());
        std::memcpy(out, &h, sizeof h);
    });
}

int umc_chain_restore(umc_chain* c, const void* buffer, uint64_t bytes)
{
    return guarded([&] {
        if (!c || !buffer) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (bytes < kCheckpointHeaderV1) throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint too short");
        CheckpointHeader h{};
        std::memcpy(&h, buffer, kCheckpointHeaderV1);
        if (std::memcmp(h.magic, kCheckpointMagic, 8) != 0 || (h.version != 1 && h.version != 2))
            throw Error(UMC_ERR_INVALID_ARGUMENT, "not a chain checkpoint (magic or version)");
        // a version-1 image has no Wolff statistics: mean_cluster_size restarts from zero
        const size_t hb = h.version == 1 ? kCheckpointHeaderV1 : sizeof h;
        if (bytes < hb) throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint too short");
        std::memcpy(&h, buffer, hb);
        if (h.model != c->model || h.components != c->N || h.n != c->n)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint is of another model, component count or lattice size");
        if (h.field_bytes != host_field_bytes(c) || bytes < hb + h.field_bytes)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint field size does not match the chain");
        if (h.coupling != c->desc.coupling)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "checkpoint coupling differs from the chain's");
        validate_proposal(c, h.proposal, h.width, h.hits);
        validate_axis(c, h.wolff_axis);
        const int st = umc_chain_set_field(c, static_cast<const uint8_t*>(buffer) + hb);
        if (st != UMC_OK) throw Error(st, umc_last_error());
        c->wolff_flips_done = h.wolff_flips_done;
        c->wolff_size_sum = h.wolff_size_sum;
        c->desc.proposal = h.proposal;
        c->desc.width = h.width;
        c->desc.hits = h.hits;
        c->desc.wolff_axis = h.wolff_axis;
        c->desc.seed = h.seed;
        c->sweeps = h.sweeps;
        c->flips = h.flips;
    });
}

int umc_chain_upload_async(umc_chain* c, const void* host_field)
{
    return guarded([&] {
        if (!c || !host_field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        if (!is_spin(c)) throw Error(UMC_ERR_UNSUPPORTED, "asynchronous upload is provided for spin models");
        device_scope(c);
        if (!c->up_stream) {
            cuda_check(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking), "upload stream");
            for (int q = 0; q < 2; ++q) {
                cuda_check(cudaEventCreateWithFlags(&c->up_copied[q], cudaEventDisableTiming), "upload event");
                cuda_check(cudaEventCreateWithFlags(&c->up_consumed[q], cudaEventDisableTiming), "upload event");
                c->up_staging[q].alloc(c->field_bytes, "upload staging");
                cuda_check(cudaEventRecord(c->up_consumed[q], c->stream), "upload event");
            }
        }
        const int q = c->up_next;
        c->up_next ^= 1;
        // the copy into buffer q waits until the layout pass that last read it has run
        cuda_check(cudaStreamWaitEvent(c->up_stream, c->up_consumed[q], 0), "upload order");
        cuda_check(cudaMemcpyAsync(c->up_staging[q].p, host_field, c->field_bytes, cudaMemcpyHostToDevice, c->up_stream),
                   "upload field");
        cuda_check(cudaEventRecord(c->up_copied[q], c->up_stream), "upload event");
        cuda_check(cudaStreamWaitEvent(c->stream, c->up_copied[q], 0), "upload order");
        const uint32_t g = grid_for(c, c->n);
        {
            LaunchScope ls(c, UMC_KERNEL_OTHER);
            if (c->elem_bytes == 1)
                scatter_field<int8_t><<<g, kBlock, 0, c->stream>>>(c->up_staging[q].as<int8_t>(), c->field.as<int8_t>(),
                                                                   uint32_t(c->n), 1, placement(c), false);
            else
                scatter_field<float><<<g, kBlock, 0, c->stream>>>(c->up_staging[q].as<float>(), c->field.as<float>(),
                                                                  uint32_t(c->n), c->comps, placement(c),
                                                                  c->model == UMC_MODEL_XY_ANGLE);
            launch_check("scatter field");
        }
        cuda_check(cudaEventRecord(c->up_consumed[q], c->stream), "upload event");
    });
}

int umc_chain_set_record_streaming(umc_chain* c, int enable)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        if (c->rec_pending) throw Error(UMC_ERR_STATE, "fetch pending records before switching record streaming");
        c->stream_records = enable != 0;
        c->streamed = 0;
    });
}

int umc_chain_get_field(umc_chain* c, void* host_field)
{
    return guarded([&] {
        if (!c || !host_field) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        device_scope(c);
        if (!is_spin(c)) {
            gauge_get_field(c, host_field);
            return;
        }
        if (!c->staging.p) c->staging.alloc(c->field_bytes, "staging");
        const uint32_t g = grid_for(c, c->n);
        {
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        if (c->elem_bytes == 1)
            gather_field<int8_t><<<g, kBlock, 0, c->stream>>>(c->field.as<int8_t>(), c->staging.as<int8_t>(), uint32_t(c->n), 1, placement(c));
        else
            gather_field<float><<<g, kBlock, 0, c->stream>>>(c->field.as<float>(), c->staging.as<float>(), uint32_t(c->n), c->comps, placement(c));
        }
        launch_check("gather field");
        cuda_check(cudaMemcpyAsync(host_field, c->staging.p, c->field_bytes, cudaMemcpyDeviceToHost, c->stream), "download field");
        cuda_check(cudaStreamSynchronize(c->stream), "download field");
    });
}

int umc_chain_randomize(umc_chain* c, uint64_t seed)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        if (!is_spin(c)) {
            gauge_randomize(c, seed);
            return;
        }
        const uint32_t g = grid_for(c, c->n);
        const uint32_t n = uint32_t(c->n);
        LaunchScope ls(c, UMC_KERNEL_OTHER);
        if (c->model == UMC_MODEL_ISING) randomize_spins<0><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c));
        else if (c->model == UMC_MODEL_XY_ANGLE) randomize_spins<-1><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c));
        else
            switch (c->N) {
            case 1: randomize_spins<1><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c)); break;
            case 2: randomize_spins<2><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c)); break;
            case 3: randomize_spins<3><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c)); break;
            case 4: randomize_spins<4><<<g, kBlock, 0, c->stream>>>(c->field.p, n, seed, placement(c)); break;
            }
        launch_check("randomize");
        cuda_check(cudaStreamSynchronize(c->stream), "randomize");
    });
}

int umc_chain_set_proposal(umc_chain* c, int32_t proposal, double width, uint32_t hits)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        validate_proposal(c, proposal, width, hits);
        c->desc.proposal = proposal;
        c->desc.width = width;
        c->desc.hits = hits;
    });
}

int umc_chain_set_wolff_axis(umc_chain* c, int32_t axis)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        validate_axis(c, axis);
        c->desc.wolff_axis = axis;
    });
}

int umc_chain_set_seed(umc_chain* c, uint64_t seed)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        c->desc.seed = seed;
    });
}

int umc_chain_counters(const umc_chain* c, uint64_t* sweeps, uint64_t* flips)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        if (sweeps) *sweeps = c->sweeps;
        if (flips) *flips = c->flips;
    });
}

int umc_chain_set_counters(umc_chain* c, uint64_t sweeps, uint64_t flips)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        c->sweeps = sweeps;
        c->flips = flips;
    });
}

void* umc_chain_stream(const umc_chain* c) { return c ? static_cast<void*>(c->stream) : nullptr; }

int umc_chain_sync(umc_chain* c)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        check_status(c);
    });
}

int umc_chain_observe(umc_chain* c, double* record)
{
    return guarded([&] {
        if (!c || !record) throw Error(UMC_ERR_INVALID_ARGUMENT, "null argument");
        device_scope(c);
        if (c->rec_pending) fetch(c, nullptr, nullptr, 0, nullptr);
        const uint64_t r = next_record(c);
        if (is_spin(c)) observe_into(c, record_ptr(c, r), nullptr);
        else gauge_observe(c, record_ptr(c, r));
        uint64_t got = 0;
        std::vector<double> buf(kObs);
        fetch(c, buf.data(), nullptr, 1, &got);
        std::copy(buf.begin(), buf.end(), record);
    });
}

int umc_metropolis_run(umc_chain* c, double beta, uint64_t n_sweeps, double* records)
{
    return guarded([&] {
        NvtxRange range("umc_metropolis_run");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        run_chunked(c, n_sweeps, records, nullptr, false, [&](uint64_t m) { enqueue_sweeps(c, beta, m); });
    });
}

int umc_wolff_run(umc_chain* c, double beta, uint64_t n_flips, uint64_t* sizes, double* records)
{
    return guarded([&] {
        NvtxRange range("umc_wolff_run");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        run_chunked(c, n_flips, records, sizes, true, [&](uint64_t m) { enqueue_flips(c, beta, m, records != nullptr); });
    });
}

int umc_hybrid_run(umc_chain* c, double beta, uint64_t n_steps, uint64_t* sizes, double* records)
{
    return guarded([&] {
        NvtxRange range("umc_hybrid_run");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        run_chunked(c, n_steps, records, sizes, true, [&](uint64_t m) { enqueue_hybrid(c, beta, m); });
    });
}

int umc_metropolis_enqueue(umc_chain* c, double beta, uint64_t n_sweeps)
{
    return guarded([&] {
        NvtxRange range("umc_metropolis_enqueue");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        enqueue_sweeps(c, beta, n_sweeps);
    });
}

int umc_wolff_enqueue(umc_chain* c, double beta, uint64_t n_flips)
{
    return guarded([&] {
        NvtxRange range("umc_wolff_enqueue");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        enqueue_flips(c, beta, n_flips, true);
    });
}

int umc_hybrid_enqueue(umc_chain* c, double beta, uint64_t n_steps)
{
    return guarded([&] {
        NvtxRange range("umc_hybrid_enqueue");
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        enqueue_hybrid(c, beta, n_steps);
    });
}

int umc_chain_fetch(umc_chain* c, double* records, uint64_t* sizes, uint64_t capacity, uint64_t* n_records)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        fetch(c, records, sizes, capacity, n_records);
    });
}

int umc_chain_set_fused(umc_chain* c, int enable)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        c->fused = enable != 0;
    });
}

int umc_chain_set_timing(umc_chain* c, int enable)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        c->timing = enable != 0;
    });
}

int umc_chain_kernel_stats(umc_chain* c, uint64_t* launches, double* device_ms, int reset)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        device_scope(c);
        collect_kernel_times(c);
        for (int k = 0; k < UMC_KERNEL_KINDS; ++k) {
            if (launches) launches[k] = c->launches[k];
            if (device_ms) device_ms[k] = c->device_ms[k];
            if (reset) {
                c->launches[k] = 0;
                c->device_ms[k] = 0.0;
            }
        }
    });
}

int umc_wolff_stats(const umc_chain* c, uint64_t* flips, double* size_sum)
{
    return guarded([&] {
        if (!c) throw Error(UMC_ERR_INVALID_ARGUMENT, "null chain");
        if (flips) *flips = c->wolff_flips_done;
        if (size_sum) *size_sum = c->wolff_size_sum;
    });
}

}  // extern "C"
