// umc_noalloc.cu -- a single-cluster Wolff flip that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code embedded in a host
// framework whose pool allocator owns all device memory and forbids side
// allocations, or code on a latency-critical path where cudaMalloc's implicit
// device synchronisation is not acceptable.  They keep their field and graph in
// memory they already own and pass device pointers in; the union-find labels
// and the status/size words this flip needs live in one file-scope device
// array instead of chain-owned buffers.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxSites sites per call (larger graphs are rejected);
//  * the array (2 label arrays + a control block, about 8 MiB) is a static
//    __device__ object, so every GPU that loads this library holds it until
//    the process exits;
//  * all calls on a device share it and it keeps the last call's contents --
//    each call re-initialises the parts that must start from a known value, and
//    calls that overlap on the GPU (two streams, or two host threads) race;
//  * every call looks up the array's device address with cudaGetSymbolAddress
//    on the current device (cheap once the module is loaded, and never stale
//    after a device reset re-creates the context);
//  * the call is synchronous: it checks the graph and reads the cluster size
//    back with stream synchronisations, so it must never be made while its
//    stream is being captured into a CUDA graph.
//
// Before the flip a check kernel verifies the caller's CSR over n sites:
// offset[0] = 0, non-decreasing offsets, every neighbour id below n and not
// the site itself, and every bond stored from both ends the same number of
// times.  A graph that fails is refused with UMC_ERR_INVALID_ARGUMENT and the
// flip kernels are not launched, so a bad id never reaches the labels.  The
// check reads offset[0..n] and bonds[offset[0]..offset[n]); those arrays must
// have that many entries.
//
// The kernels are the chain's own Wolff kernels (bond activation + union-find,
// then the cluster flip), so a call reproduces umc_wolff_run on the same field,
// table order, seed and flip counter.

#include <cuda_runtime.h>

#include <cmath>

#include "umc_chain.hpp"
#include "umc_spin_kernels.cuh"

namespace umc {
namespace {

constexpr uint32_t kNoAllocMaxSites = 1u << 20;  // 1,048,576 sites: 8 MiB of labels

struct NoAllocScratch
{
    uint32_t labels[2][kNoAllocMaxSites];
    DevCtl ctl;
    unsigned long long size;
    uint32_t csr_fault;  // bits set by noalloc_check_csr
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the scratch array on the current device.  Resolved on
// every call: a cached address would outlive a cudaDeviceReset that reloads
// the module.
NoAllocScratch* scratch_on_current_device()
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        throw Error(UMC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    return static_cast<NoAllocScratch*>(p);
}

constexpr uint32_t kCsrOffsets = 1u;    // offset[0] != 0 or a decreasing offset
constexpr uint32_t kCsrNeighbour = 2u;  // a neighbour id >= n, or a self-loop
constexpr uint32_t kCsrAsymmetric = 4u; // bond i-j stored a different number of times at i and at j

// Checks the caller's CSR before any kernel indexes labels with it.  One
// thread per site; a bond's multiplicity is counted at its first slot in row i
// against row j.
__global__ void noalloc_check_csr(const uint32_t* off, const uint32_t* adj, uint32_t n, uint32_t* fault)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t bad = 0;
        const uint32_t a0 = off[i], a1 = off[i + 1];
        if (i == 0 && a0 != 0) bad |= kCsrOffsets;
        if (a0 > a1) {
            atomicOr(fault, bad | kCsrOffsets);
            continue;
        }
        for (uint32_t q = a0; q < a1; ++q) {
            const uint32_t j = adj[q];
            if (j >= n || j == i) {
                bad |= kCsrNeighbour;
                continue;
            }
            bool first = true;
            uint32_t here = 1;
            for (uint32_t p = a0; p < a1; ++p) {
                if (p == q || adj[p] != j) continue;
                if (p < q) {
                    first = false;
                    break;
                }
                ++here;
            }
            if (!first) continue;
            const uint32_t b0 = off[j], b1 = off[j + 1];
            if (b0 > b1) continue;  // reported by site j's own thread
            uint32_t there = 0;
            for (uint32_t p = b0; p < b1; ++p) there += adj[p] == i ? 1u : 0u;
            if (there != here) bad |= kCsrAsymmetric;
        }
        if (bad) atomicOr(fault, bad);
    }
}

__global__ void noalloc_reset(NoAllocScratch* s, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s->labels[0][i] = i;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s->ctl.status = 0u;
        s->size = 0ull;
    }
}

template <int MODEL>
void launch_flip(const WolffArgs& a, uint32_t grid, cudaStream_t st)
{
    wolff_union<MODEL><<<grid, kBlock, 0, st>>>(a);
    wolff_flip<MODEL><<<grid, kBlock, 0, st>>>(a);
}

}  // namespace
}  // namespace umc

using namespace umc;

extern "C" int umc_wolff_flip_noalloc(int32_t model, int32_t components, void* field, uint64_t n_sites,
                                      const uint32_t* offset, const uint32_t* bonds, const uint32_t* slot_edge,
                                      double coupling, double beta, uint64_t seed, uint64_t flip,
                                      uint64_t* cluster_size, void* stream)
{
    try {
        set_last_error("");
        if (!field || !offset || !bonds || !slot_edge) throw Error(UMC_ERR_INVALID_ARGUMENT, "null device pointer");
        if (n_sites == 0) throw Error(UMC_ERR_INVALID_ARGUMENT, "empty graph");
        if (n_sites > kNoAllocMaxSites)
            throw Error(UMC_ERR_UNSUPPORTED, "umc_wolff_flip_noalloc: more than 1,048,576 sites (the scratch array's size)");
        if (!std::isfinite(beta) || !std::isfinite(coupling)) throw Error(UMC_ERR_INVALID_ARGUMENT, "beta and J must be finite");
        int mk;
        if (model == UMC_MODEL_ISING) {
            if (coupling != std::floor(coupling) || std::fabs(coupling) > 1e6)
                throw Error(UMC_ERR_INVALID_ARGUMENT, "Ising coupling J must be an integer");
            mk = 0;
        } else if (model == UMC_MODEL_VECTOR) {
            if (components < 1 || components > 4) throw Error(UMC_ERR_UNSUPPORTED, "VectorSpin<N>: N must be 1..4");
            mk = components;
        } else {
            throw Error(UMC_ERR_UNSUPPORTED, "Wolff is defined for Ising and VectorSpin");
        }
        int device = 0;
        cuda_check(cudaGetDevice(&device), "cudaGetDevice");
        NoAllocScratch* s = scratch_on_current_device();
        int sms = 0;
        cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
        const uint64_t blocks = (n_sites + kBlock - 1) / kBlock;
        const uint32_t grid = uint32_t(blocks < uint64_t(sms) * 8 ? blocks : uint64_t(sms) * 8);
        cudaStream_t st = static_cast<cudaStream_t>(stream);

        // the graph is checked before any kernel indexes the labels with it
        uint32_t fault = 0;
        cuda_check(cudaMemsetAsync(&s->csr_fault, 0, sizeof fault, st), "clear CSR check");
        noalloc_check_csr<<<grid, kBlock, 0, st>>>(offset, bonds, uint32_t(n_sites), &s->csr_fault);
        cuda_check(cudaGetLastError(), "CSR check");
        cuda_check(cudaMemcpyAsync(&fault, &s->csr_fault, sizeof fault, cudaMemcpyDeviceToHost, st), "read CSR check");
        cuda_check(cudaStreamSynchronize(st), "CSR check");
        if (fault & kCsrOffsets)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "umc_wolff_flip_noalloc: offsets must start at 0 and never decrease");
        if (fault & kCsrNeighbour)
            throw Error(UMC_ERR_INVALID_ARGUMENT, "umc_wolff_flip_noalloc: a neighbour id is >= n_sites or a self-loop");
        if (fault & kCsrAsymmetric)
            throw Error(UMC_ERR_INVALID_ARGUMENT,
                        "umc_wolff_flip_noalloc: the CSR is not symmetric (a bond is not stored equally at both ends)");

        WolffArgs a{};
        a.field = field;
        a.n = uint32_t(n_sites);
        a.off = offset;
        a.adj = bonds;
        a.slot = slot_edge;
        a.lab = s->labels[0];
        a.lab_next = s->labels[1];
        a.seed = seed;
        a.flip = flip;
        a.J = float(coupling);
        a.beta = float(beta);
        a.J64 = coupling;
        a.beta64 = beta;
        a.err = vector_wolff_err(beta, coupling, mk == 0 ? 1 : mk);
        if (mk == 0) ising_wolff_thresholds(int32_t(coupling), beta, a.cw);
        a.ctl = &s->ctl;
        a.size_slot = &s->size;

        noalloc_reset<<<grid, kBlock, 0, st>>>(s, a.n);
        switch (mk) {
        case 0: launch_flip<0>(a, grid, st); break;
        case 1: launch_flip<1>(a, grid, st); break;
        case 2: launch_flip<2>(a, grid, st); break;
        case 3: launch_flip<3>(a, grid, st); break;
        default: launch_flip<4>(a, grid, st); break;
        }
        cuda_check(cudaGetLastError(), "Wolff flip (no-alloc)");
        unsigned long long size = 0;
        unsigned int status = 0;
        cuda_check(cudaMemcpyAsync(&size, &s->size, sizeof size, cudaMemcpyDeviceToHost, st), "read cluster size");
        cuda_check(cudaMemcpyAsync(&status, &s->ctl.status, sizeof status, cudaMemcpyDeviceToHost, st), "read status");
        cuda_check(cudaStreamSynchronize(st), "Wolff flip (no-alloc)");
        if (status) throw Error(UMC_ERR_DEVICE_TIMEOUT, "device-side bound exhausted: union-find");
        if (cluster_size) *cluster_size = size;
        return UMC_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return UMC_ERR_INVALID_ARGUMENT;
    }
}
