/*
 * umc_b200.h -- C ABI of the B200 local-update engine.
 *
 * This is the boundary the C++23 facade (include/umc/) and any other host
 * language bind to: plain pointers and sizes, integer status codes, opaque
 * handles, no C++ or torch types.  It replaces the reference library's
 * header-only hot path (universal_monte_carlo):
 *
 *   tables      PairGraph / square_lattice     lattice/pair_graph.hpp, lattice/square.hpp
 *               CellComplex / hypercubic_plaquettes  lattice/cell_complex.hpp, lattice/hypercubic.hpp
 *   models      Ising, VectorSpin<N>, U1Gauge, SUGauge<N>  example/ headers
 *               PairModel / CellModel + terms   model/ and term/ headers
 *   proposals   Flip, FixedAxis, UniformSphereN, LocalRotation, U1Shift, SUShift  dof/ headers
 *   drivers     Metropolis<M,Q,R>, Wolff<M,A,R>  driver.hpp
 *   RNG         Pcg32                           rng.hpp
 *
 * Errors: every function returns umc_status (0 = OK).  The reference's table
 * builders throw std::invalid_argument / std::out_of_range / std::overflow_error;
 * here those become UMC_ERR_INVALID_ARGUMENT / _OUT_OF_RANGE / _OVERFLOW with
 * the same messages available from umc_last_error() (thread-local).
 *
 * Random numbers: every update opens its own reference-semantics Pcg32 keyed by
 * (seed, counter, tag, id) -- see include/umc/keyed_pcg.cuh -- so a chain
 * is a pure function of (field, seed, counters) and can be replayed by the
 * reference driver on the CPU.
 */
#ifndef UMC_B200_H
#define UMC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UMC_ABI_VERSION 2

typedef enum umc_status {
    UMC_OK = 0,
    UMC_ERR_INVALID_ARGUMENT = 1, /* std::invalid_argument in the reference builders */
    UMC_ERR_OUT_OF_RANGE = 2,     /* std::out_of_range                               */
    UMC_ERR_OVERFLOW = 3,         /* std::overflow_error                             */
    UMC_ERR_UNSUPPORTED = 4,      /* combination this engine does not provide        */
    UMC_ERR_CUDA = 5,             /* CUDA runtime error (incl. no device)            */
    UMC_ERR_DEVICE_TIMEOUT = 6,   /* a bounded device-side wait ran out              */
    UMC_ERR_OUT_OF_MEMORY = 7,
    UMC_ERR_STATE = 8             /* call out of order (e.g. records overflowed)     */
} umc_status;

/* Message of the last failing call on this thread ("" if none). */
const char* umc_last_error(void);
int umc_abi_version(void);
/* Number of visible CUDA devices (0 on a host without GPUs). */
int umc_device_count(int* count);

/* ===================================================================== tables */

typedef struct umc_graph umc_graph;

/* PairGraph(n, edges, symmetric) -- lattice/pair_graph.hpp:49-83.  CSR rows in
 * edge-list order, duplicates kept, self-loops rejected (INVALID_ARGUMENT),
 * endpoints >= n rejected (OUT_OF_RANGE), n or 2E beyond uint32 (OVERFLOW). */
int umc_graph_create(uint64_t n_sites, const uint32_t* edge_i, const uint32_t* edge_j,
                     uint64_t n_edges, int symmetric, umc_graph** out);
/* PairGraph<P>(n, edges, symmetric) with a per-bond payload -- lattice/
 * pair_graph.hpp:13-83 (Bond<P>::c, Edge::c): edge e's payload is the
 * payload_bytes record at payload + e * payload_bytes (a trivially copyable P,
 * 1 to UMC_MAX_PAYLOAD_BYTES bytes), copied into both directed slots as the
 * reference copies Edge::c.  Same checks and errors as umc_graph_create.  The
 * built-in models take NoPayload graphs only (as the reference's Ising and
 * VectorSpin take PairGraph<>); weighted models are user models over the
 * device tables (umc/device.cuh BondTables<P>). */
#define UMC_MAX_PAYLOAD_BYTES 256
int umc_graph_create_payload(uint64_t n_sites, const uint32_t* edge_i, const uint32_t* edge_j,
                             uint64_t n_edges, int symmetric, const void* payload, uint32_t payload_bytes,
                             umc_graph** out);
/* Bytes per payload record; 0 for a NoPayload graph. */
uint32_t umc_graph_payload_bytes(const umc_graph* g);
/* Bond<P>::c of every CSR slot (lattice/pair_graph.hpp:98-102), in the slot
 * order of umc_graph_csr: slots x payload_bytes bytes. */
int umc_graph_payloads(const umc_graph* g, void* out);
/* The input edge of every CSR slot (slots entries): the reference fills rows
 * in edge order, so this maps bonds(i)[a] back to its Edge. */
int umc_graph_slot_edges(const umc_graph* g, uint32_t* out);
/* square_lattice(Lx, Ly) -- lattice/square.hpp:15-38. */
int umc_graph_square(uint64_t Lx, uint64_t Ly, umc_graph** out);
/* Periodic Lx*Ly*Lz cubic lattice with square_lattice's conventions (site
 * (z*Ly+y)*Lx+x; per site a +x, +y, +z edge when that extent exceeds 1).  The
 * reference has no 3D builder; users build the same edge list by hand. */
int umc_graph_cubic(uint64_t Lx, uint64_t Ly, uint64_t Lz, umc_graph** out);
void umc_graph_destroy(umc_graph* g);
/* PairGraph::sites / degree / bonds -- lattice/pair_graph.hpp:86-102. */
uint64_t umc_graph_sites(const umc_graph* g);
uint64_t umc_graph_slots(const umc_graph* g);
int umc_graph_csr(const umc_graph* g, uint32_t* offset /* n+1 */, uint32_t* bonds /* slots */);
/* Colouring used by the colour passes (no reference counterpart: the reference
 * sweeps sites in index order, driver.hpp:34).  colour[i] in [0, n_colours);
 * position[i] = index of site i in colour-major order, which is the order in
 * which the reference driver reproduces the GPU's updates and the id that keys
 * site i's random stream.  Any pointer may be NULL. */
int umc_graph_colouring(const umc_graph* g, uint32_t* n_colours, uint32_t* colour,
                        uint32_t* position);

typedef struct umc_cells umc_cells;

/* CellComplex<A>(sites, cells) -- lattice/cell_complex.hpp:36-63 (cells is
 * n_cells*arity site ids, arity in [1, 255]). */
int umc_cells_create(uint64_t n_sites, uint32_t arity, const uint32_t* cells, uint64_t n_cells,
                     umc_cells** out);
/* hypercubic_plaquettes(L) -- lattice/hypercubic.hpp:15-64. */
int umc_cells_hypercubic(uint64_t L, umc_cells** out);
/* Periodic 2D plaquettes with the same orientation rule (links mu*L^2+y*L+x,
 * plaquette [U_0(c), U_1(c+x), U_0(c+y), U_1(c)]); no reference builder. */
int umc_cells_square_plaquettes(uint64_t L, umc_cells** out);
void umc_cells_destroy(umc_cells* c);
/* CellComplex::sites / cells / cell(c) / incident(i) -- lattice/cell_complex.hpp:65-80. */
uint64_t umc_cells_sites(const umc_cells* c);
uint64_t umc_cells_count(const umc_cells* c);
uint32_t umc_cells_arity(const umc_cells* c);
int umc_cells_table(const umc_cells* c, uint32_t* cells /* n_cells*arity */);
int umc_cells_incidence(const umc_cells* c, uint64_t* offset /* sites+1 */, uint32_t* inc_cell,
                        uint8_t* inc_which);
/* Colouring of the links (no two links of one colour share a cell). */
int umc_cells_colouring(const umc_cells* c, uint32_t* n_colours, uint32_t* colour,
                        uint32_t* position);

/* ===================================================================== chains */

/* Models (example/ and model/ headers). */
#define UMC_MODEL_ISING 1    /* Ising, example/ising.hpp:14-76 (int8 spins, integer J)     */
#define UMC_MODEL_VECTOR 2   /* VectorSpin<N>, example/vector_spin.hpp:14-83 (N = 1..4)     */
#define UMC_MODEL_XY_ANGLE 3 /* PairModel<U1Dof, -J cos(ti-tj)>, model/pair.hpp:17-83     */
#define UMC_MODEL_U1 4       /* U1Gauge / CellModel<U1Dof,U1PlaquetteTerm>, example/u1_gauge.hpp */
#define UMC_MODEL_SU 5       /* SUGauge<N> / CellModel<SUDof,SUPlaquetteTerm>, example/sun_gauge.hpp */

/* Metropolis proposals (dof/ headers). */
#define UMC_PROPOSAL_FLIP 1     /* Flip, dof/ising.hpp:27-38                 */
#define UMC_PROPOSAL_SPHERE 2   /* UniformSphereN<N>, dof/vector.hpp:35-61     */
#define UMC_PROPOSAL_ROTATION 3 /* LocalRotation<N>{delta}, dof/vector.hpp:70-122 */
#define UMC_PROPOSAL_U1SHIFT 4  /* U1Shift{width}, dof/u1.hpp:35-50          */
#define UMC_PROPOSAL_SUSHIFT 5  /* SUShift<N>{width}, dof/sun.hpp:163-204     */

/* Wolff reflection axes. */
#define UMC_AXIS_NONE 0
#define UMC_AXIS_FIXED 1  /* FixedAxis, dof/ising.hpp:41-49      */
#define UMC_AXIS_SPHERE 2 /* UniformSphereN<N> as the axis        */

typedef struct umc_chain_desc {
    int32_t model;          /* UMC_MODEL_*                                        */
    int32_t components;     /* N of VectorSpin<N> or SU(N); 1 for the others      */
    const umc_graph* graph; /* spin models                                        */
    const umc_cells* cells; /* gauge models (arity 4)                              */
    double coupling;        /* J (Ising: an integer value), or the gauge beta     */
    int32_t proposal;       /* UMC_PROPOSAL_*                                     */
    double width;           /* LocalRotation delta, U1Shift / SUShift width       */
    uint32_t hits;          /* Metropolis hits per site and sweep (>= 1)          */
    int32_t wolff_axis;     /* UMC_AXIS_*                                         */
    uint64_t seed;          /* RNG key seed                                       */
    int32_t device;         /* CUDA device ordinal                                */
    void* stream;           /* cudaStream_t to run on; NULL: the chain owns one    */
    uint64_t max_records;   /* per-sweep observable slots on the device (0: 4096) */
} umc_chain_desc;

typedef struct umc_chain umc_chain;

/* One observable record per sweep (Metropolis) or flip (Wolff), FP64:
 *   spin models:  [0] E = 0.5 * sum_i energy_at(i)  [1..N] magnetisation sum
 *                 [7] accepted proposals in the sweep (Wolff: cluster size)
 *   gauge models: [0] action S = beta * sum_p (1 - P_p)  [1] mean plaquette
 *                 [2] topological charge (2D U(1))      [7] accepted proposals */
#define UMC_OBS_STRIDE 8

/* Creates the device chain: the model's field (cold start exactly as the
 * reference constructors: Ising all +1 example/ising.hpp:24, VectorSpin along
 * the last axis example/vector_spin.hpp:27-28, gauge links identity
 * example/sun_gauge.hpp:26 / zero angles), its tables and workspace. */
int umc_chain_create(const umc_chain_desc* desc, umc_chain** out);
int umc_chain_destroy(umc_chain* c);
/* Writes the whole field from host memory in the reference's data() layout:
 * Ising int8[n]; VectorSpin float[n*N]; XY / U(1) float[n] angles; SU(N)
 * float[n*N*N*2] (row-major, interleaved re/im).  Equivalent to update(i, .)
 * for every site. */
int umc_chain_set_field(umc_chain* c, const void* host_field);
/* Reads the field back in the same layout (the reference's data()). */
int umc_chain_get_field(umc_chain* c, void* host_field);
/* Asynchronous umc_chain_set_field (spin models): the copy runs on a second
 * stream into one of two staging buffers and the layout pass follows on the
 * chain's stream, so the upload of the next configuration overlaps the work
 * queued before it.  Returns at once; host_field (pinned memory, for the copy
 * to be asynchronous) must stay unchanged until the next synchronising call
 * (umc_chain_sync, _fetch, _get_field, a *_run).  The reference sets a field
 * only through its model's update(i, .) (model.hpp:70-86). */
int umc_chain_upload_async(umc_chain* c, const void* host_field);
/* Chain checkpoints: a self-describing byte image of a chain -- a 104-byte
 * header (magic "UMCCHK01", version 2, model, components, lattice size, seed,
 * sweep and flip counters, coupling, proposal, width, hits, Wolff axis, and
 * the Wolff flips done with the sum of their cluster sizes) and then the field
 * in the reference's data() layout.  Restoring it into a chain of the same
 * model, components, lattice size and coupling (for instance in a new process)
 * sets the field, the key seed, the counters, the proposal and the Wolff
 * statistics, so the chain continues exactly as the checkpointed one would
 * have, mean_cluster_size included.  Version-1 images (an 88-byte header
 * without the Wolff statistics) are still accepted; their restore resets
 * mean_cluster_size to start from the restored flip.  The
 * reference has no checkpoint format: its user copies data() by hand
 * (model.hpp:70-86); this is the engine's own. */
int umc_chain_checkpoint_bytes(const umc_chain* c, uint64_t* bytes);
int umc_chain_checkpoint(umc_chain* c, void* buffer, uint64_t capacity);
int umc_chain_restore(umc_chain* c, const void* buffer, uint64_t bytes);
/* With streaming on, every record (and cluster size) is copied to pinned host
 * memory as soon as its step has run, on the chain's stream; umc_chain_fetch
 * then only waits.  This is how the reference's sample(n, observe) sees each
 * sweep's observables as it ends (driver.hpp:54-61, :182-190). */
int umc_chain_set_record_streaming(umc_chain* c, int enable);
/* Random start from keyed draws (tag 3, id = site): uniform on the sphere,
 * uniform angles in [0, 2pi), Haar-random SU(N), random Ising signs. */
int umc_chain_randomize(umc_chain* c, uint64_t seed);
/* A driver brings its own proposal and RNG to a model (Metropolis(M&, Q, R,
 * beta), driver.hpp:22-25; Wolff(M&, A, R, beta), driver.hpp:96-101): these
 * set the chain's proposal (with its width and hits per site), its Wolff axis
 * and the seed that keys every random stream. */
int umc_chain_set_proposal(umc_chain* c, int32_t proposal, double width, uint32_t hits);
int umc_chain_set_wolff_axis(umc_chain* c, int32_t axis);
int umc_chain_set_seed(umc_chain* c, uint64_t seed);
/* Sweep and flip counters (they key the random streams). */
int umc_chain_counters(const umc_chain* c, uint64_t* sweeps, uint64_t* flips);
int umc_chain_set_counters(umc_chain* c, uint64_t sweeps, uint64_t flips);
/* The stream the chain's kernels run on (cudaStream_t). */
void* umc_chain_stream(const umc_chain* c);
/* Waits for the chain's queued work and reports any device-side error. */
int umc_chain_sync(umc_chain* c);
/* Observables of the current field (one record, see UMC_OBS_STRIDE). */
int umc_chain_observe(umc_chain* c, double* record);

/* Metropolis::sweep x n -- driver.hpp:29-61.  beta is the driver's beta: the
 * exponent is -beta * dE (for gauge models put the physical beta in the model
 * coupling and pass 1.0 here).  records: n x UMC_OBS_STRIDE doubles or NULL.
 * Blocks until done. */
int umc_metropolis_run(umc_chain* c, double beta, uint64_t n_sweeps, double* records);
/* Wolff::flip x n -- driver.hpp:104-190 (single-cluster, reflection axis from
 * desc.wolff_axis).  sizes: n cluster sizes or NULL; records: n x stride or NULL. */
int umc_wolff_run(umc_chain* c, double beta, uint64_t n_flips, uint64_t* sizes, double* records);
/* n x (one Wolff flip, then one Metropolis sweep); one record per step, taken
 * after the sweep. */
int umc_hybrid_run(umc_chain* c, double beta, uint64_t n_steps, uint64_t* sizes, double* records);
/* Asynchronous forms: enqueue on the chain's stream and return.  Records stay
 * in the device ring (capacity desc.max_records) until umc_chain_fetch. */
int umc_metropolis_enqueue(umc_chain* c, double beta, uint64_t n_sweeps);
int umc_wolff_enqueue(umc_chain* c, double beta, uint64_t n_flips);
int umc_hybrid_enqueue(umc_chain* c, double beta, uint64_t n_steps);
/* Copies (and releases) the records queued since the last fetch. *n_records
 * receives their count; records / sizes may be NULL.  Synchronises. */
int umc_chain_fetch(umc_chain* c, double* records, uint64_t* sizes, uint64_t capacity,
                    uint64_t* n_records);
/* Execution strategy on regular lattices (no reference counterpart): with
 * fusion on (the default) a Metropolis sweep, a Wolff flip or a hybrid step of
 * a VectorSpin chain runs as one cooperative kernel whose phases are separated
 * by a bounded grid barrier; off, each phase is its own kernel.  Both give the
 * same field; the FP64 observable sums may differ in the last bits. */
int umc_chain_set_fused(umc_chain* c, int enable);
/* Kernel accounting (no reference counterpart).  Every kernel the chain
 * launches is counted by kind; with timing enabled each launch is also
 * bracketed by CUDA events on the chain's stream.  umc_chain_kernel_stats
 * synchronises and reports, per kind, launches and device milliseconds
 * (timed launches only); reset != 0 clears both. */
#define UMC_KERNEL_METROPOLIS 0 /* spin-model colour pass           */
#define UMC_KERNEL_WOLFF_UNION 1 /* bond activation + union-find     */
#define UMC_KERNEL_WOLFF_FLIP 2  /* cluster flip                     */
#define UMC_KERNEL_OBSERVE 3     /* full observable recomputation    */
#define UMC_KERNEL_GAUGE 4       /* gauge-link colour pass           */
#define UMC_KERNEL_BATCH 5       /* batched-chain kernels            */
#define UMC_KERNEL_LEARNED 6     /* learned-proposal kernels         */
#define UMC_KERNEL_OTHER 7       /* layout, start, reduction helpers */
#define UMC_KERNEL_WOLFF_MERGE 8 /* union of tile-crossing bonds     */
#define UMC_KERNEL_FUSED 9       /* fused step (Wolff + sweep)       */
#define UMC_KERNEL_KINDS 10
int umc_chain_set_timing(umc_chain* c, int enable);
int umc_chain_kernel_stats(umc_chain* c, uint64_t* launches, double* device_ms, int reset);
/* Wolff::mean_cluster_size bookkeeping -- driver.hpp:193-196. */
int umc_wolff_stats(const umc_chain* c, uint64_t* flips, double* size_sum);

/* ============================================================ batched chains */

/* Many independent XY chains (the angle model of UMC_MODEL_XY_ANGLE with
 * U1Shift) on periodic L x L lattices, organised in replica-exchange ladders.
 * No reference counterpart: the reference runs one chain per driver object
 * (driver.hpp:17-68).  Chain c = ladder * replicas + k starts at temperature
 * slot k of its ladder; every segment runs sweeps_per_exchange Metropolis
 * sweeps of every chain at the beta of the slot it holds, then one exchange
 * round per ladder: slots (k, k+1), k of the round's parity, swap their chains
 * iff (beta_k - beta_{k+1})(E_k - E_{k+1}) >= 0 or log(u) < that product. */
typedef struct umc_batch_desc {
    uint32_t n_ladders;
    uint32_t replicas;            /* temperature slots per ladder (<= 64)        */
    const uint32_t* L;            /* side per ladder: even, in [2, 4096]         */
    const double* betas;          /* n_ladders * replicas inverse temperatures   */
    double coupling;              /* J                                           */
    double width;                 /* U1Shift width                               */
    uint32_t sweeps_per_exchange; /* 0: 10                                       */
    uint64_t seed;
    int32_t device;
    void* stream;                 /* NULL: the batch owns one                    */
    uint64_t max_records;         /* segments kept on the device (0: 1024)       */
    uint32_t first_ladder;        /* global index of ladder 0 (sharding, below)   */
} umc_batch_desc;

/* Sharding a batch over ranks (one process per GPU): the ladders are
 * independent units, so rank r of W creates a batch of its contiguous range of
 * ladders [l0, l1) with first_ladder = l0 and the same seed; ladder l and the
 * chains in it draw from the keys of global ladder l0 + l (chain seeds from
 * global chain index, ladder seeds from global ladder index), so the union of
 * the ranks' batches runs exactly the chains and exchanges of one unsharded
 * batch.  No data-path collective is needed; records are gathered at the end. */

typedef struct umc_batch umc_batch;

int umc_batch_create(const umc_batch_desc* desc, umc_batch** out);
int umc_batch_destroy(umc_batch* b);
/* Uniform angles 2 pi u on every chain (keys derived from seed and chain). */
int umc_batch_randomize(umc_batch* b, uint64_t seed);
/* One chain's angles in natural site order y*L + x. */
int umc_batch_set_field(umc_batch* b, uint32_t chain, const float* theta);
int umc_batch_get_field(umc_batch* b, uint32_t chain, float* theta);
/* Queue n segments (a captured CUDA graph per segment). */
int umc_batch_enqueue(umc_batch* b, uint64_t n_segments);
/* Copy the records of the segments queued since the last fetch:
 * n_records x (n_ladders * replicas) x UMC_OBS_STRIDE doubles, by temperature
 * slot: [E, Mx, My, chain, beta, swap of (k, k+1) accepted, accepted
 * updates, 0] taken at the end of the segment, before the exchange. */
int umc_batch_fetch(umc_batch* b, double* records, uint64_t capacity, uint64_t* n_records);
/* enqueue + fetch in chunks of max_records; records may be NULL. */
int umc_batch_run(umc_batch* b, uint64_t n_segments, double* records);
int umc_batch_counters(const umc_batch* b, uint64_t* sweeps, uint64_t* rounds, uint64_t* swaps_accepted);
/* holder[l * replicas + k] = chain at slot k of ladder l. */
int umc_batch_temperature_map(const umc_batch* b, uint32_t* holder);
/* Sets the counters and the temperature map (holder as above, a permutation
 * of each ladder's chains), so that a batch created with the same description
 * and given the same fields continues a saved run exactly (engine extension;
 * the reference has no batches). */
int umc_batch_set_state(umc_batch* b, uint64_t sweeps, uint64_t rounds, uint64_t swaps_accepted, const uint32_t* holder);
/* chain_seeds[c] keys chain c's site streams; ladder_seeds[l] its swaps. */
int umc_batch_seeds(const umc_batch* b, uint64_t* chain_seeds, uint64_t* ladder_seeds);
/* Launch shape the autotuner chose for the ladders of side L. */
int umc_batch_config(const umc_batch* b, uint32_t L, uint32_t* chains_per_cta, uint32_t* ctas_per_chain,
                     uint32_t* block);
int umc_batch_sites(const umc_batch* b, uint64_t* total_sites, uint64_t* kernel_launches);
/* A segment runs in one of two forms; both run the same chains and
 * exchanges.  Persistent (enable = 1): one kernel whose resident CTAs of 1024
 * threads in clusters take work items largest first -- a chain with at least
 * 2 x 8192 sites per colour whose rows split into cluster-many bands of at
 * least 2 is swept by a whole cluster, smaller chains are packed into CTA
 * items of up to 8192 sites per colour -- and the CTA that completes a ladder
 * runs its exchange; its cluster size (1, 4 or 8: with 1 a big chain is one
 * CTA's item) and CTAs per SM (1 or 2) are tuned.  Grouped (enable = 0): one kernel per lattice-size group (tuned
 * launch shapes, umc_batch_config) plus an exchange kernel, as parallel
 * branches of the segment's graph.  At creation both forms are timed on the
 * batch itself (state restored) and the faster one is selected; the choice
 * is cached like the group shapes.  This call overrides it. */
int umc_batch_set_persistent(umc_batch* b, int enable);
/* Selects the persistent form with a given cluster size (1, 4 or 8) and CTAs
 * per SM (1 or 2) instead of the tuned ones. */
int umc_batch_set_persistent_config(umc_batch* b, uint32_t cluster, uint32_t ctas_per_sm);
int umc_batch_persistent_info(const umc_batch* b, int* enabled, uint32_t* grid, uint32_t* big_items, uint32_t* items,
                              uint32_t* cluster, uint32_t* ctas_per_sm);
/* The stream the batch's segments run on (cudaStream_t). */
void* umc_batch_stream(const umc_batch* b);

/* ==================================================== one lattice over ranks */

/* Slab domain decomposition of the regular-lattice Metropolis sweep, for a
 * lattice larger than one GPU (no reference counterpart: the reference runs
 * one chain in one process, driver.hpp:17-68).  The lattice Lx x Ly x Lz
 * (Lz = 1 in 2D; Lx, Ly even, Lz 1 or even) is cut along z in 3D, along y in
 * 2D, into planes; a rank holds planes [first_plane, first_plane + planes)
 * plus a halo plane on each side in a caller-owned device array (natural
 * order, x fastest, except the rows of 2D Ising slabs that umc_slab_row_split
 * reports split by colour; Ising int8, VectorSpin<N> one float array per
 * component with stride umc_slab_local_sites).  umc_slab_pass runs one checkerboard
 * colour over the owned planes; the caller refreshes both halos from the
 * neighbouring ranks after each pass (the planes at local index 1 and
 * `planes` are the ones they need).  Sites draw from the keys of their global
 * colour-major index and sum neighbours in the single-GPU kernels' order, so
 * the ranks together run exactly the single-GPU chain (Ising bit for bit).
 * Wolff flips across slabs: umc_slab_wolff_* below. */
typedef struct umc_slab_desc {
    int32_t model;        /* UMC_MODEL_ISING (Flip) or UMC_MODEL_VECTOR       */
    int32_t components;   /* VectorSpin<N>: 1..4                              */
    uint32_t Lx, Ly, Lz;  /* the whole lattice                                */
    uint32_t first_plane; /* this rank's first plane along z (3D) or y (2D)   */
    uint32_t planes;      /* its plane count (>= 1)                           */
    double coupling;      /* J (integer for Ising)                            */
    int32_t proposal;     /* UMC_PROPOSAL_FLIP / _SPHERE / _ROTATION          */
    double width;         /* LocalRotation delta                              */
    uint64_t seed;        /* the chain's key seed (the same on every rank)    */
    int32_t device;
} umc_slab_desc;
typedef struct umc_slab umc_slab;
int umc_slab_create(const umc_slab_desc* desc, umc_slab** out);
int umc_slab_destroy(umc_slab* s);
/* (planes + 2) x plane sites: halo, owned planes, halo. */
uint64_t umc_slab_local_sites(const umc_slab* s);
/* 1 when each row is stored split by colour instead of in x order: 2D Ising
 * with Lx / 2 a multiple of 16 (the packed 16-sites-per-thread pass).  Row y
 * then holds its colour-0 sites, x in increasing order, then its colour-1
 * sites; the site at x has colour (x + y) & 1 and sits at x / 2 in its half. */
uint32_t umc_slab_row_split(const umc_slab* s);
/* Colour pass `colour` (0 then 1 make sweep `sweep`) of the owned sites of
 * `field` (device pointer) on `stream` (cudaStream_t, NULL = default). */
int umc_slab_pass(umc_slab* s, void* field, double beta, uint64_t sweep, uint32_t colour, void* stream);
/* This rank's part of the last completed sweep's record: [E (bonds whose
 * colour-1 end it owns), M_0..M_{N-1}, 0.., accepted]; the ranks' parts add up
 * to the single-GPU record.  Synchronises `stream`. */
int umc_slab_record(umc_slab* s, double* out, void* stream);
/* Wolff flip `flip` across slabs (the single-GPU flip of the same counter:
 * the same seed, axis, bond keys and reflection).  1. umc_slab_wolff_local:
 * decides every forward bond of the owned sites (the halos must be current)
 * and labels the slab's clusters; 2. umc_slab_wolff_boundary: the root (a
 * global natural site id) of every site of the first and last owned planes,
 * and which last-plane sites have an activated bond into the next plane (the
 * next rank's first); 3. umc_slab_wolff_seed: the seed site and, on the rank
 * that owns it, its root (else 0xFFFFFFFF); 4. every rank gathers all ranks'
 * boundaries (world x plane sites each, rank order) and the seed root, and
 * umc_slab_wolff_merge picks this rank's roots in the seed's cluster (at most
 * 2 x plane sites + 1); 5. umc_slab_wolff_flip reflects those clusters and
 * counts this rank's flipped sites (the ranks' counts add up to the cluster
 * size).  Then refresh the halos. */
int umc_slab_wolff_local(umc_slab* s, void* field, double beta, uint64_t flip, void* stream);
int umc_slab_wolff_boundary(umc_slab* s, uint32_t* first_roots, uint32_t* last_roots, uint8_t* last_up,
                            void* stream);
int umc_slab_wolff_seed(umc_slab* s, uint64_t flip, uint32_t* seed_nat, uint32_t* seed_root, void* stream);
/* Host only.  first_roots, last_roots, last_up: world x plane_sites, rank r's
 * at [r * plane_sites]; rank_roots_first/last and rank_seed_root: this
 * rank's own (the seed root 0xFFFFFFFF where it does not own the seed). */
int umc_slab_wolff_merge(uint32_t world, uint32_t plane_sites, const uint32_t* first_roots, const uint32_t* last_roots,
                         const uint8_t* last_up, uint32_t seed_root, uint32_t rank, const uint32_t* rank_roots_first,
                         const uint32_t* rank_roots_last, uint32_t rank_seed_root, uint32_t* roots, uint32_t* n_roots);
int umc_slab_wolff_flip(umc_slab* s, void* field, uint64_t flip, const uint32_t* roots, uint32_t n_roots,
                        uint64_t* flipped, void* stream);

/* Gauge slabs: the U(1) and SU(N) link sweeps of a plaquette complex split
 * over ranks (no reference counterpart, as above; the motivating case is an
 * SU(3) lattice beyond one GPU).  The caller assigns every link to a rank
 * (`owner`, in the reference's link numbering; for hypercubic_plaquettes a
 * range of the slowest coordinate t per rank).  A rank keeps its owned links
 * and the halo links that its owned links' plaquettes touch, in a
 * caller-owned device array of comps planes x umc_gslab_info's n_local floats
 * (comps = 1 for U(1) angles, 2N^2 for SU(N): plane q holds scalar q of every
 * local link, the reference's data() scalars).  Local links are ordered as
 * the single-GPU chain orders them (colour classes, then the halo); each link
 * draws from the key of its global colour-major index and sums its
 * plaquettes in the single-GPU order, so the ranks together run exactly the
 * single-GPU chain.  A sweep: for each colour class c, umc_gslab_pass, then
 * for every peer p the links of class c to send (umc_gslab_pack) and to
 * receive (umc_gslab_unpack); after the last class umc_gslab_record. */
typedef struct umc_gslab_desc {
    int32_t model;            /* UMC_MODEL_U1 or UMC_MODEL_SU                    */
    int32_t N;                /* SU(N): 2 or 3 (ignored for U(1))                 */
    const umc_cells* cells;   /* the whole lattice's plaquettes (arity 4)         */
    const uint32_t* owner;    /* owner rank of each link, n_sites entries         */
    uint32_t rank, world;
    double coupling;          /* the model's beta                                 */
    double width;             /* U1Shift / SUShift width                          */
    uint32_t hits;            /* Metropolis hits per link and sweep (>= 1)        */
    uint64_t seed;            /* the chain's key seed (the same on every rank)    */
    int32_t device;
} umc_gslab_desc;
typedef struct umc_gslab umc_gslab;
int umc_gslab_create(const umc_gslab_desc* desc, umc_gslab** out);
int umc_gslab_destroy(umc_gslab* s);
/* Local links (owned first), owned links, colour classes, floats per link. */
int umc_gslab_info(const umc_gslab* s, uint32_t* n_local, uint32_t* n_owned, uint32_t* n_classes, uint32_t* comps);
/* The reference link id of every local link (n_local entries). */
int umc_gslab_local_links(const umc_gslab* s, uint32_t* ref_ids);
/* How many links of class `colour` go to `peer` and come from it. */
int umc_gslab_exchange_counts(const umc_gslab* s, uint32_t peer, uint32_t colour, uint32_t* n_send,
                              uint32_t* n_recv);
/* Copies the class-`colour` links that `peer` holds as halo into buf (comps x
 * n_send floats, device), or the ones it owns from buf into this rank's halo. */
int umc_gslab_pack(umc_gslab* s, const float* field, uint32_t peer, uint32_t colour, float* buf, void* stream);
int umc_gslab_unpack(umc_gslab* s, float* field, uint32_t peer, uint32_t colour, const float* buf, void* stream);
/* Colour class `colour` of sweep `sweep` over the owned links. */
int umc_gslab_pass(umc_gslab* s, float* field, double beta, uint64_t sweep, uint32_t colour, void* stream);
/* Ends the sweep: the plaquettes whose first link this rank owns (all their
 * links are local) into this rank's part of the record [S, <P>, Q, 0..,
 * accepted]; the parts add up to the single-GPU record.  Synchronises. */
int umc_gslab_record(umc_gslab* s, const float* field, double* out, void* stream);

/* ================================================= allocation-free Wolff flip */

/* No counterpart in the reference: an extra entry point for callers that cannot
 * call cudaMalloc (a host framework whose pool owns all device memory, or a
 * latency-critical path that must not pay cudaMalloc's device synchronisation).
 * One single-cluster Wolff flip -- the same kernels and random streams as
 * umc_wolff_run -- on caller-owned device memory:
 *   field      Ising int8[n] or VectorSpin<N> float (component c of site k at
 *              field[c*n + k]), updated in place;
 *   offset/bonds/slot_edge  symmetric CSR over the same site order (slot_edge =
 *              index of the input edge that produced each slot, which keys the
 *              bond draws; the seed site is drawn in this site order);
 *   model      UMC_MODEL_ISING (FixedAxis) or UMC_MODEL_VECTOR (UniformSphereN axis).
 * Its scratch (union-find labels and a status word) is a file-scope device
 * array sized for at most 1,048,576 sites; larger graphs return
 * UMC_ERR_UNSUPPORTED.  Every GPU that loads the library holds that array
 * (about 8 MiB) until the process exits.  Each call resolves the array's
 * address (cudaGetSymbolAddress) on the current device.  All calls share the
 * array: each call resets what must start from a known value, and calls that
 * overlap on the GPU race.  Before flipping, a device check verifies the CSR
 * (offset[0] = 0, non-decreasing offsets, neighbour ids < n_sites and no
 * self-loops, each bond stored equally often at both ends) and refuses a graph
 * that fails with UMC_ERR_INVALID_ARGUMENT, launching no flip; offset must
 * hold n_sites + 1 entries and bonds/slot_edge offset[n_sites].  The call is
 * synchronous (it synchronises `stream` twice and returns the cluster size), so
 * it must never be made while `stream` is being captured. */
int umc_wolff_flip_noalloc(int32_t model, int32_t components, void* field, uint64_t n_sites,
                           const uint32_t* offset, const uint32_t* bonds, const uint32_t* slot_edge,
                           double coupling, double beta, uint64_t seed, uint64_t flip,
                           uint64_t* cluster_size, void* stream);

/* ======================================= batched 2D U(1) chains, learned proposal */

/* No counterpart in the reference (which has one chain per driver object and no
 * learned proposals).  A chain is the reference's U(1) plaquette model
 * (model/cell.hpp:64-78 with term/plaquette.hpp:34-47, S = beta sum_p (1 -
 * cos theta_p)) on the periodic L x L square-plaquette complex (links
 * mu L^2 + y L + x; plaquette (x, y) = [(0,x,y), (1,x+1,y), (0,x,y+1), (1,x,y)])
 * under the Metropolis rule of driver.hpp:29-42.  Chain c draws with seed
 * mix64(seed + 0x9E3779B97F4A7C15 (c + 1)), so with the plain proposal
 * (U1Shift, dof/u1.hpp:36-52) it replays the single-chain U(1) sweep of that
 * seed on the colour-major relabelled complex.  With a network the proposal is
 * a 4-component von Mises mixture the network computes from the link's staple,
 * accepted with min(1, exp(-beta dE + log q(old) - log q(new))) in FP64 (the
 * Proposal contract of dof/proposal.hpp:5-12). */
typedef struct umc_u1batch umc_u1batch;
typedef struct umc_mlp umc_mlp;

typedef struct umc_u1batch_desc {
    uint32_t n_chains;
    uint32_t L;            /* even, 4 .. 96 (a chain is held in shared memory) */
    double beta;           /* Wilson coupling */
    double width;          /* U1Shift width of the plain proposal */
    uint64_t seed;
    int32_t device;
    void* stream;          /* cudaStream_t, NULL = own stream */
    uint64_t max_records;  /* record slots (sweeps) between fetches; 0 = 1024 */
    uint32_t first_chain;  /* global index of chain 0: chain c draws as global chain first_chain + c
                              (sharding over ranks, as first_ladder of umc_batch_desc) */
} umc_u1batch_desc;

/* Record per sweep and chain: [S, mean plaquette, topological charge
 * Q = sum_p remainder(theta_p, 2 pi) / 2 pi, accepted updates], laid out
 * [sweep][chain][4]. */
#define UMC_U1_RECORD 4

int umc_u1batch_create(const umc_u1batch_desc* desc, umc_u1batch** out);
int umc_u1batch_destroy(umc_u1batch* b);
/* Hot start: link i of chain c = pi (2u - 1), u the first draw of key
 * (mix64(seed + golden (c + 1)), 0, init tag, i).  Creation leaves a cold start. */
int umc_u1batch_randomize(umc_u1batch* b, uint64_t seed);
/* Angles of one chain in the natural link order (2 L^2 floats). */
int umc_u1batch_set_field(umc_u1batch* b, uint32_t chain, const float* theta);
int umc_u1batch_get_field(umc_u1batch* b, uint32_t chain, float* theta);
/* n sweeps of every chain: plain U1Shift when net is NULL, else the learned proposal. */
int umc_u1batch_enqueue(umc_u1batch* b, uint64_t n_sweeps, const umc_mlp* net);
int umc_u1batch_fetch(umc_u1batch* b, double* records, uint64_t max_sweeps, uint64_t* n_sweeps);
int umc_u1batch_run(umc_u1batch* b, uint64_t n_sweeps, const umc_mlp* net, double* records);
/* One learned sweep; outputs receives chain 0's 16 network outputs per link
 * (natural link order), as the sweep computed them. */
int umc_u1batch_run_dump(umc_u1batch* b, const umc_mlp* net, float* outputs);
int umc_u1batch_counters(const umc_u1batch* b, uint64_t* sweeps, uint64_t* kernel_launches);
int umc_u1batch_set_counter(umc_u1batch* b, uint64_t sweeps);
int umc_u1batch_seeds(const umc_u1batch* b, uint64_t* chain_seeds);
/* Resident CTAs of the plain and learned kernels (one chain per CTA at a time). */
int umc_u1batch_config(const umc_u1batch* b, uint32_t* plain_grid, uint32_t* learned_grid);
void* umc_u1batch_stream(const umc_u1batch* b);

/* The proposal network: x = (cos a, sin a, |S|) of the staple sum S -> ReLU 64
 * -> ReLU 64 -> 16 outputs, component k = (logit, u, v, rho): weight
 * softmax(logit), mean atan2(v, u), concentration clamp(softplus(rho), 1e-4,
 * 80).  BF16 tensor-core products with FP32 accumulation; FP32 master
 * parameters packed W1[3][64], b1[64], W2[64][64], b2[64], W3[64][16], b3[16]. */
#define UMC_MLP_PARAMS 5456

typedef struct umc_mlp_desc {
    uint64_t seed;         /* initial parameters and training minibatches */
    int32_t device;
    void* stream;
    uint64_t max_configs;  /* training configurations held on the device (0 = none) */
    uint32_t L;            /* their lattice side */
} umc_mlp_desc;

int umc_mlp_create(const umc_mlp_desc* desc, umc_mlp** out);
int umc_mlp_destroy(umc_mlp* n);
int umc_mlp_set_params(umc_mlp* n, const float* params);  /* also resets Adam */
int umc_mlp_get_params(umc_mlp* n, float* params);
/* out[n][16] for inputs x[n][3] (host arrays). */
int umc_mlp_forward(umc_mlp* n, const float* x, uint64_t count, float* out);
/* Mean negative log-likelihood of angles theta[n] given inputs x[n][3], and its
 * gradient (UMC_MLP_PARAMS floats); either output may be NULL. */
int umc_mlp_loss_grad(umc_mlp* n, const float* x, const float* theta, uint64_t count, double* loss, float* grad);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) with a given gradient. */
int umc_mlp_apply_gradient(umc_mlp* n, const float* grad, double lr);
/* Appends the batch's current configurations (one per chain) to the dataset. */
int umc_mlp_add_configs(umc_mlp* n, umc_u1batch* b);
int umc_mlp_configs(const umc_mlp* n, uint64_t* count);
int umc_mlp_clear_configs(umc_mlp* n);
/* steps Adam steps on minibatches of `batch` links drawn uniformly from the
 * dataset (key (seed, step, learn tag, sample)); losses[step] = minibatch mean
 * NLL before the step (may be NULL).  Do not train a network while a batch
 * that uses it is still running. */
int umc_mlp_train(umc_mlp* n, uint64_t steps, uint32_t batch, double lr, double* losses);
int umc_mlp_counters(const umc_mlp* n, uint64_t* steps, uint64_t* kernel_launches);
void* umc_mlp_stream(const umc_mlp* n);

/* ================================================================ self-test */

/* No counterpart in the reference.  Every device-side wait of the engine (grid
 * barrier, union-find, tensor-core mbarriers) has an iteration limit; on expiry
 * the kernel records a status bit and returns, and the call that launched it
 * returns UMC_ERR_DEVICE_TIMEOUT with the context still usable.  This runs the
 * engine's grid barrier on a barrier whose generation never advances (about
 * 0.3 s), reports the status bits the kernel left (8 = grid barrier) and
 * returns UMC_ERR_DEVICE_TIMEOUT after checking that the device still answers. */
int umc_selftest_barrier_timeout(int32_t device, uint32_t* status_bits);

/* ================================================= series statistics (host) */

/* No counterpart in the reference (its tests compare chain means against fixed
 * tolerances, test/model_check.cpp:171-222).  Integrated autocorrelation time
 * of a series with Sokal's automatic window: tau(W) = 1/2 + sum_{t<=W} rho(t),
 * W the first window with W >= c * tau(W) (c <= 0 selects 6).  tau_err is the
 * Madras-Sokal estimate tau * sqrt(2 (2W+1) / n).  Any output may be NULL. */
int umc_tau_int(const double* x, uint64_t n, double c, double* tau, double* tau_err, uint64_t* window);
/* The same for `series` independent chains of `length` values each (x laid out
 * [series][length]): every series is centred on its own mean and the
 * autocovariances are averaged over the series (a chain frozen at a constant
 * value contributes nothing; all frozen gives tau = 0.5, window 0).  The error
 * uses the pooled count series * length. */
int umc_tau_int_multi(const double* x, uint64_t series, uint64_t length, double c, double* tau, double* tau_err,
                      uint64_t* window);
/* Mean and its standard error from the means of floor(n/bin) bins of `bin`
 * consecutive values (at least two bins). */
int umc_binning_error(const double* x, uint64_t n, uint64_t bin, double* mean, double* err);

/* Observable streams: a per-sweep or per-flip FP64 series on disk for offline
 * autocorrelation analysis (no reference counterpart: the reference's observe
 * callbacks keep nothing, driver.hpp:54-61).  The file is a 56-byte header
 * (magic "UMCOBS01", version 1, columns, records, seed, first counter, model,
 * beta), columns x 32-byte NUL-padded names, then records x columns doubles,
 * little-endian.  The record count is rewritten after every append, so a run
 * cut short still reads back every counted record.  Not thread-safe per
 * handle. */
typedef struct umc_obs_stream umc_obs_stream;
int umc_obs_stream_create(const char* path, uint32_t columns, const char* const* names, uint64_t seed,
                          uint64_t first, int32_t model, double beta, umc_obs_stream** out);
/* Appends n records (n x columns doubles, row-major). */
int umc_obs_stream_append(umc_obs_stream* s, const double* records, uint64_t n);
int umc_obs_stream_close(umc_obs_stream* s);
/* Header of a stream file; names (columns x 32 bytes) may be NULL, as may any output. */
int umc_obs_stream_info(const char* path, uint32_t* columns, uint64_t* records, uint64_t* seed, uint64_t* first,
                        int32_t* model, double* beta, char* names);
/* Records [first_record, first_record + n) into out (n x columns). */
int umc_obs_stream_read(const char* path, uint64_t first_record, uint64_t n, double* out);

#ifdef __cplusplus
}
#endif
#endif /* UMC_B200_H */
