/* parex_b200 — B200-native random-walk expander decomposition, C ABI.
 *
 * Every entry point replaces one member of the reference's drop-in class
 * CudaDeviceManager (cuda/interface.h:16-57); the reference member is named
 * beside each declaration.  Plain pointers and sizes only: no CUDA, C++ or
 * torch types cross this boundary.  Host buffers are ordinary host memory
 * unless a function says otherwise.
 *
 * Threading: a handle is used by one host thread at a time.  All device work
 * of a handle runs on the handle's stream, in call order.
 * Errors: every function returns a pxr_status; pxr_last_error() gives the
 * message of the last failure on that handle.
 */
#ifndef PAREX_B200_H
#define PAREX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PXR_ABI_VERSION 1
#define PXR_INVALID_EDGE 0xFFFFFFFFu   /* disabled CSR slot, lib/core/definitions.h:52 */

typedef enum {
    PXR_OK = 0,
    PXR_INVALID_ARG = 1,     /* bad pointer, size or state                           */
    PXR_OUT_OF_MEMORY = 2,   /* device allocation failed                              */
    PXR_ITER_CAP = 3,        /* round cap reached before every cluster was certified  */
    PXR_CUDA_ERROR = 4,      /* a CUDA runtime call failed                            */
    PXR_DEVICE_FAULT = 5,    /* a device-side bounded wait or invariant check failed  */
    PXR_NOT_INITIALIZED = 6  /* no graph uploaded yet                                 */
} pxr_status;

/* Division used for the sweep's sparsity ratio. */
enum {
    PXR_DIV_IEEE = 0,        /* correctly rounded float division (default)                */
    PXR_DIV_REFERENCE = 1    /* the approximate division the reference's fast-math build
                                uses; reproduces its tie-breaking on equal ratios        */
};

/* Round driver. */
enum {
    PXR_DRIVER_GRAPH = 0,    /* rounds replayed from a captured CUDA graph (default)      */
    PXR_DRIVER_STREAM = 1    /* rounds launched kernel by kernel from the host            */
};

typedef struct {
    uint32_t seed;           /* randSeed, lib/core/definitions.h:46 (6582)              */
    float sc_threshold;      /* sweep sparsity threshold, definitions.h:50 (0.3)          */
    float rw_threshold;      /* potential threshold, definitions.h:49 (1e-4)              */
    uint32_t max_rounds;     /* MAX_NUM_ITER, cuda/device.h:371 (200000)                  */
    int32_t device;          /* CUDA device ordinal                                       */
    uint32_t division;       /* PXR_DIV_*                                                 */
    uint32_t driver;         /* PXR_DRIVER_*                                              */
    uint32_t tune;           /* PXR_TUNE_* (row plan: lanes per row and row bins)          */
    uint32_t components;     /* PXR_COMPONENTS_* (union-find schedule of the cut stage)    */
    uint32_t memory_cap_mib; /* device memory a handle may hold, in MiB (0: no cap); an
                                initialisation that needs more fails with
                                PXR_OUT_OF_MEMORY before any allocation is kept           */
    uint32_t reserved[6];
} pxr_config;

/* Union-find schedule of the connected-components stage (no counterpart in
 * the reference, which hooks every edge).  Both give the same components. */
enum {
    PXR_COMPONENTS_AUTO = 0,    /* sampled from mean degree 16 on, plain below (default)  */
    PXR_COMPONENTS_PLAIN = 1,   /* first-neighbour links, then every edge once            */
    PXR_COMPONENTS_SAMPLED = 2  /* first-neighbour links, one hashed neighbour per vertex,
                                   then full rows only outside each label's largest set   */
};

/* How the row plan of a graph is chosen (no counterpart in the reference,
 * whose kernels use one warp per vertex for every row). */
enum {
    PXR_TUNE_AUTO = 0,       /* time the walk step under each candidate plan on the graph
                                itself at initialisation, keep the fastest; the choice is
                                cached per degree histogram for the life of the process   */
    PXR_TUNE_HEURISTIC = 1   /* lanes per row from the mean degree, default bins           */
};

/* Row plan: rows of at most light_max slots are handled by lanes_per_row
 * lanes each (1, 4, 8, 16 or 32; 4 slot loads in flight per lane), rows up
 * to wide_max slots by a warp each, longer rows by a 256-thread CTA each.
 * The plan changes speed only: every result is the same under any plan. */
typedef struct {
    uint32_t lanes_per_row;
    uint32_t light_max;
    uint32_t wide_max;
    uint32_t wide_rows;      /* rows in the warp-per-row bin (set by the library)            */
    uint32_t heavy_rows;     /* rows in the CTA-per-row bin (set by the library)             */
    uint32_t source;         /* 0 heuristic, 1 tuned now, 2 tuned earlier (cache), 3 forced   */
    uint32_t candidates;     /* plans timed by the last tuning                               */
    float walk_us;           /* walk-step time of the chosen plan when tuned (microseconds)  */
} pxr_row_plan;

/* Sort plan of the sweep's global radix sort (no counterpart in the
 * reference, which calls CUB's SortPairs): keys per thread of a tile (16, 12
 * or 8; tiles of 256 x items) and the CTAs per SM the pass kernel's register
 * budget is sized for (2, 3 or 4), as plan 0, 1 or 2.  Digits are 8 bits
 * wide; passes whose digit is constant over the keys are skipped.  Every plan
 * gives the same order, item for item. */
typedef struct {
    uint32_t plan;           /* 0, 1 or 2                                                    */
    uint32_t items_per_thread;
    uint32_t ctas_per_sm;
    uint32_t source;         /* 0 default, 1 tuned now, 2 tuned earlier (cache), 3 forced      */
    uint32_t candidates;     /* plans timed by the last tuning                               */
    float sort_us[3];        /* time of one sort of the first round's keys under each plan   */
} pxr_sort_plan;

/* One sweep cut per active cluster: SweepCutData, lib/core/definitions.h:57-61. */
typedef struct { int32_t label; float sparsity; uint32_t offset; } pxr_sweep_cut;

/* Sweep order entry: NodeData, lib/core/definitions.h:68-78. */
typedef struct {
    uint32_t nix;
    uint32_t prefix_volume;
    int32_t prefix_edge_diff;
    uint32_t offset_in_cluster;
} pxr_node_data;

typedef struct {
    uint32_t rounds;             /* rounds run by the last pxr_decompose                 */
    uint32_t active_vertices;    /* numActiveNodes                                        */
    uint32_t active_clusters;    /* numActiveClusters                                     */
    uint32_t clusters_with_cut;  /* numClustersWithCut of the last sweep                  */
    uint64_t device_bytes;       /* device memory held by the handle                      */
    double last_decompose_ms;    /* device time of the last pxr_decompose (CUDA events)    */
    uint64_t kernel_launches;    /* kernels this handle has launched since creation        */
    uint64_t walk_vertices;      /* vertex updates done by walk steps since initialization */
    uint64_t walk_slots;         /* CSR slots read by walk steps since initialization      */
    uint64_t walk_gathers;       /* valid-neighbour gathers by walk steps                  */
    uint64_t sort_items;         /* items x passes moved by the sweep sort                 */
    uint64_t sort_passes;        /* digit passes the sweep sort ran (constant digits skip)  */
    uint64_t swept_items;        /* sweep input vertices summed over rounds                */
    uint64_t skipped_sweeps;     /* cluster-rounds the learned schedule did not sweep      */
    uint64_t false_stops;        /* skipped sweeps that would have cut (audit mode only)    */
} pxr_stats;

/* Per-phase device time, recorded with CUDA events when profiling is on
 * (pxr_set_profiling) and the stream driver runs the rounds. */
typedef struct {
    char name[24];
    double ms;                   /* summed device time                                    */
    uint64_t launches;           /* kernel launches in this phase                         */
} pxr_phase_stat;

/* ---- learned sweep schedule (no counterpart in the reference) -------------
 *
 * The reference sweeps every active cluster in every round.  The learned
 * schedule lets a cluster skip the sweep (sort, scan, cut, components,
 * recentering) for a number of rounds predicted by a small MLP from the
 * cluster's features; its vertices keep walking.  The MLP never decides a cut
 * or a certificate: cuts are chosen and scored by the exact sweep when the
 * cluster is next swept, and a cluster is certified only by the plain check
 * (potential spread below rw_threshold, or fewer than 2 vertices).
 * Network: 16 features -> 32 -> 32 -> 1 (ReLU), bf16 weights and inputs,
 * float accumulation; output y = predicted log2(1 + rounds the cluster can
 * skip); the schedule skips floor(safety * (2^y - 1)) rounds, at most
 * max_skip.  Parameter layout (PXR_MLP_PARAMS bf16 values): W1[32][16], b1[32],
 * W2[32][32], b2[32], W3[32], b3.  norm: 16 input means then 16 scales;
 * the MLP reads bf16((feature - mean) * scale). */
#define PXR_MLP_FEATURES 16
#define PXR_MLP_HIDDEN 32
#define PXR_MLP_PARAMS 1633

enum {
    PXR_SCHEDULE_PLAIN = 0,    /* every active cluster swept every round (the reference's method)  */
    PXR_SCHEDULE_LEARNED = 1,  /* clusters skip the sweep for the rounds the MLP predicts           */
    PXR_SCHEDULE_AUDIT = 2     /* as LEARNED, but skipped clusters are still swept (not acted on)
                                  and those whose sweep would have cut are counted (false_stops);
                                  the partition is the same as with LEARNED                          */
};

typedef struct {
    uint32_t mode;             /* PXR_SCHEDULE_*                                                    */
    uint32_t trace;            /* nonzero: keep one pxr_cluster_record per active cluster per round */
    float safety;              /* fraction of the predicted skips taken                             */
    uint32_t max_skip;         /* cap on consecutive skipped rounds                                 */
    float cut_gate;            /* a round that cuts more than cut_gate x its clusters skips no sweep
                                  in the next round (every cluster swept, as in PLAIN); 0: off      */
    uint32_t due_period;       /* > 1: clusters under 1/1024 of the active vertices come due only in
                                  rounds whose index is a multiple of due_period, so their sweeps
                                  share rounds and the others only walk; 0 or 1: off              */
    uint32_t reserved[2];
} pxr_schedule;

/* One active cluster after the last round (trace mode).  origin: 1 swept and
 * not split, 2 new from a split (swept next round), 3 carried unswept. */
typedef struct {
    uint32_t root, size, volume, origin;
    float potential;           /* max - min of the potentials at this round's sweep              */
    float sparsity;            /* best sweep sparsity of this round (of the parent for origin 2) */
    float prev_potential, prev_sparsity;
    uint32_t prev_round;       /* round of the previous sweep of the same vertex set             */
    uint32_t age;              /* earlier sweeps of the same vertex set                          */
    uint32_t round;            /* rounds completed before this one                                */
    uint32_t skip;             /* rounds the schedule carries the cluster next                    */
    float prediction;          /* MLP output y (learned modes)                                    */
    uint32_t has_prev;
    uint32_t reserved[2];
    float features[PXR_MLP_FEATURES];
} pxr_cluster_record;

typedef struct { float delta; float over_weight; } pxr_mlp_loss;       /* asymmetric Huber */
typedef struct { float lr, beta1, beta2, eps; } pxr_mlp_adam;

void pxr_config_default(pxr_config* cfg);
const char* pxr_status_string(pxr_status s);
const char* pxr_last_error(const void* handle);

typedef struct pxr_handle pxr_handle;

/* CudaDeviceManager::CudaDeviceManager() (cuda/interface.h:18). */
pxr_status pxr_create(const pxr_config* cfg, pxr_handle** out);
/* CudaDeviceManager::~CudaDeviceManager() (cuda/interface.h:19). */
void pxr_destroy(pxr_handle* h);

/* Run the handle's device work on the caller's stream (a cudaStream_t passed
 * as void*); NULL restores the handle's own stream.  No counterpart in the
 * reference, which uses the legacy default stream throughout. */
pxr_status pxr_set_stream(pxr_handle* h, void* stream);

/* CudaDeviceManager::initialize(const Graph&) (cuda/interface.h:24;
 * cuda/device.h:86-100).  Uploads the CSR (n+1 offsets, 2m columns), resets
 * the partition to one cluster and seeds the potentials from cfg.seed.
 * Offsets are 32-bit (the reference's EdgeIx) or 64-bit; the starting
 * cluster's volume 2m must be below 2^32 (32-bit prefix volumes, as the
 * reference's NodeData). */
pxr_status pxr_initialize(pxr_handle* h, uint32_t n, uint64_t m,
                          const uint32_t* offsets, const uint32_t* cols);
pxr_status pxr_initialize64(pxr_handle* h, uint32_t n, uint64_t m,
                            const uint64_t* offsets, const uint32_t* cols);
/* The same with the CSR already in device memory (device pointers on the
 * handle's device; offsets 64-bit when offsets_are_64bit, else 32-bit).  The
 * arrays are copied; the caller keeps ownership.  Repeated initialisation
 * with the same n and m reuses the handle's device memory. */
pxr_status pxr_initialize_device(pxr_handle* h, uint32_t n, uint64_t m,
                                 const void* offsets, int offsets_are_64bit,
                                 const uint32_t* cols);

/* Batched independent instances.  No counterpart in the reference, which
 * decomposes one graph per CudaDeviceManager.  The CSR (host arrays, 64-bit
 * offsets) is the disjoint union of n_instances graphs; instance i owns the
 * vertices [instance_start[i], instance_start[i+1]) (instance_start has
 * n_instances + 1 entries, runs from 0 to n, every instance non-empty) and no
 * edge may join two instances (PXR_INVALID_ARG otherwise).  Every instance
 * starts as its own cluster, so the whole batch, from a handful of vertices
 * to millions per instance, advances through the same rounds: one walk
 * launch, one sort, one scan and one components pass per round for all of
 * them.  The volume of each instance must be below 2^32 (the reference's
 * 32-bit prefix volumes); the batch as a whole may exceed it.  Potentials are
 * seeded as pxr_initialize does, by global vertex id. */
pxr_status pxr_initialize_batched(pxr_handle* h, uint32_t n, uint64_t m,
                                  const uint64_t* offsets, const uint32_t* cols,
                                  uint32_t n_instances, const uint32_t* instance_start);

/* The row plan in use (pxr_row_plan).  No counterpart in the reference. */
pxr_status pxr_get_row_plan(pxr_handle* h, pxr_row_plan* out);
/* Force a row plan (lanes_per_row, light_max, wide_max are read; the rest is
 * ignored) for this and later initialisations; NULL returns to cfg.tune.
 * Applied at once when a graph is loaded. */
pxr_status pxr_set_row_plan(pxr_handle* h, const pxr_row_plan* plan);

/* The sweep sort's plan in use (pxr_sort_plan).  With PXR_TUNE_AUTO the
 * library times the global sort of the first round's keys (every active
 * vertex, cluster 0) under each plan when a graph of at least 2^16 vertices
 * is loaded and keeps the fastest; choices are cached per vertex count.  No
 * counterpart in the reference. */
pxr_status pxr_get_sort_plan(pxr_handle* h, pxr_sort_plan* out);
/* Force a sort plan (plan is read) from the next round on; NULL returns to
 * cfg.tune from the next initialisation. */
pxr_status pxr_set_sort_plan(pxr_handle* h, const pxr_sort_plan* plan);

/* pxr_initialize_batched with the CSR in device memory (offsets 64-bit when
 * offsets_are_64bit, else 32-bit); instance_start stays a host array. */
pxr_status pxr_initialize_batched_device(pxr_handle* h, uint32_t n, uint64_t m, const void* offsets,
                                         int offsets_are_64bit, const uint32_t* cols, uint32_t n_instances,
                                         const uint32_t* instance_start);

/* CudaDeviceManager::iterateRandomWalk() (cuda/interface.h:29). */
pxr_status pxr_walk_step(pxr_handle* h);
/* CudaDeviceManager::computeSweepCuts() (cuda/interface.h:32). */
pxr_status pxr_sweep(pxr_handle* h);
/* CudaDeviceManager::cutClusters() (cuda/interface.h:36). */
pxr_status pxr_cut_clusters(pxr_handle* h);
/* CudaDeviceManager::expanderDecomposition() (cuda/interface.h:40). *rounds may be NULL. */
pxr_status pxr_decompose(pxr_handle* h, uint32_t* rounds);

/* CudaDeviceManager::readRandomWalkValues() (cuda/interface.h:30): n floats. */
pxr_status pxr_read_potentials(pxr_handle* h, float* out);
/* CudaDeviceManager::readSweepCuts() (cuda/interface.h:34): labels and
 * per-cluster argmin cuts of every active cluster (before thresholding).
 * Writes min(cap, count) entries and sets *count. */
pxr_status pxr_read_sweep_cuts(pxr_handle* h, int32_t* labels, pxr_sweep_cut* cuts,
                               uint32_t cap, uint32_t* count);
/* CudaDeviceManager::downloadPartition() (cuda/interface.h:27): the sweep
 * order with prefix sums, active vertices only.  Writes min(cap, count). */
pxr_status pxr_download_partition(pxr_handle* h, pxr_node_data* out, uint32_t cap,
                                  uint32_t* count);
/* CudaDeviceManager::getFinalPartition() (cuda/interface.h:42): dense ids
 * 0..k-1 ordered by label value, n entries. */
pxr_status pxr_final_partition(pxr_handle* h, int32_t* ids, int32_t* num_clusters);
/* CudaDeviceManager::getNumCutEdges() (cuda/interface.h:38). */
pxr_status pxr_num_cut_edges(pxr_handle* h, uint64_t* out);
/* CudaDeviceManager::downloadGraph() (cuda/interface.h:25): the CSR with
 * disabled slots set to PXR_INVALID_EDGE.  offsets: n+1 entries (32-bit
 * variant fails with PXR_INVALID_ARG when 2m >= 2^32). */
pxr_status pxr_download_graph(pxr_handle* h, uint32_t* offsets, uint32_t* cols);
pxr_status pxr_download_graph64(pxr_handle* h, uint64_t* offsets, uint32_t* cols);
/* CudaDeviceManager::downloadDegrees() (cuda/interface.h:26): internal degrees. */
pxr_status pxr_download_degrees(pxr_handle* h, uint32_t* out);
/* CudaDeviceManager::downloadLabels() (cuda/interface.h:45). */
pxr_status pxr_download_labels(pxr_handle* h, int32_t* out);
/* CudaDeviceManager::downloadActiveEdgeMap() (cuda/interface.h:44): 2m ints. */
pxr_status pxr_active_edge_map(pxr_handle* h, int32_t* out);
/* Cut edges of the current partition, recounted on the device: undirected
 * edges of the graph as uploaded whose ends carry different labels, i.e.
 * different getFinalPartition ids.  This is the count the reference's
 * application makes on the host after getFinalPartition
 * (Partition::splitByIndices and getNumCutEdges, main.cpp:54-60), which the
 * library's getNumCutEdges (m - valid/2, cuda/devPartition.h:741-759) does
 * not give once clusters are certified (their rows are no longer updated).
 * PXR_INVALID_ARG after pxr_set_state loaded disabled slots, whose
 * neighbours are unknown. */
pxr_status pxr_count_cut_edges(pxr_handle* h, uint64_t* out);
/* Certificate record, n uint32 (no counterpart in the reference, which
 * keeps none).  0 while the vertex is active.  When its cluster is certified
 * - deactivated by the keep test (potential spread below rw_threshold or
 * fewer than 2 vertices, cuda/devPartition.h:173-184) - the round in which
 * that happened, plus 1, with bit 31 set when the certified set is not the
 * whole set swept in that round (the swept cluster was cut, or fell apart
 * into components).  A certified vertex neither walks nor recentres again,
 * so pxr_read_potentials returns the potentials the keep test saw; with the
 * final partition this lets a caller re-check every certificate
 * (parex_b200/certificate.py). */
pxr_status pxr_download_certificates(pxr_handle* h, uint32_t* out);
/* CudaDeviceManager::getNumClusters() (cuda/interface.h:46; the reference
 * returns 0 unconditionally, cuda/device.h:120-123): here the number of
 * active clusters. */
pxr_status pxr_num_active_clusters(pxr_handle* h, uint32_t* out);

pxr_status pxr_get_stats(pxr_handle* h, pxr_stats* out);
/* Turn per-phase CUDA-event timing on (1) or off (0); it applies to rounds
 * run by the stream driver.  Resets the accumulated phase times. */
pxr_status pxr_set_profiling(pxr_handle* h, int enable);
/* Accumulated phase times; writes min(cap, count) entries, sets *count. */
pxr_status pxr_phase_stats(pxr_handle* h, pxr_phase_stat* out, uint32_t cap, uint32_t* count);

/* Final partition for callers that cannot allocate device memory.  No
 * counterpart in the reference.
 *
 * Some callers may not call cudaMalloc/cudaFree where they need the cluster
 * ids: their device memory is owned by a pooling allocator that must account
 * for every byte, or they cannot afford the device-wide synchronisation those
 * calls may imply.  This entry point allocates nothing: labels (n int32) is
 * the caller's device array of cluster labels, as pxr_download_labels returns
 * them; ids (n int32) and num_clusters (one int32) are the caller's device
 * outputs, filled exactly as pxr_final_partition fills its host outputs
 * (dense ids ordered by label value).  Work is enqueued on `stream` (a
 * cudaStream_t as void*, NULL for the legacy default stream) and the call
 * returns without waiting.
 *
 * Limit: n <= PXR_STATIC_SCRATCH_MAX_LABELS; larger n returns
 * PXR_INVALID_ARG (use pxr_final_partition).  The working memory is a fixed
 * ~1.1 MB array inside the library, held on every GPU that loads it until
 * the process exits.  Every call looks up that array's device address
 * (cudaGetSymbolAddress) with the caller's device current, so a
 * cudaDeviceReset between calls is harmless; the first call on a device also
 * loads the library's kernels there, so make it before any stream capture.  All calls share the array: calls
 * whose work may overlap on the GPU race and must be ordered by the caller.
 * *num_clusters is -1 if a device-side bounded wait ran out. */
#define PXR_STATIC_SCRATCH_MAX_LABELS 65536u
pxr_status pxr_final_partition_static(const int32_t* labels, uint32_t n, int32_t* ids,
                                      int32_t* num_clusters, void* stream);

/* Test hooks with no counterpart in the reference: overwrite the potentials
 * (n doubles, rounded to the product's float storage), or the whole round
 * state.  act holds the n_act active vertex ids in the order their keys are
 * emitted; labels of active vertices must be dense in [0, n_clusters). */
pxr_status pxr_set_potentials(pxr_handle* h, const double* x);
pxr_status pxr_set_state(pxr_handle* h, const int32_t* labels, const uint32_t* act, uint32_t n_act,
                         const double* x, const uint32_t* internal_degrees, const uint32_t* cols,
                         uint32_t n_clusters, int32_t smallest_label, int full_components);

/* Test hook with no counterpart in the reference: run the library's two
 * bounded device-side waits - the decoupled look-back of the scans and the
 * sort's tile-status wait - on a flag that nothing sets, with at most
 * spin_limit polls (1 .. 2^20), on scratch memory of their own.  Both must
 * give up, set their error bits and return; the call then reports
 * PXR_DEVICE_FAULT the way a round that timed out does, *err_bits gets the
 * bits, and the handle stays usable.  Nothing of the handle's state is
 * touched. */
pxr_status pxr_test_bounded_waits(pxr_handle* h, uint32_t spin_limit, uint32_t* err_bits);

/* ---- graph construction on the device ------------------------------------
 * The CSR the reference builds on the host (readDynGraph +
 * DynamicGraph::finalize, lib/utils/graph_io.h:49-84, lib/core/graph.h:147-184),
 * built on the GPU from an edge list in device memory: self-loops dropped,
 * duplicate edges merged, both directions stored, rows sorted by neighbour.
 * u, v: n_edges vertex ids (< n); offsets: n + 1 entries; cols: room for
 * 2 * n_edges entries; scratch: pxr_build_csr_scratch_bytes(n_edges) bytes of
 * device memory.  Needs 2 * n_edges < 2^32.  Synchronises the stream; *m_out
 * is the number of undirected edges kept.  No counterpart in the reference's
 * GPU code. */
size_t pxr_build_csr_scratch_bytes(uint64_t n_edges);
pxr_status pxr_build_csr(uint32_t n, uint64_t n_edges, const uint32_t* u, const uint32_t* v, void* scratch,
                         uint32_t* offsets, uint32_t* cols, uint64_t* m_out, void* stream);
/* The CSR of the reference's own input path, on the device:
 * DynamicGraph::finalize (lib/core/graph.h:147-184) keeps the edge list as it
 * stands - duplicate edges and self-loops included (a self-loop gives two
 * slots in its row) - and stores both directions, rows sorted by neighbour.
 * Same arguments and scratch as pxr_build_csr; the graph has m = n_edges.
 * Needs 2 * n_edges < 2^32 (the reference's 32-bit EdgeIx). */
pxr_status pxr_build_csr_finalize(uint32_t n, uint64_t n_edges, const uint32_t* u, const uint32_t* v, void* scratch,
                                  uint32_t* offsets, uint32_t* cols, void* stream);
/* The body of a Matrix Market file (device memory: the bytes after the size
 * line) parsed as readDynGraph (lib/utils/graph_io.h:49-84) reads it: a stream
 * of decimal integers, two per edge, 1-based, line breaks not significant;
 * the first 2 * n_edges numbers give u[i], v[i] (0-based).  The caller
 * parses the header (comment lines, then "rows n n_edges") on the host.
 * scratch: pxr_parse_mtx_scratch_bytes(text_bytes) bytes of device memory.
 * *tokens_out: the numbers found.  PXR_INVALID_ARG when fewer than
 * 2 * n_edges numbers are found or an id lies outside 1..n (the reference
 * would read past its edge array or wrap).  Synchronises the stream. */
size_t pxr_parse_mtx_scratch_bytes(uint64_t text_bytes);
pxr_status pxr_parse_mtx_body(const char* text, uint64_t text_bytes, uint32_t n, uint64_t n_edges, uint32_t* u,
                              uint32_t* v, void* scratch, uint64_t* tokens_out, void* stream);
/* One level of the expander hierarchy on the device
 * (ExpanderHierarchy::contract, lib/algorithms/expander_hierarchy.h:34-88):
 * the graph whose vertices are the k clusters of `ids` (n int32 in [0, k),
 * e.g. pxr_final_partition's ids) and whose edges are the cut edges of the
 * level graph (offsets/cols: n + 1 and offsets[n] 32-bit entries), one per cut
 * edge, multi-edges kept, rows sorted (the reference leaves them in its
 * clusters' vertex order).  cut_sizes[c]: cut slots leaving cluster c;
 * volumes[c]: sum over its vertices of level_volumes (k 64-bit entries; at the
 * first level pass NULL to take the vertices' degrees).  out_offsets: k + 1
 * entries; out_cols: room for offsets[n] entries; *out_m: edges of the
 * contracted graph.  All arrays in device memory; scratch:
 * pxr_contract_scratch_bytes(offsets[n]) bytes.  Synchronises the stream. */
size_t pxr_contract_scratch_bytes(uint64_t slots);
pxr_status pxr_contract(uint32_t n, const uint32_t* offsets, const uint32_t* cols, const int32_t* ids, uint32_t k,
                        const uint64_t* level_volumes, void* scratch, uint32_t* out_offsets, uint32_t* out_cols,
                        uint64_t* out_m, uint64_t* cut_sizes, uint64_t* volumes, void* stream);
/* One block pair of a planted-partition instance: candidate pairs
 * (base_u + i, base_v + j), i < su, j < sv (intra: i < j < su, base_u == base_v),
 * each an edge with probability p.  key names the task's random stream: a
 * task's edges depend on (seed, key, su, sv, p) only, not on the task's place
 * in the list, so a subset of a batch (one shard) draws the same edges. */
typedef struct {
    uint32_t base_u, base_v, su, sv;
    double p;
    uint32_t intra;
    uint32_t key;
} pxr_sbm_task;
/* Planted-partition edges on the device by geometric skipping: the candidate
 * range of task t is cut into segments of segment_len candidates;
 * seg_prefix[t] is the first global segment of task t (n_tasks + 1 entries,
 * ending with n_segments).  Two calls, all arrays in device memory: with
 * seg_offset == NULL the number of edges of every segment goes to
 * seg_count[n_segments]; then, with seg_offset the exclusive prefix of those
 * counts, the edges go to u, v (segment by segment, in candidate order).
 * Deterministic in seed; pxr_build_csr turns the list into the CSR. */
pxr_status pxr_sbm_edges(const pxr_sbm_task* tasks, uint32_t n_tasks, const uint64_t* seg_prefix, uint64_t n_segments,
                         uint64_t segment_len, uint64_t seed, uint32_t* seg_count, const uint64_t* seg_offset,
                         uint32_t* u, uint32_t* v, void* stream);
/* R-MAT edge samples on the device: samples (u, v) pairs over 2^scale
 * vertices, quadrant probabilities a, b, c (d = 1 - a - b - c), from the
 * counter-based hash of parex_b200/graphs.py rmat() (same seed, same edges). */
pxr_status pxr_rmat_edges(uint32_t scale, uint64_t samples, double a, double b, double c, uint64_t seed,
                          uint32_t* u, uint32_t* v, void* stream);

/* Learned sweep schedule: mode, trace and, for the learned modes, the MLP
 * (weights: PXR_MLP_PARAMS bf16 bit patterns, norm: 32 floats; host memory).
 * Takes effect from the next round; every cluster is due at (re)initialisation. */
pxr_status pxr_set_schedule(pxr_handle* h, const pxr_schedule* cfg, const uint16_t* weights, const float* norm);
/* Records of the active clusters after the last round (trace mode): writes
 * min(cap, count) and sets *count. */
pxr_status pxr_read_cluster_records(pxr_handle* h, pxr_cluster_record* out, uint32_t cap, uint32_t* count);

/* MLP kernels on device arrays (the caller's stream; NULL = legacy stream).
 * features: n x 16 floats; weights: PXR_MLP_PARAMS bf16; norm: 32 floats. */
pxr_status pxr_mlp_forward(const float* features, uint32_t n, const uint16_t* weights, const float* norm,
                           float* out, void* stream);
/* Floats of scratch pxr_mlp_gradient needs for n samples. */
size_t pxr_mlp_scratch_floats(uint32_t n);
/* Mean loss and its gradient over n samples (targets: n floats): asymmetric
 * Huber on e = y - target, weight over_weight when e > 0, quadratic for
 * |e| <= delta.  grad: PXR_MLP_PARAMS floats; loss_out: 1 float. */
pxr_status pxr_mlp_gradient(const float* features, const float* targets, uint32_t n, const uint16_t* weights,
                            const float* norm, const pxr_mlp_loss* loss, float* scratch, float* grad,
                            float* loss_out, void* stream);
/* One Adam step on float master weights (m, v: moments; step counts from 1),
 * then weights = bf16(master). */
pxr_status pxr_mlp_adam_step(float* master, float* m, float* v, const float* grad, uint16_t* weights,
                             uint32_t step, const pxr_mlp_adam* opt, void* stream);

#ifdef __cplusplus
}
#endif
#endif
