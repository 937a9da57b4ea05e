/* CPU oracle for the random-walk expander decomposition round (test infrastructure).
 *
 * A plain-C restatement of the reference's GPU decomposition
 * (cuda/device.h:101-168 and 301-350 with the managers in cuda/dev*.h),
 * used only by the tests, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg, as the checker.  The product never links or calls it.
 *
 * Two arithmetic modes share every integer stage (sort order, sweep scan,
 * cut, components, relabelling, edge disabling):
 *
 *   ORC_MODE_REF  potentials in double, walk sums in the reference's warp
 *                 order, per-cluster sums in float as the reference does;
 *                 pinned against traces of the reference's own GPU binary.
 *   ORC_MODE_PXR  the CUDA product's arithmetic: float potentials, exact
 *                 fixed-point walk and cluster sums, so that the product and
 *                 this mode agree bit for bit, end to end.
 *
 * Types mirror the reference's PODs (lib/core/definitions.h:57-107).
 */
#ifndef PXR_ORACLE_H
#define PXR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_INVALID_EDGE 0xFFFFFFFFu

enum { ORC_MODE_REF = 0, ORC_MODE_PXR = 1 };

typedef struct { uint32_t nix; int32_t label; } orc_lnode;              /* LabeledNode */
typedef struct {                                                         /* NodeData    */
    uint32_t nix;
    uint32_t prefix_volume;
    int32_t prefix_edge_diff;
    uint32_t offset;
} orc_node_data;
typedef struct { int32_t label; float sparsity; uint32_t offset; } orc_sweep_cut;  /* SweepCutData */
typedef struct { float sum; float max; float min; uint32_t count; } orc_cluster_data; /* ClusterData */

typedef struct orc_state orc_state;

orc_state* orc_create(uint32_t n, uint64_t m, const uint64_t* offsets, const uint32_t* cols,
                      int mode, float sc_threshold, float rw_threshold);
void orc_destroy(orc_state* s);

/* x0[v] ~ N(0, sqrt(deg v)) as the reference seeds it (cuda/devRandomWalk.h:22-48),
 * evaluated with this file's own inverse complementary error function. */
void orc_initial_potentials(uint32_t n, const uint64_t* offsets, uint32_t seed, float* out);

/* Replace the current potentials (all n vertices). */
void orc_set_potentials(orc_state* s, const double* x);

/* Replace the whole round state (per-stage parity from a recorded trace). */
void orc_set_state(orc_state* s, const int32_t* labels, const orc_lnode* act, uint32_t n_act,
                   const double* x, const uint32_t* internal_degrees, const uint32_t* cols,
                   uint32_t n_clusters, int32_t smallest_label);

/* Stages of one round, in the reference's order. */
void orc_walk(orc_state* s);
void orc_sweep(orc_state* s);
void orc_cut_stage(orc_state* s);
void orc_components_stage(orc_state* s);
void orc_cluster_data_stage(orc_state* s);
void orc_recenter_stage(orc_state* s);
void orc_disable_stage(orc_state* s);
void orc_cut_clusters(orc_state* s);   /* the five stages above */
/* Re-emit the walk's sort keys from the current potentials. */
void orc_rekey(orc_state* s);

/* One round with a sweep schedule: due[c] != 0 for the active clusters
 * (labels 0..n_clusters-1) that are swept this round; the others only walk
 * and are relabelled.  No reference counterpart (the learned stop
 * predictor's schedule); with every cluster due it is the plain round. */
void orc_scheduled_round(orc_state* s, const uint8_t* due);

/* Rounds until no active cluster is left (cuda/device.h:363-404). Returns the
 * number of rounds that ran a walk step. */
uint32_t orc_decompose(orc_state* s, uint32_t max_rounds);

/* FinalPartition: dense ids ordered by label value (cuda/devPartition.h:798-823). */
int32_t orc_final_partition(const orc_state* s, int32_t* ids);
/* m - (valid slots)/2 (cuda/devPartition.h:741-759). */
uint64_t orc_num_cut_edges(const orc_state* s);

/* Accessors (pointers stay valid until the next call that changes the state). */
uint32_t orc_n_active(const orc_state* s);
uint32_t orc_n_clusters(const orc_state* s);
uint32_t orc_n_sweep_clusters(const orc_state* s);
uint32_t orc_n_cuts(const orc_state* s);
uint32_t orc_n_data_clusters(const orc_state* s);
int32_t orc_smallest_label(const orc_state* s);
const int32_t* orc_labels(const orc_state* s);
const orc_lnode* orc_active(const orc_state* s);
const uint32_t* orc_internal_degrees(const orc_state* s);
const uint32_t* orc_cols(const orc_state* s);
const uint64_t* orc_keys(const orc_state* s);
const orc_node_data* orc_sorted(const orc_state* s);
const int32_t* orc_sweep_labels(const orc_state* s);
const uint32_t* orc_sweep_volumes(const orc_state* s);
const orc_sweep_cut* orc_all_cuts(const orc_state* s);
const orc_sweep_cut* orc_cuts(const orc_state* s);
const int32_t* orc_data_labels(const orc_state* s);
const orc_cluster_data* orc_cluster_values(const orc_state* s);
/* Certificate record per vertex (no reference counterpart): 0 while the
 * vertex is active; once its cluster is certified, (round + 1) with bit 31
 * set when the certified set differs from the set swept in that round. */
const uint32_t* orc_certificates(const orc_state* s);
/* current potentials widened to double */
void orc_get_potentials(const orc_state* s, double* out);

#ifdef __cplusplus
}
#endif
#endif
