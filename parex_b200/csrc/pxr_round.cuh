// Device state and kernels of one decomposition round (sm_100a).
//
// The round follows the reference's stage order (cuda/device.h:101-168,
// 363-404): walk step, sweep (edge differences, stable sort by
// (cluster, potential), prefix scan, sparsest prefix per cluster), cut,
// connected components, per-cluster reductions, deactivation and recentering,
// edge disabling.  Layout and arithmetic are this project's own:
//
//  * potentials are float; the walk and the per-cluster sums accumulate
//    exactly in int64 fixed point (scale 2^e chosen from the largest |x| and
//    the largest term count), so results do not depend on the order in which
//    threads add terms;
//  * per-cluster tables (start, size, volume, start volume, root vertex) are
//    produced at the end of a round, so the next sweep is a single
//    unsegmented look-back scan: the edge differences of a cluster sum to
//    zero and its start volume is known;
//  * components use lock-free union-find (hook the larger root under the
//    smaller with atomicCAS, path halving), which labels every component by
//    its minimum vertex id, the reference's canonical root;
//  * active vertices are kept twice: `act` in the order of the last sort (the
//    stable sort's tie order) and `ids` in vertex order (coalesced row work).
#pragma once

#include "pxr_common.cuh"
#include "pxr_sort.cuh"

namespace pxr {

// Sweep history of a cluster, carried across relabelling (the learned
// schedule's features).
struct SchedHist {
    float pot;            // potential spread (max - min) at the last sweep
    float sp;             // best sweep sparsity at the last sweep (2 when none)
    uint32_t round;       // round of the last sweep
    uint32_t age;         // sweeps since the cluster was created
};

struct ClusterTables {
    uint32_t* start;      // first sorted position of the cluster
    uint32_t* size;       // vertices
    uint32_t* vol;        // internal volume (sum of internal degrees)
    uint32_t* vol_start;  // exclusive prefix of vol over labels
    uint32_t* root;       // minimum vertex id
    uint64_t* best;       // packed (sparsity bits, ~position) argmin
    uint16_t* skip;       // learned schedule: rounds left before the next sweep
    SchedHist* hist;      // learned schedule: sweep history
};

// Origin of a cluster after the round, stored at its root vertex
// (Dev::rootc): kind << 30 | label of the cluster it came from.
enum : uint32_t { kOriginSwept = 1u, kOriginChild = 2u, kOriginCarried = 3u };
constexpr uint32_t kOriginLabelMask = 0x3FFFFFFFu;

// What the end of a round does with the rows of a cluster (Dev::nflag):
// a cluster born from a split rescans its rows (disables the slots that now
// cross clusters, recounts degrees); one swept but not split keeps its rows
// and only refreshes x / degree after recentring; a carried one is unchanged.
enum : uint8_t { kRowsScan = 0, kRowsKept = 1, kRowsCarried = 2 };

template <typename OffT>
struct Dev {
    // graph
    const OffT* off;
    uint32_t* cols;
    uint32_t n;
    uint32_t nb_bits;     // bit length of max(n, max row length)
    float sc_threshold;
    float rw_threshold;
    uint32_t division;    // PXR_DIV_*
    // per vertex
    int32_t* lab;
    uint32_t* ideg;
    float* x;
    int2* dv;             // {edge difference, internal degree}
    uint32_t* parent;
    uint32_t* acc_max;    // ordered float bits, by root vertex
    uint32_t* acc_min;
    int64_t* acc_sum;
    uint32_t* acc_cnt;
    int32_t* newlab;      // by root vertex
    double* avg;          // by root vertex
    uint32_t* cert;       // per vertex: certificate record (round + 1, bit 31: not the whole swept set)
    // per sorted position
    int32_t* pdif;
    uint32_t* pvol;
    // per cluster
    uint32_t* cut_off;
    uint32_t* rep[2];     // per split cluster: root of its first / last sorted vertex (sampled union)
    unsigned long long* walk_stats;   // [kStatSlots][3]: walk vertices, slots, gathers
    uint32_t union_sampled;   // components by sampled linking (graphs of mean degree >= kSampledDegree)
    uint8_t* split;
    void* allcuts;        // pxr_sweep_cut[]
    // roots after the components stage: a bitmap over vertex ids (zero
    // between rounds), compacted into roots[0] in id order
    uint32_t* roots[2];
    uint32_t* rootmap;
    uint32_t n_words;
    LookbackState lb_roots;
    // look-back state
    LookbackState lb_scan, lb_relabel, lb_apply, lb_ids, lb_cvol;
    uint32_t* lb_epoch;   // [8] current epoch per look-back site
    RoundCtr* ctr;
    SortState sort;
    uint32_t* sort_end_bit;   // main sort bits
    uint32_t light_max;       // rows up to this many slots: W lanes per row in the round kernels
    const uint32_t* wide;     // vertices with light_max < row <= wide_max slots (one warp each)
    uint32_t n_wide;
    const uint32_t* heavy;    // vertices with longer rows (one CTA each)
    uint32_t n_heavy;
    // learned sweep schedule (all zero / null in the plain form)
    uint32_t sched;           // PXR_SCHEDULE_*
    uint32_t trace;           // write per-cluster records each round
    uint8_t* sflag;           // per label this round: bit 0 acted on (due), bit 1 in the sweep,
                              // bit 2 carried with its potential spread already below rw_threshold
    uint32_t* smax;           // per label: max / min ordered potential bits after this round's walk
    uint32_t* smin;           // (learned schedule; identity between rounds)
    uint8_t* nflag;           // per label of the next round: kRows* (rows to rescan or not)
    uint32_t* rootc;          // per root vertex: kind << 30 | old label
    LookbackState lb_sched, lb_emit, lb_carry;
    const float* mlp;         // bf16 weights widened to float, then input mean and scale
    float safety;             // skip = floor(safety * (2^y - 1))
    float cut_gate;           // a round cutting more than cut_gate x its clusters: no skip next round
    uint32_t due_period;      // > 1: clusters come due only in rounds whose index is a multiple of it
    uint32_t max_skip;
    void* records;            // pxr_cluster_record[] when trace is on
};

// Default row bins: rows up to kLightRow slots go W lanes per row, up to
// kWideRow a warp per row, longer rows a CTA per row.
constexpr uint32_t kLightRow = 64;
// Slots a lane loads before it gathers their neighbours' values (loads in
// flight per lane in the row kernels).
#ifndef PXR_SLOT_UNROLL
#define PXR_SLOT_UNROLL 4
#endif
constexpr int kSlotUnroll = PXR_SLOT_UNROLL;
constexpr uint32_t kWideRow = 4096;
// Largest previous-round cluster for which a round's sort runs chunk by
// chunk in shared memory (pxr_chunk.cuh).
constexpr uint32_t kChunkCapRows = 4096;

// look-back sites (index into Dev::lb_epoch and RoundCtr::tile_counter)
enum : int {
    kSiteScan = 0, kSiteRelabel = 1, kSiteApply = 2, kSiteIds = 3, kSiteCvol = 4,
    kSiteFinal = 5, kSiteSched = 6, kSiteEmit = 7, kSiteCarry = 8, kSiteRoots = 9
};

__device__ __forceinline__ uint32_t bitlen(uint32_t v) { return v ? 32u - __clz(v) : 0u; }

// Learned schedule: this round cut more than cut_gate x its clusters, so the
// next round sweeps every cluster (read after the cut, before the round ends).
template <typename OffT>
__device__ __forceinline__ bool cut_gate_on(const Dev<OffT>& d) {
    return d.cut_gate > 0.0f &&
           __uint2float_rn(d.ctr->n_cut_swept) > __fmul_rn(d.cut_gate, __uint2float_rn(d.ctr->n_clusters));
}

// Learned schedule: the next round's skip sk of a cluster of `size`
// vertices.  A small cluster (under 1/kDueSmallShare of the active vertices)
// is held at 1 while the next round's index is not a multiple of
// due_period: the sweeps of small clusters, which each cost a round its
// passes over every active vertex, gather into fewer rounds and the rest
// only walk.  Larger clusters keep their own timing (holding them back lets
// the walk mix past cuts they would have made); after a gated round every
// cluster stays due.
constexpr uint32_t kDueSmallShare = 1024;

template <typename OffT>
__device__ __forceinline__ uint16_t due_aligned(const Dev<OffT>& d, uint32_t sk, uint32_t size) {
    const uint32_t P = d.due_period;
    if (sk == 0 && P > 1 && (d.ctr->rounds + 1u) % P != 0u && (uint64_t)size * kDueSmallShare < d.ctr->n_active &&
        !cut_gate_on(d))
        return 1u;
    return (uint16_t)sk;
}

}  // namespace pxr
