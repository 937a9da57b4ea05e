// Kernels of one decomposition round (sm_100a).  See pxr_round.cuh for the
// data layout.  Every kernel reads its item counts from RoundCtr, so launches
// use host-side capacities and a round can be captured in a CUDA graph.
#pragma once

#include "pxr_round.cuh"
#include "../../include/parex_b200.h"

namespace pxr {

constexpr int kBlock = 256;
// Walk kernels: CTAs per SM their register budget is sized for, and whether
// the long-row kernels load the next row's head while gathering this row.
// The walk is latency-bound (its gathers wait on L2); eight 256-thread CTAs
// per SM (32 registers, a few bytes spilled) beat five (44 registers): on
// R-MAT 24 one walk step took 2.11 instead of 2.32 ms, and the prefetch made
// it slower at either bound (measured on a B200).
#ifndef PXR_WALK_PREFETCH
#define PXR_WALK_PREFETCH 0
#endif
#ifndef PXR_WALK_MIN_BLOCKS
#define PXR_WALK_MIN_BLOCKS 8
#endif
#if PXR_WALK_MIN_BLOCKS > 0
#define PXR_WALK_BOUNDS __launch_bounds__(kBlock, PXR_WALK_MIN_BLOCKS)
#else
#define PXR_WALK_BOUNDS __launch_bounds__(kBlock)
#endif
constexpr int kScanItems = 8;                        // items per thread in look-back kernels
constexpr int kScanTile = kBlock * kScanItems;
// k_relabel runs over the roots, often far fewer than the vertices: smaller
// tiles keep more of its latency-bound gathers in flight
constexpr int kRelabelItems = 2;
constexpr int kRelabelTile = kBlock * kRelabelItems;

// ---------------------------------------------------------------------------
// Run aggregation: a thread holds the aggregates of the runs of equal keys in
// its consecutive items; the interior runs are emitted by the caller, the
// first and last fragments here.  A warp (or the whole block) whose threads
// all hold one run of the same key emits a single combined atomic.

template <class Agg>
__device__ __forceinline__ void emit_fragments(bool has, bool single, uint32_t k_first,
                                               typename Agg::T a_first, uint32_t k_last,
                                               typename Agg::T a_last, const Agg& agg) {
    using T = typename Agg::T;
    __shared__ uint32_t s_uni[kBlock / 32];
    __shared__ uint32_t s_key[kBlock / 32];
    __shared__ T s_agg[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t k0 = __shfl_sync(0xFFFFFFFFu, k_first, 0);
    const bool uni = __all_sync(0xFFFFFFFFu, has && single && k_first == k0);
    T w = uni ? a_first : Agg::identity();
    if (uni) w = Agg::warp_reduce(w);
    if (lane == 0) { s_uni[warp] = uni; s_key[warp] = k0; s_agg[warp] = w; }
    __syncthreads();
    bool block_uni = true;
#pragma unroll
    for (int i = 0; i < kBlock / 32; ++i) block_uni &= s_uni[i] && s_key[i] == s_key[0];
    if (block_uni) {
        if (threadIdx.x == 0) {
            T t = s_agg[0];
            for (int i = 1; i < kBlock / 32; ++i) t = Agg::combine(t, s_agg[i]);
            agg.emit(s_key[0], t);
        }
    } else if (uni) {
        if (lane == 0) agg.emit(k0, w);
    } else if (has) {
        agg.emit(k_first, a_first);
        if (!single) agg.emit(k_last, a_last);
    }
    __syncthreads();
}

// argmin of packed (sparsity bits << 32 | ~position): smaller sparsity wins,
// equal sparsity goes to the later position (the reference's ArgMinOp keeps
// its right operand on ties, cuda/devSweepCut.h:356-361).
struct ArgminAgg {
    using T = unsigned long long;
    unsigned long long* best;
    __device__ static T identity() { return ~0ull; }
    __device__ static T combine(T a, T b) { return a < b ? a : b; }
    __device__ static T warp_reduce(T v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const T u = __shfl_xor_sync(0xFFFFFFFFu, v, o);
            v = u < v ? u : v;
        }
        return v;
    }
    __device__ void emit(uint32_t key, T v) const { atomicMin(&best[key], v); }
};

struct ClusterAcc {
    uint32_t mx, mn;
    int64_t sum;
    uint32_t cnt;
};

struct DataAgg {
    using T = ClusterAcc;
    uint32_t* acc_max;
    uint32_t* acc_min;
    int64_t* acc_sum;
    uint32_t* acc_cnt;
    __device__ static T identity() { return {0u, 0xFFFFFFFFu, 0, 0u}; }
    __device__ static T combine(T a, T b) {
        return {a.mx > b.mx ? a.mx : b.mx, a.mn < b.mn ? a.mn : b.mn, a.sum + b.sum, a.cnt + b.cnt};
    }
    __device__ static T warp_reduce(T v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            T u;
            u.mx = __shfl_xor_sync(0xFFFFFFFFu, v.mx, o);
            u.mn = __shfl_xor_sync(0xFFFFFFFFu, v.mn, o);
            u.sum = __shfl_xor_sync(0xFFFFFFFFu, v.sum, o);
            u.cnt = __shfl_xor_sync(0xFFFFFFFFu, v.cnt, o);
            v = combine(v, u);
        }
        return v;
    }
    __device__ void emit(uint32_t key, T v) const {
        atomicMax(&acc_max[key], v.mx);
        atomicMin(&acc_min[key], v.mn);
        atomic_add_i64(&acc_sum[key], v.sum);
        atomicAdd(&acc_cnt[key], v.cnt);
    }
};

struct CountAgg {
    using T = uint32_t;
    uint32_t* dst;
    __device__ static T identity() { return 0u; }
    __device__ static T combine(T a, T b) { return a + b; }
    __device__ static T warp_reduce(T v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        return v;
    }
    __device__ void emit(uint32_t key, T v) const { atomicAdd(&dst[key], v); }
};

// ---------------------------------------------------------------------------
// dynamic tile id + epoch for a look-back site

__device__ __forceinline__ uint32_t fetch_tile(RoundCtr* ctr, int site) {
    __shared__ uint32_t s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctr->tile_counter[site], 1u);
    __syncthreads();
    return s_tile;
}

__device__ __forceinline__ uint32_t sorted_sel(const SortState& s) { return s.pass_info[kMaxPasses]; }


// Column indices are read once per round and stream through: load them with
// an evict-first hint so that the potentials the gathers read stay in L2.
__device__ __forceinline__ uint32_t stream_col(const uint32_t* p) { return __ldcs(p); }

// ---------------------------------------------------------------------------
// round bookkeeping

// stage: 0 before the walk, 1 before the sweep, 2 before the cut
// In the graph driver, the global sort and the chunked sort of stage 1 sit
// under two IF nodes whose conditions (gsort, chunk) are set here.
template <typename OffT>
__global__ void k_round_prep(Dev<OffT> d, int stage, cudaGraphConditionalHandle gsort = 0,
                             cudaGraphConditionalHandle chunk = 0) {
    pdl_wait();
    pdl_launch_next();
    RoundCtr* c = d.ctr;
    // one warp: lane i resets look-back site i, lane 0 does the rest (the
    // sites' dependent read-modify-writes in one thread took ~4 us)
    const uint32_t lane = threadIdx.x;
    if (lane < (uint32_t)kSites) {
        c->tile_counter[lane] = 0;
        d.lb_epoch[lane] += 1;
    }
    if (lane != 0) return;
    if (stage == 2) c->n_cut_swept = c->n_cut;   // the sweep's count, read by the cut stage
    c->n_cut = 0;
    c->n_roots = 0;
    if (stage == 0) {
        c->xmax_walk_bits = 0;
        c->walk_only = 0;
    }
    c->smallest_next = 0;
    c->n_keep = 0;
    c->n_active_next = 0;
    if (stage == 1) {
        c->n_due_items = 0;
        c->any_split = 0;
        if (d.sched) c->n_sweep = 0;   // set by k_due_scan
    }
    if (!d.sched) c->n_sweep = c->n_active;
    if (stage == 1) {
        // every previous cluster fits a chunk: sort in shared memory (pxr_chunk.cuh)
        c->chunk_path = (!d.sched && c->max_parent <= kChunkCapRows && c->n_active > 0) ? 1u : 0u;
        c->n_gsort = c->chunk_path ? 0u : c->n_sweep;
        if (c->chunk_path) {   // the chunked sort reads and writes every item once
            c->stat_sort_items += c->n_sweep;
            c->stat_sort_passes += 1;
        }
        // the chunked sort leaves its output in buffer 0 (the global sort,
        // when it runs with no items, selects buffer 0 as well)
        if (c->chunk_path) d.sort.pass_info[kMaxPasses] = 0u;
        if (gsort) {
            cudaGraphSetConditional(gsort, c->chunk_path ? 0u : 1u);
            cudaGraphSetConditional(chunk, c->chunk_path ? 1u : 0u);
            if (c->chunk_path) c->stat_chunk_slots += 1; else c->stat_gsort_slots += 1;
        }
    }
    if (stage == 2) c->max_csize_next = 0;
    const uint32_t k = c->n_clusters;
    *d.sort_end_bit = 32u + bitlen(k > 0 ? k - 1 : 0);
}

template <typename OffT>
__global__ void k_after_walk(Dev<OffT> d) {
    pdl_wait();
    pdl_launch_next();
    d.ctr->xmax_bits = d.ctr->xmax_walk_bits;
}

template <typename OffT>
__global__ void k_round_end(Dev<OffT> d) {
    pdl_wait();
    pdl_launch_next();
    RoundCtr* c = d.ctr;
    if (c->n_active > 0) {
        c->rounds += 1;
        c->stat_swept_items += c->n_sweep;
    }
    // the next active list holds this round's clusters as contiguous runs
    // (the learned schedule appends carried clusters: no chunk path)
    c->max_parent = d.sched ? 0xFFFFFFFFu : c->max_csize;
    c->max_csize = c->max_csize_next;
    c->n_active = c->n_active_next;
    c->n_clusters = c->n_keep;
    c->smallest = c->smallest_next;
    c->full_components = 0;
    c->done = (c->n_active == 0 || c->n_clusters == 0) ? 1u : 0u;
}

// device-driven round loop: keep looping while clusters remain and the cap allows
template <typename OffT>
__global__ void k_loop_cond(Dev<OffT> d, cudaGraphConditionalHandle cond) {
    pdl_wait();
    const RoundCtr* c = d.ctr;
    const bool more = !c->done && c->err == 0 && (c->rounds - c->loop_start) < c->loop_cap;
    cudaGraphSetConditional(cond, more ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// walk: x'[v] = 0.9 * sum_{u ~ v, valid} x[u]/d(u) + 0.1 * x[v]
// (fusedRandomWalk_WarpParallel, cuda/devRandomWalk.h:117-203), W lanes per
// vertex, vertices in id order, exact fixed-point sum.

// Block-wide max of v, then one atomicMax per block on `addr` (atomics from
// every warp on one word queue behind each other at its L2 slice).  Every
// thread of the block must call it.
__device__ __forceinline__ void block_atomic_max(uint32_t* addr, uint32_t v) {
    __shared__ uint32_t s_m[kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    if ((threadIdx.x & 31u) == 0) s_m[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t q = 1; q < blockDim.x / 32; ++q) v = max(v, s_m[q]);
        if (v) atomicMax(addr, v);
    }
    __syncthreads();
}

// The walk's max |x'| and traffic counters: summed per block, then one
// atomic per counter and block, the counters spread over kStatSlots slots
// (per-warp atomics on four words cost 3 of 27 ms on the 128^3 grid).
template <typename OffT>
__device__ __forceinline__ void walk_block_totals(const Dev<OffT>& d, uint32_t vmax, unsigned long long st_v,
                                                  unsigned long long st_s, unsigned long long st_g) {
    __shared__ uint32_t s_vmax[kBlock / 32];
    __shared__ unsigned long long s_st[3][kBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
        st_v += __shfl_xor_sync(0xFFFFFFFFu, st_v, o);
        st_s += __shfl_xor_sync(0xFFFFFFFFu, st_s, o);
        st_g += __shfl_xor_sync(0xFFFFFFFFu, st_g, o);
    }
    const uint32_t w = threadIdx.x >> 5;
    if ((threadIdx.x & 31u) == 0) {
        s_vmax[w] = vmax;
        s_st[0][w] = st_v;
        s_st[1][w] = st_s;
        s_st[2][w] = st_g;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t q = 1; q < blockDim.x / 32; ++q) {
            vmax = max(vmax, s_vmax[q]);
            st_v += s_st[0][q];
            st_s += s_st[1][q];
            st_g += s_st[2][q];
        }
        if (vmax) atomicMax(&d.ctr->xmax_walk_bits, vmax);
        unsigned long long* slot = d.walk_stats + 3 * (blockIdx.x % kStatSlots);
        if (st_v) atomicAdd(&slot[0], st_v);
        if (st_s) atomicAdd(&slot[1], st_s);
        if (st_g) atomicAdd(&slot[2], st_g);
    }
}

template <typename OffT, int W>
__global__ void PXR_WALK_BOUNDS k_walk(Dev<OffT> d, const uint32_t* ids, const float* xt_in,
                                                 float* xt_out) {
    pdl_wait();
    const uint32_t count = d.ctr->n_active;
    const int e = fixed_exponent(d.ctr->xmax_bits, d.nb_bits);
    const double scale = pow2(e), inv = pow2(-e);
    const uint32_t gl = threadIdx.x & (W - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / W;
    const uint32_t warp0 = ((blockIdx.x * blockDim.x + threadIdx.x) & ~31u) / W;
    uint32_t vmax = 0;
    unsigned long long st_v = 0, st_s = 0, st_g = 0;
    for (uint32_t j0 = warp0; j0 < count; j0 += groups) {
        const uint32_t j = j0 + (threadIdx.x & 31u) / W;
        const bool valid = j < count;
        uint32_t v = valid ? ids[j] : 0u;
        OffT beg = valid ? d.off[v] : 0, end = valid ? d.off[v + 1] : 0;
        const bool light = valid && (uint64_t)(end - beg) <= d.light_max;
        if (!light) beg = end;      // long rows: k_walk_long
        int64_t acc = 0;
        for (OffT s = beg + gl; s < end; s += kSlotUnroll * W) {
            uint32_t nb[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) nb[u] = s + u * W < end ? stream_col(d.cols + s + u * W) : kInvalidEdge;
            float xv[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) xv[u] = slot_valid(nb[u]) ? xt_in[nb[u]] : 0.0f;
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) {
                st_s += s + u * W < end ? 1 : 0;
                if (slot_valid(nb[u])) { acc += to_fixed(xv[u], scale); ++st_g; }
            }
        }
        st_v += (light && gl == 0) ? 1 : 0;
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o, W);
        if (light && gl == 0) {
            const double sum = __dmul_rn(__ll2double_rn(acc), inv);
            const double val = __dadd_rn(__dmul_rn(sum, 0.9), __dmul_rn((double)d.x[v], 0.1));
            const float xv = __double2float_rn(val);
            d.x[v] = xv;
            const uint32_t dg = d.ideg[v];
            xt_out[v] = dg ? __double2float_rn(__ddiv_rn((double)xv, (double)dg)) : 0.0f;
            const uint32_t b = __float_as_uint(fabsf(xv));
            vmax = b > vmax ? b : vmax;
        }
    }
    walk_block_totals(d, vmax, st_v, st_s, st_g);
}

// ---------------------------------------------------------------------------
// edge differences (nodeDiffKernel_Sparse_WarpParallel, cuda/devSweepCut.h:20-112):
// +1 per valid neighbour after v in (potential, id) order, -1 per neighbour before.

// A sweep set at most 1 / kSweepListShare of the active list is walked as a list.
constexpr uint32_t kSweepListShare = 8;

// ids: the active list in vertex order (count n_active), or with sweep_list
// the sweep set as the learned schedule's emit compacted it (count n_sweep,
// every entry swept).
//
// The learned schedule launches both forms; one returns at once: the sweep
// set (in the last sort's order, so its rows are scattered) when it is a
// small part of the active list, the vertex-order scan (coalesced) when it
// holds a large cluster.
template <typename OffT, int W>
__global__ void __launch_bounds__(kBlock) k_nodediff(Dev<OffT> d, const uint32_t* ids, int sweep_list = 0) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    if (d.sched) {
        const bool small = (uint64_t)d.ctr->n_sweep * kSweepListShare <= d.ctr->n_active;
        if (sweep_list ? !small : small) return;
    }
    const uint32_t count = sweep_list ? d.ctr->n_sweep : d.ctr->n_active;
    const uint32_t gl = threadIdx.x & (W - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / W;
    const uint32_t warp0 = ((blockIdx.x * blockDim.x + threadIdx.x) & ~31u) / W;
    for (uint32_t j0 = warp0; j0 < count; j0 += groups) {
        const uint32_t j = j0 + (threadIdx.x & 31u) / W;
        const bool valid = j < count;
        uint32_t v = valid ? ids[j] : 0u;
        const bool in = valid && (sweep_list || !d.sched || ((uint32_t)d.lab[v] < d.n && (d.sflag[d.lab[v]] & 2u)));
        if (!in) v = 0u;
        const uint32_t mine = in ? ordered_bits(d.x[v]) : 0u;
        OffT beg = in ? d.off[v] : 0, end = in ? d.off[v + 1] : 0;
        const bool light = in && (uint64_t)(end - beg) <= d.light_max;
        if (!light) beg = end;      // long rows: k_nodediff_long
        int32_t c = 0;
        for (OffT s = beg + gl; s < end; s += kSlotUnroll * W) {
            uint32_t nb[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) nb[u] = s + u * W < end ? stream_col(d.cols + s + u * W) : kInvalidEdge;
            float xn[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) xn[u] = slot_valid(nb[u]) ? d.x[nb[u]] : 0.0f;
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) {
                if (!slot_valid(nb[u])) continue;
                const uint32_t o = ordered_bits(xn[u]);
                const bool before = o < mine || (o == mine && nb[u] < v);
                c += before ? -1 : 1;
            }
        }
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o, W);
        if (light && gl == 0) d.dv[v] = make_int2(c, (int)d.ideg[v]);
    }
}

// sort keys in the order of the last sort: (label << 32) | ordered potential
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_emit(Dev<OffT> d, const uint32_t* act, uint64_t* keys,
                                                 uint32_t* vals, uint64_t* best) {
    pdl_wait();
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    const bool emit = !d.ctr->chunk_path;   // the chunk path reads the active list itself
    const uint32_t lim = emit ? max(count, k) : k;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
        if (emit && i < count) {
            const uint32_t v = act[i];
            keys[i] = ((uint64_t)(uint32_t)d.lab[v] << 32) | ordered_bits(d.x[v]);
            vals[i] = v;
        }
        if (i < k) best[i] = ~0ull;
    }
}

// ---------------------------------------------------------------------------
// sweep scan: inclusive prefix of (edge difference, volume) over the sorted
// order with a decoupled look-back, then the sparsity of every prefix and the
// per-cluster argmin (SweepCutTransform + ArgMinOp, cuda/devSweepCut.h:374-433, 665-688).

__device__ __forceinline__ float sweep_ratio(uint32_t num, uint32_t den, uint32_t division) {
    if (division == PXR_DIV_REFERENCE) return __fdividef((float)num, (float)den);
    return __fdiv_rn((float)num, (float)den);
}

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_sweep_scan(Dev<OffT> d, ClusterTables t, const uint64_t* keys0,
                                                       const uint64_t* keys1, const uint32_t* vals0,
                                                       const uint32_t* vals1) {
    pdl_wait();
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_sweep;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteScan);
    if (tile >= ntiles) return;
    const uint32_t sel = sorted_sel(d.sort);
    if (tile == 0 && threadIdx.x == 0) {
        d.ctr->main_sel = sel;
        d.ctr->sweep_n = count;
        d.ctr->sweep_k = d.ctr->n_clusters;
    }
    const uint64_t* keys = sel ? keys1 : keys0;
    const uint32_t* vals = sel ? vals1 : vals0;
    const uint32_t epoch = d.lb_epoch[kSiteScan];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;

    uint32_t lab[kScanItems];
    uint64_t pre[kScanItems];
    uint64_t run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        uint64_t val = 0;
        lab[k] = 0;
        if (i < count) {
            lab[k] = (uint32_t)(keys[i] >> 32);
            const int2 dv = d.dv[vals[i]];
            val = ((uint64_t)(uint32_t)dv.y << 32) | (uint32_t)dv.x;
        }
        run = PairAdd::combine(run, val);
        pre[k] = run;
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<PairAdd>(run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<PairAdd>(d.lb_scan, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    // exclusive prefix of this thread = tile exclusive + (block inclusive - own run)
    const uint32_t lo = (uint32_t)incl - (uint32_t)run;
    const uint32_t hi = (uint32_t)(incl >> 32) - (uint32_t)(run >> 32);
    const uint64_t texcl = PairAdd::combine(s_excl, ((uint64_t)hi << 32) | lo);

    bool has = false, single = true;
    uint32_t k_first = 0, k_last = 0;
    unsigned long long a_first = ~0ull, a_last = ~0ull;
    ArgminAgg am{reinterpret_cast<unsigned long long*>(t.best)};
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        if (i >= count) break;
        const uint64_t p = PairAdd::combine(texcl, pre[k]);
        const uint32_t c = lab[k];
        const int32_t ldif = (int32_t)(uint32_t)p;
        const uint32_t lvol = (uint32_t)(p >> 32) - t.vol_start[c];
        const uint32_t tot = t.vol[c];
        const uint32_t denom = lvol >= tot ? 0u : (lvol < tot - lvol ? lvol : tot - lvol);
        const float sp = denom > 0 ? sweep_ratio((uint32_t)ldif, denom, d.division) : 2.0f;
        d.pdif[i] = ldif;
        d.pvol[i] = lvol;
        const unsigned long long cand = ((unsigned long long)__float_as_uint(sp) << 32) | (uint32_t)~i;
        if (!has) {
            has = true; k_first = c; a_first = cand; k_last = c; a_last = cand;
        } else if (c == k_last) {
            a_last = cand < a_last ? cand : a_last;
            if (single) a_first = a_last;
        } else {
            if (!single) am.emit(k_last, a_last);
            single = false;
            k_last = c;
            a_last = cand;
        }
    }
    emit_fragments<ArgminAgg>(has, single, k_first, a_first, k_last, a_last, am);
}

// per cluster: the best cut, the threshold test (CheckThreshold,
// cuda/devSweepCut.h:321-331, 701-709) and the components plan.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cluster_cut(Dev<OffT> d, ClusterTables t) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t full = d.ctr->full_components;
    pxr_sweep_cut* cuts = reinterpret_cast<pxr_sweep_cut*>(d.allcuts);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < k; c += gridDim.x * blockDim.x) {
        const uint32_t fl = d.sched ? d.sflag[c] : 3u;   // bit 0 acted on, bit 1 swept
        const bool acted = fl & 1u, swept = fl & 2u;
        const uint64_t b = t.best[c];
        const uint32_t pos = ~(uint32_t)b;
        const float sp = swept ? __uint_as_float((uint32_t)(b >> 32)) : 2.0f;
        const uint32_t off = swept ? pos - t.start[c] + 1u : 0u;
        cuts[c].label = (int32_t)c;
        cuts[c].sparsity = sp;
        cuts[c].offset = off;
        const bool cut = acted && sp < d.sc_threshold;
        d.cut_off[c] = cut ? off : kNoCut;
        const bool split = acted && (cut || full);
        d.split[c] = split ? 1 : 0;
        const uint32_t am = __activemask();
        const uint32_t splits = __ballot_sync(am, split);
        if (split && (splits & lanemask_lt()) == 0u) d.ctr->any_split = 1u;   // one store per warp
        const uint32_t cuts_in_warp = __ballot_sync(__activemask(), cut);
        if (cut && (cuts_in_warp & lanemask_lt()) == 0u) atomicAdd(&d.ctr->n_cut, (uint32_t)__popc(cuts_in_warp));
        if (!acted && swept && sp < d.sc_threshold) atomicAdd(&d.ctr->stat_false_stops, 1ull);
        if (acted && !split) d.rootc[t.root[c]] = (kOriginSwept << 30) | c;
        if (acted && !split) {
            const uint32_t r = t.root[c];
            d.acc_max[r] = 0u;
            d.acc_min[r] = 0xFFFFFFFFu;
            d.acc_sum[r] = 0;
            d.acc_cnt[r] = 0u;
        }
    }
}

// ---------------------------------------------------------------------------
// cut (PartitionManager::cutClusters, cuda/devPartition.h:545-622): in a cut
// cluster, positions past the chosen prefix take a fresh label; every vertex
// of a split cluster becomes its own union-find root.

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cut_init(Dev<OffT> d, ClusterTables t, const uint32_t* vals0,
                                                     const uint32_t* vals1, const uint64_t* keys0,
                                                     const uint64_t* keys1) {
    pdl_wait();
    const uint32_t count = d.ctr->n_sweep;
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t sel = d.ctr->main_sel;
    const uint32_t* vals = sel ? vals1 : vals0;
    const uint64_t* keys = sel ? keys1 : keys0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t c = (uint32_t)(keys[i] >> 32);
        if (!d.split[c]) continue;
        const uint32_t v = vals[i];
        const uint32_t co = d.cut_off[c];
        const uint32_t pos = i - t.start[c] + 1u;
        d.lab[v] = (co != kNoCut && pos > co) ? (int32_t)(k + c) : (int32_t)c;
    }
}

// cluster a vertex belonged to this round, or k when it is not in a split
// cluster (after k_cut_init, labels of a split cluster c are c or k + c)
template <typename OffT>
__device__ __forceinline__ bool in_split(const Dev<OffT>& d, uint32_t k, int32_t lv) {
    const uint32_t c = (uint32_t)lv >= k ? (uint32_t)lv - k : (uint32_t)lv;
    return lv >= 0 && c < k && d.split[c];
}

// Every parent pointer points to a smaller id (roots are hooked under smaller
// roots), so a component's root is its minimum vertex and atomicMin can only
// move a pointer closer to the root.  find() splits the path as it walks
// with atomicMin, so a stored root is never replaced by a non-root ancestor.
__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t v) {
    uint32_t p = ld_relaxed(&parent[v]);
    while (p != v) {
        const uint32_t gp = ld_relaxed(&parent[p]);
        if (gp < p) atomicMin(&parent[v], gp);
        v = p;
        p = gp;
    }
    return v;
}

// Root of v, left in parent[v] (the atomic only where v's parent is not the root).
__device__ __forceinline__ uint32_t uf_find_flat(uint32_t* parent, uint32_t v) {
    const uint32_t p0 = ld_relaxed(&parent[v]);
    const uint32_t r = p0 == v ? v : uf_find(parent, p0);
    if (r != p0) atomicMin(&parent[v], r);
    return r;
}

// The three linking kernels walk this round's active list in vertex order
// (the walk's list), so rows, labels and parent words of neighbouring ids are
// read together; the forest they build does not depend on the order.
//
// First linking pass: each vertex of a split cluster points to its smallest
// same-label neighbour below it (rows are sorted, so the first one found), or
// to itself.  Only the owning thread writes parent[v] here; the vertex's
// accumulators for the component data start from the identity.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_link_first(Dev<OffT> d, const uint32_t* ids) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    if (!d.ctr->any_split) return;   // no cluster split: no components to find
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const uint32_t v = ids[j];
        const int32_t lv = d.lab[v];
        if (!in_split(d, k, lv)) continue;
        const OffT beg = d.off[v], end = d.off[v + 1];
        uint32_t p = v;
        for (OffT s = beg; s < end; ++s) {
            const uint32_t nb = d.cols[s];
            if (!slot_valid(nb)) continue;  // disabled slots keep their place in the sorted row
            if (nb >= v) break;                // no smaller neighbour left
            if (d.lab[nb] == lv) { p = nb; break; }
        }
        d.parent[v] = p;
        d.acc_max[v] = 0u;
        d.acc_min[v] = 0xFFFFFFFFu;
        d.acc_sum[v] = 0;
        d.acc_cnt[v] = 0u;
    }
}

// Flatten the linked forest: every vertex of a split cluster points at its root.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_compress(Dev<OffT> d, const uint32_t* ids) {
    pdl_wait();
    if (d.ctr->walk_only) return;
    if (!d.ctr->any_split) return;   // no cluster split: no components to find
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const uint32_t v = ids[j];
        if (!in_split(d, k, d.lab[v])) continue;
        uf_find_flat(d.parent, v);
    }
}

// Join the sets of v and nb (both in a split cluster, same label).  hint is
// a word of v's set: when nb's parent is it, the two are joined already.
__device__ __forceinline__ void uf_join(uint32_t* parent, uint32_t* err, uint32_t v, uint32_t nb, uint32_t& hint) {
    if (ld_relaxed(&parent[nb]) == hint) return;
    uint32_t a = v, b = nb;
    for (uint32_t tries = 0;; ++tries) {
        if (tries > kSpinLimit) { atomicOr(err, kErrUnionFind); return; }
        const uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
        if (ra == rb) { hint = ra; return; }
        const uint32_t hi = ra > rb ? ra : rb, lo = ra > rb ? rb : ra;
        if (atomicCAS(&parent[hi], hi, lo) == hi) { hint = lo; return; }
        a = hi;
        b = lo;
    }
}

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16; x *= 0x7FEB352Du; x ^= x >> 15; x *= 0x846CA68Bu; x ^= x >> 16;
    return x;
}

// Sampled linking: each vertex of a split cluster joins one more same-label
// neighbour, picked by a hash of its id.  With the first-link forest this
// usually leaves one large set per label.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_union_sample(Dev<OffT> d, const uint32_t* ids) {
    pdl_wait();
    if (d.ctr->walk_only) return;
    if (!d.ctr->any_split) return;   // no cluster split: no components to find
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const uint32_t v = ids[j];
        const int32_t lv = d.lab[v];
        if (!in_split(d, k, lv)) continue;
        const OffT beg = d.off[v], end = d.off[v + 1];
        if (end == beg) continue;
        const uint32_t nb = d.cols[beg + (OffT)(mix32(v) % (uint64_t)(end - beg))];
        if (!slot_valid(nb) || d.lab[nb] != lv) continue;
        uint32_t hint = ld_relaxed(&d.parent[v]);
        uf_join(d.parent, &d.ctr->err, v, nb, hint);
    }
}

// Representatives: per split cluster, the root of its first sorted vertex
// (label c) and, when cut, of its last (label k + c).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_union_reps(Dev<OffT> d, ClusterTables t, const uint32_t* vals0,
                                                       const uint32_t* vals1) {
    pdl_wait();
    if (d.ctr->walk_only || !d.ctr->any_split) return;
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t* vals = d.ctr->main_sel ? vals1 : vals0;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < k; c += gridDim.x * blockDim.x) {
        if (!d.split[c]) continue;
        const uint32_t st = t.start[c], sz = t.size[c];
        d.rep[0][c] = uf_find(d.parent, vals[st]);
        if (d.cut_off[c] != kNoCut && sz > 0) d.rep[1][c] = uf_find(d.parent, vals[st + sz - 1]);
    }
}

// union over same-label valid edges (ConsolidationManager::consolidate,
// cuda/devConsolidate.h:46-112, 168-204), each undirected edge once (from its
// larger end; rows are sorted, so a lane stops at the first neighbour >= v).
// With the sampled linking (d.union_sampled), a vertex whose set is its
// label's representative set skips its row, and the others join every
// same-label neighbour: an edge is then either joined from an end outside
// that set or has both ends inside it.  Without it, every edge is joined
// once, from its larger end.
template <typename OffT>
__device__ __forceinline__ bool union_skip_row(const Dev<OffT>& d, uint32_t k, uint32_t v, int32_t lv,
                                               uint32_t& hint) {
    if (!d.union_sampled) {
        hint = ld_relaxed(&d.parent[v]);
        return false;
    }
    const uint32_t c = (uint32_t)lv >= k ? (uint32_t)lv - k : (uint32_t)lv;
    const uint32_t rep = (uint32_t)lv >= k ? d.rep[1][c] : d.rep[0][c];
    hint = uf_find(d.parent, v);
    return hint == rep;
}

template <typename OffT, int W>
__global__ void __launch_bounds__(kBlock) k_union(Dev<OffT> d, const uint32_t* ids) {
    pdl_wait();
    if (d.ctr->walk_only || !d.ctr->any_split) return;
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t gl = threadIdx.x & (W - 1);
    const uint32_t groups = (gridDim.x * blockDim.x) / W;
    for (uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) / W; j < count; j += groups) {
        const uint32_t v = ids[j];
        const int32_t lv = d.lab[v];
        if (!in_split(d, k, lv)) continue;
        const OffT beg = d.off[v], end = d.off[v + 1];
        if ((uint64_t)(end - beg) > d.light_max) continue;   // k_union_long
        uint32_t hint;
        if (union_skip_row(d, k, v, lv, hint)) continue;
        for (OffT s = beg + gl; s < end; s += W) {
            const uint32_t nb = d.cols[s];
            if (!slot_valid(nb) || nb == v) continue;
            if (!d.union_sampled && nb > v) break;   // each edge once, from its larger end
            if (d.lab[nb] == lv) uf_join(d.parent, &d.ctr->err, v, nb, hint);
        }
    }
}

// root registry: one bit per vertex id
template <typename OffT>
__device__ __forceinline__ void mark_root(const Dev<OffT>& d, uint32_t r) {
    atomicOr(&d.rootmap[r >> 5], 1u << (r & 31u));
}

// roots, per-cluster data (computeClusterData, cuda/devPartition.h:380-411)
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_components_data(Dev<OffT> d, ClusterTables t, const uint32_t* vals0,
                                                            const uint32_t* vals1, const uint64_t* keys0,
                                                            const uint64_t* keys1) {
    pdl_wait();
    // the sorted order: a cluster's items are contiguous, so runs of one root
    // are long and the per-root atomics few
    const uint32_t count = d.ctr->n_sweep;
    const uint32_t sel = d.ctr->main_sel;
    const uint32_t* vals = sel ? vals1 : vals0;
    const uint64_t* keys = sel ? keys1 : keys0;
    const int e = fixed_exponent(d.ctr->xmax_walk_bits, d.nb_bits);
    const double scale = pow2(e);
    DataAgg agg{d.acc_max, d.acc_min, d.acc_sum, d.acc_cnt};
    const uint32_t stride = gridDim.x * kScanTile;
    for (uint32_t base = blockIdx.x * kScanTile; base < count; base += stride) {
        const uint32_t first = base + threadIdx.x * kScanItems;
        bool has = false, single = true;
        uint32_t k_first = 0, k_last = 0;
        ClusterAcc a_first = DataAgg::identity(), a_last = DataAgg::identity();
        for (int k = 0; k < kScanItems; ++k) {
            const uint32_t i = first + k;
            if (i >= count) break;
            const uint32_t c = (uint32_t)(keys[i] >> 32);
            if (d.sched && !(d.sflag[c] & 1u)) continue;   // carried (swept for the audit only)
            const uint32_t v = vals[i];
            uint32_t r;
            if (d.split[c]) {
                r = uf_find_flat(d.parent, v);
                if (r == v) {
                    mark_root(d, r);
                    d.rootc[r] = (kOriginChild << 30) | c;
                }
            } else {
                r = t.root[c];
                if (i == t.start[c]) mark_root(d, r);
            }
            const float xv = d.x[v];
            const uint32_t ob = ordered_bits(xv);
            const ClusterAcc cur{ob, ob, to_fixed(xv, scale), 1u};
            if (!has) {
                has = true; k_first = r; a_first = cur; k_last = r; a_last = cur;
            } else if (r == k_last) {
                a_last = DataAgg::combine(a_last, cur);
                if (single) a_first = a_last;
            } else {
                if (!single) agg.emit(k_last, a_last);
                single = false;
                k_last = r;
                a_last = cur;
            }
        }
        emit_fragments<DataAgg>(has, single, k_first, a_first, k_last, a_last, agg);
    }
}

// ---------------------------------------------------------------------------
// roots in vertex-id order: the root bitmap compacted with a decoupled
// look-back over tiles of kRootWords words per thread; the words are cleared
// as they are read, so the bitmap is zero again for the next round.

constexpr int kRootWords = 4;
constexpr uint32_t kRootTileWords = kBlock * kRootWords;

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_root_compact(Dev<OffT> d, uint32_t* roots) {
    pdl_wait();
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    const uint32_t nw = d.n_words;
    const uint32_t ntiles = (nw + kRootTileWords - 1) / kRootTileWords;
    const uint32_t tile = fetch_tile(d.ctr, kSiteRoots);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteRoots];
    const uint32_t w0 = tile * kRootTileWords + threadIdx.x * kRootWords;
    uint32_t words[kRootWords];
    uint32_t cnt = 0;
#pragma unroll
    for (int q = 0; q < kRootWords; ++q) {
        const uint32_t w = w0 + q;
        words[q] = w < nw ? d.rootmap[w] : 0u;
        if (words[q]) d.rootmap[w] = 0u;
        cnt += __popc(words[q]);
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)cnt, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_roots, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) {
            s_excl = ex;
            if (tile == ntiles - 1) d.ctr->n_roots = (uint32_t)(ex + tile_total);
        }
    }
    __syncthreads();
    uint32_t pos = (uint32_t)(s_excl + incl - cnt);
#pragma unroll
    for (int q = 0; q < kRootWords; ++q) {
        uint32_t bits = words[q];
        while (bits) {
            roots[pos++] = ((w0 + q) << 5) + (uint32_t)(__ffs(bits) - 1);
            bits &= bits - 1u;
        }
    }
}

// ---------------------------------------------------------------------------
// keep / deactivate and dense relabel (recenterAndDeactivateClusters,
// cuda/devPartition.h:624-711): roots sorted by vertex id; kept clusters get
// dense labels in root order, dropped ones smallest - index - 1.

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_relabel(Dev<OffT> d, const uint32_t* roots, ClusterTables t,
                                                    ClusterTables nt) {
    pdl_wait();
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_roots;
    const uint32_t ntiles = (count + kRelabelTile - 1) / kRelabelTile;
    const uint32_t epoch = d.lb_epoch[kSiteRelabel];
    const int e = fixed_exponent(d.ctr->xmax_walk_bits, d.nb_bits);
    const double inv = pow2(-e);
    const int32_t smallest = d.ctr->smallest;
    int32_t most_negative = 0;
    uint32_t biggest = 0;
    // tiles in the order they are taken (look-back), several per block
    for (;;) {
        const uint32_t tile = fetch_tile(d.ctr, kSiteRelabel);
        if (tile >= ntiles) break;
        const uint32_t first = tile * kRelabelTile + threadIdx.x * kRelabelItems;
        uint64_t vals[kRelabelItems];
        uint64_t run = 0;
#pragma unroll
        for (int k = 0; k < kRelabelItems; ++k) {
            const uint32_t j = first + k;
            uint64_t v = 0;
            if (j < count) {
                const uint32_t r = roots[j];
                const uint32_t cnt = d.acc_cnt[r];
                const float pot = __fsub_rn(from_ordered_bits(d.acc_max[r]), from_ordered_bits(d.acc_min[r]));
                const bool keep = pot >= d.rw_threshold && cnt >= 2;
                v = keep ? (((uint64_t)cnt << 32) | 1u) : 0ull;
            }
            vals[k] = v;
            run = PairAdd::combine(run, v);
        }
        uint64_t tile_total;
        const uint64_t incl = block_inclusive<PairAdd>(run, warp_tot, &tile_total);
        if (threadIdx.x < 32) {
            const uint64_t ex = lookback_tile<PairAdd>(d.lb_relabel, tile, epoch, tile_total, &d.ctr->err);
            if (threadIdx.x == 0) s_excl = ex;
            if (threadIdx.x == 0 && tile == ntiles - 1) {
                const uint64_t all = PairAdd::combine(ex, tile_total);
                d.ctr->n_keep = (uint32_t)all;
                d.ctr->n_active_next = (uint32_t)(all >> 32);
            }
        }
        __syncthreads();
        const uint32_t lo = (uint32_t)incl - (uint32_t)run;
        const uint32_t hi = (uint32_t)(incl >> 32) - (uint32_t)(run >> 32);
        uint64_t p = PairAdd::combine(s_excl, ((uint64_t)hi << 32) | lo);
#pragma unroll
        for (int k = 0; k < kRelabelItems; ++k) {
            const uint32_t j = first + k;
            if (j >= count) break;
            const uint32_t r = roots[j];
            if (vals[k]) {
                const uint32_t nl = (uint32_t)p;
                const uint32_t cnt = (uint32_t)(vals[k] >> 32);
                biggest = cnt > biggest ? cnt : biggest;
                d.newlab[r] = (int32_t)nl;
                d.avg[r] = __ddiv_rn(__dmul_rn(__ll2double_rn(d.acc_sum[r]), inv), (double)cnt);
                nt.size[nl] = cnt;
                nt.start[nl] = (uint32_t)(p >> 32);
                nt.root[nl] = r;
                nt.best[nl] = ~0ull;
                // a cluster that was not split keeps its rows, degrees and volume:
                // only the clusters born from a split rescan their rows
                const uint32_t info = d.rootc[r];
                const uint32_t kind = info >> 30;
                const uint32_t c = info & kOriginLabelMask;
                d.nflag[nl] = kind == kOriginCarried ? kRowsCarried : kind == kOriginSwept ? kRowsKept : kRowsScan;
                nt.vol[nl] = kind == kOriginChild ? 0u : t.vol[c];
                if (kind == kOriginCarried) {
                    const uint16_t sk = t.skip[c];
                    // due next round once its spread is below the threshold (k_due_scan),
                    // or after a round that cut many clusters
                    nt.skip[nl] = due_aligned(d, (sk > 0 && !(d.sflag[c] & 4u) && !cut_gate_on(d)) ? sk - 1u : 0u, cnt);
                    nt.hist[nl] = t.hist[c];
                }
            } else {
                const int32_t nl = (int32_t)((uint32_t)smallest - j - 1u);
                d.newlab[r] = nl;
                most_negative = nl < most_negative ? nl : most_negative;
            }
            p = PairAdd::combine(p, vals[k]);
        }
        __syncthreads();   // s_excl and warp_tot are reused by the next tile
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) most_negative = min(most_negative, __shfl_xor_sync(0xFFFFFFFFu, most_negative, o));
    if ((threadIdx.x & 31u) == 0 && most_negative < 0) atomicMin(&d.ctr->smallest_next, most_negative);
    block_atomic_max(&d.ctr->max_csize_next, biggest);
}

// Certificate record of a vertex whose cluster is certified this round: the
// round (+1), and bit 31 when the certified set (the component of root r,
// acc_cnt[r] vertices) is not the whole cluster c swept this round, i.e. c
// was cut or fell apart into components.  Certified vertices neither walk nor
// recentre afterwards, so their potentials stay the ones this test saw.
template <typename OffT>
__device__ __forceinline__ void record_certificate(const Dev<OffT>& d, const ClusterTables& t, uint32_t v,
                                                   uint32_t c, uint32_t r) {
    const bool whole = d.cut_off[c] == kNoCut && d.acc_cnt[r] == t.size[c];
    d.cert[v] = (d.ctr->rounds + 1u) | (whole ? 0u : 0x80000000u);
}

// Plain form: new labels and recentering (x -= cluster mean) over the
// active list in vertex order, so labels, parents and potentials are read
// and written in runs (k_apply then only compacts the sorted order).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_newlab(Dev<OffT> d, ClusterTables t, const uint32_t* ids) {
    pdl_wait();
    if (d.ctr->walk_only || d.sched) return;
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < count; j += gridDim.x * blockDim.x) {
        const uint32_t v = ids[j];
        const uint32_t lv = (uint32_t)d.lab[v];   // c, or k + c past a cut
        const uint32_t c = lv >= k ? lv - k : lv;
        // k_components_data left parent[v] at the root
        const uint32_t r = d.split[c] ? d.parent[v] : t.root[c];
        const int32_t nl = d.newlab[r];
        d.lab[v] = nl;
        if (nl >= 0) d.x[v] = __double2float_rn(__dsub_rn((double)d.x[v], d.avg[r]));
        else record_certificate(d, t, v, c, r);
    }
}

// new labels and recentering (learned schedule only), and the stable
// compaction of the sorted order into the next round's active list.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_apply(Dev<OffT> d, ClusterTables t, const uint32_t* vals0,
                                                  const uint32_t* vals1, const uint64_t* keys0,
                                                  const uint64_t* keys1, uint32_t* act_next, uint32_t* par_next) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_sweep;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteApply);
    if (tile == 0 && threadIdx.x == 0) d.ctr->xmax_bits = 0;
    if (tile >= ntiles) return;
    const uint32_t sel = d.ctr->main_sel;
    const uint32_t* vals = sel ? vals1 : vals0;
    const uint64_t* keys = sel ? keys1 : keys0;
    const uint32_t epoch = d.lb_epoch[kSiteApply];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t vv[kScanItems], cc[kScanItems];
    uint32_t keepmask = 0, run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        vv[k] = 0;
        cc[k] = 0;
        if (i >= count) continue;
        const uint32_t c = (uint32_t)(keys[i] >> 32);
        cc[k] = c;
        const uint32_t v = vals[i];
        vv[k] = v;
        if (!d.sched) {   // k_newlab wrote the new labels in vertex order
            if (d.lab[v] >= 0) { keepmask |= 1u << k; ++run; }
            continue;
        }
        if (!(d.sflag[c] & 1u)) continue;   // carried: k_carry_vertices
        // k_components_data left parent[v] at the root (atomicMin stores only
        // ever move a pointer towards the root)
        const uint32_t r = d.split[c] ? d.parent[v] : t.root[c];
        const int32_t nl = d.newlab[r];
        d.lab[v] = nl;
        if (nl >= 0) {
            d.x[v] = __double2float_rn(__dsub_rn((double)d.x[v], d.avg[r]));
            keepmask |= 1u << k;
            ++run;
        } else {
            record_certificate(d, t, v, c, r);
        }
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_apply, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    uint32_t pos = (uint32_t)(s_excl + incl - run);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (keepmask & (1u << k)) {
            act_next[pos] = vv[k];
            par_next[pos] = cc[k];   // the cluster the vertex was swept in: runs of the next list
            ++pos;
        }
}

// next round's vertex-order list, edge disabling (disableEdgesKernel_node,
// cuda/devPartition.h:80-146), internal degrees, x/d, cluster volumes.
template <typename OffT, int W>
__global__ void __launch_bounds__(kBlock) k_ids_disable(Dev<OffT> d, const uint32_t* ids, uint32_t* ids_next,
                                                        float* xt, ClusterTables nt) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_list[kScanTile];
    __shared__ uint32_t s_hkey[kScanTile];
    __shared__ uint32_t s_hval[kScanTile];
    __shared__ uint32_t s_n;
    const uint32_t count = d.ctr->n_active;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteIds);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteIds];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t vv[kScanItems];
    uint32_t keepmask = 0, run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t j = first + k;
        vv[k] = 0;
        if (j >= count) continue;
        const uint32_t v = ids[j];
        vv[k] = v;
        if (d.lab[v] >= 0) { keepmask |= 1u << k; ++run; }
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_ids, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) {
            s_excl = ex;
            s_n = (uint32_t)tile_total;
        }
    }
    __syncthreads();
    uint32_t lpos = (uint32_t)(incl - run);
    const uint32_t gpos = (uint32_t)s_excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
        if (keepmask & (1u << k)) {
            ids_next[gpos + lpos] = vv[k];
            s_list[lpos] = vv[k];
            ++lpos;
        }
    __syncthreads();
    // row pass over this tile's kept vertices, W lanes per vertex; cluster
    // volumes are summed per tile in a shared hash table keyed by label
    for (uint32_t q = threadIdx.x; q < kScanTile; q += kBlock) { s_hkey[q] = 0xFFFFFFFFu; s_hval[q] = 0u; }
    __syncthreads();
    const uint32_t nkept = s_n;
    const uint32_t gl = threadIdx.x & (W - 1);
    uint32_t vmax = 0;
    for (uint32_t q0 = (threadIdx.x & ~31u) / W; q0 < nkept; q0 += kBlock / W) {
        const uint32_t q = q0 + (threadIdx.x & 31u) / W;
        const bool valid = q < nkept;
        const uint32_t v = valid ? s_list[q] : 0u;
        const int32_t lv = valid ? d.lab[v] : 0;
        const uint32_t rows = valid ? d.nflag[lv] : kRowsScan;
        const bool noscan = rows != kRowsScan;   // not split: no slot can have become inter-cluster
        OffT beg = valid ? d.off[v] : 0, end = valid ? d.off[v + 1] : 0;
        const bool light = valid && (uint64_t)(end - beg) <= d.light_max;
        if (!light || noscan) beg = end;      // long rows: k_disable_long
        uint32_t deg = 0;
        for (OffT s = beg + gl; s < end; s += kSlotUnroll * W) {
            uint32_t nb[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) nb[u] = s + u * W < end ? stream_col(d.cols + s + u * W) : kInvalidEdge;
            int32_t ln[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) ln[u] = slot_valid(nb[u]) ? d.lab[nb[u]] : lv;
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) {
                if (!slot_valid(nb[u])) continue;
                if (ln[u] != lv) d.cols[s + u * W] = nb[u] | kDisabledBit;
                else ++deg;
            }
        }
#pragma unroll
        for (int o = W / 2; o > 0; o >>= 1) deg += __shfl_xor_sync(0xFFFFFFFFu, deg, o, W);
        if (valid && noscan && gl == 0) {
            const float xv = d.x[v];
            if (rows == kRowsKept) {   // recentred: refresh x / degree
                const uint32_t dg = d.ideg[v];
                xt[v] = dg ? __double2float_rn(__ddiv_rn((double)xv, (double)dg)) : 0.0f;
            }
            const uint32_t b = __float_as_uint(fabsf(xv));
            vmax = b > vmax ? b : vmax;
        }
        if (light && !noscan && gl == 0) {
            d.ideg[v] = deg;
            const float xv = d.x[v];
            xt[v] = deg ? __double2float_rn(__ddiv_rn((double)xv, (double)deg)) : 0.0f;
            const uint32_t b = __float_as_uint(fabsf(xv));
            vmax = b > vmax ? b : vmax;
            uint32_t h = ((uint32_t)lv * 2654435761u) & (kScanTile - 1);
            for (;;) {
                const uint32_t prev = atomicCAS(&s_hkey[h], 0xFFFFFFFFu, (uint32_t)lv);
                if (prev == 0xFFFFFFFFu || prev == (uint32_t)lv) { atomicAdd(&s_hval[h], deg); break; }
                h = (h + 1) & (kScanTile - 1);
            }
        }
    }
    block_atomic_max(&d.ctr->xmax_bits, vmax);
    for (uint32_t q = threadIdx.x; q < kScanTile; q += kBlock)
        if (s_hkey[q] != 0xFFFFFFFFu && s_hval[q]) atomicAdd(&nt.vol[s_hkey[q]], s_hval[q]);
}

// ---------------------------------------------------------------------------
// Long rows.  Rows longer than Dev::light_max slots are binned once per graph
// into two static lists: "wide" rows (up to Dev::wide_max slots) get one warp
// each, "heavy" rows one CTA each (G = 32 or kBlock lanes per row, slots
// strided by G with kSlotUnroll independent loads per step, group reduction).
// Every accumulation is order-independent, so the binning does not change
// any result.

template <typename T>
__device__ __forceinline__ T block_sum(T v, T* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    T t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kBlock / 32; ++w) t += sh[w];
    return t;  // valid in thread 0
}

// sum over the G lanes of a row group; valid in the group's first lane
template <int G, typename T>
__device__ __forceinline__ T group_sum(T v, T* sh) {
    if constexpr (G == 32) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
        return v;
    } else {
        return block_sum<T>(v, sh);
    }
}

// the rows of one list that a group visits: group index, group count, lane
template <int G>
struct RowGroups {
    uint32_t first, step, lane;
    __device__ __forceinline__ RowGroups() {
        if constexpr (G == 32) {
            first = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
            step = (gridDim.x * blockDim.x) >> 5;
            lane = threadIdx.x & 31u;
        } else {
            first = blockIdx.x;
            step = gridDim.x;
            lane = threadIdx.x;
        }
    }
};

// Rows of a long-row list that pass `pred`, each handed to `body` with the
// whole group.  With `windows` a warp-per-row group tests a window of 32
// rows at once, one per lane, and then works the passing rows one after
// another: lists whose rows mostly fail (clusters not split, not swept) cost
// one load chain per 32 rows instead of per row.  Where most rows pass, the
// row-by-row order spreads the rows over the warps more evenly.  pred(v)
// runs per lane; body(v) on every lane.
template <int G, class Pred, class Body>
__device__ __forceinline__ void for_each_row(const uint32_t* list, uint32_t cnt, const RowGroups<G>& rg, Pred pred,
                                             Body body, bool windows = true) {
    if (G == 32 && windows) {
        for (uint32_t h0 = rg.first * 32u; h0 < cnt; h0 += rg.step * 32u) {
            const uint32_t h = h0 + rg.lane;
            const uint32_t v = h < cnt ? list[h] : 0u;
            uint32_t pass = __ballot_sync(0xFFFFFFFFu, h < cnt && pred(v));
            while (pass) {
                const int src = __ffs(pass) - 1;
                pass &= pass - 1u;
                body(__shfl_sync(0xFFFFFFFFu, v, src));
            }
        }
    } else {
        for (uint32_t h = rg.first; h < cnt; h += rg.step) {
            const uint32_t v = list[h];
            if (pred(v)) body(v);
        }
    }
}

template <typename OffT>
__device__ __forceinline__ const uint32_t* row_list(const Dev<OffT>& d, int G, uint32_t* count) {
    *count = G == 32 ? d.n_wide : d.n_heavy;
    return G == 32 ? d.wide : d.heavy;
}

// A long row's head: vertex, label and slot bounds (label -1 past the list).
template <typename OffT>
struct RowHead {
    uint32_t v;
    int32_t lab;
    OffT beg, end;
};

template <typename OffT>
__device__ __forceinline__ RowHead<OffT> row_head(const Dev<OffT>& d, const uint32_t* list, uint32_t h, uint32_t cnt) {
    RowHead<OffT> r{0u, -1, 0, 0};
    if (h < cnt) {
        r.v = list[h];
        r.lab = d.lab[r.v];
        r.beg = d.off[r.v];
        r.end = d.off[r.v + 1];
    }
    return r;
}

template <typename OffT, int G>
__global__ void PXR_WALK_BOUNDS k_walk_long(Dev<OffT> d, const float* xt_in,
                                                                          float* xt_out) {
    pdl_wait();
    __shared__ int64_t sh[kBlock / 32];
    const int e = fixed_exponent(d.ctr->xmax_bits, d.nb_bits);
    const double scale = pow2(e), inv = pow2(-e);
    uint32_t cnt;
    const uint32_t* list = row_list(d, G, &cnt);
    const RowGroups<G> rg;
    uint32_t vmax = 0;
    unsigned long long st_v = 0, st_s = 0, st_g = 0;
    // With PXR_WALK_PREFETCH the next row's id, label and bounds are loaded
    // before this row's slots are gathered, so a row's setup loads overlap
    // the previous row's gathers.
    RowHead<OffT> nx = row_head(d, list, rg.first, cnt);
    for (uint32_t h = rg.first; h < cnt; h += rg.step) {
        RowHead<OffT> cur;
        if (PXR_WALK_PREFETCH) {
            cur = nx;
            nx = row_head(d, list, h + rg.step, cnt);
        } else {
            cur = row_head(d, list, h, cnt);
        }
        if (cur.lab < 0) continue;
        const uint32_t v = cur.v;
        const OffT beg = cur.beg, end = cur.end;
        int64_t acc = 0;
        unsigned long long g = 0;
        for (OffT s = beg + rg.lane; s < end; s += kSlotUnroll * G) {
            uint32_t nb[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) nb[u] = s + u * G < end ? stream_col(d.cols + s + u * G) : kInvalidEdge;
            float xv[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) xv[u] = slot_valid(nb[u]) ? xt_in[nb[u]] : 0.0f;
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u)
                if (slot_valid(nb[u])) { acc += to_fixed(xv[u], scale); ++g; }
        }
        acc = group_sum<G, int64_t>(acc, sh);
        st_g += g;
        if (rg.lane == 0) {
            const double sum = __dmul_rn(__ll2double_rn(acc), inv);
            const double val = __dadd_rn(__dmul_rn(sum, 0.9), __dmul_rn((double)d.x[v], 0.1));
            const float xv = __double2float_rn(val);
            d.x[v] = xv;
            const uint32_t dg = d.ideg[v];
            xt_out[v] = dg ? __double2float_rn(__ddiv_rn((double)xv, (double)dg)) : 0.0f;
            const uint32_t b = __float_as_uint(fabsf(xv));
            vmax = b > vmax ? b : vmax;
            st_v += 1;
            st_s += (unsigned long long)(end - beg);
        }
    }
    walk_block_totals(d, vmax, st_v, st_s, st_g);
}

template <typename OffT, int G>
__global__ void __launch_bounds__(kBlock) k_nodediff_long(Dev<OffT> d) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ int32_t sh[kBlock / 32];
    uint32_t cnt;
    const uint32_t* list = row_list(d, G, &cnt);
    const RowGroups<G> rg;
    auto swept = [&](uint32_t v) {
        const int32_t lv = d.lab[v];
        return lv >= 0 && (!d.sched || (d.sflag[lv] & 2u));
    };
    for_each_row<G>(list, cnt, rg, swept, [&](uint32_t v) {
        const uint32_t mine = ordered_bits(d.x[v]);
        const OffT beg = d.off[v], end = d.off[v + 1];
        int32_t c = 0;
        for (OffT s = beg + rg.lane; s < end; s += kSlotUnroll * G) {
            uint32_t nb[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) nb[u] = s + u * G < end ? stream_col(d.cols + s + u * G) : kInvalidEdge;
            float xn[kSlotUnroll];
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) xn[u] = slot_valid(nb[u]) ? d.x[nb[u]] : 0.0f;
#pragma unroll
            for (int u = 0; u < kSlotUnroll; ++u) {
                if (!slot_valid(nb[u])) continue;
                const uint32_t o = ordered_bits(xn[u]);
                c += (o < mine || (o == mine && nb[u] < v)) ? -1 : 1;
            }
        }
        c = group_sum<G, int32_t>(c, sh);
        if (rg.lane == 0) d.dv[v] = make_int2(c, (int)d.ideg[v]);
    }, d.sched != 0);   // the plain form takes the edge differences of every row
}

template <typename OffT, int G>
__global__ void __launch_bounds__(kBlock) k_union_long(Dev<OffT> d) {
    pdl_wait();
    if (d.ctr->walk_only || !d.ctr->any_split) return;   // nothing due, or nothing split
    const uint32_t k = d.ctr->n_clusters;
    uint32_t cnt;
    const uint32_t* list = row_list(d, G, &cnt);
    const RowGroups<G> rg;
    auto in_split_cluster = [&](uint32_t v) {
        const int32_t lv = d.lab[v];
        if (lv < 0) return false;
        const uint32_t c = (uint32_t)lv >= k ? (uint32_t)lv - k : (uint32_t)lv;   // cut labels are c or K + c
        return c < k && d.split[c] != 0;
    };
    for_each_row<G>(list, cnt, rg, in_split_cluster, [&](uint32_t v) {
        const int32_t lv = d.lab[v];
        const OffT beg = d.off[v], end = d.off[v + 1];
        uint32_t hint;
        if (union_skip_row(d, k, v, lv, hint)) return;
        for (OffT s = beg + rg.lane; s < end; s += G) {
            const uint32_t nb = d.cols[s];
            if (!slot_valid(nb) || nb == v) continue;
            if (!d.union_sampled && nb > v) break;
            if (d.lab[nb] == lv) uf_join(d.parent, &d.ctr->err, v, nb, hint);
        }
    });
}

template <typename OffT, int G>
__global__ void __launch_bounds__(kBlock) k_disable_long(Dev<OffT> d, float* xt, ClusterTables nt) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint32_t sh[kBlock / 32];
    uint32_t cnt;
    const uint32_t* list = row_list(d, G, &cnt);
    const RowGroups<G> rg;
    uint32_t vmax = 0;
    // rows of clusters born from a split only: k_ids_disable refreshed x / degree of the others
    auto rescanned = [&](uint32_t v) {
        const int32_t lv = d.lab[v];
        return lv >= 0 && d.nflag[lv] == kRowsScan;
    };
    for_each_row<G>(list, cnt, rg, rescanned, [&](uint32_t v) {
        const int32_t lv = d.lab[v];
        const OffT beg = d.off[v], end = d.off[v + 1];
        uint32_t deg = 0;
        for (OffT s = beg + rg.lane; s < end; s += G) {
            const uint32_t nb = d.cols[s];
            if (!slot_valid(nb)) continue;
            if (d.lab[nb] != lv) d.cols[s] = nb | kDisabledBit;
            else ++deg;
        }
        deg = group_sum<G, uint32_t>(deg, sh);
        if (rg.lane == 0) {
            d.ideg[v] = deg;
            const float xv = d.x[v];
            xt[v] = deg ? __double2float_rn(__ddiv_rn((double)xv, (double)deg)) : 0.0f;
            const uint32_t b = __float_as_uint(fabsf(xv));
            vmax = b > vmax ? b : vmax;
            atomicAdd(&nt.vol[lv], deg);
        }
    });
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
    if ((threadIdx.x & 31u) == 0 && vmax) atomicMax(&d.ctr->xmax_bits, vmax);
}

// exclusive prefix of cluster volumes over labels
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cvol_scan(Dev<OffT> d, ClusterTables nt) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_keep;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteCvol);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteCvol];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint64_t run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t j = first + k;
        v[k] = j < count ? nt.vol[j] : 0u;
        run += v[k];
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>(run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_cvol, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    uint64_t p = s_excl + incl - run;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t j = first + k;
        if (j >= count) break;
        nt.vol_start[j] = (uint32_t)p;
        p += v[k];
    }
}

// ---------------------------------------------------------------------------
// initial potentials (RandomWalkManager::initRandomWalk, cuda/devRandomWalk.h:22-48, 509-519)
void launch_initial_potentials(const void* off, bool off64, uint32_t n, uint32_t seed, float* x,
                               uint32_t* xmax_bits, cudaStream_t stream);

}  // namespace pxr
