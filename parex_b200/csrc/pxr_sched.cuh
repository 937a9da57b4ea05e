// Kernels of the learned sweep schedule (sm_100a).  No reference
// counterpart: the reference sweeps every active cluster every round.
//
// A cluster whose skip counter is non-zero is "carried" through the round:
// its vertices walk with the rest, but it is left out of the sort, the scan,
// the cut, components and recentering.  The clusters that are due go through
// the unchanged plain kernels, restricted to the sweep set by the tables this
// file builds (start and start volume of the due clusters only), so every cut
// is still chosen and scored by the exact sweep.  Carried clusters keep their
// vertices and rows and take part in the dense relabelling (root order over
// all clusters).  After the round a per-cluster kernel evaluates the MLP on
// the cluster's features and sets how many rounds it is carried next.
// In audit mode every cluster is swept, the schedule only decides which
// sweeps are acted on, and a skipped sweep that finds a cut is counted as a
// false stop; the partition is the same as without the audit.
#pragma once

#include "pxr_kernels.cuh"
#include "pxr_mlp.cuh"

namespace pxr {

// Potential spread per cluster after the walk, over the active list in vertex
// order (runs of one label give few atomics).  A carried cluster whose spread
// is already below rw_threshold is swept in the next round instead of
// walking until its skip counter runs out: the keep test would certify it,
// and every further walk step over it is wasted.
struct SpreadAgg {
    using T = uint2;              // x: max ordered bits, y: min ordered bits
    uint32_t* smax;
    uint32_t* smin;
    __device__ static T identity() { return make_uint2(0u, 0xFFFFFFFFu); }
    __device__ static T combine(T a, T b) { return make_uint2(a.x > b.x ? a.x : b.x, a.y < b.y ? a.y : b.y); }
    __device__ static T warp_reduce(T v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            T u;
            u.x = __shfl_xor_sync(0xFFFFFFFFu, v.x, o);
            u.y = __shfl_xor_sync(0xFFFFFFFFu, v.y, o);
            v = combine(v, u);
        }
        return v;
    }
    __device__ void emit(uint32_t key, T v) const {
        atomicMax(&smax[key], v.x);
        atomicMin(&smin[key], v.y);
    }
};

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_cluster_spread(Dev<OffT> d, const uint32_t* ids) {
    pdl_wait();
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    SpreadAgg agg{d.smax, d.smin};
    const uint32_t stride = gridDim.x * kScanTile;
    for (uint32_t base = blockIdx.x * kScanTile; base < count; base += stride) {
        const uint32_t first = base + threadIdx.x * kScanItems;
        bool has = false, single = true;
        uint32_t k_first = 0, k_last = 0;
        uint2 a_first = SpreadAgg::identity(), a_last = SpreadAgg::identity();
        for (int q = 0; q < kScanItems; ++q) {
            const uint32_t j = first + q;
            if (j >= count) break;
            const uint32_t v = ids[j];
            const uint32_t c = (uint32_t)d.lab[v];
            if (c >= k) continue;
            const uint32_t ob = ordered_bits(d.x[v]);
            const uint2 cur = make_uint2(ob, ob);
            if (!has) {
                has = true; k_first = c; a_first = cur; k_last = c; a_last = cur;
            } else if (c == k_last) {
                a_last = SpreadAgg::combine(a_last, cur);
                if (single) a_first = a_last;
            } else {
                if (!single) agg.emit(k_last, a_last);
                single = false;
                k_last = c;
                a_last = cur;
            }
        }
        emit_fragments<SpreadAgg>(has, single, k_first, a_first, k_last, a_last, agg);
    }
}

// per cluster: due / in-sweep flags and the start tables of the sweep set
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_due_scan(Dev<OffT> d, ClusterTables t) {
    pdl_wait();
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_clusters;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteSched);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteSched];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint64_t vals[kScanItems];
    uint64_t run = 0;
    uint32_t due_items = 0, skipped = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t c = first + k;
        uint64_t v = 0;
        if (c < count) {
            const bool due = t.skip[c] == 0;
            const bool swept = due || d.sched == 2u;
            const float spread = __fsub_rn(from_ordered_bits(d.smax[c]), from_ordered_bits(d.smin[c]));
            const bool settled = !due && d.smin[c] != 0xFFFFFFFFu && spread < d.rw_threshold;
            d.smax[c] = 0u;              // identity again for the next round
            d.smin[c] = 0xFFFFFFFFu;
            d.sflag[c] = (uint8_t)((due ? 1u : 0u) | (swept ? 2u : 0u) | (settled ? 4u : 0u));
            if (swept) v = ((uint64_t)t.vol[c] << 32) | t.size[c];
            if (due) due_items += t.size[c]; else ++skipped;
        }
        vals[k] = v;
        run = PairAdd::combine(run, v);
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<PairAdd>(run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<PairAdd>(d.lb_sched, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
        if (threadIdx.x == 0 && tile == ntiles - 1) d.ctr->n_sweep = (uint32_t)PairAdd::combine(ex, tile_total);
    }
    __syncthreads();
    const uint32_t lo = (uint32_t)incl - (uint32_t)run;
    const uint32_t hi = (uint32_t)(incl >> 32) - (uint32_t)(run >> 32);
    uint64_t p = PairAdd::combine(s_excl, ((uint64_t)hi << 32) | lo);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t c = first + k;
        if (c >= count) break;
        if (vals[k]) {
            t.start[c] = (uint32_t)p;
            t.vol_start[c] = (uint32_t)(p >> 32);
        }
        p = PairAdd::combine(p, vals[k]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        due_items += __shfl_xor_sync(0xFFFFFFFFu, due_items, o);
        skipped += __shfl_xor_sync(0xFFFFFFFFu, skipped, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        if (due_items) atomicAdd(&d.ctr->n_due_items, due_items);
        if (skipped) atomicAdd(&d.ctr->stat_skipped, (unsigned long long)skipped);
    }
}

// sort keys of the sweep set, compacted from the last sort order
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_emit_sched(Dev<OffT> d, const uint32_t* act, uint64_t* keys,
                                                       uint32_t* vals, uint64_t* best) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < k; c += gridDim.x * blockDim.x) best[c] = ~0ull;
    const uint32_t count = d.ctr->n_active;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteEmit);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteEmit];
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint64_t kk[kScanItems];
    uint32_t vv[kScanItems];
    uint32_t mask = 0, run = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const uint32_t i = first + q;
        kk[q] = 0;
        vv[q] = 0;
        if (i >= count) continue;
        const uint32_t v = act[i];
        const uint32_t c = (uint32_t)d.lab[v];
        if (c < k && (d.sflag[c] & 2u)) {
            kk[q] = ((uint64_t)c << 32) | ordered_bits(d.x[v]);
            vv[q] = v;
            mask |= 1u << q;
            ++run;
        }
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_emit, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    uint32_t pos = (uint32_t)(s_excl + incl - run);
#pragma unroll
    for (int q = 0; q < kScanItems; ++q)
        if (mask & (1u << q)) {
            keys[pos] = kk[q];
            vals[pos] = vv[q];
            ++pos;
        }
}

// After the due scan: a round in which no cluster is due only walks.
template <typename OffT>
__global__ void k_walk_only_check(Dev<OffT> d) {
    pdl_wait();
    d.ctr->walk_only = (d.ctr->n_sweep == 0 && d.ctr->n_active > 0) ? 1u : 0u;
}

// A round that only walked: every cluster, label, row and list stays; the
// next round's buffers take copies and every skip counter goes down by one.
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_carry_all(Dev<OffT> d, ClusterTables t, ClusterTables nt,
                                                      const uint32_t* act, uint32_t* act_next, const uint32_t* ids,
                                                      uint32_t* ids_next) {
    pdl_wait();
    if (!d.ctr->walk_only) return;
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t na = d.ctr->n_active;
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    for (uint32_t c = tid; c < k; c += stride) {
        nt.start[c] = t.start[c];
        nt.size[c] = t.size[c];
        nt.vol[c] = t.vol[c];
        nt.vol_start[c] = t.vol_start[c];
        nt.root[c] = t.root[c];
        nt.best[c] = ~0ull;
        const uint16_t sk = t.skip[c];
        nt.skip[c] = due_aligned(d, (sk > 0 && !(d.sflag[c] & 4u)) ? sk - 1u : 0u, t.size[c]);
        nt.hist[c] = t.hist[c];
        if (d.trace) {
            pxr_cluster_record& o = static_cast<pxr_cluster_record*>(d.records)[c];
            o.origin = kOriginCarried;
            o.skip = nt.skip[c];
            o.round = d.ctr->rounds;
        }
    }
    for (uint32_t i = tid; i < na; i += stride) {
        act_next[i] = act[i];
        ids_next[i] = ids[i];
    }
    if (tid == 0) {
        d.ctr->n_keep = k;
        d.ctr->n_active_next = na;
    }
}

// Carried clusters: register their roots for the relabelling with data that
// keeps them (count = size, spread 2, sum 0).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_carry_roots(Dev<OffT> d, ClusterTables t) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    const uint32_t k = d.ctr->n_clusters;
    for (uint32_t c0 = blockIdx.x * blockDim.x; c0 < k; c0 += gridDim.x * blockDim.x) {
        const uint32_t c = c0 + threadIdx.x;
        const bool carried = c < k && !(d.sflag[c] & 1u);
        if (carried) {
            const uint32_t r = t.root[c];
            d.acc_cnt[r] = t.size[c];
            d.acc_max[r] = ordered_bits(1.0f);
            d.acc_min[r] = ordered_bits(-1.0f);
            d.acc_sum[r] = 0;
            d.rootc[r] = (kOriginCarried << 30) | c;
            mark_root(d, r);
        }
    }
}

// Carried vertices: new label, and their place in the next active list after
// the swept ones (in the order of the last sort).
template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_carry_vertices(Dev<OffT> d, ClusterTables t, const uint32_t* act,
                                                           uint32_t* act_next) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = d.ctr->n_active;
    const uint32_t k = d.ctr->n_clusters;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(d.ctr, kSiteCarry);
    if (tile >= ntiles) return;
    const uint32_t epoch = d.lb_epoch[kSiteCarry];
    const uint32_t base = d.ctr->n_active_next - (count - d.ctr->n_due_items);
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t vv[kScanItems];
    uint32_t mask = 0, run = 0;
#pragma unroll
    for (int q = 0; q < kScanItems; ++q) {
        const uint32_t i = first + q;
        vv[q] = 0;
        if (i >= count) continue;
        const uint32_t v = act[i];
        const uint32_t c = (uint32_t)d.lab[v];   // due vertices may carry cut labels k + c here
        if (c < k && !(d.sflag[c] & 1u)) {
            d.lab[v] = d.newlab[t.root[c]];
            vv[q] = v;
            mask |= 1u << q;
            ++run;
        }
    }
    uint64_t tile_total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &tile_total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(d.lb_carry, tile, epoch, tile_total, &d.ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
    }
    __syncthreads();
    uint32_t pos = base + (uint32_t)(s_excl + incl - run);
#pragma unroll
    for (int q = 0; q < kScanItems; ++q)
        if (mask & (1u << q)) {
            if (pos < d.n) act_next[pos] = vv[q];
            else atomicOr(&d.ctr->err, kErrLabelRange);   // sizes and active list disagree
            ++pos;
        }
}

// After the round, per cluster of the next round: features, the sweep
// history and, in the learned modes, the MLP's skip count.  Carried clusters
// were already handled by k_relabel (counter decremented, history kept).
// Inference keeps only the layer-1 activations live (mlp_infer): 128
// registers with a few spilled, two CTAs per SM (the training forward's
// 144 stored values held it to one).
template <typename OffT>
__global__ void __launch_bounds__(kBlock, 2) k_schedule(Dev<OffT> d, ClusterTables t, ClusterTables nt) {
    pdl_wait();
    if (d.ctr->walk_only) return;   // nothing due: the round only walks
    __shared__ float img[kMlpImage];
    if (d.sched)
        for (int p = threadIdx.x; p < kMlpImage; p += blockDim.x) img[p] = d.mlp[p];
    __syncthreads();
    const uint32_t k = d.ctr->n_keep;
    const uint32_t round = d.ctr->rounds;
    pxr_cluster_record* rec = static_cast<pxr_cluster_record*>(d.records);
    for (uint32_t nl = blockIdx.x * blockDim.x + threadIdx.x; nl < k; nl += gridDim.x * blockDim.x) {
        const uint32_t r = nt.root[nl];
        const uint32_t info = d.rootc[r];
        const uint32_t kind = info >> 30;
        const uint32_t c = info & kOriginLabelMask;
        if (kind == kOriginCarried) {
            if (d.trace) {
                rec[nl].root = r;
                rec[nl].size = nt.size[nl];
                rec[nl].volume = nt.vol[nl];
                rec[nl].origin = kind;
                rec[nl].skip = nt.skip[nl];
                rec[nl].round = round;
            }
            continue;
        }
        const uint32_t size = nt.size[nl];
        const uint32_t vol = nt.vol[nl];
        const float pot = __fsub_rn(from_ordered_bits(d.acc_max[r]), from_ordered_bits(d.acc_min[r]));
        const float sp = __uint_as_float((uint32_t)(t.best[c] >> 32));
        SchedHist h{0.0f, 2.0f, 0u, 0u};
        if (kind == kOriginSwept) h = t.hist[c];
        const bool has_prev = kind == kOriginSwept && h.age > 0;
        const uint32_t dr = has_prev ? round - h.round : 0u;
        const uint32_t age = kind == kOriginSwept ? h.age : 0u;
        float y = 0.0f;
        uint32_t sk = 0;
        if (d.sched && kind == kOriginSwept) {
            float f[kMlpIn];
            cluster_features(f, size, vol, pot, sp, has_prev, h.pot, h.sp, dr, age, round, d.rw_threshold,
                             d.sc_threshold);
            y = mlp_infer(img, f);
            sk = cut_gate_on(d) ? 0u : skip_from_prediction(y, d.safety, d.max_skip);
        }
        if (d.sched) {
            sk = due_aligned(d, sk, size);
            nt.skip[nl] = (uint16_t)sk;
        }
        const SchedHist nh{pot, sp, round, kind == kOriginSwept ? h.age + 1u : 0u};
        nt.hist[nl] = nh;
        if (d.trace) {
            pxr_cluster_record& o = rec[nl];
            o.root = r;
            o.size = size;
            o.volume = vol;
            o.origin = kind;
            o.potential = pot;
            o.sparsity = sp;
            o.prev_potential = h.pot;
            o.prev_sparsity = h.sp;
            o.prev_round = h.round;
            o.age = kind == kOriginSwept ? h.age : 0u;
            o.round = round;
            o.skip = sk;
            o.prediction = y;
            o.has_prev = has_prev ? 1u : 0u;
            // the features again (the same function of the same values): not kept live across the MLP
            float f[kMlpIn];
            cluster_features(f, size, vol, pot, sp, has_prev, h.pot, h.sp, dr, age, round, d.rw_threshold,
                             d.sc_threshold);
#pragma unroll
            for (int i = 0; i < kMlpIn; ++i) o.features[i] = f[i];
        }
    }
}

}  // namespace pxr
