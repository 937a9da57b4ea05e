// Host side of parex_b200: the handle, device memory, the round drivers and
// the C ABI declared in include/parex_b200.h.
#include <algorithm>
#include <array>
#include <cstdio>
#include <map>
#include <mutex>
#include <cstring>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "pxr_sched.cuh"
#include "pxr_chunk.cuh"

using namespace pxr;

namespace pxr {
constexpr uint32_t kMaxGrid = 148u * 32u;
#ifndef PXR_UNION_LANES
#define PXR_UNION_LANES 1
#endif
constexpr int kUnionLanes = PXR_UNION_LANES;   // lanes per light row in k_union
constexpr uint32_t kSampledDegree = 16;        // mean degree from which k_union uses sampled linking

// ---------------------------------------------------------------------------
// final partition on the device (PartitionManager::finalizePartition,
// cuda/devPartition.h:798-823): sort (label, vertex) pairs, rank the distinct
// labels, scatter the rank back to each vertex.

__global__ void k_fp_keys(const int32_t* lab, uint32_t n, uint32_t* keys, uint32_t* vals) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        keys[i] = (uint32_t)lab[i] ^ 0x80000000u;
        vals[i] = i;
    }
}

__global__ void __launch_bounds__(kBlock) k_fp_rank(const uint32_t* keys0, const uint32_t* keys1,
                                                    const uint32_t* vals0, const uint32_t* vals1,
                                                    const uint32_t* sel_ptr, const uint32_t* n_ptr, int32_t* ids,
                                                    LookbackState lb, const uint32_t* epoch_ptr, RoundCtr* ctr,
                                                    int32_t* num_out) {
    __shared__ uint64_t warp_tot[kBlock / 32];
    __shared__ uint64_t s_excl;
    const uint32_t count = *n_ptr;
    const uint32_t ntiles = (count + kScanTile - 1) / kScanTile;
    const uint32_t tile = fetch_tile(ctr, kSiteFinal);
    if (tile >= ntiles) return;
    const uint32_t sel = *sel_ptr;
    const uint32_t* keys = sel ? keys1 : keys0;
    const uint32_t* vals = sel ? vals1 : vals0;
    const uint32_t epoch = *epoch_ptr;
    const uint32_t first = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t heads = 0, run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        if (i < count && (i == 0 || keys[i] != keys[i - 1])) { heads |= 1u << k; ++run; }
    }
    uint64_t total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)run, warp_tot, &total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(lb, tile, epoch, total, &ctr->err);
        if (threadIdx.x == 0) s_excl = ex;
        if (threadIdx.x == 0 && tile == ntiles - 1) *num_out = (int32_t)(ex + total);
    }
    __syncthreads();
    uint32_t r = (uint32_t)(s_excl + incl - run);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = first + k;
        if (i >= count) break;
        if (heads & (1u << k)) ++r;
        ids[vals[i]] = (int32_t)r - 1;
    }
}

__global__ void k_count_valid(const uint32_t* cols, uint64_t slots, unsigned long long* out) {
    uint32_t c = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < slots; j += (uint64_t)gridDim.x * blockDim.x)
        c += slot_valid(cols[j]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31u) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

// Test hook kernels: the look-back and the sort-status wait on flags that
// nothing sets.  One warp each; scratch holds 2 look-back tiles and one
// status word, all zero (epoch 0), and the waits ask for epoch 1.
__global__ void k_test_lookback_wait(uint32_t* flags, uint64_t* agg, uint64_t* inc, uint32_t spin_limit,
                                     uint32_t* err) {
    LookbackState s{flags, agg, inc};
    lookback_exclusive<Add64>(s, 1u, 1u, err, spin_limit);   // tile 0 never publishes
}

__global__ void k_test_sort_wait(const uint64_t* word, uint32_t spin_limit, uint32_t* err) {
    if (threadIdx.x == 0) wait_sort_status(word, 1u, err, spin_limit);
}

// Cut edges of the partition given by the labels: CSR slots (both directions
// of every edge) whose ends carry different labels, over the graph as
// uploaded (a disabled slot still holds its neighbour under kDisabledBit).
// Final ids are a bijection of label values, so these are the edges whose
// ends carry different final ids.  A tile of kCountTile slots finds its
// first and last rows once; each slot's row is then a binary search between
// them.  bad is set when a slot's neighbour is unknown (pxr_set_state may
// load disabled slots without one).
constexpr uint32_t kCountTile = 4096;

template <typename OffT>
__global__ void __launch_bounds__(kBlock) k_count_cut(const OffT* off, const uint32_t* cols, const int32_t* lab,
                                                      uint32_t n, uint64_t slots, unsigned long long* out,
                                                      uint32_t* bad) {
    __shared__ uint32_t s_rows[2];
    __shared__ unsigned long long s_sum[kBlock / 32];
    const uint64_t ntiles = (slots + kCountTile - 1) / kCountTile;
    unsigned long long cnt = 0;
    uint32_t unknown = 0;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t s0 = tile * kCountTile;
        const uint64_t s1 = s0 + kCountTile < slots ? s0 + kCountTile : slots;
        if (threadIdx.x < 2) {
            // last row r with off[r] <= target (rows are non-decreasing, off[n] = slots > target)
            const uint64_t target = threadIdx.x == 0 ? s0 : s1 - 1;
            uint32_t lo = 0, hi = n - 1;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo + 1) / 2;
                if ((uint64_t)off[mid] <= target) lo = mid; else hi = mid - 1;
            }
            s_rows[threadIdx.x] = lo;
        }
        __syncthreads();
        const uint32_t r0 = s_rows[0], r1 = s_rows[1];
        __syncthreads();
        for (uint64_t sl = s0 + threadIdx.x; sl < s1; sl += blockDim.x) {
            uint32_t lo = r0, hi = r1;
            while (lo < hi) {
                const uint32_t mid = lo + (hi - lo + 1) / 2;
                if ((uint64_t)off[mid] <= sl) lo = mid; else hi = mid - 1;
            }
            const uint32_t u = cols[sl] & ~kDisabledBit;
            if (u >= n) { unknown = 1; continue; }
            cnt += lab[lo] != lab[u] ? 1ull : 0ull;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    if ((threadIdx.x & 31u) == 0) s_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += s_sum[w];
        if (t) atomicAdd(out, t);
    }
    if (unknown) atomicOr(bad, 1u);
}


template <typename OffT>
__global__ void k_degrees(const OffT* off, uint32_t n, uint32_t* ideg, int32_t* lab, uint32_t* act, uint32_t* ids) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        ideg[v] = (uint32_t)(off[v + 1] - off[v]);
        lab[v] = 0;
        act[v] = v;
        ids[v] = v;
    }
}

// Batched instances: label = index of the instance that owns the vertex
// (binary search of the instance starts), the instance volumes, and a flag
// when an edge leaves its instance.
template <typename OffT>
__global__ void k_batch_setup(const OffT* off, const uint32_t* cols, const uint32_t* ideg, const uint32_t* starts,
                              uint32_t n, uint32_t n_inst, int32_t* lab, unsigned long long* vol, uint32_t* bad) {
    for (uint32_t v0 = blockIdx.x * blockDim.x; v0 < n; v0 += gridDim.x * blockDim.x) {
        const uint32_t v = v0 + threadIdx.x;
        const bool valid = v < n;
        uint32_t inst = 0;
        if (valid) {
            uint32_t lo = 0, hi = n_inst;   // starts[0] = 0 <= v < starts[n_inst] = n
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (starts[mid] <= v) lo = mid; else hi = mid;
            }
            inst = lo;
            lab[v] = (int32_t)inst;
            const uint32_t a = starts[inst], b = starts[inst + 1];
            bool out = false;
            for (OffT e = off[v]; e < off[v + 1]; ++e) {
                const uint32_t u = cols[e];
                out |= slot_valid(u) && (u < a || u >= b);
            }
            if (out) atomicOr(bad, 1u);
        }
        // one atomic per warp when the whole warp lies in one instance
        const unsigned long long dg = valid ? ideg[v] : 0ull;
        const uint32_t first = __shfl_sync(0xFFFFFFFFu, inst, 0);
        if (__all_sync(0xFFFFFFFFu, !valid || inst == first)) {
            unsigned long long sum = dg;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xFFFFFFFFu, sum, o);
            if ((threadIdx.x & 31u) == 0 && sum) atomicAdd(&vol[first], sum);
        } else if (valid && dg) {
            atomicAdd(&vol[inst], dg);
        }
    }
}

// x~ = x / internal degree for every vertex, and max |x| over every vertex
__global__ void k_refresh_scaled(const float* x, const uint32_t* ideg, uint32_t n, float* xt, uint32_t* xmax_bits) {
    uint32_t vmax = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float xv = x[v];
        const uint32_t dg = ideg[v];
        xt[v] = dg ? __double2float_rn(__ddiv_rn((double)xv, (double)dg)) : 0.0f;
        const uint32_t b = __float_as_uint(fabsf(xv));
        vmax = b > vmax ? b : vmax;
    }
    for (int o = 16; o > 0; o >>= 1) vmax = max(vmax, __shfl_xor_sync(0xFFFFFFFFu, vmax, o));
    if ((threadIdx.x & 31u) == 0 && vmax) atomicMax(xmax_bits, vmax);
}

// input checks for a CSR already on the device: offsets[0] == 0, offsets[n]
// == 2m, non-decreasing offsets, columns < n; also the maximum row length.
template <typename OffT>
__global__ void k_validate(const OffT* off, const uint32_t* cols, uint32_t n, uint64_t slots, uint32_t* bad,
                           uint32_t* maxdeg) {
    uint32_t b = 0, mx = 0;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t v = tid; v < n; v += stride) {
        const OffT a = off[v], z = off[v + 1];
        if (z < a) b |= 1u;
        else {
            const uint64_t len = (uint64_t)(z - a);
            mx = max(mx, (uint32_t)min(len, (uint64_t)0xFFFFFFFFu));
        }
    }
    if (tid == 0 && ((uint64_t)off[0] != 0 || (uint64_t)off[n] != slots)) b |= 2u;
    for (uint64_t j = tid; j < slots; j += stride)
        if (cols[j] >= n) b |= 4u;
    for (int o = 16; o > 0; o >>= 1) {
        b |= __shfl_xor_sync(0xFFFFFFFFu, b, o);
        mx = max(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    }
    if ((threadIdx.x & 31u) == 0) {
        if (b) atomicOr(bad, b);
        if (mx) atomicMax(maxdeg, mx);
    }
}

// Static row bins: rows longer than light_max slots go to the wide list (up
// to wide_max slots, a warp each) or the heavy list (a CTA each); the order
// inside a list is irrelevant.
template <typename OffT>
__global__ void k_bin_rows(const OffT* off, uint32_t n, uint32_t light_max, uint32_t wide_max, uint32_t* wide,
                           uint32_t* heavy, uint32_t* counts) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint64_t len = (uint64_t)(off[v + 1] - off[v]);
        if (len <= light_max) continue;
        if (len <= wide_max) wide[atomicAdd(&counts[0], 1u)] = v;
        else heavy[atomicAdd(&counts[1], 1u)] = v;
    }
}

// rows per bit length of their size (0: empty rows, 32: 2^31 slots or more)
template <typename OffT>
__global__ void k_degree_hist(const OffT* off, uint32_t n, uint32_t* hist) {
    __shared__ uint32_t sh[33];
    for (int i = threadIdx.x; i < 33; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint64_t len = (uint64_t)(off[v + 1] - off[v]);
        const uint32_t b = len >= (1ull << 31) ? 32u : (len ? 32u - __clz((uint32_t)len) : 0u);
        atomicAdd(&sh[b], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 33; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Profiling aid: hold the stream for a moment so the host can queue a whole
// op before the device starts it; the phase events then time device work
// rather than host launch latency.
__global__ void k_hold(uint32_t ns) {
    for (uint32_t t = 0; t < ns; t += 1000) __nanosleep(1000);
}

__global__ void k_bump_site(uint32_t* epoch, RoundCtr* ctr, int site) {
    epoch[site] += 1;
    ctr->tile_counter[site] = 0;
}

inline uint32_t grid_for(uint64_t threads) {
    const uint64_t g = (threads + kBlock - 1) / kBlock;
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g, kMaxGrid));
}

inline uint32_t host_bitlen(uint64_t v) {
    uint32_t b = 0;
    while (v) { ++b; v >>= 1; }
    return b;
}

}  // namespace pxr

// ---------------------------------------------------------------------------

struct pxr_handle {
    pxr_config cfg{};
    std::string err;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t side_stream = nullptr;   // captures the bodies of IF nodes
    cudaStream_t walk_side[2] = {};       // the wide- and heavy-row walk kernels, beside the light-row one
    cudaEvent_t walk_ev[3] = {};          // fork, and the two joins
    cudaStream_t stream = nullptr;
    bool initialized = false;
    bool off64 = false;
    uint32_t n = 0;
    uint64_t m = 0, slots = 0;
    uint32_t maxdeg = 0;
    uint32_t W = 8;
    uint32_t nb_bits = 0;
    std::vector<void*> allocs;
    size_t bytes = 0;

    void* off = nullptr;
    uint32_t* cols = nullptr;
    int32_t* lab = nullptr;
    uint32_t* ideg = nullptr;
    float* x = nullptr;
    float* xt[2] = {nullptr, nullptr};
    int2* dv = nullptr;
    uint32_t *parent = nullptr, *acc_max = nullptr, *acc_min = nullptr, *acc_cnt = nullptr;
    int64_t* acc_sum = nullptr;
    int32_t* newlab = nullptr;
    double* avg = nullptr;
    uint32_t* cert = nullptr;
    int32_t* pdif = nullptr;
    uint32_t* pvol = nullptr;
    uint32_t* act[2] = {nullptr, nullptr};
    uint32_t* ids[2] = {nullptr, nullptr};
    uint32_t* par[2] = {nullptr, nullptr};   // per active-list position: cluster it was last swept in
    uint64_t* keys[2] = {nullptr, nullptr};
    uint32_t* vals[2] = {nullptr, nullptr};
    ClusterTables tab[2]{};
    uint32_t* cut_off = nullptr;
    uint8_t* split = nullptr;
    pxr_sweep_cut* allcuts = nullptr;
    unsigned long long* walk_stats = nullptr;
    uint32_t* rep[2] = {nullptr, nullptr};
    uint32_t* roots[2] = {nullptr, nullptr};
    LookbackState lb[kSiteRoots + 1]{};
    uint32_t* rootmap = nullptr;
    uint32_t* lb_epoch = nullptr;
    RoundCtr* ctr = nullptr;
    SortState sort{};
    uint32_t* sort_end_bit = nullptr;
    uint32_t* fp_end_bit = nullptr;
    uint32_t* d_n = nullptr;
    int32_t* d_num = nullptr;
    unsigned long long* d_valid = nullptr;
    RoundCtr* h_ctr = nullptr;  // pinned mirror

    uint32_t* d_check = nullptr;   // [3]: invalid-input bits, max row length, heavy rows
    RoundCtr* probe_ctr = nullptr;    // scratch counters for the tuner's timed walk steps
    bool plan_forced = false;
    pxr_row_plan plan_info{};         // last plan chosen (pxr_get_row_plan)
    bool sort_forced = false;
    pxr_sort_plan sort_info{0, 16, 2, 0, 0, {0.0f, 0.0f, 0.0f}};   // sweep sort plan (pxr_get_sort_plan)
    uint32_t light_max = kLightRow;   // row bins (see k_bin_rows)
    uint32_t wide_max = kWideRow;
    uint32_t* wide = nullptr;
    uint32_t n_wide = 0;
    uint32_t* hist = nullptr;         // [33] rows per bit length of the row size
    uint32_t* heavy = nullptr;
    uint32_t n_heavy = 0;
    // learned sweep schedule
    pxr_schedule sched{};
    uint8_t* sflag = nullptr;
    uint32_t* smax = nullptr;
    uint32_t* smin = nullptr;
    uint8_t* nflag = nullptr;
    uint32_t* rootc = nullptr;
    float* mlp = nullptr;             // kMlpImage floats
    std::vector<float> mlp_img;       // host copy (set before or after allocation)
    pxr_cluster_record* records = nullptr;   // n entries, allocated when trace is first enabled
    uint32_t records_n = 0;
    int xcur = 0, tcur = 0, acur = 0;
    int sweep_tab = 0;
    cudaGraphExec_t graphs[8] = {};  // device-driven loop, one per parity combination
    cudaGraphConditionalHandle conds[8] = {};
    uint64_t body_launches[8] = {};  // kernels per replay of the loop body
    bool sort_regions = false;       // set while capturing: the body holds the sort IF nodes
    bool body_regions[8] = {};
    uint32_t last_rounds = 0;
    double last_ms = 0.0;
    uint64_t launches = 0;
    // per-phase profiling (stream driver)
    bool profiling = false;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    std::vector<cudaEvent_t> event_pool;
    double phase_ms[16] = {};
    uint64_t phase_launches[16] = {};
};

namespace {

pxr_status fail(pxr_handle* h, pxr_status s, const std::string& msg) {
    if (h) h->err = msg;
    return s;
}

pxr_status cuda_fail(pxr_handle* h, cudaError_t e, const char* where) {
    return fail(h, e == cudaErrorMemoryAllocation ? PXR_OUT_OF_MEMORY : PXR_CUDA_ERROR,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define PXR_CUDA(h, call)                                        \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail((h), e_, #call); \
    } while (0)

template <typename T>
cudaError_t dalloc(pxr_handle* h, T** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    // the handle's memory cap (pxr_config.memory_cap_mib) refuses like a full device
    if (h->cfg.memory_cap_mib && h->bytes + bytes > ((size_t)h->cfg.memory_cap_mib << 20))
        return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return e;
    h->allocs.push_back(q);
    h->bytes += bytes;
    *p = static_cast<T*>(q);
    return cudaSuccess;
}

void drop_graphs(pxr_handle* h) {
    for (auto& g : h->graphs)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

void release(pxr_handle* h) {
    drop_graphs(h);
    for (void* p : h->allocs) cudaFree(p);
    h->allocs.clear();
    h->records = nullptr;
    h->records_n = 0;
    h->bytes = 0;
    h->initialized = false;
}

template <typename OffT>
Dev<OffT> make_dev(pxr_handle* h) {
    Dev<OffT> d{};
    d.off = static_cast<const OffT*>(h->off);
    d.cols = h->cols;
    d.n = h->n;
    d.nb_bits = h->nb_bits;
    d.sc_threshold = h->cfg.sc_threshold;
    d.rw_threshold = h->cfg.rw_threshold;
    d.division = h->cfg.division;
    d.lab = h->lab;
    d.ideg = h->ideg;
    d.x = h->x;
    d.dv = h->dv;
    d.parent = h->parent;
    d.acc_max = h->acc_max;
    d.acc_min = h->acc_min;
    d.acc_sum = h->acc_sum;
    d.acc_cnt = h->acc_cnt;
    d.newlab = h->newlab;
    d.avg = h->avg;
    d.cert = h->cert;
    d.pdif = h->pdif;
    d.pvol = h->pvol;
    d.cut_off = h->cut_off;
    d.walk_stats = h->walk_stats;
    d.rep[0] = h->rep[0];
    d.rep[1] = h->rep[1];
    // sampled linking pays where rows are long (measured: 16k planted
    // partition and 3D grids slower with it, 512-instance batch faster)
    d.union_sampled = h->cfg.components == PXR_COMPONENTS_SAMPLED ? 1u
                      : h->cfg.components == PXR_COMPONENTS_PLAIN ? 0u
                      : (h->slots >= (uint64_t)kSampledDegree * h->n ? 1u : 0u);
    d.split = h->split;
    d.allcuts = h->allcuts;
    d.roots[0] = h->roots[0];
    d.roots[1] = h->roots[1];
    d.lb_scan = h->lb[kSiteScan];
    d.lb_relabel = h->lb[kSiteRelabel];
    d.lb_apply = h->lb[kSiteApply];
    d.lb_ids = h->lb[kSiteIds];
    d.lb_cvol = h->lb[kSiteCvol];
    d.lb_epoch = h->lb_epoch;
    d.ctr = h->ctr;
    d.sort = h->sort;
    d.sort_end_bit = h->sort_end_bit;
    d.light_max = h->light_max;
    d.wide = h->wide;
    d.n_wide = h->n_wide;
    d.heavy = h->heavy;
    d.n_heavy = h->n_heavy;
    d.sched = h->sched.mode;
    d.trace = (h->sched.trace && h->records) ? 1u : 0u;
    d.sflag = h->sflag;
    d.smax = h->smax;
    d.smin = h->smin;
    d.nflag = h->nflag;
    d.rootc = h->rootc;
    d.lb_sched = h->lb[kSiteSched];
    d.lb_emit = h->lb[kSiteEmit];
    d.lb_carry = h->lb[kSiteCarry];
    d.lb_roots = h->lb[kSiteRoots];
    d.rootmap = h->rootmap;
    d.n_words = (h->n + 31u) / 32u;
    d.mlp = h->mlp;
    d.safety = h->sched.safety;
    d.max_skip = h->sched.max_skip;
    d.cut_gate = h->sched.cut_gate;
    d.due_period = h->sched.due_period;
    d.records = h->records;
    return d;
}

// ---------------------------------------------------------------------------
// phase profiling: CUDA events around each phase of a round (stream driver)

enum Phase {
    kPhWalk, kPhNodeDiff, kPhEmit, kPhSort, kPhScan, kPhClusterCut, kPhCutInit, kPhUnion,
    kPhComponents, kPhRootSort, kPhRelabel, kPhApply, kPhDisable, kPhCvol, kPhBook, kPhSched, kPhaseCount
};
const char* kPhaseNames[kPhaseCount] = {"walk", "nodediff", "emit_keys", "sort", "sweep_scan", "cluster_cut",
                                        "cut_init", "union", "components", "root_sort", "relabel", "apply",
                                        "disable", "cvol_scan", "bookkeeping", "schedule"};

cudaEvent_t take_event(pxr_handle* h) {
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

template <class F>
void phase(pxr_handle* h, Phase ph, int nlaunch, F&& launch) {
    h->launches += nlaunch;
    h->phase_launches[ph] += nlaunch;
    if (!h->profiling) { launch(); return; }
    cudaEvent_t a = take_event(h), b = take_event(h);
    cudaEventRecord(a, h->stream);
    launch();
    cudaEventRecord(b, h->stream);
    h->marks.push_back({ph, {a, b}});
}

void collect_phases(pxr_handle* h) {
    for (auto& mk : h->marks) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, mk.second.first, mk.second.second) == cudaSuccess) h->phase_ms[mk.first] += ms;
        h->event_pool.push_back(mk.second.first);
        h->event_pool.push_back(mk.second.second);
    }
    h->marks.clear();
}

// ---------------------------------------------------------------------------
// stages

// launches of the long-row kernels: warp per wide row, CTA per heavy row
int long_launches(const pxr_handle* h) { return (h->n_wide ? 1 : 0) + (h->n_heavy ? 1 : 0); }
uint32_t wide_grid(const pxr_handle* h) { return std::min((h->n_wide + kBlock / 32 - 1) / (kBlock / 32), 148u * 16u); }
uint32_t heavy_grid(const pxr_handle* h) { return std::min(h->n_heavy, 148u * 16u); }
#define PXR_LONG(h, kern, ...)                                                                         \
    do {                                                                                               \
        if ((h)->n_wide) launch_pdl(kern<OffT, 32>, wide_grid(h), kBlock, 0, s, __VA_ARGS__);          \
        if ((h)->n_heavy) launch_pdl(kern<OffT, kBlock>, heavy_grid(h), kBlock, 0, s, __VA_ARGS__);    \
    } while (0)

// Launch with programmatic stream serialization: the kernel may be scheduled
// while its predecessor in the stream drains, and waits in pdl_wait() before
// it reads anything.  Launch errors surface through cudaGetLastError().
template <typename... KArgs, typename... Args>
void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

void hold_for_profiling(pxr_handle* h) {
    if (h->profiling) k_hold<<<1, 1, 0, h->stream>>>(300000u);
}

#define PXR_TRY(call)                      \
    do {                                   \
        const cudaError_t e_ = (call);     \
        if (e_ != cudaSuccess) return e_;  \
    } while (0)

constexpr cudaGraphConditionalHandle kNoCond = 0;   // round preparation outside the IF-node form

// kernels of the global sort (histogram, plan, 8 digit passes)
constexpr uint64_t kGsortLaunches = 2 + kMaxPasses;

// The graph being captured on h->stream, or null outside capture.
cudaGraph_t capture_graph(pxr_handle* h) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    if (cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &g) != cudaSuccess) return nullptr;
    return cs == cudaStreamCaptureStatusActive ? g : nullptr;
}

// Run body(stream) under an IF node of the graph being captured on h->stream;
// `cond` is set on the device by an earlier kernel of the same graph.
// Without a handle, body runs on h->stream (its kernels guard themselves).
template <class F>
cudaError_t if_region(pxr_handle* h, cudaGraphConditionalHandle cond, F&& body) {
    if (!cond) return body(h->stream);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaError_t e = cudaStreamGetCaptureInfo(h->stream, &cs, nullptr, &g, &deps, &ndeps);
    if (e != cudaSuccess) return e;
    if (cs != cudaStreamCaptureStatusActive) return cudaErrorStreamCaptureInvalidated;
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = cond;
    params.conditional.type = cudaGraphCondTypeIf;
    params.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, g, deps, ndeps, &params);
    if (e != cudaSuccess) return e;
    e = cudaStreamBeginCaptureToGraph(h->side_stream, params.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    const cudaError_t eb = body(h->side_stream);
    cudaGraph_t captured = nullptr;
    e = cudaStreamEndCapture(h->side_stream, &captured);
    if (e == cudaSuccess) e = eb;
    if (e != cudaSuccess) return e;
    return cudaStreamUpdateCaptureDependencies(h->stream, &node, 1, cudaStreamSetCaptureDependencies);
}

// A row kernel in its three parts, which work disjoint rows: light(st)
// launches the light-row kernel(s) on s, wide(st) and heavy(st) the
// warp- and CTA-per-row kernels on the handle's two side streams, forked
// from s and joined back into it.  Running side by side, each part fills the
// SMs the others leave idle in their last wave (in a captured graph the three
// are parallel branches).  With no long rows, light(s) alone.
template <class Light, class Wide, class Heavy>
void launch_row_parts(pxr_handle* h, cudaStream_t s, Light light, Wide wide, Heavy heavy) {
    if (!h->n_wide && !h->n_heavy) {
        light(s);
        return;
    }
    cudaEventRecord(h->walk_ev[0], s);
    if (h->n_wide) {
        cudaStreamWaitEvent(h->walk_side[0], h->walk_ev[0], 0);
        wide(h->walk_side[0]);
        cudaEventRecord(h->walk_ev[1], h->walk_side[0]);
    }
    if (h->n_heavy) {
        cudaStreamWaitEvent(h->walk_side[1], h->walk_ev[0], 0);
        heavy(h->walk_side[1]);
        cudaEventRecord(h->walk_ev[2], h->walk_side[1]);
    }
    light(s);
    if (h->n_wide) cudaStreamWaitEvent(s, h->walk_ev[1], 0);
    if (h->n_heavy) cudaStreamWaitEvent(s, h->walk_ev[2], 0);
}

// One walk step: light rows of the active list (W lanes each), the wide list
// (a warp per row) and the heavy list (a CTA per row).
template <typename OffT, int W>
void launch_walk(pxr_handle* h, const Dev<OffT>& d, cudaStream_t s, const float* xt_in, float* xt_out) {
    launch_row_parts(
        h, s,
        [&](cudaStream_t st) {
            k_walk<OffT, W><<<grid_for((uint64_t)h->n * W), kBlock, 0, st>>>(d, h->ids[h->acur], xt_in, xt_out);
        },
        [&](cudaStream_t st) { k_walk_long<OffT, 32><<<wide_grid(h), kBlock, 0, st>>>(d, xt_in, xt_out); },
        [&](cudaStream_t st) { k_walk_long<OffT, kBlock><<<heavy_grid(h), kBlock, 0, st>>>(d, xt_in, xt_out); });
}

template <typename OffT, int W>
cudaError_t op_walk(pxr_handle* h, bool in_round = false) {
    Dev<OffT> d = make_dev<OffT>(h);
    cudaStream_t s = h->stream;
    hold_for_profiling(h);
    phase(h, kPhBook, 1, [&] { launch_pdl(k_round_prep<OffT>, 1, 32, 0, s, d, 0, kNoCond, kNoCond); });
    phase(h, kPhWalk, 1 + long_launches(h), [&] { launch_walk<OffT, W>(h, d, s, h->xt[h->xcur], h->xt[h->xcur ^ 1]); });
    // the next walk's fixed-point scale follows max |x'|; inside a plain round
    // the cut stage recomputes it over the recentred potentials anyway
    if (!in_round || h->sched.mode) phase(h, kPhBook, 1, [&] { launch_pdl(k_after_walk<OffT>, 1, 1, 0, s, d); });
    h->xcur ^= 1;
    return cudaGetLastError();
}

template <typename OffT, int W>
cudaError_t op_sweep(pxr_handle* h) {
    Dev<OffT> d = make_dev<OffT>(h);
    cudaStream_t s = h->stream;
    const ClusterTables& t = h->tab[h->tcur];
    hold_for_profiling(h);
    // graph driver, plain form: the global sort and the chunked sort become
    // IF nodes, so a round launches only the sort it uses
    cudaGraphConditionalHandle c_gsort = 0, c_chunk = 0;
    if (!h->sched.mode) {
        if (cudaGraph_t g = capture_graph(h)) {
            PXR_TRY(cudaGraphConditionalHandleCreate(&c_gsort, g, 1u, cudaGraphCondAssignDefault));
            PXR_TRY(cudaGraphConditionalHandleCreate(&c_chunk, g, 1u, cudaGraphCondAssignDefault));
            h->sort_regions = true;
        }
    }
    phase(h, kPhBook, 1, [&] { launch_pdl(k_round_prep<OffT>, 1, 32, 0, s, d, 1, c_gsort, c_chunk); });
    const uint32_t tiles = std::max((h->n + kScanTile - 1) / kScanTile, 1u);
    if (h->sched.mode)
        phase(h, kPhSched, 3, [&] {
            launch_pdl(k_cluster_spread<OffT>, std::min(tiles, kMaxGrid), kBlock, 0, s, d, h->ids[h->acur]);
            launch_pdl(k_due_scan<OffT>, tiles, kBlock, 0, s, d, t);
            launch_pdl(k_walk_only_check<OffT>, 1, 1, 0, s, d);
        });
    // learned schedule: the sweep set is compacted first and the edge
    // differences are taken over it alone (carried clusters need none)
    if (h->sched.mode) {
        phase(h, kPhEmit, 1, [&] {
            launch_pdl(k_emit_sched<OffT>, tiles, kBlock, 0, s, d, h->act[h->acur], h->keys[0], h->vals[0], t.best);
        });
        phase(h, kPhNodeDiff, 2 + long_launches(h), [&] {
            launch_row_parts(
                h, s,
                [&](cudaStream_t st) {
                    k_nodediff<OffT, W><<<grid_for((uint64_t)h->n * W), kBlock, 0, st>>>(d, h->vals[0], 1);
                    k_nodediff<OffT, W><<<grid_for((uint64_t)h->n * W), kBlock, 0, st>>>(d, h->ids[h->acur], 0);
                },
                [&](cudaStream_t st) { k_nodediff_long<OffT, 32><<<wide_grid(h), kBlock, 0, st>>>(d); },
                [&](cudaStream_t st) { k_nodediff_long<OffT, kBlock><<<heavy_grid(h), kBlock, 0, st>>>(d); });
        });
    } else {
        phase(h, kPhNodeDiff, 1 + long_launches(h), [&] {
            launch_row_parts(
                h, s,
                [&](cudaStream_t st) {
                    k_nodediff<OffT, W><<<grid_for((uint64_t)h->n * W), kBlock, 0, st>>>(d, h->ids[h->acur], 0);
                },
                [&](cudaStream_t st) { k_nodediff_long<OffT, 32><<<wide_grid(h), kBlock, 0, st>>>(d); },
                [&](cudaStream_t st) { k_nodediff_long<OffT, kBlock><<<heavy_grid(h), kBlock, 0, st>>>(d); });
        });
        phase(h, kPhEmit, 1, [&] {
            launch_pdl(k_emit<OffT>, grid_for(h->n), kBlock, 0, s, d, h->act[h->acur], h->keys[0], h->vals[0], t.best);
        });
    }
    SortBuffers<uint64_t> b{};
    b.keys[0] = h->keys[0]; b.keys[1] = h->keys[1];
    b.vals[0] = h->vals[0]; b.vals[1] = h->vals[1];
    // the learned schedule sets the sweep size after the round's preparation
    b.count = h->sched.mode ? &h->ctr->n_sweep : &h->ctr->n_gsort;
    b.end_bit = h->sort_end_bit;
    b.capacity = h->n;
    cudaError_t e = cudaSuccess;
    // per-phase timing (stream driver): read the round's choice and launch
    // only that sort, as the graph driver's IF nodes do
    bool run_gsort = true, run_chunk = true;
    if (h->profiling && !c_gsort) {
        uint32_t chunk_path = 0;
        PXR_TRY(cudaMemcpyAsync(&chunk_path, &h->ctr->chunk_path, 4, cudaMemcpyDeviceToHost, s));
        PXR_TRY(cudaStreamSynchronize(s));
        run_gsort = chunk_path == 0;
        run_chunk = chunk_path != 0;
    }
    phase(h, kPhSort, (run_gsort ? kGsortLaunches : 0) + (run_chunk ? 1 : 0), [&] {
        if (run_gsort)
            e = if_region(h, c_gsort, [&](cudaStream_t st) {
                return radix_sort<uint64_t>(b, h->sort, &h->ctr->err, st, 64, (int)h->sort_info.plan);
            });
        // the chunked sort writes buffer 0, which round preparation selects
        if (e == cudaSuccess && run_chunk)
            e = if_region(h, c_chunk, [&](cudaStream_t st) {
                k_chunk_sort<OffT><<<std::min(std::max((h->n + kChunk - 1) / kChunk, 1u), 148u), kChunkThreads,
                                     chunk_sort_smem(), st>>>(d, t, h->act[h->acur], h->par[h->acur], h->keys[0],
                                                              h->vals[0]);
                return cudaGetLastError();
            });
    });
    if (e != cudaSuccess) return e;
    phase(h, kPhScan, 1, [&] {
        k_sweep_scan<OffT><<<tiles, kBlock, 0, s>>>(d, t, h->keys[0], h->keys[1], h->vals[0], h->vals[1]);
    });
    phase(h, kPhClusterCut, 1, [&] { launch_pdl(k_cluster_cut<OffT>, grid_for(h->n), kBlock, 0, s, d, t); });
    h->sweep_tab = h->tcur;
    return cudaGetLastError();
}

template <typename OffT, int W>
cudaError_t op_cut(pxr_handle* h) {
    Dev<OffT> d = make_dev<OffT>(h);
    cudaStream_t s = h->stream;
    const ClusterTables& t = h->tab[h->tcur];
    const ClusterTables& nt = h->tab[h->tcur ^ 1];
    const uint32_t tiles = std::max((h->n + kScanTile - 1) / kScanTile, 1u);
    hold_for_profiling(h);
    phase(h, kPhBook, 1, [&] { launch_pdl(k_round_prep<OffT>, 1, 32, 0, s, d, 2, kNoCond, kNoCond); });
    if (h->sched.mode)
        phase(h, kPhSched, 2, [&] {
            launch_pdl(k_carry_all<OffT>, grid_for(h->n), kBlock, 0, s, d, t, nt, h->act[h->acur], h->act[h->acur ^ 1],
                                                                 h->ids[h->acur], h->ids[h->acur ^ 1]);
            launch_pdl(k_carry_roots<OffT>, grid_for(h->n), kBlock, 0, s, d, t);
        });
    phase(h, kPhCutInit, 1, [&] {
        launch_pdl(k_cut_init<OffT>, grid_for(h->n), kBlock, 0, s, d, t, h->vals[0], h->vals[1], h->keys[0], h->keys[1]);
    });
    phase(h, kPhUnion, 3 + (d.union_sampled ? 3 : 0) + long_launches(h), [&] {
        launch_pdl(k_link_first<OffT>, grid_for(h->n), kBlock, 0, s, d, h->ids[h->acur]);
        launch_pdl(k_compress<OffT>, grid_for(h->n), kBlock, 0, s, d, h->ids[h->acur]);
        if (d.union_sampled) {
            launch_pdl(k_union_sample<OffT>, grid_for(h->n), kBlock, 0, s, d, h->ids[h->acur]);
            launch_pdl(k_compress<OffT>, grid_for(h->n), kBlock, 0, s, d, h->ids[h->acur]);
            launch_pdl(k_union_reps<OffT>, grid_for(h->n), kBlock, 0, s, d, t, h->vals[0], h->vals[1]);
        }
        // lock-free unions over disjoint rows: the three parts side by side
        launch_row_parts(
            h, s,
            [&](cudaStream_t st) {
                k_union<OffT, kUnionLanes><<<grid_for((uint64_t)h->n * kUnionLanes), kBlock, 0, st>>>(d, h->ids[h->acur]);
            },
            [&](cudaStream_t st) { k_union_long<OffT, 32><<<wide_grid(h), kBlock, 0, st>>>(d); },
            [&](cudaStream_t st) { k_union_long<OffT, kBlock><<<heavy_grid(h), kBlock, 0, st>>>(d); });
    });
    phase(h, kPhComponents, 1, [&] {
        launch_pdl(k_components_data<OffT>, std::min(tiles, kMaxGrid), kBlock, 0, s, d, t, h->vals[0], h->vals[1],
                                                                              h->keys[0], h->keys[1]);
    });
    // roots in vertex-id order (the order of the reference's root sort)
    const uint32_t root_tiles = (uint32_t)(((h->n + 31u) / 32u + kRootTileWords - 1) / kRootTileWords);
    phase(h, kPhRootSort, 1, [&] { launch_pdl(k_root_compact<OffT>, std::max(root_tiles, 1u), kBlock, 0, s, d, h->roots[0]); });
    const uint32_t relabel_tiles = std::min(std::max((h->n + kRelabelTile - 1) / kRelabelTile, 1u), 148u * 8u);
    phase(h, kPhRelabel, 1, [&] { launch_pdl(k_relabel<OffT>, relabel_tiles, kBlock, 0, s, d, h->roots[0], t, nt); });
    if (h->sched.mode)
        phase(h, kPhSched, 1, [&] {
            launch_pdl(k_carry_vertices<OffT>, tiles, kBlock, 0, s, d, t, h->act[h->acur], h->act[h->acur ^ 1]);
        });
    phase(h, kPhApply, 2, [&] {
        launch_pdl(k_newlab<OffT>, grid_for(h->n), kBlock, 0, s, d, t, h->ids[h->acur]);
        launch_pdl(k_apply<OffT>, tiles, kBlock, 0, s, d, t, h->vals[0], h->vals[1], h->keys[0], h->keys[1],
                                               h->act[h->acur ^ 1], h->par[h->acur ^ 1]);
    });
    phase(h, kPhDisable, 1 + long_launches(h), [&] {
        // disjoint rows; shared results are atomics (volumes, max |x|): side by side
        launch_row_parts(
            h, s,
            [&](cudaStream_t st) {
                k_ids_disable<OffT, W><<<tiles, kBlock, 0, st>>>(d, h->ids[h->acur], h->ids[h->acur ^ 1], h->xt[h->xcur], nt);
            },
            [&](cudaStream_t st) { k_disable_long<OffT, 32><<<wide_grid(h), kBlock, 0, st>>>(d, h->xt[h->xcur], nt); },
            [&](cudaStream_t st) { k_disable_long<OffT, kBlock><<<heavy_grid(h), kBlock, 0, st>>>(d, h->xt[h->xcur], nt); });
    });
    phase(h, kPhCvol, 1, [&] { launch_pdl(k_cvol_scan<OffT>, tiles, kBlock, 0, s, d, nt); });
    if (h->sched.mode || d.trace)
        phase(h, kPhSched, 1, [&] { launch_pdl(k_schedule<OffT>, std::min(grid_for(h->n), 148u * 8u), kBlock, 0, s, d, t, nt); });
    phase(h, kPhBook, 1, [&] { launch_pdl(k_round_end<OffT>, 1, 1, 0, s, d); });
    h->tcur ^= 1;
    h->acur ^= 1;
    return cudaGetLastError();
}

template <typename OffT, int W>
cudaError_t op_round(pxr_handle* h) {
    cudaError_t e = op_walk<OffT, W>(h, true);
    if (e == cudaSuccess) e = op_sweep<OffT, W>(h);
    if (e == cudaSuccess) e = op_cut<OffT, W>(h);
    return e;
}

// two rounds (the parities return to their start) and the loop condition
template <typename OffT, int W>
cudaError_t op_loop_body(pxr_handle* h, cudaGraphConditionalHandle cond) {
    cudaError_t e = op_round<OffT, W>(h);
    if (e == cudaSuccess) e = op_round<OffT, W>(h);
    if (e != cudaSuccess) return e;
    Dev<OffT> d = make_dev<OffT>(h);
    phase(h, kPhBook, 1, [&] { launch_pdl(k_loop_cond<OffT>, 1, 1, 0, h->stream, d, cond); });
    return cudaGetLastError();
}

enum Op { kOpWalk, kOpSweep, kOpCut, kOpRound, kOpLoopBody };

template <typename OffT>
cudaError_t dispatch_w(pxr_handle* h, Op op, cudaGraphConditionalHandle cond) {
#define PXR_OPS(WV)                                              \
    switch (op) {                                                \
        case kOpWalk: return op_walk<OffT, WV>(h);               \
        case kOpSweep: return op_sweep<OffT, WV>(h);             \
        case kOpCut: return op_cut<OffT, WV>(h);                 \
        case kOpLoopBody: return op_loop_body<OffT, WV>(h, cond); \
        default: return op_round<OffT, WV>(h);                   \
    }
    switch (h->W) {
        case 1: PXR_OPS(1)
        case 4: PXR_OPS(4)
        case 16: PXR_OPS(16)
        case 32: PXR_OPS(32)
        default: PXR_OPS(8)
    }
#undef PXR_OPS
}

cudaError_t dispatch(pxr_handle* h, Op op, cudaGraphConditionalHandle cond = 0) {
    return h->off64 ? dispatch_w<uint64_t>(h, op, cond) : dispatch_w<uint32_t>(h, op, cond);
}

pxr_status check_device_errors(pxr_handle* h) {
    if (h->h_ctr->err) {
        const uint32_t e = h->h_ctr->err;
        h->h_ctr->err = 0;
        cudaMemsetAsync(&h->ctr->err, 0, sizeof(uint32_t), h->stream);
        return fail(h, PXR_DEVICE_FAULT, "device-side bounded wait or invariant failed (bits " + std::to_string(e) + ")");
    }
    return PXR_OK;
}

pxr_status sync_ctr(pxr_handle* h) {
    PXR_CUDA(h, cudaMemcpyAsync(h->h_ctr, h->ctr, sizeof(RoundCtr), cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    collect_phases(h);
    return check_device_errors(h);
}

pxr_status run_op(pxr_handle* h, Op op) {
    if (!h) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    cudaError_t e = dispatch(h, op);
    if (e != cudaSuccess) return cuda_fail(h, e, "kernel launch");
    return sync_ctr(h);
}

// Capture the two-round loop body under a conditional while node; the whole
// decomposition then runs as one graph launch with no host round trip.
pxr_status build_loop_graph(pxr_handle* h, int key) {
    cudaGraph_t g = nullptr;
    PXR_CUDA(h, cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle cond = 0;
    cudaError_t e = cudaGraphConditionalHandleCreate(&cond, g, 1u, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(h, e, "cudaGraphConditionalHandleCreate"); }
    cudaGraphNodeParams params{};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = cond;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &params);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(h, e, "cudaGraphAddNode(conditional)"); }
    cudaGraph_t body = params.conditional.phGraph_out[0];
    cudaStream_t user = h->stream;
    h->stream = h->own_stream;
    const bool prof = h->profiling;
    h->profiling = false;
    const uint64_t launches_before = h->launches;
    h->sort_regions = false;
    e = cudaStreamBeginCaptureToGraph(h->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    cudaError_t e2 = e == cudaSuccess ? dispatch(h, kOpLoopBody, cond) : e;
    h->body_launches[key] = h->launches - launches_before;
    h->body_regions[key] = h->sort_regions;
    h->launches = launches_before;   // counted when the graph runs
    cudaGraph_t captured = nullptr;
    if (e == cudaSuccess) e = cudaStreamEndCapture(h->stream, &captured);
    h->stream = user;
    h->profiling = prof;
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) { cudaGraphDestroy(g); return cuda_fail(h, e, "round capture"); }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    h->graphs[key] = exec;
    h->conds[key] = cond;
    return PXR_OK;
}

__global__ void k_loop_begin(RoundCtr* c, uint32_t cap) {
    c->loop_start = c->rounds;
    c->loop_cap = cap;
}

pxr_status decompose_graph(pxr_handle* h) {
    const int key = h->xcur | (h->tcur << 1) | (h->acur << 2);
    if (!h->graphs[key]) {
        pxr_status st = build_loop_graph(h, key);
        if (st != PXR_OK) return st;
    }
    k_loop_begin<<<1, 1, 0, h->stream>>>(h->ctr, h->cfg.max_rounds);
    PXR_CUDA(h, cudaGetLastError());
    const uint32_t before = h->h_ctr->rounds;
    const uint64_t g0 = h->h_ctr->stat_gsort_slots, c0 = h->h_ctr->stat_chunk_slots;
    PXR_CUDA(h, cudaGraphLaunch(h->graphs[key], h->stream));
    pxr_status st = sync_ctr(h);
    // the body (two rounds) ran ceil(rounds / 2) times, at least once; of the
    // two sort IF nodes of each round slot only one ran
    const uint32_t ran = h->h_ctr->rounds - before;
    const uint64_t iters = std::max<uint64_t>(1, (ran + 1) / 2);
    if (h->body_regions[key]) {
        const uint64_t dg = h->h_ctr->stat_gsort_slots - g0, dc = h->h_ctr->stat_chunk_slots - c0;
        h->launches += 1 + iters * (h->body_launches[key] - 2 * (kGsortLaunches + 1)) + dg * kGsortLaunches + dc;
    } else {
        h->launches += 1 + h->body_launches[key] * iters;
    }
    return st;
}

pxr_status decompose_stream(pxr_handle* h) {
    pxr_status st = sync_ctr(h);
    const uint32_t start = h->h_ctr->rounds;
    while (st == PXR_OK && !h->h_ctr->done && h->h_ctr->rounds - start < h->cfg.max_rounds) {
        cudaError_t e = dispatch(h, kOpRound);
        if (e != cudaSuccess) return cuda_fail(h, e, "round launch");
        st = sync_ctr(h);
    }
    return st;
}

// ---------------------------------------------------------------------------

// every cluster due, no sweep history (after any change of the partition state)
pxr_status reset_schedule_state(pxr_handle* h) {
    const size_t N = std::max<uint32_t>(h->n, 1);
    for (int i = 0; i < 2; ++i) {
        PXR_CUDA(h, cudaMemsetAsync(h->tab[i].skip, 0, N * sizeof(uint16_t), h->stream));
        PXR_CUDA(h, cudaMemsetAsync(h->tab[i].hist, 0, N * sizeof(SchedHist), h->stream));
    }
    return PXR_OK;
}

pxr_status setup_tables_initial(pxr_handle* h) {
    // one cluster with every vertex: start 0, size n, volume 2m, root 0
    std::vector<uint32_t> one = {0u, h->n, (uint32_t)h->slots, 0u, 0u};
    const ClusterTables& t = h->tab[h->tcur];
    PXR_CUDA(h, cudaMemcpyAsync(t.start, &one[0], 4, cudaMemcpyHostToDevice, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(t.size, &one[1], 4, cudaMemcpyHostToDevice, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(t.vol, &one[2], 4, cudaMemcpyHostToDevice, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(t.vol_start, &one[3], 4, cudaMemcpyHostToDevice, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(t.root, &one[4], 4, cudaMemcpyHostToDevice, h->stream));
    PXR_CUDA(h, cudaMemsetAsync(t.best, 0xFF, 8, h->stream));
    return PXR_OK;
}

template <typename OffT>
pxr_status allocate(pxr_handle* h, uint32_t n, uint64_t m) {
    release(h);
    h->n = n;
    h->m = m;
    h->slots = 2 * m;
    h->off64 = sizeof(OffT) == 8;
    const size_t N = std::max<uint32_t>(n, 1);
    // look-back state per site, sized for the smallest tile (k_relabel's)
    const uint32_t scan_tiles = (uint32_t)((N + kRelabelTile - 1) / kRelabelTile) + 1;
    const uint32_t sort_tiles = (uint32_t)((N + kSortMinTile - 1) / kSortMinTile) + 1;   // any sort plan's tiles
    cudaError_t e = cudaSuccess;
#define A(ptr, cnt) if (e == cudaSuccess) e = dalloc(h, ptr, cnt)
    A(reinterpret_cast<OffT**>(&h->off), (size_t)n + 1);
    A(&h->cols, std::max<uint64_t>(h->slots, 1));
    A(&h->lab, N); A(&h->ideg, N); A(&h->x, N); A(&h->xt[0], N); A(&h->xt[1], N);
    A(&h->dv, N); A(&h->parent, N); A(&h->acc_max, N); A(&h->acc_min, N); A(&h->acc_cnt, N);
    A(&h->acc_sum, N); A(&h->newlab, N); A(&h->avg, N); A(&h->pdif, N); A(&h->pvol, N); A(&h->cert, N);
    for (int i = 0; i < 2; ++i) {
        A(&h->act[i], N); A(&h->ids[i], N); A(&h->par[i], N); A(&h->keys[i], N); A(&h->vals[i], N); A(&h->roots[i], N);
        A(&h->tab[i].start, N); A(&h->tab[i].size, N); A(&h->tab[i].vol, N); A(&h->tab[i].vol_start, N);
        A(&h->tab[i].root, N); A(&h->tab[i].best, N); A(&h->tab[i].skip, N); A(&h->tab[i].hist, N);
    }
    A(&h->sflag, N); A(&h->nflag, N); A(&h->rootc, N); A(&h->mlp, (size_t)kMlpImage);
    A(&h->smax, N); A(&h->smin, N);
    if (h->sched.trace) { A(&h->records, N); }
    A(&h->cut_off, N); A(&h->split, N); A(&h->allcuts, N); A(&h->rep[0], N); A(&h->rep[1], N);
    A(&h->walk_stats, 3 * kStatSlots);
    for (int i = 0; i <= kSiteRoots; ++i) {
        A(&h->lb[i].flags, scan_tiles); A(&h->lb[i].agg, scan_tiles); A(&h->lb[i].inc, scan_tiles);
    }
    A(&h->rootmap, N / 32 + 1);
    A(&h->lb_epoch, kSites); A(&h->ctr, 1);
    A(&h->sort.hist, kMaxPasses * kRadix); A(&h->sort.bases, kMaxPasses * kRadix);
    A(&h->sort.pass_info, kMaxPasses + 1); A(&h->sort.tile_ctr, kMaxPasses); A(&h->sort.epoch, 1);
    A(&h->sort.status, (size_t)sort_tiles * kRadix);
    A(&h->sort_end_bit, 1); A(&h->fp_end_bit, 1); A(&h->d_n, 1);
    A(&h->d_num, 1); A(&h->d_valid, 1); A(&h->d_check, 4); A(&h->heavy, N); A(&h->wide, N);
    A(&h->probe_ctr, 1); A(&h->hist, 33);
#undef A
    if (e != cudaSuccess) {
        const size_t held = h->bytes;
        release(h);
        if (e == cudaErrorMemoryAllocation)
            return fail(h, PXR_OUT_OF_MEMORY, "device memory exhausted after " + std::to_string(held >> 20) +
                                                  " MiB" + (h->cfg.memory_cap_mib ? " (the handle's memory cap is " +
                                                  std::to_string(h->cfg.memory_cap_mib) + " MiB)" : std::string()));
        return cuda_fail(h, e, "cudaMalloc");
    }
    h->sort.max_tiles = sort_tiles;
    h->sort.items_moved = &h->ctr->stat_sort_items;
    // look-back flags and sort status words carry epochs that only grow, so
    // they are cleared once here and never again
    cudaStream_t s = h->stream;
    for (int i = 0; i <= kSiteRoots; ++i) PXR_CUDA(h, cudaMemsetAsync(h->lb[i].flags, 0, scan_tiles * 4, s));
    PXR_CUDA(h, cudaMemsetAsync(h->rootmap, 0, (N / 32 + 1) * 4, s));
    PXR_CUDA(h, cudaMemsetAsync(h->smax, 0, N * 4, s));      // per-label spread: identity
    PXR_CUDA(h, cudaMemsetAsync(h->smin, 0xFF, N * 4, s));
    PXR_CUDA(h, cudaMemsetAsync(h->walk_stats, 0, 3 * kStatSlots * sizeof(unsigned long long), s));
    PXR_CUDA(h, cudaMemsetAsync(h->lb_epoch, 0, kSites * 4, s));
    h->records_n = h->records ? (uint32_t)N : 0u;
    if (!h->mlp_img.empty())
        PXR_CUDA(h, cudaMemcpyAsync(h->mlp, h->mlp_img.data(), kMlpImage * 4, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemsetAsync(h->ctr, 0, sizeof(RoundCtr), s));
    PXR_CUDA(h, cudaMemsetAsync(h->sort.hist, 0, kMaxPasses * kRadix * 4, s));
    PXR_CUDA(h, cudaMemsetAsync(h->sort.epoch, 0, 4, s));
    PXR_CUDA(h, cudaMemsetAsync(h->sort.status, 0, (size_t)sort_tiles * kRadix * 8, s));
    PXR_CUDA(h, cudaMemsetAsync(h->sort.pass_info, 0, (kMaxPasses + 1) * 4, s));
    const uint32_t consts[2] = {32u, n};
    PXR_CUDA(h, cudaMemcpyAsync(h->fp_end_bit, &consts[0], 4, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(h->d_n, &consts[1], 4, cudaMemcpyHostToDevice, s));
    return PXR_OK;
}

// Lanes per light row and the row-bin bounds.
struct RowPlan {
    uint32_t W, light_max, wide_max;
};

// Without tuning: one thread per row for sparse graphs (4 independent slots
// per step), more lanes as the mean degree grows.
RowPlan default_row_plan(const pxr_handle* h, uint32_t n, uint64_t m) {
    (void)h;
    const double mean = n ? (double)(2 * m) / n : 0.0;
    const uint32_t W = mean <= 16.0 ? 1u : mean <= 32.0 ? 4u : mean <= 64.0 ? 8u : 32u;
    return RowPlan{W, kLightRow, kWideRow};
}

template <typename OffT>
pxr_status bin_rows(pxr_handle* h, const RowPlan& p, uint32_t* counts) {
    cudaStream_t s = h->stream;
    PXR_CUDA(h, cudaMemsetAsync(&h->d_check[2], 0, 8, s));
    if (h->n) {
        k_bin_rows<OffT><<<grid_for(h->n), kBlock, 0, s>>>(static_cast<const OffT*>(h->off), h->n, p.light_max,
                                                           p.wide_max, h->wide, h->heavy, &h->d_check[2]);
        ++h->launches;
    }
    PXR_CUDA(h, cudaMemcpyAsync(counts, &h->d_check[2], 8, cudaMemcpyDeviceToHost, s));
    PXR_CUDA(h, cudaStreamSynchronize(s));
    return PXR_OK;
}

// ---------------------------------------------------------------------------
// Row-plan autotuner: time one walk step (the light-row kernel plus the
// warp- and CTA-per-row kernels) of the whole graph under each candidate
// plan, on the graph's own rows and potentials, and keep the fastest.  The
// walk writes only scratch (a copy of x, a scratch x / degree and scratch
// counters), so the state is untouched.  Plans are cached per (n, m, offset
// width, row-size histogram) for the life of the process.

std::mutex g_plan_mu;
std::map<std::vector<uint64_t>, RowPlan> g_plan_cache;

template <typename OffT, int W>
cudaError_t probe_walk(pxr_handle* h, Dev<OffT> d, float* xt_out) {
    launch_walk<OffT, W>(h, d, h->stream, h->xt[h->xcur], xt_out);
    return cudaGetLastError();
}

template <typename OffT>
cudaError_t probe_walk_w(pxr_handle* h, const Dev<OffT>& d, float* xt_out) {
    switch (h->W) {
        case 1: return probe_walk<OffT, 1>(h, d, xt_out);
        case 4: return probe_walk<OffT, 4>(h, d, xt_out);
        case 16: return probe_walk<OffT, 16>(h, d, xt_out);
        case 32: return probe_walk<OffT, 32>(h, d, xt_out);
        default: return probe_walk<OffT, 8>(h, d, xt_out);
    }
}

template <typename OffT>
pxr_status tune_row_plan(pxr_handle* h, const std::array<uint32_t, 33>& hist, RowPlan* best, uint32_t* tried,
                         float* best_us) {
    cudaStream_t s = h->stream;
    const uint32_t n = h->n;
    // rows of the largest size class decide which bin bounds can differ
    int top = 0;
    for (int b = 0; b < 33; ++b)
        if (hist[b]) top = b;
    const uint64_t maxlen = top == 0 ? 0 : (1ull << top) - 1;   // upper bound of the largest class
    std::vector<RowPlan> cands;
    const uint32_t lanes[] = {1, 4, 8, 16, 32};
    const uint32_t lights[] = {16, 32, 64, 128};
    const uint32_t wides[] = {1024, 4096, 16384};
    // a bound above the previous one that already holds every row gives the same bins: skip it
    for (uint32_t W : lanes)
        for (int i = 0; i < 4; ++i) {
            if (i > 0 && (uint64_t)lights[i - 1] >= maxlen) continue;
            for (int j = 0; j < 3; ++j) {
                if (j > 0 && (uint64_t)wides[j - 1] >= maxlen) continue;
                cands.push_back(RowPlan{W, lights[i], wides[j]});
            }
        }
    // scratch: x copy in keys[0], x / degree in keys[1], counters in probe_ctr
    float* xs = reinterpret_cast<float*>(h->keys[0]);
    float* xo = reinterpret_cast<float*>(h->keys[1]);
    PXR_CUDA(h, cudaMemcpyAsync(xs, h->x, (size_t)n * 4, cudaMemcpyDeviceToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(h->probe_ctr, h->ctr, sizeof(RoundCtr), cudaMemcpyDeviceToDevice, s));
    cudaEvent_t e0 = take_event(h), e1 = take_event(h);
    float best_ms = 0.0f;
    bool have = false;
    for (const RowPlan& p : cands) {
        uint32_t bins[2];
        pxr_status st = bin_rows<OffT>(h, p, bins);
        if (st != PXR_OK) return st;
        h->W = p.W;
        h->light_max = p.light_max;
        h->wide_max = p.wide_max;
        h->n_wide = bins[0];
        h->n_heavy = bins[1];
        Dev<OffT> d = make_dev<OffT>(h);
        d.x = xs;
        d.ctr = h->probe_ctr;
        PXR_CUDA(h, probe_walk_w<OffT>(h, d, xo));     // warm-up
        cudaEventRecord(e0, s);
        for (int r = 0; r < 3; ++r) PXR_CUDA(h, probe_walk_w<OffT>(h, d, xo));
        cudaEventRecord(e1, s);
        PXR_CUDA(h, cudaEventSynchronize(e1));
        float ms = 0.0f;
        PXR_CUDA(h, cudaEventElapsedTime(&ms, e0, e1));
        h->launches += 4ull * (1 + long_launches(h));
        if (!have || ms < best_ms) { best_ms = ms; *best = p; have = true; }
    }
    h->event_pool.push_back(e0);
    h->event_pool.push_back(e1);
    *tried = (uint32_t)cands.size();
    *best_us = best_ms * 1000.0f / 3.0f;
    return PXR_OK;
}

// The plan for the graph just uploaded: forced, cached, tuned or heuristic.
// Rebins the rows and drops captured graphs when the plan changed.
template <typename OffT>
pxr_status choose_row_plan(pxr_handle* h, bool reuse, uint32_t nb_bits) {
    const RowPlan old{h->W, h->light_max, h->wide_max};
    const uint32_t old_wide = h->n_wide, old_heavy = h->n_heavy, old_bits = h->nb_bits;
    RowPlan plan = default_row_plan(h, h->n, h->m);
    uint32_t source = 0, tried = 0;
    float us = 0.0f;
    if (h->plan_forced) {
        plan = RowPlan{h->plan_info.lanes_per_row, h->plan_info.light_max, h->plan_info.wide_max};
        source = 3;
    } else if (h->cfg.tune == PXR_TUNE_AUTO && h->n > 0) {
        cudaStream_t s = h->stream;
        std::array<uint32_t, 33> hist{};
        PXR_CUDA(h, cudaMemsetAsync(h->hist, 0, 33 * 4, s));
        k_degree_hist<OffT><<<std::min(grid_for(h->n), 148u * 4u), kBlock, 0, s>>>(static_cast<const OffT*>(h->off),
                                                                                   h->n, h->hist);
        ++h->launches;
        PXR_CUDA(h, cudaMemcpyAsync(hist.data(), h->hist, 33 * 4, cudaMemcpyDeviceToHost, s));
        PXR_CUDA(h, cudaStreamSynchronize(s));
        std::vector<uint64_t> key{h->n, h->m, sizeof(OffT)};
        key.insert(key.end(), hist.begin(), hist.end());
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_plan_mu);
            auto it = g_plan_cache.find(key);
            if (it != g_plan_cache.end()) { plan = it->second; hit = true; }
        }
        if (hit) {
            source = 2;
        } else {
            pxr_status st = tune_row_plan<OffT>(h, hist, &plan, &tried, &us);
            if (st != PXR_OK) return st;
            source = 1;
            std::lock_guard<std::mutex> lk(g_plan_mu);
            g_plan_cache[key] = plan;
        }
    }
    uint32_t bins[2] = {0, 0};
    pxr_status bst = bin_rows<OffT>(h, plan, bins);
    if (bst != PXR_OK) return bst;
    // captured round graphs bake in buffers, nb_bits and the row plan: keep them only if all are unchanged
    if (!reuse || nb_bits != old_bits || plan.W != old.W || plan.light_max != old.light_max ||
        plan.wide_max != old.wide_max || bins[0] != old_wide || bins[1] != old_heavy)
        drop_graphs(h);
    h->nb_bits = nb_bits;
    h->W = plan.W;
    h->light_max = plan.light_max;
    h->wide_max = plan.wide_max;
    h->n_wide = bins[0];
    h->n_heavy = bins[1];
    h->plan_info.lanes_per_row = plan.W;
    h->plan_info.light_max = plan.light_max;
    h->plan_info.wide_max = plan.wide_max;
    h->plan_info.wide_rows = bins[0];
    h->plan_info.heavy_rows = bins[1];
    h->plan_info.source = source;
    if (source == 1) {
        h->plan_info.candidates = tried;
        h->plan_info.walk_us = us;
    }
    return PXR_OK;
}

// ---------------------------------------------------------------------------
// Sort-plan autotuner: time the global sort of the first round's keys (label
// 0, the ordered bits of every vertex's potential, values the vertex ids) under
// each plan of kSortPlans and keep the fastest.  The keys live in the sort
// buffers, which hold nothing before the first round.  Cached per vertex
// count for the life of the process.

std::map<uint64_t, std::pair<uint32_t, std::array<float, 3>>> g_sort_cache;
constexpr uint32_t kSortTuneMinVertices = 1u << 16;

__global__ void k_tune_sort_keys(const float* x, uint32_t n, uint64_t* keys, uint32_t* vals) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        keys[v] = ordered_bits(x[v]);
        vals[v] = v;
    }
}

pxr_status tune_sort_plan(pxr_handle* h, uint32_t* best, std::array<float, 3>* us) {
    cudaStream_t s = h->stream;
    const uint32_t n = h->n;
    SortBuffers<uint64_t> b{};
    b.keys[0] = h->keys[0]; b.keys[1] = h->keys[1];
    b.vals[0] = h->vals[0]; b.vals[1] = h->vals[1];
    b.count = h->d_n;
    b.end_bit = h->fp_end_bit;   // 32 bits: the potential part of a cluster-0 key
    b.capacity = n;
    SortState st = h->sort;
    st.items_moved = nullptr;    // the probe sorts stay out of the traffic counters
    cudaEvent_t e0 = take_event(h), e1 = take_event(h);
    constexpr int kReps = 3;
    float best_ms = 0.0f;
    for (int p = 0; p < kSortPlanCount; ++p) {
        float total = 0.0f;
        for (int r = 0; r <= kReps; ++r) {   // the first run warms up
            k_tune_sort_keys<<<grid_for(n), kBlock, 0, s>>>(h->x, n, h->keys[0], h->vals[0]);
            cudaEventRecord(e0, s);
            PXR_CUDA(h, radix_sort<uint64_t>(b, st, &h->ctr->err, s, 32, p));
            cudaEventRecord(e1, s);
            PXR_CUDA(h, cudaEventSynchronize(e1));
            float ms = 0.0f;
            PXR_CUDA(h, cudaEventElapsedTime(&ms, e0, e1));
            if (r > 0) total += ms;
            h->launches += 1 + 2 + 4;
        }
        (*us)[p] = total * 1000.0f / kReps;
        if (p == 0 || total < best_ms) { best_ms = total; *best = (uint32_t)p; }
    }
    h->event_pool.push_back(e0);
    h->event_pool.push_back(e1);
    return PXR_OK;
}

// The sweep sort's plan for the graph just uploaded: forced, cached, tuned or
// the default.  Drops captured graphs when the plan changed.
pxr_status choose_sort_plan(pxr_handle* h) {
    const uint32_t old = h->sort_info.plan;
    uint32_t plan = 0, source = 0, tried = 0;
    std::array<float, 3> us{0.0f, 0.0f, 0.0f};
    if (h->sort_forced) {
        plan = h->sort_info.plan;
        source = 3;
    } else if (h->cfg.tune == PXR_TUNE_AUTO && h->n >= kSortTuneMinVertices) {
        bool hit = false;
        {
            std::lock_guard<std::mutex> lk(g_plan_mu);
            auto it = g_sort_cache.find(h->n);
            if (it != g_sort_cache.end()) { plan = it->second.first; us = it->second.second; hit = true; }
        }
        if (hit) {
            source = 2;
        } else {
            pxr_status st = tune_sort_plan(h, &plan, &us);
            if (st != PXR_OK) return st;
            source = 1;
            tried = kSortPlanCount;
            std::lock_guard<std::mutex> lk(g_plan_mu);
            g_sort_cache[h->n] = {plan, us};
        }
    }
    if (plan != old) drop_graphs(h);
    h->sort_info.plan = plan;
    h->sort_info.items_per_thread = (uint32_t)kSortPlans[plan].items;
    h->sort_info.ctas_per_sm = (uint32_t)kSortPlans[plan].ctas;
    h->sort_info.source = source;
    if (source != 3) h->sort_info.candidates = tried;
    for (int p = 0; p < 3; ++p) h->sort_info.sort_us[p] = us[p];
    return PXR_OK;
}

// offsets/cols: host pointers (kind = cudaMemcpyHostToDevice) or device pointers
template <typename OffT>
pxr_status initialize_impl(pxr_handle* h, uint32_t n, uint64_t m, const OffT* offsets, const uint32_t* cols,
                           cudaMemcpyKind kind, bool batched = false) {
    if (!h) return PXR_INVALID_ARG;
    if (!offsets || (m > 0 && !cols)) return fail(h, PXR_INVALID_ARG, "null graph pointer");
    if (n >= 0x7FFFFFFFu) return fail(h, PXR_INVALID_ARG, "n must be below 2^31 - 1");
    // cluster volumes are 32-bit (NodeData::prefix_volume, lib/core/definitions.h)
    if (!batched && 2 * m >= (1ull << 32))
        return fail(h, PXR_INVALID_ARG, "the volume 2m of the starting cluster must be below 2^32");
    PXR_CUDA(h, cudaSetDevice(h->device));
    h->initialized = false;
    const bool reuse = !h->allocs.empty() && h->n == n && h->m == m && h->off64 == (sizeof(OffT) == 8);
    if (!reuse) {
        pxr_status st = allocate<OffT>(h, n, m);
        if (st != PXR_OK) return st;
    }
    cudaStream_t s = h->stream;
    h->xcur = h->tcur = h->acur = 0;
    PXR_CUDA(h, cudaMemcpyAsync(h->off, offsets, ((size_t)n + 1) * sizeof(OffT), kind, s));
    if (m) PXR_CUDA(h, cudaMemcpyAsync(h->cols, cols, h->slots * 4, kind, s));
    PXR_CUDA(h, cudaMemsetAsync(h->d_check, 0, 16, s));
    k_validate<OffT><<<grid_for(std::max<uint64_t>(h->slots, n)), kBlock, 0, s>>>(
        static_cast<const OffT*>(h->off), h->cols, n, h->slots, &h->d_check[0], &h->d_check[1]);
    ++h->launches;
    uint32_t check[4] = {0, 0, 0, 0};
    PXR_CUDA(h, cudaMemcpyAsync(check, h->d_check, 16, cudaMemcpyDeviceToHost, s));
    PXR_CUDA(h, cudaStreamSynchronize(s));
    if (check[0] & 2u) return fail(h, PXR_INVALID_ARG, "offsets must start at 0 and end at 2m");
    if (check[0] & 1u) return fail(h, PXR_INVALID_ARG, "offsets must be non-decreasing");
    if (check[0] & 4u) return fail(h, PXR_INVALID_ARG, "column index out of range");
    h->maxdeg = check[1];
    const uint32_t nb_bits = host_bitlen(std::max<uint64_t>(n, h->maxdeg));
    // round state: one cluster, every vertex active; keep the growing epochs
    RoundCtr c;
    PXR_CUDA(h, cudaMemcpyAsync(&c, h->ctr, sizeof(RoundCtr), cudaMemcpyDeviceToHost, s));
    PXR_CUDA(h, cudaStreamSynchronize(s));
    const RoundCtr old = c;
    std::memset(&c, 0, sizeof(c));
    c.n_active = n;
    c.n_clusters = n ? 1u : 0u;
    c.full_components = 1;
    c.done = n ? 0u : 1u;
    c.main_sel = old.main_sel;
    c.max_parent = 0xFFFFFFFFu;   // the first round sorts globally (the list is in vertex order)
    c.max_csize = n;
    PXR_CUDA(h, cudaMemcpyAsync(h->ctr, &c, sizeof(RoundCtr), cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemsetAsync(h->cert, 0, (size_t)std::max<uint32_t>(n, 1) * 4, s));
    if (n) {
        k_degrees<OffT><<<grid_for(n), kBlock, 0, s>>>(static_cast<const OffT*>(h->off), n, h->ideg, h->lab,
                                                      h->act[0], h->ids[0]);
        launch_initial_potentials(h->off, h->off64, n, h->cfg.seed, h->x, &h->ctr->xmax_bits, s);
        k_refresh_scaled<<<grid_for(n), kBlock, 0, s>>>(h->x, h->ideg, n, h->xt[0], &h->ctr->xmax_bits);
        PXR_CUDA(h, cudaMemcpyAsync(&h->ctr->xmax_walk_bits, &h->ctr->xmax_bits, 4, cudaMemcpyDeviceToDevice, s));
        h->launches += 3;
    }
    pxr_status st = setup_tables_initial(h);
    if (st == PXR_OK) st = reset_schedule_state(h);
    if (st == PXR_OK) st = choose_row_plan<OffT>(h, reuse, nb_bits);
    if (st == PXR_OK) st = choose_sort_plan(h);
    if (st != PXR_OK) return st;
    PXR_CUDA(h, cudaGetLastError());
    if (batched) return PXR_OK;   // batch_setup completes the state
    h->initialized = true;
    return sync_ctr(h);
}

// Every instance becomes its own cluster: labels, cluster tables and the
// round counters replace the one-cluster state that initialize_impl left.
template <typename OffT>
pxr_status batch_setup(pxr_handle* h, uint32_t n_inst, const uint32_t* starts) {
    const uint32_t n = h->n;
    cudaStream_t s = h->stream;
    // scratch in the sort key buffers, free until the first round (every
    // instance holds a vertex, so n_inst + 1 <= 2n words and n_inst <= n)
    uint32_t* d_starts = reinterpret_cast<uint32_t*>(h->keys[0]);
    unsigned long long* d_vol = reinterpret_cast<unsigned long long*>(h->keys[1]);
    cudaError_t e = cudaMemcpyAsync(d_starts, starts, ((size_t)n_inst + 1) * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_vol, 0, (size_t)n_inst * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&h->d_check[3], 0, 4, s);
    if (e == cudaSuccess) {
        k_batch_setup<OffT><<<grid_for(n), kBlock, 0, s>>>(static_cast<const OffT*>(h->off), h->cols, h->ideg, d_starts,
                                                           n, n_inst, h->lab, d_vol, &h->d_check[3]);
        ++h->launches;
        e = cudaGetLastError();
    }
    std::vector<unsigned long long> vol(n_inst);
    uint32_t bad = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(vol.data(), d_vol, (size_t)n_inst * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, &h->d_check[3], 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(h, e, "batched set-up");
    if (bad) return fail(h, PXR_INVALID_ARG, "an edge joins two instances");
    std::vector<uint32_t> start(n_inst), size(n_inst), vol32(n_inst), vol_start(n_inst), root(n_inst);
    uint64_t acc = 0;
    for (uint32_t i = 0; i < n_inst; ++i) {
        if (vol[i] >= (1ull << 32)) return fail(h, PXR_INVALID_ARG, "instance volume must be below 2^32");
        start[i] = starts[i];
        size[i] = starts[i + 1] - starts[i];
        root[i] = starts[i];
        vol32[i] = (uint32_t)vol[i];
        vol_start[i] = (uint32_t)acc;   // prefixes are used modulo 2^32, per cluster
        acc += vol[i];
    }
    const ClusterTables& t = h->tab[h->tcur];
    PXR_CUDA(h, cudaMemcpyAsync(t.start, start.data(), n_inst * 4ull, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(t.size, size.data(), n_inst * 4ull, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(t.vol, vol32.data(), n_inst * 4ull, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(t.vol_start, vol_start.data(), n_inst * 4ull, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemcpyAsync(t.root, root.data(), n_inst * 4ull, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemsetAsync(t.best, 0xFF, n_inst * 8ull, s));
    PXR_CUDA(h, cudaMemcpyAsync(&h->ctr->n_clusters, &n_inst, 4, cudaMemcpyHostToDevice, s));
    h->initialized = true;
    return sync_ctr(h);
}

}  // namespace

// ===========================================================================
// C ABI

extern "C" {

void pxr_config_default(pxr_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->seed = 6582u;
    cfg->sc_threshold = 0.3f;
    cfg->rw_threshold = 1e-4f;
    cfg->max_rounds = 200000u;
    cfg->device = 0;
    cfg->division = PXR_DIV_IEEE;
    cfg->driver = PXR_DRIVER_GRAPH;
}

const char* pxr_status_string(pxr_status s) {
    switch (s) {
        case PXR_OK: return "ok";
        case PXR_INVALID_ARG: return "invalid argument";
        case PXR_OUT_OF_MEMORY: return "out of device memory";
        case PXR_ITER_CAP: return "round cap reached";
        case PXR_CUDA_ERROR: return "CUDA error";
        case PXR_DEVICE_FAULT: return "device-side check failed";
        case PXR_NOT_INITIALIZED: return "not initialized";
    }
    return "unknown status";
}

const char* pxr_last_error(const void* handle) {
    return handle ? static_cast<const pxr_handle*>(handle)->err.c_str() : "null handle";
}

pxr_status pxr_create(const pxr_config* cfg, pxr_handle** out) {
    if (!out) return PXR_INVALID_ARG;
    *out = nullptr;
    pxr_handle* h = new (std::nothrow) pxr_handle();
    if (!h) return PXR_OUT_OF_MEMORY;
    if (cfg) h->cfg = *cfg; else pxr_config_default(&h->cfg);
    if (h->cfg.division > PXR_DIV_REFERENCE || h->cfg.driver > PXR_DRIVER_STREAM ||
        h->cfg.components > PXR_COMPONENTS_SAMPLED) {
        delete h;
        return PXR_INVALID_ARG;
    }
    h->device = h->cfg.device;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) { delete h; return PXR_CUDA_ERROR; }
    if (h->device < 0 || h->device >= count) { delete h; return PXR_INVALID_ARG; }
    if (cudaSetDevice(h->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->walk_side[0], cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&h->walk_side[1], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->walk_ev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->walk_ev[1], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&h->walk_ev[2], cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&h->h_ctr, sizeof(RoundCtr)) != cudaSuccess) {
        delete h;
        return PXR_CUDA_ERROR;
    }
    std::memset(h->h_ctr, 0, sizeof(RoundCtr));
    h->stream = h->own_stream;
    static bool attrs_set[64] = {};   // function attributes are per device
    if (h->device < 64 && !attrs_set[h->device]) {
        radix_sort_prepare<uint64_t>();
        radix_sort_prepare<uint32_t>();
        cudaFuncSetAttribute(k_chunk_sort<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chunk_sort_smem());
        cudaFuncSetAttribute(k_chunk_sort<uint64_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chunk_sort_smem());
        attrs_set[h->device] = true;
    }
    *out = h;
    return PXR_OK;
}

void pxr_destroy(pxr_handle* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->stream);
    release(h);
    collect_phases(h);
    for (cudaEvent_t e : h->event_pool) cudaEventDestroy(e);
    if (h->h_ctr) cudaFreeHost(h->h_ctr);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    if (h->side_stream) cudaStreamDestroy(h->side_stream);
    for (cudaStream_t st : h->walk_side)
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : h->walk_ev)
        if (ev) cudaEventDestroy(ev);
    delete h;
}

pxr_status pxr_set_stream(pxr_handle* h, void* stream) {
    if (!h) return PXR_INVALID_ARG;
    h->stream = stream ? static_cast<cudaStream_t>(stream) : h->own_stream;
    return PXR_OK;
}

pxr_status pxr_initialize(pxr_handle* h, uint32_t n, uint64_t m, const uint32_t* offsets, const uint32_t* cols) {
    if (2 * m >= (1ull << 32)) return fail(h, PXR_INVALID_ARG, "32-bit offsets need 2m < 2^32");
    return initialize_impl<uint32_t>(h, n, m, offsets, cols, cudaMemcpyHostToDevice);
}

pxr_status pxr_initialize64(pxr_handle* h, uint32_t n, uint64_t m, const uint64_t* offsets, const uint32_t* cols) {
    if (offsets && 2 * m < (1ull << 32)) {
        // keep 32-bit offsets on the device when they fit: half the offset traffic
        std::vector<uint32_t> o32((size_t)n + 1);
        for (size_t i = 0; i <= n; ++i) o32[i] = (uint32_t)offsets[i];
        return initialize_impl<uint32_t>(h, n, m, o32.data(), cols, cudaMemcpyHostToDevice);
    }
    return initialize_impl<uint64_t>(h, n, m, offsets, cols, cudaMemcpyHostToDevice);
}

pxr_status pxr_initialize_device(pxr_handle* h, uint32_t n, uint64_t m, const void* offsets, int offsets_are_64bit,
                                 const uint32_t* cols) {
    if (offsets_are_64bit)
        return initialize_impl<uint64_t>(h, n, m, static_cast<const uint64_t*>(offsets), cols, cudaMemcpyDeviceToDevice);
    if (2 * m >= (1ull << 32)) return fail(h, PXR_INVALID_ARG, "32-bit offsets need 2m < 2^32");
    return initialize_impl<uint32_t>(h, n, m, static_cast<const uint32_t*>(offsets), cols, cudaMemcpyDeviceToDevice);
}

pxr_status pxr_initialize_batched(pxr_handle* h, uint32_t n, uint64_t m, const uint64_t* offsets, const uint32_t* cols,
                                  uint32_t n_instances, const uint32_t* instance_start) {
    if (!h) return PXR_INVALID_ARG;
    if (!instance_start || n_instances == 0) return fail(h, PXR_INVALID_ARG, "no instances");
    if (instance_start[0] != 0 || instance_start[n_instances] != n)
        return fail(h, PXR_INVALID_ARG, "instance starts must run from 0 to n");
    for (uint32_t i = 0; i < n_instances; ++i)
        if (instance_start[i + 1] <= instance_start[i])
            return fail(h, PXR_INVALID_ARG, "every instance needs at least one vertex");
    pxr_status st;
    if (offsets && 2 * m < (1ull << 32)) {
        std::vector<uint32_t> o32((size_t)n + 1);
        for (size_t i = 0; i <= n; ++i) o32[i] = (uint32_t)offsets[i];
        st = initialize_impl<uint32_t>(h, n, m, o32.data(), cols, cudaMemcpyHostToDevice, true);
        if (st != PXR_OK) return st;
        return batch_setup<uint32_t>(h, n_instances, instance_start);
    }
    st = initialize_impl<uint64_t>(h, n, m, offsets, cols, cudaMemcpyHostToDevice, true);
    if (st != PXR_OK) return st;
    return batch_setup<uint64_t>(h, n_instances, instance_start);
}

pxr_status pxr_initialize_batched_device(pxr_handle* h, uint32_t n, uint64_t m, const void* offsets,
                                         int offsets_are_64bit, const uint32_t* cols, uint32_t n_instances,
                                         const uint32_t* instance_start) {
    if (!h) return PXR_INVALID_ARG;
    if (!instance_start || n_instances == 0) return fail(h, PXR_INVALID_ARG, "no instances");
    if (instance_start[0] != 0 || instance_start[n_instances] != n)
        return fail(h, PXR_INVALID_ARG, "instance starts must run from 0 to n");
    for (uint32_t i = 0; i < n_instances; ++i)
        if (instance_start[i + 1] <= instance_start[i])
            return fail(h, PXR_INVALID_ARG, "every instance needs at least one vertex");
    pxr_status st;
    if (offsets_are_64bit) {
        st = initialize_impl<uint64_t>(h, n, m, static_cast<const uint64_t*>(offsets), cols, cudaMemcpyDeviceToDevice,
                                       true);
        if (st != PXR_OK) return st;
        return batch_setup<uint64_t>(h, n_instances, instance_start);
    }
    if (2 * m >= (1ull << 32)) return fail(h, PXR_INVALID_ARG, "32-bit offsets need 2m < 2^32");
    st = initialize_impl<uint32_t>(h, n, m, static_cast<const uint32_t*>(offsets), cols, cudaMemcpyDeviceToDevice, true);
    if (st != PXR_OK) return st;
    return batch_setup<uint32_t>(h, n_instances, instance_start);
}

pxr_status pxr_walk_step(pxr_handle* h) { return run_op(h, kOpWalk); }
pxr_status pxr_sweep(pxr_handle* h) { return run_op(h, kOpSweep); }
pxr_status pxr_cut_clusters(pxr_handle* h) { return run_op(h, kOpCut); }

pxr_status pxr_decompose(pxr_handle* h, uint32_t* rounds_out) {
    if (!h) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    cudaEvent_t e0, e1;
    PXR_CUDA(h, cudaEventCreate(&e0));
    PXR_CUDA(h, cudaEventCreate(&e1));
    pxr_status st = sync_ctr(h);
    const uint32_t start_rounds = h->h_ctr->rounds;
    PXR_CUDA(h, cudaEventRecord(e0, h->stream));
    if (st == PXR_OK) st = h->cfg.driver == PXR_DRIVER_GRAPH ? decompose_graph(h) : decompose_stream(h);
    PXR_CUDA(h, cudaEventRecord(e1, h->stream));
    PXR_CUDA(h, cudaEventSynchronize(e1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->last_ms = ms;
    h->last_rounds = h->h_ctr->rounds - start_rounds;
    if (rounds_out) *rounds_out = h->last_rounds;
    if (st != PXR_OK) return st;
    if (!h->h_ctr->done) return fail(h, PXR_ITER_CAP, "round cap reached before every cluster was certified");
    return PXR_OK;
}

pxr_status pxr_read_potentials(pxr_handle* h, float* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    PXR_CUDA(h, cudaMemcpyAsync(out, h->x, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return PXR_OK;
}

pxr_status pxr_read_sweep_cuts(pxr_handle* h, int32_t* labels, pxr_sweep_cut* cuts, uint32_t cap, uint32_t* count) {
    if (!h || !count) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    pxr_status st = sync_ctr(h);
    if (st != PXR_OK) return st;
    const uint32_t k = h->h_ctr->sweep_k;
    *count = k;
    const uint32_t c = std::min(cap, k);
    if (c && cuts) {
        PXR_CUDA(h, cudaMemcpyAsync(cuts, h->allcuts, (size_t)c * sizeof(pxr_sweep_cut), cudaMemcpyDeviceToHost, h->stream));
        PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    if (labels)
        for (uint32_t i = 0; i < c; ++i) labels[i] = (int32_t)i;
    return PXR_OK;
}

pxr_status pxr_download_partition(pxr_handle* h, pxr_node_data* out, uint32_t cap, uint32_t* count) {
    if (!h || !count) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    pxr_status st = sync_ctr(h);
    if (st != PXR_OK) return st;
    const uint32_t na = h->h_ctr->sweep_n;
    *count = na;
    const uint32_t c = std::min(cap, na);
    if (!c || !out) return PXR_OK;
    const uint32_t sel = h->h_ctr->main_sel;
    std::vector<uint64_t> keys(c);
    std::vector<uint32_t> vals(c), pvol(c), starts(h->n ? h->n : 1);
    std::vector<int32_t> pdif(c);
    PXR_CUDA(h, cudaMemcpyAsync(keys.data(), h->keys[sel], c * 8ull, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(vals.data(), h->vals[sel], c * 4ull, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(pdif.data(), h->pdif, c * 4ull, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(pvol.data(), h->pvol, c * 4ull, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(starts.data(), h->tab[h->sweep_tab].start, (size_t)h->n * 4, cudaMemcpyDeviceToHost,
                                h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    for (uint32_t i = 0; i < c; ++i) {
        const uint32_t lab = (uint32_t)(keys[i] >> 32);
        out[i].nix = vals[i];
        out[i].prefix_volume = pvol[i];
        out[i].prefix_edge_diff = pdif[i];
        out[i].offset_in_cluster = i - starts[lab] + 1;
    }
    return PXR_OK;
}

pxr_status pxr_final_partition(pxr_handle* h, int32_t* ids, int32_t* num_clusters) {
    if (!h || !ids || !num_clusters) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    const uint32_t n = h->n;
    if (n == 0) { *num_clusters = 0; return PXR_OK; }
    cudaStream_t s = h->stream;
    // reuse idle buffers: roots[] as keys, the idle parity of act[] / ids[] as values
    uint32_t* k0 = h->roots[0];
    uint32_t* k1 = h->roots[1];
    uint32_t* v0 = h->act[h->acur ^ 1];
    uint32_t* v1 = h->ids[h->acur ^ 1];
    int32_t* out = reinterpret_cast<int32_t*>(h->dv);
    k_fp_keys<<<grid_for(n), kBlock, 0, s>>>(h->lab, n, k0, v0);
    h->launches += 4 + 2 + 4;
    SortBuffers<uint32_t> b{};
    b.keys[0] = k0; b.keys[1] = k1; b.vals[0] = v0; b.vals[1] = v1;
    b.count = h->d_n;
    b.end_bit = h->fp_end_bit;
    b.capacity = n;
    cudaError_t e = radix_sort<uint32_t>(b, h->sort, &h->ctr->err, s, 32);
    if (e != cudaSuccess) return cuda_fail(h, e, "final partition sort");
    k_bump_site<<<1, 1, 0, s>>>(h->lb_epoch, h->ctr, kSiteFinal);
    const uint32_t tiles = (n + kScanTile - 1) / kScanTile;
    k_fp_rank<<<tiles, kBlock, 0, s>>>(k0, k1, v0, v1, &h->sort.pass_info[kMaxPasses], h->d_n, out, h->lb[kSiteFinal],
                                       &h->lb_epoch[kSiteFinal], h->ctr, h->d_num);
    PXR_CUDA(h, cudaGetLastError());
    PXR_CUDA(h, cudaMemcpyAsync(ids, out, (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    PXR_CUDA(h, cudaMemcpyAsync(num_clusters, h->d_num, 4, cudaMemcpyDeviceToHost, s));
    return sync_ctr(h);
}

pxr_status pxr_num_cut_edges(pxr_handle* h, uint64_t* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    unsigned long long valid = 0;
    PXR_CUDA(h, cudaMemsetAsync(h->d_valid, 0, 8, h->stream));
    if (h->slots) k_count_valid<<<grid_for(h->slots), kBlock, 0, h->stream>>>(h->cols, h->slots, h->d_valid);
    PXR_CUDA(h, cudaGetLastError());
    PXR_CUDA(h, cudaMemcpyAsync(&valid, h->d_valid, 8, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    *out = h->m - valid / 2;
    return PXR_OK;
}

}  // extern "C"

namespace {
// The CSR columns into host memory with disabled slots as INVALID_EDGE (the
// reference's mutated graph).
pxr_status download_cols(pxr_handle* h, uint32_t* cols) {
    if (!h->slots) return PXR_OK;
    PXR_CUDA(h, cudaMemcpyAsync(cols, h->cols, h->slots * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    for (uint64_t j = 0; j < h->slots; ++j)
        if (!slot_valid(cols[j])) cols[j] = PXR_INVALID_EDGE;
    return PXR_OK;
}
}  // namespace

extern "C" {

pxr_status pxr_download_graph64(pxr_handle* h, uint64_t* offsets, uint32_t* cols) {
    if (!h || !offsets || (h->slots && !cols)) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    if (h->off64) {
        PXR_CUDA(h, cudaMemcpyAsync(offsets, h->off, ((size_t)h->n + 1) * 8, cudaMemcpyDeviceToHost, h->stream));
    } else {
        std::vector<uint32_t> o((size_t)h->n + 1);
        PXR_CUDA(h, cudaMemcpyAsync(o.data(), h->off, o.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        PXR_CUDA(h, cudaStreamSynchronize(h->stream));
        for (size_t i = 0; i < o.size(); ++i) offsets[i] = o[i];
    }
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return download_cols(h, cols);
}

pxr_status pxr_download_graph(pxr_handle* h, uint32_t* offsets, uint32_t* cols) {
    if (!h || !offsets) return PXR_INVALID_ARG;
    if (h->off64) return fail(h, PXR_INVALID_ARG, "graph has 64-bit offsets");
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    PXR_CUDA(h, cudaMemcpyAsync(offsets, h->off, ((size_t)h->n + 1) * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return download_cols(h, cols);
}

pxr_status pxr_download_degrees(pxr_handle* h, uint32_t* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    PXR_CUDA(h, cudaMemcpyAsync(out, h->ideg, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return PXR_OK;
}

pxr_status pxr_download_labels(pxr_handle* h, int32_t* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    PXR_CUDA(h, cudaMemcpyAsync(out, h->lab, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return PXR_OK;
}

pxr_status pxr_active_edge_map(pxr_handle* h, int32_t* out) {
    if (!h || (h->slots && !out)) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    std::vector<uint32_t> c(h->slots);
    if (h->slots) PXR_CUDA(h, cudaMemcpyAsync(c.data(), h->cols, h->slots * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    for (uint64_t j = 0; j < h->slots; ++j) out[j] = slot_valid(c[j]) ? 1 : 0;
    return PXR_OK;
}

pxr_status pxr_test_bounded_waits(pxr_handle* h, uint32_t spin_limit, uint32_t* err_bits) {
    if (!h || !err_bits || spin_limit == 0 || spin_limit > kSpinLimit) return PXR_INVALID_ARG;
    PXR_CUDA(h, cudaSetDevice(h->device));
    // flags[2] | pad | agg[2] | inc[2] | status word | error word
    unsigned char* scratch = nullptr;
    constexpr size_t kBytes = 64;
    PXR_CUDA(h, cudaMalloc(&scratch, kBytes));
    uint32_t* flags = reinterpret_cast<uint32_t*>(scratch);
    uint64_t* agg = reinterpret_cast<uint64_t*>(scratch + 8);
    uint64_t* inc = reinterpret_cast<uint64_t*>(scratch + 24);
    uint64_t* word = reinterpret_cast<uint64_t*>(scratch + 40);
    uint32_t* err = reinterpret_cast<uint32_t*>(scratch + 48);
    cudaError_t e = cudaMemsetAsync(scratch, 0, kBytes, h->stream);
    if (e == cudaSuccess) {
        k_test_lookback_wait<<<1, 32, 0, h->stream>>>(flags, agg, inc, spin_limit, err);
        k_test_sort_wait<<<1, 32, 0, h->stream>>>(word, spin_limit, err);
        h->launches += 2;
        e = cudaGetLastError();
    }
    uint32_t bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, err, 4, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    cudaFree(scratch);
    if (e != cudaSuccess) return cuda_fail(h, e, "bounded-wait test");
    *err_bits = bits;
    if (bits) return fail(h, PXR_DEVICE_FAULT, "device-side bounded wait ran out (bits " + std::to_string(bits) + ")");
    return PXR_OK;
}

pxr_status pxr_download_certificates(pxr_handle* h, uint32_t* out) {
    if (!h || (h->n && !out)) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    if (h->n) PXR_CUDA(h, cudaMemcpyAsync(out, h->cert, (size_t)h->n * 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    return PXR_OK;
}

pxr_status pxr_count_cut_edges(pxr_handle* h, uint64_t* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    unsigned long long both = 0;
    uint32_t bad = 0;
    PXR_CUDA(h, cudaMemsetAsync(h->d_valid, 0, 8, h->stream));
    PXR_CUDA(h, cudaMemsetAsync(h->d_check, 0, 4, h->stream));
    if (h->slots) {
        const uint32_t grid = (uint32_t)std::min<uint64_t>((h->slots + kCountTile - 1) / kCountTile, 148u * 16u);
        if (h->off64)
            k_count_cut<uint64_t><<<grid, kBlock, 0, h->stream>>>(static_cast<const uint64_t*>(h->off), h->cols,
                                                                  h->lab, h->n, h->slots, h->d_valid, h->d_check);
        else
            k_count_cut<uint32_t><<<grid, kBlock, 0, h->stream>>>(static_cast<const uint32_t*>(h->off), h->cols,
                                                                  h->lab, h->n, h->slots, h->d_valid, h->d_check);
        ++h->launches;
    }
    PXR_CUDA(h, cudaGetLastError());
    PXR_CUDA(h, cudaMemcpyAsync(&both, h->d_valid, 8, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaMemcpyAsync(&bad, h->d_check, 4, cudaMemcpyDeviceToHost, h->stream));
    PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    if (bad) return fail(h, PXR_INVALID_ARG, "a disabled slot's neighbour is unknown (slots loaded by pxr_set_state)");
    *out = both / 2;
    return PXR_OK;
}

pxr_status pxr_num_active_clusters(pxr_handle* h, uint32_t* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    pxr_status st = sync_ctr(h);
    *out = h->h_ctr->n_clusters;
    return st;
}

pxr_status pxr_get_stats(pxr_handle* h, pxr_stats* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->device_bytes = h->bytes;
    out->rounds = h->last_rounds;
    out->last_decompose_ms = h->last_ms;
    out->kernel_launches = h->launches;
    if (!h->initialized) return PXR_OK;
    pxr_status st = sync_ctr(h);
    out->active_vertices = h->h_ctr->n_active;
    out->active_clusters = h->h_ctr->n_clusters;
    out->clusters_with_cut = h->h_ctr->n_cut;
    unsigned long long ws[3 * kStatSlots] = {};
    if (h->walk_stats) {
        PXR_CUDA(h, cudaMemcpyAsync(ws, h->walk_stats, sizeof(ws), cudaMemcpyDeviceToHost, h->stream));
        PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    out->walk_vertices = out->walk_slots = out->walk_gathers = 0;
    for (uint32_t q = 0; q < kStatSlots; ++q) {
        out->walk_vertices += ws[3 * q];
        out->walk_slots += ws[3 * q + 1];
        out->walk_gathers += ws[3 * q + 2];
    }
    out->sort_items = h->h_ctr->stat_sort_items;
    out->sort_passes = h->h_ctr->stat_sort_passes;
    out->swept_items = h->h_ctr->stat_swept_items;
    out->skipped_sweeps = h->h_ctr->stat_skipped;
    out->false_stops = h->h_ctr->stat_false_stops;
    return st;
}

pxr_status pxr_set_profiling(pxr_handle* h, int enable) {
    if (!h) return PXR_INVALID_ARG;
    h->profiling = enable != 0;
    std::memset(h->phase_ms, 0, sizeof(h->phase_ms));
    std::memset(h->phase_launches, 0, sizeof(h->phase_launches));
    return PXR_OK;
}

pxr_status pxr_phase_stats(pxr_handle* h, pxr_phase_stat* out, uint32_t cap, uint32_t* count) {
    if (!h || !count) return PXR_INVALID_ARG;
    *count = kPhaseCount;
    for (uint32_t i = 0; i < std::min<uint32_t>(cap, kPhaseCount) && out; ++i) {
        std::memset(&out[i], 0, sizeof(out[i]));
        std::strncpy(out[i].name, kPhaseNames[i], sizeof(out[i].name) - 1);
        out[i].ms = h->phase_ms[i];
        out[i].launches = h->phase_launches[i];
    }
    return PXR_OK;
}

pxr_status pxr_set_potentials(pxr_handle* h, const double* x) {
    if (!h || !x) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    std::vector<float> xf(h->n);
    for (uint32_t v = 0; v < h->n; ++v) xf[v] = (float)x[v];
    PXR_CUDA(h, cudaMemcpyAsync(h->x, xf.data(), (size_t)h->n * 4, cudaMemcpyHostToDevice, h->stream));
    // the walk and the per-cluster sums both take their fixed-point scale from
    // the max |x| over every vertex, as after initialisation
    PXR_CUDA(h, cudaMemsetAsync(&h->ctr->xmax_bits, 0, 8, h->stream));
    if (h->n)
        k_refresh_scaled<<<grid_for(h->n), kBlock, 0, h->stream>>>(h->x, h->ideg, h->n, h->xt[h->xcur],
                                                                    &h->ctr->xmax_bits);
    PXR_CUDA(h, cudaGetLastError());
    PXR_CUDA(h, cudaMemcpyAsync(&h->ctr->xmax_walk_bits, &h->ctr->xmax_bits, 4, cudaMemcpyDeviceToDevice, h->stream));
    return sync_ctr(h);
}

pxr_status pxr_set_state(pxr_handle* h, const int32_t* labels, const uint32_t* act, uint32_t n_act, const double* x,
                         const uint32_t* ideg, const uint32_t* cols, uint32_t n_clusters, int32_t smallest,
                         int full_components) {
    if (!h || !labels || (n_act && !act) || !x || !ideg || (h->slots && !cols)) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    const uint32_t n = h->n;
    if (n_act > n) return fail(h, PXR_INVALID_ARG, "n_act exceeds n");
    std::vector<uint32_t> size(std::max<uint32_t>(n_clusters, 1), 0), vol(std::max<uint32_t>(n_clusters, 1), 0),
        root(std::max<uint32_t>(n_clusters, 1), 0xFFFFFFFFu);
    for (uint32_t i = 0; i < n_act; ++i) {
        const uint32_t v = act[i];
        if (v >= n) return fail(h, PXR_INVALID_ARG, "active vertex out of range");
        const int32_t l = labels[v];
        if (l < 0 || (uint32_t)l >= n_clusters) return fail(h, PXR_INVALID_ARG, "active labels must lie in [0, n_clusters)");
        size[l] += 1;
        vol[l] += ideg[v];
        root[l] = std::min(root[l], v);
    }
    std::vector<uint32_t> start(size.size(), 0), vol_start(size.size(), 0);
    for (uint32_t c = 1; c < n_clusters; ++c) {
        start[c] = start[c - 1] + size[c - 1];
        vol_start[c] = vol_start[c - 1] + vol[c - 1];
    }
    std::vector<uint32_t> ids(act, act + n_act);
    std::sort(ids.begin(), ids.end());
    cudaStream_t s = h->stream;
    h->tcur = 0;
    h->acur = 0;
    const ClusterTables& t = h->tab[0];
    PXR_CUDA(h, cudaMemcpyAsync(h->lab, labels, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    if (n_act) {
        PXR_CUDA(h, cudaMemcpyAsync(h->act[0], act, (size_t)n_act * 4, cudaMemcpyHostToDevice, s));
        PXR_CUDA(h, cudaMemcpyAsync(h->ids[0], ids.data(), (size_t)n_act * 4, cudaMemcpyHostToDevice, s));
    }
    PXR_CUDA(h, cudaMemcpyAsync(h->ideg, ideg, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    if (h->slots) PXR_CUDA(h, cudaMemcpyAsync(h->cols, cols, h->slots * 4, cudaMemcpyHostToDevice, s));
    PXR_CUDA(h, cudaMemsetAsync(h->cert, 0, (size_t)std::max<uint32_t>(n, 1) * 4, s));
    if (n_clusters) {
        PXR_CUDA(h, cudaMemcpyAsync(t.start, start.data(), n_clusters * 4ull, cudaMemcpyHostToDevice, s));
        PXR_CUDA(h, cudaMemcpyAsync(t.size, size.data(), n_clusters * 4ull, cudaMemcpyHostToDevice, s));
        PXR_CUDA(h, cudaMemcpyAsync(t.vol, vol.data(), n_clusters * 4ull, cudaMemcpyHostToDevice, s));
        PXR_CUDA(h, cudaMemcpyAsync(t.vol_start, vol_start.data(), n_clusters * 4ull, cudaMemcpyHostToDevice, s));
        PXR_CUDA(h, cudaMemcpyAsync(t.root, root.data(), n_clusters * 4ull, cudaMemcpyHostToDevice, s));
    }
    PXR_CUDA(h, cudaStreamSynchronize(s));
    RoundCtr* c = h->h_ctr;
    PXR_CUDA(h, cudaMemcpyAsync(c, h->ctr, sizeof(RoundCtr), cudaMemcpyDeviceToHost, s));
    PXR_CUDA(h, cudaStreamSynchronize(s));
    c->n_active = n_act;
    c->n_clusters = n_clusters;
    c->smallest = smallest;
    c->full_components = full_components ? 1u : 0u;
    c->done = (n_act == 0 || n_clusters == 0) ? 1u : 0u;
    c->max_parent = 0xFFFFFFFFu;   // the given list has no run structure: sort globally first
    c->max_csize = n;
    PXR_CUDA(h, cudaMemcpyAsync(h->ctr, c, sizeof(RoundCtr), cudaMemcpyHostToDevice, s));
    pxr_status rs = reset_schedule_state(h);
    if (rs != PXR_OK) return rs;
    return pxr_set_potentials(h, x);
}

pxr_status pxr_set_schedule(pxr_handle* h, const pxr_schedule* cfg, const uint16_t* weights, const float* norm) {
    if (!h || !cfg) return PXR_INVALID_ARG;
    if (cfg->mode > PXR_SCHEDULE_AUDIT) return fail(h, PXR_INVALID_ARG, "unknown schedule mode");
    if (cfg->mode != PXR_SCHEDULE_PLAIN) {
        if (!weights || !norm) return fail(h, PXR_INVALID_ARG, "the learned schedule needs weights and norm");
        if (!(cfg->safety >= 0.0f) || cfg->max_skip > 0xFFFFu)
            return fail(h, PXR_INVALID_ARG, "safety must be >= 0 and max_skip below 65536");
        if (!(cfg->cut_gate >= 0.0f) || !(cfg->cut_gate <= 1.0f))
            return fail(h, PXR_INVALID_ARG, "cut_gate must lie in [0, 1]");
        if (cfg->due_period > 1024u) return fail(h, PXR_INVALID_ARG, "due_period must be at most 1024");
        std::vector<float> img(kMlpImage);
        for (int p = 0; p < kMlpParams; ++p) {
            const uint32_t b = (uint32_t)weights[p] << 16;
            std::memcpy(&img[p], &b, 4);
        }
        for (int i = 0; i < 2 * kMlpIn; ++i) img[kMlpParams + i] = norm[i];
        h->mlp_img = std::move(img);
    }
    const bool mode_changed = cfg->mode != h->sched.mode || (cfg->trace != 0) != (h->sched.trace != 0);
    h->sched = *cfg;
    if (mode_changed) drop_graphs(h);   // the captured round depends on the mode
    if (!h->allocs.empty()) {
        PXR_CUDA(h, cudaSetDevice(h->device));
        if (!h->mlp_img.empty())
            PXR_CUDA(h, cudaMemcpyAsync(h->mlp, h->mlp_img.data(), kMlpImage * 4, cudaMemcpyHostToDevice, h->stream));
        if (cfg->trace && !h->records) {
            const size_t N = std::max<uint32_t>(h->n, 1);
            cudaError_t e = dalloc(h, &h->records, N);
            if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc");
            h->records_n = (uint32_t)N;
            drop_graphs(h);
        }
        PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    return PXR_OK;
}

pxr_status pxr_read_cluster_records(pxr_handle* h, pxr_cluster_record* out, uint32_t cap, uint32_t* count) {
    if (!h || !count || (cap && !out)) return PXR_INVALID_ARG;
    if (!h->initialized) return fail(h, PXR_NOT_INITIALIZED, "no graph uploaded");
    if (!h->sched.trace || !h->records) return fail(h, PXR_INVALID_ARG, "trace is off");
    pxr_status st = sync_ctr(h);
    if (st != PXR_OK) return st;
    const uint32_t k = h->h_ctr->n_clusters;
    *count = k;
    const uint32_t w = std::min(cap, k);
    if (w) {
        PXR_CUDA(h, cudaMemcpyAsync(out, h->records, (size_t)w * sizeof(pxr_cluster_record), cudaMemcpyDeviceToHost,
                                    h->stream));
        PXR_CUDA(h, cudaStreamSynchronize(h->stream));
    }
    return PXR_OK;
}

pxr_status pxr_get_row_plan(pxr_handle* h, pxr_row_plan* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    *out = h->plan_info;
    return PXR_OK;
}

pxr_status pxr_get_sort_plan(pxr_handle* h, pxr_sort_plan* out) {
    if (!h || !out) return PXR_INVALID_ARG;
    *out = h->sort_info;
    return PXR_OK;
}

pxr_status pxr_set_sort_plan(pxr_handle* h, const pxr_sort_plan* plan) {
    if (!h) return PXR_INVALID_ARG;
    if (plan) {
        if (plan->plan >= (uint32_t)kSortPlanCount) return fail(h, PXR_INVALID_ARG, "sort plan must be 0, 1 or 2");
        if (plan->plan != h->sort_info.plan) drop_graphs(h);
        h->sort_forced = true;
        h->sort_info.plan = plan->plan;
        h->sort_info.items_per_thread = (uint32_t)kSortPlans[plan->plan].items;
        h->sort_info.ctas_per_sm = (uint32_t)kSortPlans[plan->plan].ctas;
        h->sort_info.source = 3;
    } else {
        h->sort_forced = false;   // the tuned or default plan returns with the next graph
    }
    return PXR_OK;
}

pxr_status pxr_set_row_plan(pxr_handle* h, const pxr_row_plan* plan) {
    if (!h) return PXR_INVALID_ARG;
    if (plan) {
        const uint32_t W = plan->lanes_per_row;
        if (!(W == 1 || W == 4 || W == 8 || W == 16 || W == 32))
            return fail(h, PXR_INVALID_ARG, "lanes_per_row must be 1, 4, 8, 16 or 32");
        if (plan->light_max == 0 || plan->wide_max < plan->light_max)
            return fail(h, PXR_INVALID_ARG, "need 0 < light_max <= wide_max");
        h->plan_info.lanes_per_row = W;
        h->plan_info.light_max = plan->light_max;
        h->plan_info.wide_max = plan->wide_max;
        h->plan_forced = true;
    } else {
        h->plan_forced = false;
    }
    if (!h->initialized) return PXR_OK;
    PXR_CUDA(h, cudaSetDevice(h->device));
    return h->off64 ? choose_row_plan<uint64_t>(h, true, h->nb_bits) : choose_row_plan<uint32_t>(h, true, h->nb_bits);
}

}  // extern "C"
