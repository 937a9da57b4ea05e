// Stable LSD radix sort for the sweep (sm_100a): onesweep passes with a
// decoupled look-back per digit.
//
// Keys are 32- or 64-bit, values optional 32-bit.  The item count and the
// number of key bits are read from device memory, and the buffer holding the
// result is recorded on the device (SortState::pass_info[kMaxPasses]), so a
// sort can be launched with host-side capacities only and captured in a CUDA
// graph.  Passes whose digit is the same for every key are skipped.
//
// Per pass and tile (kSortTile items): each warp ranks its items with
// __match_any_sync against a warp-private digit histogram in shared memory;
// thread d then publishes the tile's count of digit d, looks back over the
// preceding tiles' counts of d (status words stamped with a per-pass epoch,
// so the status area needs no clearing between sorts), and the tile is
// staged in shared memory in digit order before the coalesced scatter.
#pragma once

#include "pxr_common.cuh"

namespace pxr {

constexpr int kSortThreads = 256;
#ifndef PXR_SORT_ITEMS
#define PXR_SORT_ITEMS 16
#endif
constexpr int kSortItems = PXR_SORT_ITEMS;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadix = 256;
constexpr int kMaxPasses = 8;

struct SortState {
    uint32_t* hist;       // [kMaxPasses][kRadix] digit counts (kept zero between sorts)
    uint32_t* bases;      // [kMaxPasses][kRadix] exclusive digit bases
    uint32_t* pass_info;  // [kMaxPasses + 1]: bit0 active, bit1 input buffer; [kMaxPasses]: result buffer
    uint32_t* tile_ctr;   // [kMaxPasses]
    uint32_t* epoch;      // [1]
    uint64_t* status;     // [max_tiles][kRadix]
    uint32_t max_tiles;
    unsigned long long* items_moved;  // optional: [0] += items x active passes, [1] += active passes
};

template <typename K>
struct SortBuffers {
    K* keys[2];
    uint32_t* vals[2];        // both null for keys-only sorts
    const uint32_t* count;    // device
    const uint32_t* end_bit;  // device: sort bits [0, end_bit)
    uint32_t capacity;        // host bound on *count
};

// ---------------------------------------------------------------------------

template <typename K>
__global__ void __launch_bounds__(kSortThreads) sort_histogram_kernel(SortBuffers<K> b, SortState s) {
    __shared__ uint32_t sh[kMaxPasses][kRadix];
    for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) (&sh[0][0])[i] = 0;
    __syncthreads();
    const uint32_t count = *b.count;
    const uint32_t end_bit = *b.end_bit;
    const int npasses = (int)((end_bit + 7u) / 8u);
    const K* keys = b.keys[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const K k = keys[i];
        for (int p = 0; p < npasses; ++p) atomicAdd(&sh[p][(uint32_t)(k >> (8 * p)) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npasses * kRadix; i += blockDim.x) {
        const uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&s.hist[i], c);
    }
}

// One block of kRadix threads: digit bases, pass activity, buffer parity,
// fresh epoch and tile counters; leaves the histogram zeroed.
template <typename K>
__global__ void __launch_bounds__(kRadix) sort_plan_kernel(SortBuffers<K> b, SortState s) {
    __shared__ uint64_t warp_tot[kRadix / 32];
    __shared__ uint32_t constant_digit;
    const uint32_t count = *b.count;
    const uint32_t end_bit = *b.end_bit;
    const int npasses = (int)((end_bit + 7u) / 8u);
    const uint32_t d = threadIdx.x;
    uint32_t parity = 0;
    for (int p = 0; p < kMaxPasses; ++p) {
        const uint32_t c = p < npasses ? s.hist[p * kRadix + d] : 0u;
        if (d == 0) constant_digit = 0;
        __syncthreads();
        if (c == count && count > 0) constant_digit = 1;
        uint64_t total;
        const uint64_t incl = block_inclusive<Add64>((uint64_t)c, warp_tot, &total);
        s.bases[p * kRadix + d] = (uint32_t)(incl - c);
        if (p < npasses) s.hist[p * kRadix + d] = 0;
        const bool active = p < npasses && count > 0 && !constant_digit;
        if (d == 0) s.pass_info[p] = (active ? 1u : 0u) | (parity << 1);
        if (active) parity ^= 1u;
        if (d == 0) s.tile_ctr[p] = 0;
        __syncthreads();
    }
    if (d == 0) {
        s.pass_info[kMaxPasses] = parity;
        *s.epoch = *s.epoch + kMaxPasses;
        uint32_t active = 0;
        for (int p = 0; p < kMaxPasses; ++p) active += s.pass_info[p] & 1u;
        if (s.items_moved) {
            s.items_moved[0] += (unsigned long long)count * active;
            s.items_moved[1] += active;
        }
    }
}

__device__ __forceinline__ uint64_t sort_status_word(uint32_t epoch, uint32_t flag, uint32_t cnt) {
    return ((uint64_t)((epoch << 2) | flag) << 32) | cnt;
}

// A predecessor tile's status word for this epoch, polled at most spin_limit
// times; when it never arrives the error bit is set and the stale word is
// returned.  Tile ids are taken in launch order, so a predecessor is always
// resident or done and the limit (about a second) is reached only if the
// protocol itself is broken; the host then reports PXR_DEVICE_FAULT.
__device__ __forceinline__ uint64_t wait_sort_status(const uint64_t* word, uint32_t epoch, uint32_t* err,
                                                     uint32_t spin_limit = kSpinLimit) {
    uint64_t w = ld_relaxed64(word);
    uint32_t spins = 0;
    while ((uint32_t)(w >> 34) != (epoch & 0x3FFFFFFFu) || ((w >> 32) & 3u) == 0u) {
        if (++spins > spin_limit) { atomicOr(err, kErrSortTiles); break; }
        __nanosleep(32);
        w = ld_relaxed64(word);
    }
    return w;
}

#ifndef PXR_SORT_MIN_BLOCKS
#define PXR_SORT_MIN_BLOCKS 2
#endif
// One digit pass.  ITEMS keys per thread (tile = 256 ITEMS) and the CTAs per
// SM the register budget is sized for (MINB) are the sort plan's two axes
// (pxr_sort_plan); every plan gives the same output, item for item.
template <typename K, int ITEMS = kSortItems, int MINB = PXR_SORT_MIN_BLOCKS>
__global__ void __launch_bounds__(kSortThreads, MINB) sort_pass_kernel(SortBuffers<K> b, SortState s, int pass,
                                                                       uint32_t* err) {
    constexpr int kSortItems = ITEMS;
    constexpr int kSortTile = kSortThreads * ITEMS;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* skeys = reinterpret_cast<K*>(smem_raw);
    uint32_t* svals = reinterpret_cast<uint32_t*>(skeys + kSortTile);
    uint32_t (*whist)[kRadix] = reinterpret_cast<uint32_t (*)[kRadix]>(svals + kSortTile);
    __shared__ uint32_t tpre[kRadix];
    __shared__ uint32_t gbase[kRadix];
    __shared__ uint64_t warp_tot[kSortThreads / 32];
    __shared__ uint32_t s_tile;

    const uint32_t info = s.pass_info[pass];
    if (!(info & 1u)) return;
    const int in = (info >> 1) & 1;
    const K* kin = b.keys[in];
    K* kout = b.keys[in ^ 1];
    const uint32_t* vin = b.vals[in];
    uint32_t* vout = b.vals[in ^ 1];
    const bool has_vals = vin != nullptr;
    const uint32_t count = *b.count;
    const uint32_t num_tiles = (count + kSortTile - 1) / kSortTile;
    const uint32_t epoch = *s.epoch + (uint32_t)pass;
    const int shift = 8 * pass;

    if (threadIdx.x == 0) s_tile = atomicAdd(&s.tile_ctr[pass], 1u);
    for (int i = threadIdx.x; i < (kSortThreads / 32) * kRadix; i += kSortThreads) (&whist[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= num_tiles) return;

    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t base = tile * kSortTile + warp * (32 * kSortItems);
    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        const bool valid = idx < count;
        key[k] = valid ? kin[idx] : (K)0;
        val[k] = (valid && has_vals) ? vin[idx] : 0u;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        const bool valid = idx < count;
        const uint32_t d = valid ? ((uint32_t)(key[k] >> shift) & 0xFFu) : 0x100u;
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        // the lowest lane of each digit reads and advances the warp's count,
        // the others take the old count from it
        const uint32_t leader = (uint32_t)__ffs(peers) - 1u;
        uint32_t before = 0;
        if (valid && lane == leader) {
            before = whist[warp][d];
            whist[warp][d] = before + __popc(peers);
        }
        before = __shfl_sync(0xFFFFFFFFu, before, leader);
        rank[k] = before + __popc(peers & lt);
        __syncwarp();
    }
    __syncthreads();

    // digit d = threadIdx.x: per-warp exclusive offsets, tile count, look-back
    const uint32_t d = threadIdx.x;
    uint32_t tile_cnt = 0;
#pragma unroll
    for (int w = 0; w < kSortThreads / 32; ++w) {
        const uint32_t c = whist[w][d];
        whist[w][d] = tile_cnt;
        tile_cnt += c;
    }
    // a status word carries its own count, so relaxed accesses suffice (no fences)
    uint64_t* st = s.status + (size_t)tile * kRadix + d;
    st_relaxed64(st, sort_status_word(epoch, 1u, tile_cnt));
    uint32_t excl = 0;
    for (int32_t t = (int32_t)tile - 1; t >= 0; --t) {
        const uint64_t w = wait_sort_status(s.status + (size_t)t * kRadix + d, epoch, err);
        excl += (uint32_t)w;
        if (((w >> 32) & 3u) == 2u) break;
    }
    st_relaxed64(st, sort_status_word(epoch, 2u, excl + tile_cnt));
    gbase[d] = s.bases[pass * kRadix + d] + excl;
    uint64_t total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)tile_cnt, warp_tot, &total);
    tpre[d] = (uint32_t)incl - tile_cnt;
    __syncthreads();

#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t idx = base + k * 32 + lane;
        if (idx < count) {
            const uint32_t dg = (uint32_t)(key[k] >> shift) & 0xFFu;
            const uint32_t pos = tpre[dg] + whist[warp][dg] + rank[k];
            skeys[pos] = key[k];
            svals[pos] = val[k];
        }
    }
    __syncthreads();
    const uint32_t tile_items = min((uint32_t)kSortTile, count - tile * kSortTile);
    for (uint32_t j = threadIdx.x; j < tile_items; j += kSortThreads) {
        const K kk = skeys[j];
        const uint32_t dg = (uint32_t)(kk >> shift) & 0xFFu;
        const uint32_t out = gbase[dg] + (j - tpre[dg]);
        kout[out] = kk;
        if (has_vals) vout[out] = svals[j];
    }
}

template <typename K, int ITEMS = kSortItems>
constexpr size_t sort_pass_smem() {
    return (sizeof(K) + sizeof(uint32_t)) * kSortThreads * ITEMS + sizeof(uint32_t) * (kSortThreads / 32) * kRadix;
}

// Sort plans (items per thread, CTAs per SM) the tuner chooses from; plan 0
// is the default.  The smallest tile sets how many tile status words a sort
// may need (kSortMinTile).
struct SortPlanEntry { int items, ctas; };
constexpr SortPlanEntry kSortPlans[3] = {{16, 2}, {12, 3}, {8, 4}};
constexpr int kSortPlanCount = 3;
constexpr int kSortMinTile = kSortThreads * 8;

template <typename K, int ITEMS, int MINB>
inline void launch_sort_passes(const SortBuffers<K>& b, const SortState& s, uint32_t* err, cudaStream_t stream,
                               int npasses) {
    const uint32_t tiles = (b.capacity + kSortThreads * ITEMS - 1) / (kSortThreads * ITEMS);
    for (int p = 0; p < npasses; ++p)
        sort_pass_kernel<K, ITEMS, MINB><<<tiles, kSortThreads, sort_pass_smem<K, ITEMS>(), stream>>>(b, s, p, err);
}

// Launch a full sort on `stream` with sort plan `plan` (index into
// kSortPlans).  After it, s.pass_info[kMaxPasses] on the device names the
// buffer (0/1) holding the sorted keys and values.
template <typename K>
inline cudaError_t radix_sort(const SortBuffers<K>& b, const SortState& s, uint32_t* err, cudaStream_t stream,
                              int max_end_bit, int plan = 0) {
    if (b.capacity == 0) return cudaSuccess;
    const uint32_t tiles = (b.capacity + kSortTile - 1) / kSortTile;
    const uint32_t hgrid = min(tiles * 4u, 148u * 8u);
    sort_histogram_kernel<K><<<hgrid, kSortThreads, 0, stream>>>(b, s);
    sort_plan_kernel<K><<<1, kRadix, 0, stream>>>(b, s);
    const int npasses = (max_end_bit + 7) / 8;
    switch (plan) {
        case 1: launch_sort_passes<K, 12, 3>(b, s, err, stream, npasses); break;
        case 2: launch_sort_passes<K, 8, 4>(b, s, err, stream, npasses); break;
        default: launch_sort_passes<K, 16, PXR_SORT_MIN_BLOCKS>(b, s, err, stream, npasses); break;
    }
    return cudaGetLastError();
}

template <typename K>
inline cudaError_t radix_sort_prepare() {
    cudaError_t e = cudaFuncSetAttribute(sort_pass_kernel<K, 16, PXR_SORT_MIN_BLOCKS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sort_pass_smem<K, 16>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sort_pass_kernel<K, 12, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sort_pass_smem<K, 12>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(sort_pass_kernel<K, 8, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sort_pass_smem<K, 8>());
    return e;
}

}  // namespace pxr
