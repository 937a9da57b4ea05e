// Shared device helpers for the parex_b200 kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <cuda/atomic>

namespace pxr {

constexpr uint32_t kInvalidEdge = 0xFFFFFFFFu;
// A disabled CSR slot keeps its neighbour with the top bit set (vertex ids
// are below 2^31 - 1), so the graph as uploaded stays recoverable on the
// device; downloads show the reference's INVALID_EDGE there.
constexpr uint32_t kDisabledBit = 0x80000000u;
__host__ __device__ __forceinline__ bool slot_valid(uint32_t c) { return c < kDisabledBit; }
constexpr uint32_t kNoCut = 0xFFFFFFFFu;

// Device-side error bits, OR-ed into RoundCtr::err.
enum : uint32_t {
    kErrLookback = 1u << 0,      // a look-back wait ran out of iterations
    kErrUnionFind = 1u << 1,     // a union-find retry loop ran out of iterations
    kErrLabelRange = 1u << 2,    // a label fell outside the cluster tables
    kErrSortTiles = 1u << 3,     // a sort look-back wait ran out of iterations
};

// Spin bound for every device-side wait (about a second with the back-off below).
constexpr uint32_t kSpinLimit = 1u << 20;

// Look-back sites (dynamic tile counters and epochs), one per scan kernel.
constexpr int kSites = 12;

// The walk's traffic counters (vertices, slots, gathers) are spread over
// this many slot triples (block b adds to slot b mod kStatSlots) so that
// their atomics do not queue on one L2 address; the host sums the slots.
constexpr uint32_t kStatSlots = 32;

// Per-round scalars kept on the device so rounds need no host round trip.
struct RoundCtr {
    uint32_t n_active;        // active vertices (sweep input size)
    uint32_t n_clusters;      // active clusters, dense labels [0, n_clusters)
    uint32_t n_cut;           // clusters whose best sweep cut is below the threshold
    uint32_t n_roots;         // clusters after the components stage
    uint32_t n_keep;          // clusters kept active after recentering
    uint32_t n_active_next;   // vertices kept active after recentering
    int32_t smallest;         // label the reference's sort sees first this round
    int32_t smallest_next;    // the same for the next round
    uint32_t xmax_bits;       // max |x| over the vertices last updated (float bits)
    uint32_t xmax_walk_bits;  // max |x'| written by the last walk (float bits)
    uint32_t full_components; // run components over every cluster in the next cut
    uint32_t err;             // kErr* bits
    uint32_t tile_counter[kSites]; // dynamic tile ids for look-back kernels
    uint32_t rounds;          // rounds completed
    uint32_t done;            // set when no active cluster is left
    uint32_t main_sel;        // buffer holding the last sweep's sorted keys and values
    uint32_t sweep_n;         // items of the last sweep
    uint32_t sweep_k;         // clusters of the last sweep
    uint32_t loop_start;      // rounds at the start of the device-driven loop
    uint32_t loop_cap;        // round cap of the device-driven loop
    uint32_t n_sweep;         // vertices in this round's sweep (all active ones in the plain form)
    uint32_t n_due_items;     // vertices of the clusters swept and acted on this round
    uint32_t chunk_path;      // this round's sort runs chunk by chunk in shared memory
    uint32_t n_gsort;         // items of the global sort (0 on the chunk path)
    uint32_t max_parent;      // largest cluster of the previous round (bounds the active list's runs)
    uint32_t max_csize;       // largest cluster of this round
    uint32_t max_csize_next;  // largest cluster kept for the next round
    uint32_t walk_only;       // learned schedule: no cluster is due this round, only the walk runs
    uint32_t any_split;       // some cluster of this round is split (cut, or all components): union-find runs
    uint32_t n_cut_swept;     // n_cut of this round's sweep, kept through the cut stage (learned schedule's gate)
    unsigned long long stat_sort_items;     // traffic counters since initialisation (the walk's: kStatSlots)
    unsigned long long stat_sort_passes;
    unsigned long long stat_swept_items;     // sweep input vertices, summed over rounds
    unsigned long long stat_skipped;         // cluster-rounds whose sweep the schedule skipped
    unsigned long long stat_false_stops;     // skipped sweeps that would have cut (audit mode)
    unsigned long long stat_gsort_slots;     // round slots whose global-sort branch ran (graph driver)
    unsigned long long stat_chunk_slots;     // round slots whose chunked-sort branch ran (graph driver)
};

// ---------------------------------------------------------------------------
// ordered float bits: monotone map of float onto uint32 (cuda/devRandomWalk.h:50-61)

__host__ __device__ __forceinline__ uint32_t ordered_bits(float v) {
#ifdef __CUDA_ARCH__
    const uint32_t i = __float_as_uint(v);
#else
    uint32_t i;
    __builtin_memcpy(&i, &v, 4);
#endif
    const uint32_t mask = (i & 0x80000000u) ? 0xFFFFFFFFu : 0x80000000u;
    return i ^ mask;
}

__device__ __forceinline__ float from_ordered_bits(uint32_t o) {
    const uint32_t mask = (o & 0x80000000u) ? 0x80000000u : 0xFFFFFFFFu;
    return __uint_as_float(o ^ mask);
}

// exponent e of the exact fixed-point accumulation: |x| * 2^e * terms < 2^62
__device__ __forceinline__ int fixed_exponent(uint32_t xmax_bits, uint32_t nb_bits) {
    const float xmax = __uint_as_float(xmax_bits);
    if (!(xmax > 0.0f) || isinf(xmax)) return 0;
    int ex;
    frexpf(xmax, &ex);
    int e = 62 - ex - (int)nb_bits;
    e = e > 900 ? 900 : (e < -900 ? -900 : e);
    return e;
}

__device__ __forceinline__ double pow2(int e) {
    return __longlong_as_double((long long)(e + 1023) << 52);
}

__device__ __forceinline__ int64_t to_fixed(float v, double scale) {
    return __double2ll_rn(__dmul_rn((double)v, scale));
}

// ---------------------------------------------------------------------------
// device-scope atomics with explicit ordering

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> r(*const_cast<uint32_t*>(p));
    return r.load(cuda::memory_order_acquire);
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_release);
}
__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) {
    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> r(*const_cast<uint64_t*>(p));
    return r.load(cuda::memory_order_relaxed);
}
// Programmatic dependent launch: the round kernels are launched so that they
// may be scheduled while their predecessor in the stream drains; each waits
// here, before touching memory, until that predecessor has completed and its
// writes are visible (a no-op when the launch has no programmatic dependency).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
// Let the next kernel in the stream be scheduled now (its blocks still wait
// in pdl_wait for this kernel's completion); used by the one-block
// bookkeeping kernels, which leave the rest of the GPU idle.
__device__ __forceinline__ void pdl_launch_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

__device__ __forceinline__ void st_relaxed64(uint64_t* p, uint64_t v) {
    cuda::atomic_ref<uint64_t, cuda::thread_scope_device> r(*p);
    r.store(v, cuda::memory_order_relaxed);
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> r(*const_cast<uint32_t*>(p));
    return r.load(cuda::memory_order_relaxed);
}

// ---------------------------------------------------------------------------
// Decoupled look-back over tiles for an associative operator on uint64 values.
// flags[t] holds (epoch << 2) | f with f = 1 (aggregate ready) or 2
// (inclusive prefix ready); words from an older epoch read as "not ready",
// so the state needs no clearing between launches.

struct LookbackState {
    uint32_t* flags;
    uint64_t* agg;
    uint64_t* inc;
};

__device__ __forceinline__ void lookback_publish(LookbackState s, uint32_t tile, uint32_t epoch, uint32_t f,
                                                 uint64_t v) {
    st_relaxed64(f == 1u ? &s.agg[tile] : &s.inc[tile], v);
    st_release(&s.flags[tile], (epoch << 2) | f);
}

// Exclusive prefix of tile `tile` (Op::identity() for tile 0), computed by
// one whole warp: lane i waits for tile - 1 - i (bounded), the nearest
// predecessor holding an inclusive prefix ends the window, and the lanes up
// to it are combined.  Windows of 32 tiles repeat until an inclusive prefix
// (or tile 0) is reached.  Op must be commutative.  Every lane gets the result.
template <class Op>
__device__ __forceinline__ uint64_t lookback_exclusive(LookbackState s, uint32_t tile, uint32_t epoch,
                                                       uint32_t* err, uint32_t spin_limit = kSpinLimit) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t want = epoch & 0x3FFFFFFFu;
    uint64_t excl = Op::identity();
    for (int32_t base = (int32_t)tile - 1; base >= 0; base -= 32) {
        const int32_t t = base - (int32_t)lane;
        uint32_t f = 2u;               // tiles before 0 act as an empty inclusive prefix
        uint64_t v = Op::identity();
        if (t >= 0) {
            uint32_t w = ld_acquire(&s.flags[t]);
            uint32_t spins = 0;
            while ((w >> 2) != want || (w & 3u) == 0u) {
                if (++spins > spin_limit) { atomicOr(err, kErrLookback); w = (want << 2) | 2u; break; }
                __nanosleep(32);
                w = ld_acquire(&s.flags[t]);
            }
            f = w & 3u;
            if (spins <= spin_limit) v = (f == 2u) ? ld_relaxed64(&s.inc[t]) : ld_relaxed64(&s.agg[t]);
        }
        const uint32_t inc_lanes = __ballot_sync(0xFFFFFFFFu, f == 2u);
        const uint32_t stop = inc_lanes ? (uint32_t)(__ffs(inc_lanes) - 1) : 31u;
        uint64_t part = lane <= stop ? v : Op::identity();
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part = Op::combine(part, __shfl_xor_sync(0xFFFFFFFFu, part, o));
        excl = Op::combine(part, excl);
        if (inc_lanes) break;
    }
    return excl;
}

// One tile's part of a decoupled look-back, called by warp 0 of the block:
// publish the aggregate, look back, publish the inclusive prefix.  Returns the
// exclusive prefix in every lane of warp 0.
template <class Op>
__device__ __forceinline__ uint64_t lookback_tile(LookbackState s, uint32_t tile, uint32_t epoch, uint64_t aggregate,
                                                  uint32_t* err) {
    const uint32_t lane = threadIdx.x & 31u;
    if (tile == 0) {
        if (lane == 0) lookback_publish(s, tile, epoch, 2u, aggregate);
        return Op::identity();
    }
    if (lane == 0) lookback_publish(s, tile, epoch, 1u, aggregate);
    const uint64_t ex = lookback_exclusive<Op>(s, tile, epoch, err);
    if (lane == 0) lookback_publish(s, tile, epoch, 2u, Op::combine(ex, aggregate));
    return ex;
}

// lane-wise addition of two packed uint32 lanes
struct PairAdd {
    __device__ __forceinline__ static uint64_t identity() { return 0ull; }
    __device__ __forceinline__ static uint64_t combine(uint64_t a, uint64_t b) {
        const uint32_t lo = (uint32_t)a + (uint32_t)b;
        const uint32_t hi = (uint32_t)(a >> 32) + (uint32_t)(b >> 32);
        return ((uint64_t)hi << 32) | lo;
    }
};

struct Add64 {
    __device__ __forceinline__ static uint64_t identity() { return 0ull; }
    __device__ __forceinline__ static uint64_t combine(uint64_t a, uint64_t b) { return a + b; }
};

// ---------------------------------------------------------------------------
// warp / block scans

template <class Op>
__device__ __forceinline__ uint64_t warp_inclusive(uint64_t v) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t u = __shfl_up_sync(0xFFFFFFFFu, v, o);
        if (lane >= (uint32_t)o) v = Op::combine(u, v);
    }
    return v;
}

// Block-wide inclusive scan of one value per thread.  `warp_tot` is shared
// scratch of blockDim/32 entries.  Returns the inclusive value; *total gets
// the block aggregate (valid in every thread).
template <class Op>
__device__ __forceinline__ uint64_t block_inclusive(uint64_t v, uint64_t* warp_tot, uint64_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nwarps = blockDim.x >> 5;
    v = warp_inclusive<Op>(v);
    if (lane == 31u) warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        uint64_t w = lane < nwarps ? warp_tot[lane] : Op::identity();
        w = warp_inclusive<Op>(w);
        if (lane < nwarps) warp_tot[lane] = w;
    }
    __syncthreads();
    if (warp > 0) v = Op::combine(warp_tot[warp - 1], v);
    *total = warp_tot[nwarps - 1];
    __syncthreads();
    return v;
}

// ---------------------------------------------------------------------------
// 64-bit min / max atomics on float-ordered bits and signed sums

__device__ __forceinline__ void atomic_add_i64(int64_t* p, int64_t v) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), (unsigned long long)v);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace pxr
