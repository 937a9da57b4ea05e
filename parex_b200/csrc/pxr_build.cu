// Graph construction on the device (sm_100a): the reference builds its CSR
// on the host (readDynGraph + DynamicGraph::finalize, lib/utils/graph_io.h:49-84,
// lib/core/graph.h:147-184: self-loops dropped, both directions of every edge,
// duplicates merged, rows sorted by neighbour id).  Here the same CSR comes from
// two 64-bit radix sorts with this library's onesweep sort:
//
//   1. pack every non-loop edge as (min << 32 | max) (compaction by atomic
//      counter: the order is irrelevant, a sort follows);
//   2. sort, keep the first of each run of equal keys, emit both directions
//      (src << 32 | dst);
//   3. sort again: the low words are the columns, row starts come from a
//      binary search for each vertex.
//
// Also an R-MAT edge sampler with the counter-based hash of the Python
// generator (parex_b200/graphs.py: rmat), so both produce the same graph.
#include <algorithm>
#include <cmath>

#include "pxr_sort.cuh"
#include "../../include/parex_b200.h"

namespace pxr {
namespace {

constexpr int kBuildBlock = 256;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// One quadrant choice per bit level from a 16-bit uniform; four levels per
// 64-bit hash of (seed, stream 1000 + level / 4, sample index).
__global__ void k_rmat(uint64_t samples, uint32_t scale, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t seed,
                       uint32_t* u, uint32_t* v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < samples;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t uu = 0, vv = 0;
        uint64_t h = 0;
        for (uint32_t lvl = 0; lvl < scale; ++lvl) {
            if ((lvl & 3u) == 0) {
                const uint64_t base = seed * 0x100000001B3ull + (uint64_t)(1000u + lvl / 4u) * 0x9E3779B1ull;
                h = splitmix64(splitmix64(i ^ base) + base);
            }
            const uint32_t r = (uint32_t)(h >> (16u * (lvl & 3u))) & 0xFFFFu;
            const uint32_t bit = 1u << (scale - 1u - lvl);
            if (r >= tab) uu |= bit;
            if ((r >= ta && r < tab) || r >= tabc) vv |= bit;
        }
        u[i] = uu;
        v[i] = vv;
    }
}

__global__ void k_pack_edges(const uint32_t* u, const uint32_t* v, uint64_t n_edges, uint32_t n, uint64_t* keys,
                             uint32_t* count, uint32_t* bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_edges;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = u[i], b = v[i];
        if (a >= n || b >= n) { atomicOr(bad, 1u); continue; }
        if (a == b) continue;
        const uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
        keys[atomicAdd(count, 1u)] = ((uint64_t)lo << 32) | hi;
    }
}

// first of each run of equal sorted keys -> both directions
__global__ void k_unique_both(const uint64_t* sorted0, const uint64_t* sorted1, const uint32_t* sel,
                              const uint32_t* count, uint64_t* out, uint32_t* out_count) {
    const uint64_t* k = *sel ? sorted1 : sorted0;
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t key = k[i];
        if (i > 0 && k[i - 1] == key) continue;
        const uint32_t lo = (uint32_t)(key >> 32), hi = (uint32_t)key;
        const uint32_t p = atomicAdd(out_count, 2u);
        out[p] = key;
        out[p + 1] = ((uint64_t)hi << 32) | lo;
    }
}

// columns and row starts of the sorted (src, dst) list
__global__ void k_csr_rows(const uint64_t* sorted0, const uint64_t* sorted1, const uint32_t* sel, const uint32_t* count,
                           uint32_t n, uint32_t* offsets, uint32_t* cols) {
    const uint64_t* k = *sel ? sorted1 : sorted0;
    const uint32_t total = *count;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < total; i += stride) cols[i] = (uint32_t)k[i];
    for (uint64_t v = tid; v <= n; v += stride) {
        const uint64_t target = v << 32;
        uint32_t lo = 0, hi = total;   // first position with key >= target
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (k[mid] < target) lo = mid + 1; else hi = mid;
        }
        offsets[v] = lo;
    }
}

// Planted-partition edges by geometric skipping: one thread per segment of a
// block pair's candidate range; a segment restarts the skipping (the gaps
// are memoryless).  Candidate k of an inter-block pair is (k / sv, k % sv);
// of an intra-block pair the k-th (row, col) with row < col in row order.
__device__ __forceinline__ double uniform_open(uint64_t& state) {
    state = splitmix64(state);
    return ((double)(state >> 11) + 1.0) * (1.0 / 9007199254740992.0);   // (0, 1]
}

__device__ __forceinline__ void tri_unrank(uint64_t k, uint64_t s, uint64_t* r, uint64_t* c) {
    // row r holds s - 1 - r candidates and starts at r (2s - r - 1) / 2
    const double b = 2.0 * (double)s - 1.0;
    int64_t row = (int64_t)((b - sqrt(b * b - 8.0 * (double)k)) / 2.0);
    if (row < 0) row = 0;
    auto start = [&](int64_t q) { return (uint64_t)q * (2 * s - (uint64_t)q - 1) / 2; };
    while (row > 0 && start(row) > k) --row;
    while ((uint64_t)row + 1 < s && start(row + 1) <= k) ++row;
    *r = (uint64_t)row;
    *c = k - start(row) + (uint64_t)row + 1;
}

__global__ void k_sbm_segments(const pxr_sbm_task* tasks, uint32_t n_tasks, const uint64_t* seg_prefix,
                               uint64_t n_segments, uint64_t seg_len, uint64_t seed, uint32_t* seg_count,
                               const uint64_t* seg_offset, uint32_t* u, uint32_t* v) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n_segments;
         g += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n_tasks;   // task: last t with seg_prefix[t] <= g
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (seg_prefix[mid] <= g) lo = mid; else hi = mid;
        }
        const pxr_sbm_task tk = tasks[lo];
        const uint64_t su = tk.su, sv = tk.sv;
        const uint64_t total = tk.intra ? su * (su - 1) / 2 : su * sv;
        const uint64_t k0 = (g - seg_prefix[lo]) * seg_len;
        const uint64_t k1 = min(total, k0 + seg_len);
        uint32_t drawn = 0;
        const uint64_t out = seg_offset ? seg_offset[g] : 0;
        if (tk.p > 0.0 && k0 < k1) {
            // the stream of segment (task key, segment within the task)
            const uint64_t local = g - seg_prefix[lo];
            const uint64_t sid = ((uint64_t)tk.key << 32) | local;
            uint64_t state = splitmix64(seed ^ splitmix64(sid * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull));
            const double lq = log1p(-min(tk.p, 1.0 - 1e-16));
            uint64_t k = k0;
            bool first = true;
            for (;;) {
                const double skip = floor(log(uniform_open(state)) / lq);
                if (!(skip < 1e18)) break;
                const uint64_t step = (uint64_t)skip + (first ? 0 : 1);
                first = false;
                if (step >= k1 - k) break;
                k += step;
                if (seg_offset) {
                    uint64_t a, b;
                    if (tk.intra) tri_unrank(k, su, &a, &b);
                    else { a = k / sv; b = k % sv; }
                    u[out + drawn] = tk.base_u + (uint32_t)a;
                    v[out + drawn] = tk.base_v + (uint32_t)b;
                }
                ++drawn;
            }
        }
        if (!seg_offset) seg_count[g] = drawn;
    }
}

__global__ void k_set_u32(uint32_t* p, uint32_t value) { *p = value; }

// DynamicGraph::finalize (lib/core/graph.h:147-184): both directions of every
// edge as it stands - self-loops and duplicate edges kept - sorted by
// (from, to) by the radix sort that follows.
__global__ void k_both_directions(const uint32_t* u, const uint32_t* v, uint64_t n_edges, uint32_t n, uint64_t* keys,
                                  uint32_t* bad) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_edges;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = u[i], b = v[i];
        if (a >= n || b >= n) { atomicOr(bad, 1u); keys[2 * i] = keys[2 * i + 1] = 0; continue; }
        keys[2 * i] = ((uint64_t)a << 32) | b;
        keys[2 * i + 1] = ((uint64_t)b << 32) | a;
    }
}

// ---------------------------------------------------------------------------
// Matrix Market body on the device.  readDynGraph (lib/utils/graph_io.h:49-84)
// reads the body as a stream of integers, "fx tx" per edge, 1-based, with no
// regard to lines; so does this tokenizer: a token is a maximal run of
// decimal digits, tokens 2i and 2i+1 are edge i.  Each thread owns
// kMtxBytes bytes and parses the tokens that start there (reading past its
// bytes to a token's end); a tile's tokens are numbered by a decoupled
// look-back over tile counts (tile ids taken in launch order).

constexpr uint32_t kMtxBytes = 16;
constexpr uint32_t kMtxTile = kBuildBlock * kMtxBytes;

__device__ __forceinline__ bool is_digit(unsigned char c) { return c >= '0' && c <= '9'; }

__global__ void __launch_bounds__(kBuildBlock) k_mtx_tokens(const unsigned char* text, uint64_t len, uint64_t n_edges,
                                                            uint32_t n, uint32_t* u, uint32_t* v, uint32_t* tile_ctr,
                                                            LookbackState lb, unsigned long long* tokens_out,
                                                            uint32_t* bad, uint32_t* err) {
    __shared__ uint64_t warp_tot[kBuildBlock / 32];
    __shared__ uint64_t s_excl;
    __shared__ uint32_t s_tile;
    const uint64_t ntiles = (len + kMtxTile - 1) / kMtxTile;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) return;
    const uint64_t b0 = (uint64_t)tile * kMtxTile + (uint64_t)threadIdx.x * kMtxBytes;
    uint32_t starts = 0;
    for (uint32_t q = 0; q < kMtxBytes; ++q) {
        const uint64_t i = b0 + q;
        if (i >= len) break;
        if (is_digit(text[i]) && (i == 0 || !is_digit(text[i - 1]))) starts |= 1u << q;
    }
    const uint32_t cnt = __popc(starts);
    uint64_t total;
    const uint64_t incl = block_inclusive<Add64>((uint64_t)cnt, warp_tot, &total);
    if (threadIdx.x < 32) {
        const uint64_t ex = lookback_tile<Add64>(lb, tile, 1u, total, err);
        if (threadIdx.x == 0) {
            s_excl = ex;
            if (tile == ntiles - 1) *tokens_out = ex + total;
        }
    }
    __syncthreads();
    uint64_t k = s_excl + incl - cnt;
    while (starts) {
        const uint32_t q = (uint32_t)__ffs(starts) - 1u;
        starts &= starts - 1u;
        uint64_t val = 0;
        bool big = false;
        for (uint64_t i = b0 + q; i < len && is_digit(text[i]); ++i) {
            val = val * 10u + (text[i] - '0');
            if (val > 0xFFFFFFFFull) { big = true; val = 0xFFFFFFFFull; }
        }
        if (k < 2 * n_edges) {
            // 1-based ids; 0 or ids above n have no vertex
            if (big || val == 0 || val > n) atomicOr(bad, 1u);
            const uint32_t id = (val >= 1 && val <= n) ? (uint32_t)(val - 1) : 0u;
            if (k & 1u) v[k >> 1] = id; else u[k >> 1] = id;
        }
        ++k;
    }
}

struct BuildLayout {
    size_t keys0, keys1, hist, bases, pass_info, tile_ctr, epoch, status, words, total;
    uint32_t tiles;
};

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

BuildLayout build_layout(uint64_t n_edges) {
    BuildLayout L{};
    const uint64_t cap = std::max<uint64_t>(2 * n_edges, 1);
    L.tiles = (uint32_t)((cap + kSortTile - 1) / kSortTile) + 1;
    size_t o = 0;
    L.keys0 = o; o = align256(o + cap * 8);
    L.keys1 = o; o = align256(o + cap * 8);
    L.hist = o; o = align256(o + kMaxPasses * kRadix * 4);
    L.bases = o; o = align256(o + kMaxPasses * kRadix * 4);
    L.pass_info = o; o = align256(o + (kMaxPasses + 1) * 4);
    L.tile_ctr = o; o = align256(o + kMaxPasses * 4);
    L.epoch = o; o = align256(o + 4);
    L.status = o; o = align256(o + (size_t)L.tiles * kRadix * 8);
    L.words = o; o = align256(o + 8 * 4);   // count0, count1, end_bit, err, bad
    L.total = o;
    return L;
}

// Expander hierarchy contraction (ExpanderHierarchy::contract,
// lib/algorithms/expander_hierarchy.h:34-88): one warp per vertex; every slot
// whose ends lie in different clusters becomes a (cluster, neighbour's
// cluster) key of the contracted graph and counts toward its cluster's cut;
// the cluster's volume adds the vertex's volume (its degree at the first
// level, its subtree volume above).
__global__ void k_contract_slots(uint32_t n, const uint32_t* off, const uint32_t* cols, const int32_t* ids,
                                 uint32_t k, const unsigned long long* level_vol, uint64_t* keys, uint32_t* count,
                                 unsigned long long* cut_sizes, unsigned long long* volumes, uint32_t* bad) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const int32_t c = ids[v];
        if (c < 0 || (uint32_t)c >= k) { if (lane == 0) atomicOr(bad, 1u); continue; }
        const uint32_t beg = off[v], end = off[v + 1];
        uint32_t cut = 0;
        for (uint32_t s = beg + lane; s < end; s += 32) {
            const uint32_t u = cols[s];
            if (u >= n) { atomicOr(bad, 1u); continue; }
            const int32_t cu = ids[u];
            if (cu == c) continue;
            ++cut;
            keys[atomicAdd(count, 1u)] = ((uint64_t)(uint32_t)c << 32) | (uint32_t)cu;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cut += __shfl_xor_sync(0xFFFFFFFFu, cut, o);
        if (lane == 0) {
            if (cut) atomicAdd(&cut_sizes[c], (unsigned long long)cut);
            atomicAdd(&volumes[c], level_vol ? level_vol[v] : (unsigned long long)(end - beg));
        }
    }
}

}  // namespace
}  // namespace pxr

using namespace pxr;

extern "C" {

pxr_status pxr_rmat_edges(uint32_t scale, uint64_t samples, double a, double b, double c, uint64_t seed, uint32_t* u,
                          uint32_t* v, void* stream) {
    if (scale == 0 || scale > 31 || (samples && (!u || !v))) return PXR_INVALID_ARG;
    if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return PXR_INVALID_ARG;
    if (!samples) return PXR_OK;
    // quadrant thresholds on a 16-bit uniform, rounded half to even as the Python generator does
    const uint32_t ta = (uint32_t)std::nearbyint(a * 65536.0);
    const uint32_t tab = (uint32_t)std::nearbyint((a + b) * 65536.0);
    const uint32_t tabc = (uint32_t)std::nearbyint((a + b + c) * 65536.0);
    const uint64_t blocks = std::min<uint64_t>((samples + kBuildBlock - 1) / kBuildBlock, 148u * 32u);
    k_rmat<<<(uint32_t)blocks, kBuildBlock, 0, static_cast<cudaStream_t>(stream)>>>(samples, scale, ta, tab, tabc,
                                                                                    seed, u, v);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}

pxr_status pxr_sbm_edges(const pxr_sbm_task* tasks, uint32_t n_tasks, const uint64_t* seg_prefix, uint64_t n_segments,
                         uint64_t segment_len, uint64_t seed, uint32_t* seg_count, const uint64_t* seg_offset,
                         uint32_t* u, uint32_t* v, void* stream) {
    if (!tasks || !seg_prefix || segment_len == 0 || n_tasks == 0) return PXR_INVALID_ARG;
    if (seg_offset ? (!u || !v) : !seg_count) return PXR_INVALID_ARG;
    if (!n_segments) return PXR_OK;
    const uint64_t blocks = std::min<uint64_t>((n_segments + kBuildBlock - 1) / kBuildBlock, 148u * 64u);
    k_sbm_segments<<<(uint32_t)blocks, kBuildBlock, 0, static_cast<cudaStream_t>(stream)>>>(
        tasks, n_tasks, seg_prefix, n_segments, segment_len, seed, seg_count, seg_offset, u, v);
    return cudaGetLastError() == cudaSuccess ? PXR_OK : PXR_CUDA_ERROR;
}

size_t pxr_build_csr_scratch_bytes(uint64_t n_edges) { return build_layout(n_edges).total; }

size_t pxr_parse_mtx_scratch_bytes(uint64_t text_bytes) {
    const uint64_t slots = (text_bytes + kMtxTile - 1) / kMtxTile + 1;   // look-back state per tile
    return 256 + align256(slots * 4) + 2 * align256(slots * 8);
}

pxr_status pxr_parse_mtx_body(const char* text, uint64_t text_bytes, uint32_t n, uint64_t n_edges, uint32_t* u,
                              uint32_t* v, void* scratch, uint64_t* tokens_out, void* stream) {
    if (!tokens_out || (text_bytes && (!text || !scratch)) || (n_edges && (!u || !v))) return PXR_INVALID_ARG;
    *tokens_out = 0;
    if (!text_bytes) return n_edges ? PXR_INVALID_ARG : PXR_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const uint64_t tiles = (text_bytes + kMtxTile - 1) / kMtxTile;
    if (tiles >= (1ull << 32)) return PXR_INVALID_ARG;
    unsigned char* base = static_cast<unsigned char*>(scratch);
    // words: tile counter, bad, err, pad | tokens (u64) | flags | agg | inc
    uint32_t* words = reinterpret_cast<uint32_t*>(base);
    unsigned long long* tokens = reinterpret_cast<unsigned long long*>(base + 16);
    LookbackState lb{};
    lb.flags = reinterpret_cast<uint32_t*>(base + 256);
    lb.agg = reinterpret_cast<uint64_t*>(base + 256 + align256((tiles + 1) * 4));
    lb.inc = reinterpret_cast<uint64_t*>(base + 256 + align256((tiles + 1) * 4) + align256((tiles + 1) * 8));
    if (cudaMemsetAsync(base, 0, 256 + align256((tiles + 1) * 4), s) != cudaSuccess) return PXR_CUDA_ERROR;
    k_mtx_tokens<<<(uint32_t)tiles, kBuildBlock, 0, s>>>(reinterpret_cast<const unsigned char*>(text), text_bytes,
                                                         n_edges, n, u, v, &words[0], lb, tokens, &words[1],
                                                         &words[2]);
    if (cudaGetLastError() != cudaSuccess) return PXR_CUDA_ERROR;
    uint32_t w[3] = {0, 0, 0};
    unsigned long long t = 0;
    if (cudaMemcpyAsync(w, words, 12, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaMemcpyAsync(&t, tokens, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    *tokens_out = t;
    if (w[2]) return PXR_DEVICE_FAULT;        // a look-back wait ran out
    if (t < 2 * n_edges || w[1]) return PXR_INVALID_ARG;   // too few numbers, or an id outside 1..n
    return PXR_OK;
}

pxr_status pxr_contract(uint32_t n, const uint32_t* offsets, const uint32_t* cols, const int32_t* ids, uint32_t k,
                        const uint64_t* level_volumes, void* scratch, uint32_t* out_offsets, uint32_t* out_cols,
                        uint64_t* out_m, uint64_t* cut_sizes, uint64_t* volumes, void* stream) {
    if (!offsets || !ids || !out_offsets || !out_m || !cut_sizes || !volumes || !scratch || k == 0 || k > n)
        return PXR_INVALID_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t slots = 0;
    if (cudaMemcpyAsync(&slots, offsets + n, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (slots && (!cols || !out_cols)) return PXR_INVALID_ARG;
    static bool prepared[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PXR_CUDA_ERROR;
    if (dev >= 0 && dev < 64 && !prepared[dev]) {
        if (radix_sort_prepare<uint64_t>() != cudaSuccess) return PXR_CUDA_ERROR;
        prepared[dev] = true;
    }
    // the layout of pxr_build_csr for slots / 2 edges: key buffers of `slots` entries
    const BuildLayout L = build_layout((slots + 1) / 2);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(base + L.keys0);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(base + L.keys1);
    uint32_t* words = reinterpret_cast<uint32_t*>(base + L.words);
    uint32_t *count = words, *end_bit = words + 2, *err = words + 3, *bad = words + 4;
    if (cudaMemsetAsync(base + L.hist, 0, L.total - L.hist, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaMemsetAsync(cut_sizes, 0, (size_t)k * 8, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaMemsetAsync(volumes, 0, (size_t)k * 8, s) != cudaSuccess) return PXR_CUDA_ERROR;
    uint32_t bits = 0;
    while (bits < 32 && (1ull << bits) < k) ++bits;
    k_set_u32<<<1, 1, 0, s>>>(end_bit, 32u + bits);
    const uint32_t grid = (uint32_t)std::min<uint64_t>(((uint64_t)n * 32 + kBuildBlock - 1) / kBuildBlock, 148u * 32u);
    if (n) k_contract_slots<<<grid, kBuildBlock, 0, s>>>(n, offsets, cols, ids, k,
                                                         reinterpret_cast<const unsigned long long*>(level_volumes),
                                                         k0, count, reinterpret_cast<unsigned long long*>(cut_sizes),
                                                         reinterpret_cast<unsigned long long*>(volumes), bad);
    SortState st{};
    st.hist = reinterpret_cast<uint32_t*>(base + L.hist);
    st.bases = reinterpret_cast<uint32_t*>(base + L.bases);
    st.pass_info = reinterpret_cast<uint32_t*>(base + L.pass_info);
    st.tile_ctr = reinterpret_cast<uint32_t*>(base + L.tile_ctr);
    st.epoch = reinterpret_cast<uint32_t*>(base + L.epoch);
    st.status = reinterpret_cast<uint64_t*>(base + L.status);
    st.max_tiles = L.tiles;
    st.items_moved = nullptr;
    SortBuffers<uint64_t> b{};
    b.keys[0] = k0;
    b.keys[1] = k1;
    b.count = count;
    b.end_bit = end_bit;
    b.capacity = std::max<uint32_t>(slots, 1);
    if (radix_sort<uint64_t>(b, st, err, s, 64) != cudaSuccess) return PXR_CUDA_ERROR;
    k_csr_rows<<<grid, kBuildBlock, 0, s>>>(k0, k1, st.pass_info + kMaxPasses, count, k, out_offsets,
                                            out_cols ? out_cols : reinterpret_cast<uint32_t*>(k1));
    uint32_t w[5] = {0, 0, 0, 0, 0};
    if (cudaMemcpyAsync(w, words, 20, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (w[4]) return PXR_INVALID_ARG;   // an id outside [0, k) or a column outside [0, n)
    if (w[3]) return PXR_DEVICE_FAULT;
    *out_m = w[0] / 2;
    return PXR_OK;
}

size_t pxr_contract_scratch_bytes(uint64_t slots) { return build_layout((slots + 1) / 2).total; }

pxr_status pxr_build_csr_finalize(uint32_t n, uint64_t n_edges, const uint32_t* u, const uint32_t* v, void* scratch,
                                  uint32_t* offsets, uint32_t* cols, void* stream) {
    if (!offsets || (n_edges && (!u || !v || !cols || !scratch))) return PXR_INVALID_ARG;
    if (n >= 0x7FFFFFFFu || 2 * n_edges >= (1ull << 32)) return PXR_INVALID_ARG;   // 32-bit offsets (EdgeIx)
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static bool prepared[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PXR_CUDA_ERROR;
    if (dev >= 0 && dev < 64 && !prepared[dev]) {
        if (radix_sort_prepare<uint64_t>() != cudaSuccess) return PXR_CUDA_ERROR;
        prepared[dev] = true;
    }
    const BuildLayout L = build_layout(n_edges);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(base + L.keys0);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(base + L.keys1);
    uint32_t* words = reinterpret_cast<uint32_t*>(base + L.words);
    uint32_t *count1 = words + 1, *end_bit = words + 2, *err = words + 3, *bad = words + 4;
    if (cudaMemsetAsync(base + L.hist, 0, L.total - L.hist, s) != cudaSuccess) return PXR_CUDA_ERROR;
    uint32_t bits = 0;
    while (bits < 32 && (1ull << bits) < n) ++bits;
    k_set_u32<<<1, 1, 0, s>>>(end_bit, 32u + bits);
    k_set_u32<<<1, 1, 0, s>>>(count1, (uint32_t)(2 * n_edges));
    const uint32_t grid = (uint32_t)std::min<uint64_t>((std::max<uint64_t>(n_edges, (uint64_t)n + 1) + kBuildBlock - 1) /
                                                           kBuildBlock, 148u * 32u);
    if (n_edges) k_both_directions<<<grid, kBuildBlock, 0, s>>>(u, v, n_edges, n, k0, bad);
    SortState st{};
    st.hist = reinterpret_cast<uint32_t*>(base + L.hist);
    st.bases = reinterpret_cast<uint32_t*>(base + L.bases);
    st.pass_info = reinterpret_cast<uint32_t*>(base + L.pass_info);
    st.tile_ctr = reinterpret_cast<uint32_t*>(base + L.tile_ctr);
    st.epoch = reinterpret_cast<uint32_t*>(base + L.epoch);
    st.status = reinterpret_cast<uint64_t*>(base + L.status);
    st.max_tiles = L.tiles;
    st.items_moved = nullptr;
    SortBuffers<uint64_t> b{};
    b.keys[0] = k0;
    b.keys[1] = k1;
    b.count = count1;
    b.end_bit = end_bit;
    b.capacity = (uint32_t)(2 * n_edges);
    if (radix_sort<uint64_t>(b, st, err, s, 64) != cudaSuccess) return PXR_CUDA_ERROR;
    k_csr_rows<<<grid, kBuildBlock, 0, s>>>(k0, k1, st.pass_info + kMaxPasses, count1, n, offsets, cols);
    uint32_t w[5] = {0, 0, 0, 0, 0};
    if (cudaMemcpyAsync(w, words, 20, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (w[4]) return PXR_INVALID_ARG;   // a vertex id >= n
    if (w[3]) return PXR_DEVICE_FAULT;  // a sort wait ran out
    return PXR_OK;
}

pxr_status pxr_build_csr(uint32_t n, uint64_t n_edges, const uint32_t* u, const uint32_t* v, void* scratch,
                         uint32_t* offsets, uint32_t* cols, uint64_t* m_out, void* stream) {
    if (!offsets || !m_out || (n_edges && (!u || !v || !cols || !scratch))) return PXR_INVALID_ARG;
    if (n >= 0x7FFFFFFFu || 2 * n_edges >= (1ull << 32)) return PXR_INVALID_ARG;   // 32-bit item counts and offsets
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    static bool prepared[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PXR_CUDA_ERROR;
    if (dev >= 0 && dev < 64 && !prepared[dev]) {
        if (radix_sort_prepare<uint64_t>() != cudaSuccess) return PXR_CUDA_ERROR;
        prepared[dev] = true;
    }
    const BuildLayout L = build_layout(n_edges);
    unsigned char* base = static_cast<unsigned char*>(scratch);
    uint64_t* k0 = reinterpret_cast<uint64_t*>(base + L.keys0);
    uint64_t* k1 = reinterpret_cast<uint64_t*>(base + L.keys1);
    uint32_t* words = reinterpret_cast<uint32_t*>(base + L.words);
    uint32_t *count0 = words, *count1 = words + 1, *end_bit = words + 2, *err = words + 3, *bad = words + 4;
    // sort state starts zeroed (histograms, epochs, status words)
    if (cudaMemsetAsync(base + L.hist, 0, L.total - L.hist, s) != cudaSuccess) return PXR_CUDA_ERROR;
    uint32_t bits = 0;
    while (bits < 32 && (1ull << bits) < n) ++bits;
    k_set_u32<<<1, 1, 0, s>>>(end_bit, 32u + bits);
    const uint32_t grid = (uint32_t)std::min<uint64_t>((std::max<uint64_t>(n_edges, (uint64_t)n + 1) + kBuildBlock - 1) /
                                                           kBuildBlock, 148u * 32u);
    if (n_edges) k_pack_edges<<<grid, kBuildBlock, 0, s>>>(u, v, n_edges, n, k0, count0, bad);
    SortState st{};
    st.hist = reinterpret_cast<uint32_t*>(base + L.hist);
    st.bases = reinterpret_cast<uint32_t*>(base + L.bases);
    st.pass_info = reinterpret_cast<uint32_t*>(base + L.pass_info);
    st.tile_ctr = reinterpret_cast<uint32_t*>(base + L.tile_ctr);
    st.epoch = reinterpret_cast<uint32_t*>(base + L.epoch);
    st.status = reinterpret_cast<uint64_t*>(base + L.status);
    st.max_tiles = L.tiles;
    st.items_moved = nullptr;
    SortBuffers<uint64_t> b{};
    b.keys[0] = k0;
    b.keys[1] = k1;
    b.count = count0;
    b.end_bit = end_bit;
    b.capacity = (uint32_t)n_edges;
    if (radix_sort<uint64_t>(b, st, err, s, 64) != cudaSuccess) return PXR_CUDA_ERROR;
    // the unique pass writes into the buffer the sort did not end in
    const uint32_t* sel = st.pass_info + kMaxPasses;
    uint32_t sel_host = 0;
    if (cudaMemcpyAsync(&sel_host, sel, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    uint64_t* uniq = sel_host ? k0 : k1;
    if (n_edges) k_unique_both<<<grid, kBuildBlock, 0, s>>>(k0, k1, sel, count0, uniq, count1);
    SortBuffers<uint64_t> b2{};
    b2.keys[0] = uniq;
    b2.keys[1] = sel_host ? k1 : k0;
    b2.count = count1;
    b2.end_bit = end_bit;
    b2.capacity = (uint32_t)(2 * n_edges);
    if (radix_sort<uint64_t>(b2, st, err, s, 64) != cudaSuccess) return PXR_CUDA_ERROR;
    // result buffer of the second sort relative to b2: pass_info[kMaxPasses] selects keys[0] or keys[1]
    uint32_t sel2 = 0;
    if (cudaMemcpyAsync(&sel2, sel, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    k_csr_rows<<<grid, kBuildBlock, 0, s>>>(b2.keys[0], b2.keys[1], sel, count1, n, offsets, cols);
    uint32_t w[5] = {0, 0, 0, 0, 0};
    if (cudaMemcpyAsync(w, words, 20, cudaMemcpyDeviceToHost, s) != cudaSuccess) return PXR_CUDA_ERROR;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PXR_CUDA_ERROR;
    (void)sel2;
    if (w[4]) return PXR_INVALID_ARG;   // a vertex id >= n
    if (w[3]) return PXR_DEVICE_FAULT;  // a sort wait ran out
    *m_out = w[1] / 2;
    return PXR_OK;
}

}  // extern "C"
